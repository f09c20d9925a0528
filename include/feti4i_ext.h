/*
 * Extensions of the FETI4I interface for the B200 dual solver.
 *
 * All of these are additive: none changes a reference signature.  Options
 * the reference keeps in its ECF configuration (src/config/ecf/solver/feti.h)
 * but does not expose through FETI4I (schur precision, scaling, ...) are set
 * here; data the reference computes with METIS inside API::load (the
 * subdomain partition, src/input/api/api.cpp:106) is supplied by the caller.
 */
#ifndef FETI4I_EXT_H_
#define FETI4I_EXT_H_

#include "feti4i.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Message of the last failing FETI4I call of this thread ("" if none); the
 * reference prints and calls exit() instead (src/basis/logging/logging.cpp:103-131). */
const char *FETI4IGetLastError(void);

/* Element -> subdomain map (size = number of added elements); replaces the
 * METIS partition of API::load (src/input/api/api.cpp:106).  Without it the
 * elements are split into FETI4I_SUBDOMAINS contiguous blocks. */
void FETI4ISetSubdomainPartition(FETI4IMatrix matrix, FETI4IInt size, FETI4IInt *elem2sub);

/* Subdomain -> cluster map for FETI_METHOD = 1 (HYBRID_FETI).  The reference runs
 * one cluster per MPI process (src/mesh/preprocessing/fetidata.cpp:146-188,
 * src/assembler/constraints/equalityconstraints.cpp:504-555); here one process
 * holds several clusters.  Without it HYBRID_FETI uses one cluster of all
 * subdomains, as a single reference process does. */
void FETI4ISetClusterPartition(FETI4IMatrix matrix, FETI4IInt nsubdomains, const FETI4IInt *sub2cluster);

/* Batched FETI4IAddElement (src/app/apiwrapper/wrapper.cpp:140-165): nelems
 * elements with the same node/DOF counts, arrays laid out element after element. */
void FETI4IAddElements(FETI4IMatrix matrix, FETI4IInt type, FETI4IInt nelems, FETI4IInt nodesSize, FETI4IInt *nodes,
                       FETI4IInt dofsSize, FETI4IInt *dofs, FETI4IReal *values);

/* FETI4IUpdateStiffnessMatrix with K_e := scale[e] * K_e of `matrix` (one scale per stored element),
 * e.g. the densities of a topology-optimisation step applied to unit-modulus element matrices.
 * Like FETI4IUpdateStiffnessMatrix (which here also keeps the decomposition when the element
 * structure and partition are unchanged), it repeats the subdomain factorisations and the Schur
 * complements.  No counterpart in the reference; it saves the caller building and passing scaled
 * copies of every element matrix. */
void FETI4IUpdateStiffnessMatrixScaled(FETI4IInstance instance, FETI4IMatrix matrix, FETI4IInt size,
                                       const FETI4IReal *scale);

/* Extended options, read by FETI4ICreateInstance (process-wide, like the
 * reference's global ECF configuration). */
typedef enum {
    FETI4I_EXT_SCHUR_PRECISION,  /* 0 FP64 (reference DOUBLE), 1 FP32 (reference SINGLE), 2 BF16 + per-tile scale */
    FETI4I_EXT_SCALING,          /* 1: K-diagonal B1 scaling (reference default), 0: 1/multiplicity */
    FETI4I_EXT_HOST_ONLY,        /* 1: run the host preprocessing only (no GPU; FETI4ISolve fails) */
    FETI4I_EXT_TILES_PER_ITEM,   /* work-queue granularity of the Schur SYMV (autotuned default 48) */
    FETI4I_EXT_GRAPH_CHUNK,      /* PCG iterations per captured CUDA graph (default 16) */
    FETI4I_EXT_RELIABLE_DELTA,   /* mixed precision: residual replacement threshold (default 0.003) */
    FETI4I_EXT_HOST_THREADS,     /* OpenMP threads of the preprocessing (0: all) */
    FETI4I_EXT_TILE_KERNEL,      /* Schur SYMV: 0 register-prefetch loads, 1 TMA bulk-copy pipeline */
    FETI4I_EXT_AUTOTUNE,         /* 1 (default): time both SYMV variants and the work-item sizes per size class */
    FETI4I_EXT_SYMM_TENSOR,      /* multi-RHS solves with FP32 Schur storage: 1 (default) tcgen05 tensor-core SYMM
                                    (3xTF32, 8 or more right-hand sides), 0 CUDA-core SYMM */
    FETI4I_EXT_DEVICE_PREP,      /* 1 (default): subdomain eliminations and Schur complements S_i on the GPU
                                    (batched FP64 partial Cholesky of [K_reg B^T; B 0]); 0, or HOST_ONLY: host
                                    dense path.  The reference assembles S_i on the host
                                    (SparseSolverMKL.cpp:1207) */
    FETI4I_EXT_SCHUR_EXPLICIT,   /* 1 (default): F applied through stored Schur complements S_i (the reference's
                                    use_schur_complement); 0: through the subdomains' K^+ factors, with no S_i stored
                                    (the reference's default, itersolvercpu.cpp:73-106; FP64, Total FETI, one
                                    right-hand side) */
    FETI4I_EXT_OWNED_FIRST,      /* partitioned dual problem: first subdomain of this process's block */
    FETI4I_EXT_OWNED_COUNT,      /* ... and its size (0, default: all subdomains).  The reference splits the
                                    subdomains over MPI processes and sums the shared multipliers between them
                                    (itersolver.cpp:6373-6406); here every process numbers the whole problem,
                                    prepares and uploads only its block, and a driver (espreso_b200.partitioned)
                                    runs the dual PCG with the operators below and one allreduce per apply. */
    FETI4I_EXT_TRUNCATE,         /* 1: FETI4ISolve / FETI4ISolveMulti return the solution truncated as the reference's
                                    FETISolver::solve does (FETISolver.cpp:130-147): to 1 / PRECISION places relative
                                    to 10^ceil(log10 max|u|), per load case; 0 (default): the full FP64 solution */
    FETI4I_EXT_OPTIONS_SIZE
} FETI4IExtOptions;
void FETI4ISetExtendedOption(FETI4IInt key, FETI4IReal value);

/* Extended option of one instance (the per-instance form of FETI4ISetExtendedOption, which only
 * sets the defaults of instances created afterwards).  FETI4I_EXT_RELIABLE_DELTA, GRAPH_CHUNK, TRUNCATE and
 * SYMM_TENSOR apply to the next solve; the others (Schur precision, scaling, tiles, device or host
 * preprocessing) redo the instance's preprocessing and upload with its decomposition kept. */
void FETI4ISetExtendedOptions(FETI4IInstance instance, FETI4IInt key, FETI4IReal value);

/* Statistics of an instance (indices of FETI4IStatIndex). */
typedef enum {
    FETI4I_STAT_ITERATIONS,
    FETI4I_STAT_CONVERGED,
    FETI4I_STAT_DUAL_SIZE,
    FETI4I_STAT_KERNEL_SIZE,
    FETI4I_STAT_SUBDOMAINS,
    FETI4I_STAT_PREP_SECONDS,       /* host factorisation + Schur assembly */
    FETI4I_STAT_UPLOAD_SECONDS,
    FETI4I_STAT_SOLVE_MS,           /* device time of the dual PCG */
    FETI4I_STAT_SOLVE_WALL_MS,      /* wall time of the last FETI4ISolve */
    FETI4I_STAT_FAPPLY_BYTES,       /* algorithmic bytes of one F apply (iteration precision) */
    FETI4I_STAT_REPLACEMENTS,
    FETI4I_STAT_KERNEL_LAUNCHES,
    FETI4I_STAT_DEVICE_BYTES,
    FETI4I_STAT_FINAL_NORM,
    FETI4I_STAT_TOLERANCE,
    FETI4I_STAT_ELEMENTS,           /* stored elements */
    FETI4I_STAT_PREP_DEVICE_MS,     /* device time of the GPU eliminations (FETI4I_EXT_DEVICE_PREP), else 0 */
    FETI4I_STAT_PREP_DEVICE_FLOPS,  /* their algorithmic FP64 flops */
    FETI4I_STAT_KPLUS_TILES,        /* fraction of the stored K+ factor tiles that are not all zero (applied) */
    FETI4I_STAT_SIZE
} FETI4IStatIndex;
void FETI4IGetStats(FETI4IInstance instance, FETI4IInt size, FETI4IReal *stats);

/* Result of the SYMV autotuner of an instance, e.g. "f64:ldg[48,48,128,..] low:tma[..]"
 * (pointer valid until the next call on this thread). */
const char *FETI4IGetTuning(FETI4IInstance instance);

/* Dual solution lambda (dual size) and rigid-body amplitudes (kernel size) of the last solve. */
void FETI4IGetDualSolution(FETI4IInstance instance, FETI4IReal *lambda, FETI4IReal *amplitudes);

/* Introspection of the preprocessing (host data; used by the parity tests). */
/* info: [ndofs, rows of B_i, kernel dimension, touched DOFs] */
void FETI4IGetSubdomainInfo(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *info);
/* per local multiplier: global index, local DOF, sign, B1 scale, Dirichlet value */
void FETI4IGetSubdomainMultipliers(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *lambda, FETI4IInt *dof,
                                   FETI4IReal *sign, FETI4IReal *weight, FETI4IReal *c);
/* local node -> caller node */
void FETI4IGetSubdomainNodes(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *nodes);
/* S_i = B_i K_i^+ B_i^T, rows x rows column-major */
void FETI4IGetSubdomainSchur(FETI4IInstance instance, FETI4IInt subdomain, FETI4IReal *S);
/* kernel basis R_i, ndofs x kernel column-major */
void FETI4IGetSubdomainKernel(FETI4IInstance instance, FETI4IInt subdomain, FETI4IReal *R);
/* x := K_reg^-1 x for one subdomain (host factor; local DOF order) */
void FETI4IApplySubdomainKplus(FETI4IInstance instance, FETI4IInt subdomain, FETI4IReal *x);
/* HYBRID_FETI corner rows B0 of one subdomain: cluster-local row, local DOF and sign per entry
 * (one DOF per row).  Returns the entry count; null arrays only query it. */
FETI4IInt FETI4IGetSubdomainCorners(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *rows, FETI4IInt *dofs,
                                    FETI4IReal *signs);
/* info[0] FETI method, info[1] clusters (subdomains for TOTAL_FETI), info[2] corner rows over all
 * clusters, info[3] dual kernel dimension */
void FETI4IGetClusterInfo(FETI4IInstance instance, FETI4IInt *info);
/* b (dual size) and e (kernel size) of the current right-hand side */
void FETI4IGetDualRhs(FETI4IInstance instance, FETI4IReal *b, FETI4IReal *e);

/* y = F x on the GPU with the Schur complements in the given precision (0/1/2). */
void FETI4IApplyDualOperator(FETI4IInstance instance, FETI4IInt precision, FETI4IReal *x, FETI4IReal *y);
/* y_j = F x_j for nrhs <= 32 dual vectors (vector j at j * dual size) through the multi right-hand-side
   F apply of FETI4ISolveMulti (tile SYMM in the given Schur precision; introspection) */
void FETI4IApplyDualOperatorMulti(FETI4IInstance instance, FETI4IInt precision, FETI4IInt nrhs, FETI4IReal *x,
                                  FETI4IReal *y);
/* Partitioned dual problem (FETI4I_EXT_OWNED_COUNT > 0), device memory of the caller, dual vectors in the
 * whole problem's multiplier numbering (dual size entries): y += sum over this instance's subdomains of
 * B_i S_i B_i^T x (the F apply of itersolvercpu.cpp:9-114 before All_Reduce_lambdas_compB), and
 * y += sum of W_i B_i M_i B_i^T W_i x (Apply_Prec, itersolvercpu.cpp:520-602, before its allreduce).  The
 * caller sums y over the processes.  stream: a cudaStream_t the calls are ordered after and before,
 * or NULL for the default stream. */
void FETI4IApplyDualOperatorDevice(FETI4IInstance instance, FETI4IInt precision, const FETI4IReal *x, FETI4IReal *y,
                                   void *stream);
void FETI4IApplyPreconditionerDevice(FETI4IInstance instance, const FETI4IReal *x, FETI4IReal *y, void *stream);
/* Primal recovery u_i = K_i^+ (f_i - B_i^T lambda) + R_i alpha_i of this instance's subdomains
 * (itersolver.cpp:372-431) from host lambda (whole problem's numbering) and the amplitudes of its own
 * kernel numbering (FETI4IGetStats kernel size entries), averaged into caller DOFs with the weights of
 * the whole problem: summed over the processes it is the solution. */
void FETI4IPrimalFromDual(FETI4IInstance instance, const FETI4IReal *lambda, const FETI4IReal *amplitudes,
                          FETI4IInt solution_size, FETI4IReal *solution);

/* Average device time in ms of one F apply over `reps` launches (inputs resident). */
FETI4IReal FETI4ITimeDualOperator(FETI4IInstance instance, FETI4IInt precision, FETI4IInt reps);
/* Several load cases at once (the reference has no multi-RHS path): nrhs right-hand
 * sides (1..32) in rhs[j * size + i] are solved together by a block PCG whose F apply is a
 * tile SYMM; solutions[j * size + i].  LUMPED, WEIGHT_FUNCTION or no preconditioner. */
void FETI4ISolveMulti(FETI4IInstance instance, FETI4IInt nrhs, FETI4IInt size, const FETI4IReal *rhs,
                      FETI4IReal *solutions);
/* Re-solve the last FETI4ISolveMulti right-hand sides on the device; returns the device ms. */
FETI4IReal FETI4ISolveMultiResident(FETI4IInstance instance, FETI4IInt nrhs);

/* Solve on device-resident data only (right-hand side already uploaded by a
 * previous FETI4ISolve): returns the device time in ms of the dual PCG. */
FETI4IReal FETI4ISolveResident(FETI4IInstance instance);
/* Select the operator precision of the following solves (must have been prepared). */
void FETI4ISetSolvePrecision(FETI4IInstance instance, FETI4IInt precision);

/* Element energies out[e] = v_e^T K_e u_e for every stored element (in the order
 * they were added; elements skipped by the zero-row rule are not stored), with u
 * and v caller DOF vectors of length size.  For an adjoint solve v (K v = dL/du,
 * zero Dirichlet values) this gives dL/drho_e = -(dK_e/drho_e : ...) when K_e
 * scales with a material parameter: dL/dp_e = -(dE_e/dp_e / E_e) * out[e].
 * Computed on the GPU (no counterpart in the reference). */
void FETI4IElementEnergies(FETI4IInstance instance, FETI4IInt size, const FETI4IReal *u, const FETI4IReal *v,
                           FETI4IReal *out);

/* Allocation-free batched SYMV: y_m = S_m x_m for m < nmatrices (no counterpart in
 * the reference).  For callers that manage all device memory themselves and may
 * not allocate while they run (for example a finite-element code that reserves
 * its HBM pool at start-up): every pointer is caller-owned device memory and
 * the call allocates nothing.  Layout: matrix m of order order[m] <= max_order
 * is stored from tile tile_offset[m] of `tiles` as its T(T+1)/2 upper 32x32
 * tiles, T = ceil(order/32), tile (I,J), I <= J, in row-major tile order, each
 * tile row-major FP64, diagonal tiles holding the full symmetric block, zero
 * padding beyond the order.  x and y use vector_offset[m].  If `dot` is not
 * NULL the total x.y lands there (device memory).  Limits: nmatrices <= 16384
 * and max_order <= 3200; larger values are rejected with an error (return -1,
 * message in FETI4IGetLastError).  A matrix whose order exceeds max_order (or is
 * negative) gets no product: its y range is filled with NaN and *dot is NaN.  The
 * scratch (work-queue counters, one dot partial per matrix) is a static array
 * in device memory, held by every GPU that loads the library until exit; the
 * first call on a device looks up its address, so that call should come before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * race.  stream: a cudaStream_t, or NULL for the default stream. */
int FETI4ITiledSymvNoAlloc(const FETI4IReal *tiles, const long long *tile_offset, const FETI4IInt *order,
                           const FETI4IInt *vector_offset, FETI4IInt nmatrices, FETI4IInt max_order,
                           const FETI4IReal *x, FETI4IReal *y, FETI4IReal *dot, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FETI4I_EXT_H_ */
