// Total-FETI dual PCG on one B200 (sm_100a): tiled Schur-complement SYMV
// work queue, projector, lumped/Dirichlet preconditioners and the PCG
// recurrences over replicated local dual vectors, captured in CUDA graphs.
//
// Reference behaviour restated here:
//   PCG recurrences, stop rule ........ src/solver/specific/itersolver.cpp:1406-1724
//   projector P = I - G^T (GG^T)^-1 G .. src/solver/specific/itersolver.cpp:5541-5623
//   F apply (explicit S_i) ............ src/solver/specific/cpu/itersolvercpu.cpp:49-70
//   preconditioners ................... src/solver/specific/cpu/itersolvercpu.cpp:520-602
//   FP32 Schur path (x->float, float accumulate, y->double)
//                                       src/solver/generic/SparseMatrix.cpp:1093-1160
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>

#include "common.h"
#include "dense.h"
#include "gpu_prep.h"
#include "gpu_solver.h"

#define CUDA_CHECK(x)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            throw ::feti::Error(std::string("CUDA error ") + cudaGetErrorString(e_) + " in " #x); \
    } while (0)

namespace feti {

namespace {

constexpr int KMAX = 8;        // kernel dimension bound per subdomain (elasticity: 6)
constexpr int TPB = 256;       // threads of the per-subdomain kernels
constexpr int TPB1 = 512;      // threads of the single right-hand-side w/preconditioner kernel
constexpr int TPBB = 1024;     // threads of the per-subdomain block (multi right-hand-side) kernels
constexpr int TILE = 32;       // Schur tile edge
constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------------------------
// device state shared by the kernels of one solve
struct DevState {
    int conv_iter;      // first iteration whose check passed, -1 while running
    int iter_base;      // iteration index of slot 0 of the current graph chunk
    int replace_iter;   // mixed precision: iteration that starts with r = b - F64 x (-1: none pending)
    int true_iter;      // iteration whose starting residual was computed in FP64 from x
    int replacements;
    int max_it;
    int mixed;
    int error;          // set by a kernel whose bounded wait ran out (pipeline stalled)
    double tol;
    double precision;
    double rmax;        // largest projected residual norm since the last replacement
    double delta;       // replacement threshold
    double last_norm;
};

struct DevProblem {
    int nd, NL, nK, NT, KS;     // KS: row stride of the G coefficient arrays (max kernel dimension)
    int nP;                 // partial G-products: one block per subdomain (nP = nK for Total FETI)
    const int *loff;        // nd+1
    const int *kof;         // nd+1 offsets of the subdomains' partial G-product blocks
    const int *akof;        // nd: offset of the subdomain's kernel block in the dual kernel space
    const int *toff;        // nd+1 T-space offsets
    const int *partner;     // NL: row of the other owner, -1
    const int *tidx;        // NL: global T index of the row's DOF
    const int *ptidx;       // NL: T index of the partner row, -1
    const double *ws;       // NL: B1 weight * sign
    const double *pws;      // NL: partner's weight * sign, 0
    const double *minv;     // NL: 1 / multiplicity
    const double *Gl;       // NL*KS: G coefficients of the row
    const double *Gp;       // NL*KS: G coefficients of the partner row
    const int *rkof, *rnk;  // NL: dual kernel offset / dimension of the row's subdomain
    const int *pkof, *pnk;  // NL: same for the partner's subdomain (pnk = 0 without partner)
    const int *trow_ptr;    // NT+1
    const int *trow_idx;    // rows of each T index
    const int *slice0;      // nd+1: lumped K_TT in sliced ELL (32 T rows per slice)
    const int *ell_ptr;     // per slice: offset of its column-major block
    const int *ell_w;       // per slice: width
    const unsigned short *ell_col;  // column (T index inside the subdomain)
    const double *ell_val;
    const int *tbase;       // NT: first T index of the subdomain owning each T index
    const int *tslot;       // NT: (ELL slice << 5) | row within the slice
    const double *GGtinv;   // nK x nP, row-major: (GG^T)^-1 times the sum over partial blocks
    const double *bL;       // NL replicated b
    double *x, *r, *w, *z, *y, *p, *Ap, *uT, *vT, *d, *alpha;
    double *part_w, *part_rho, *part_b, *rho_hist;
    double *scal;           // grid totals (SC_*)
    int *done;              // completion counters of the last-CTA reductions (DONE_*)
    DevState *st;
};

enum { SC_RHO = 0, SC_PAP = 1, SC_WN2 = 2, SC_BN2 = 3, SC_PN2 = 4, SC_COUNT = 8 };

// block (multi right-hand-side) solver vectors: [row][rhs]
struct BlockDev {
    int nr;              // right-hand sides (power of two <= 32)
    int lg;              // log2(nr)
    double *x, *r, *w, *z, *y, *p, *Ap, *Ax, *bL, *uT, *vT, *d, *alpha, *e;
    float *p32;          // FP32 copy of p (SYMM input in mixed precision)
    double *part;        // nd * nr partials
    double *unit_dot;    // SYMM work units * nr
    double *scal;        // SC_COUNT * nr
    double *rho_hist;    // (max_it + 64) * nr
    double *tol, *rmax, *last_norm;  // nr
    int *conv;           // nr: iteration whose stop test passed, -1
    int *done;           // DONE_COUNT counters
    int *queue;          // SYMM work queue [2]
    int n_conv_target;
};
enum { DONE_W = 0, DONE_RHO = 1, DONE_B = 2, DONE_PN = 3, DONE_PAP_IMPLICIT = 4, DONE_COUNT = 8 };

// Hybrid Total FETI cluster correction: F_c = sum_i B_i S_i B_i^T - V M V^T with, per subdomain,
// V_i = [B_i K_i^+ B0_i^T | G_i^T] (n_i x m_i, column-major) and, per cluster, the dense
// symmetric M mapping [g0; e0] to [lambda0; alpha].
struct HybDev {
    int ncl;
    int max_nc;                   // largest cluster vector
    const long long *voff;        // nd: offset of V_i
    const int *zof;               // nd+1: offsets of the subdomains' slots (m_i = zof[i+1] - zof[i])
    const int *m0;                // nd: B0 entries of the subdomain (first m0 columns of V_i)
    const int *vmap;              // per slot: index into its cluster's vector
    const int *sub_cl;            // nd: cluster of every subdomain
    const int *cof;               // ncl+1: offsets of the cluster vectors
    const long long *mof;         // ncl: offset of M_c (nc x nc)
    const double *M;
    const double *V;
    const int *mem_ptr, *mem;     // ncl+1 / nd: members of every cluster, ascending
    const int *b0dof;             // per slot of a B0 entry: local DOF (slots of e0 unused)
    const double *b0sign;
    double *z;                    // per slot: V_i^T x (or [B0 K^+ f; -R^T f])
    double *w;                    // cluster vectors M z
    double *part;                 // per CTA of the M kernel: z.w partial
    int *done;                    // completion counter of the z.w reduction
};

struct TileSetDev {
    int nitems;
    int prec;
    const int4 *items;            // (matrix, k0, k1, -)
    const int *mat_n, *mat_voff, *mat_tn;
    const long long *mat_tile0;
    const unsigned *tile_ij;      // (I << 16) | J
    const void *tiles;
    const float *scale;           // BF16 per-tile scale
    double *item_dot;
    int *queue;                   // [0] work counter, [1] finished CTAs
};

// ---------------------------------------------------------------------------------------------
// Programmatic dependent launch (opt-in, FETI4I_PDL=1).  With it a kernel launched by launch_pdl
// may be scheduled while its predecessor in the stream still drains, and pdl_enter() returns once
// the predecessor has completed and its writes are visible, so it is the first
// statement of every kernel launched that way.  For an ordinary launch it is a no-op.  Measured on
// the heat workload of 512 subdomains: 6.57 ms per solve with it against 6.55 ms without, and
// 6.9 ms when the successor was also released early (griddepcontrol.launch_dependents), so it is
// off by default.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// The dual PCG as one graph with conditional nodes (capture_loop), opt-in (FETI4I_LOOP_GRAPH=1).
// It launches only the kernels an iteration needs (no replacement kernels that return at once, no
// iterations past convergence in the last chunk): 258 instead of 300 launches per solve of the heat
// workload of 216 subdomains, but measured 3.35 ms per solve against 3.28 ms with chunked graphs of
// 16 iterations, so the chunked graphs stay the default.
bool loop_graph_enabled() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_LOOP_GRAPH");
        return e && e[0] == '1';
    }();
    return on;
}

bool pdl_enabled() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_PDL");
        return e && e[0] == '1';
    }();
    return on;
}

// kernel<<<grid, block, smem, stream>>>(args...) with the programmatic-serialization attribute
template <typename... KA, typename... A>
void launch_pdl(void (*kernel)(KA...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CUDA_CHECK(cudaLaunchKernelEx(&cfg, kernel, static_cast<KA>(args)...));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// block-wide sum; identical result in every thread; fixed order for a given blockDim
__device__ double block_sum(double v, double *sh) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < nw; ++i) s += sh[i];
    __syncthreads();
    return s;
}

// block-wide sum of KMAX values at once
__device__ void block_sum_k(double (&v)[KMAX], double *sh /* >= 32*KMAX */) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < KMAX; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < KMAX; ++k) sh[wid * KMAX + k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
        double s = 0.0;
        for (int i = 0; i < nw; ++i) s += sh[i * KMAX + k];
        v[k] = s;
    }
    __syncthreads();
}


// block-wide sum of KC values at once (KC = the kernel width of the problem)
template <int KC>
__device__ void block_sum_kc(double (&v)[KC], double *sh /* >= 32*KC */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < KC; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < KC; ++k) sh[wid * KC + k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        double s = 0.0;
        for (int i = 0; i < nw; ++i) s += sh[i * KC + k];
        v[k] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ bool skip_iter(const DevState *st, int iter) {
    int c = st->conv_iter;
    return (c >= 0 && iter > c) || iter >= st->max_it;
}

// (G^T a) at local row e: own coefficients plus the partner's
template <int KC>
__device__ __forceinline__ double gt_alpha_fixed(const DevProblem &P, int e, const double *a) {
    const int ko = __ldg(P.rkof + e), po = __ldg(P.pkof + e);
    const double *g = P.Gl + (size_t)e * KC, *gp = P.Gp + (size_t)e * KC;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < KC; ++k) s += __ldg(g + k) * a[ko + k] + __ldg(gp + k) * a[po + k];
    return s;
}
// The common kernel widths 1 (heat) and 6 (elasticity) take fixed-width loads: coefficients
// zero-padded to KS and the amplitudes padded by KS zero entries, so the loads do not depend
// on the per-row counts and overlap.
__device__ __forceinline__ double gt_alpha(const DevProblem &P, int e, const double *a) {
    if (P.KS == 1) return gt_alpha_fixed<1>(P, e, a);
    if (P.KS == 6) return gt_alpha_fixed<6>(P, e, a);
    double s = 0.0;
    const int nk = P.rnk[e], ko = P.rkof[e], pn = P.pnk[e], po = P.pkof[e];
    const double *g = P.Gl + (size_t)e * P.KS, *gp = P.Gp + (size_t)e * P.KS;
    for (int k = 0; k < nk; ++k) s += g[k] * a[ko + k];
    for (int k = 0; k < pn; ++k) s += gp[k] * a[po + k];
    return s;
}

// Every CTA contributes v (valid in thread 0); the last CTA to arrive adds the
// partials in index order and stores the total.  No CTA waits for another.
__device__ void grid_total(double v, double *partials, int *counter, double *out, double *sh) {
    __shared__ int s_last;
    __syncthreads();  // s_last may still be read from a previous call
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        s_last = (atomicAdd(counter, 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double t = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t += __ldcg(&partials[i]);
        t = block_sum(t, sh);
        if (threadIdx.x == 0) {
            *out = t;
            *counter = 0;
        }
    }
}

// G_i v over the rows [e0, e1) of one subdomain, written to d[kof..]; KC = the row stride KS of the
// coefficients (zero-padded rows), so only the problem's kernel width is reduced
template <int KC>
__device__ void g_dot_kc(const DevProblem &P, int dsub, const double *v, double *sh) {
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    const int nk = P.kof[dsub + 1] - P.kof[dsub];
    double gk[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k) gk[k] = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const double ve = v[e - e0];
        const double *g = P.Gl + (size_t)e * KC;
#pragma unroll
        for (int k = 0; k < KC; ++k) gk[k] += __ldg(g + k) * ve;
    }
    block_sum_kc<KC>(gk, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < nk; ++k) P.d[P.kof[dsub] + k] = gk[k];
}

__device__ void g_dot(const DevProblem &P, int dsub, const double *v, double *sh) {
    if (P.KS == 1) { g_dot_kc<1>(P, dsub, v, sh); return; }
    if (P.KS == 6) { g_dot_kc<6>(P, dsub, v, sh); return; }
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    const int nk = P.kof[dsub + 1] - P.kof[dsub];
    double gk[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) gk[k] = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const double ve = v[e - e0];
        const double *g = P.Gl + (size_t)e * P.KS;
#pragma unroll
        for (int k = 0; k < KMAX; ++k)
            if (k < nk) gk[k] += g[k] * ve;
    }
    block_sum_k(gk, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < nk; ++k) P.d[P.kof[dsub] + k] = gk[k];
}

// ---------------------------------------------------------------------------------------------
// Tile SYMV.  A symmetric matrix of order n is stored as its upper-triangular
// 32x32 tiles (I <= J), row-major inside a tile; diagonal tiles hold the full
// symmetric block.  A warp owns one tile at a time: every lane loads
// 32/EPC 16-byte chunks (coalesced, one 512-byte row segment per instruction),
// forms partial row sums (S x_J) and column sums (S^T x_I) and finishes both
// with shuffle reduce-scatters, so each lane ends with one row and one column.
template <int PREC>
struct TileT;
template <>
struct TileT<SCHUR_FP64> {
    using Acc = double;
    static constexpr int EPC = 2;
};
template <>
struct TileT<SCHUR_FP32> {
    using Acc = float;
    static constexpr int EPC = 4;
};
template <>
struct TileT<SCHUR_BF16> {
    using Acc = float;
    static constexpr int EPC = 8;
};

// L2 policy for data streamed once per apply: evict first, so the vectors and
// metadata of the small kernels stay resident in the 126 MB L2
__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ uint4 ld_stream(const uint4 *p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(policy_evict_first()));
    return v;
}

template <int PREC>
__device__ __forceinline__ void unpack(const uint4 &u, typename TileT<PREC>::Acc (&e)[TileT<PREC>::EPC], float sc);
template <>
__device__ __forceinline__ void unpack<SCHUR_FP64>(const uint4 &u, double (&e)[2], float) {
    e[0] = __hiloint2double(u.y, u.x);
    e[1] = __hiloint2double(u.w, u.z);
}
template <>
__device__ __forceinline__ void unpack<SCHUR_FP32>(const uint4 &u, float (&e)[4], float) {
    e[0] = __uint_as_float(u.x);
    e[1] = __uint_as_float(u.y);
    e[2] = __uint_as_float(u.z);
    e[3] = __uint_as_float(u.w);
}
template <>
__device__ __forceinline__ void unpack<SCHUR_BF16>(const uint4 &u, float (&e)[8], float sc) {
    const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        e[2 * i] = __uint_as_float(w[i] << 16) * sc;
        e[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u) * sc;
    }
}

// reduce-scatter over the M lanes that differ in lane bits [SHIFT, SHIFT+log2 M):
// afterwards v[0] of a lane holds the group sum of entry ((lane >> SHIFT) & (M-1)).
template <int M, int SHIFT, typename T>
__device__ __forceinline__ T reduce_scatter(T (&v)[M], int lane) {
#pragma unroll
    for (int half = M / 2; half >= 1; half /= 2) {
        const bool upper = (lane >> SHIFT) & half;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            T send = upper ? v[i] : v[i + half];
            T keep = upper ? v[i + half] : v[i];
            v[i] = keep + __shfl_xor_sync(FULL, send, half << SHIFT);
        }
    }
    return v[0];
}

template <int CPR>
__device__ __forceinline__ void load_tile(uint4 (&raw)[CPR], const uint4 *tiles, long long g, int lane) {
    const uint4 *tp = tiles + (size_t)g * (TILE * CPR);
#pragma unroll
    for (int q = 0; q < CPR; ++q) raw[q] = ld_stream(tp + q * 32 + lane);
}

// one 32x32 tile: row sums into the running accumulator of tile row I, column
// sums (off-diagonal tiles) straight into the shared y
template <int PREC>
__device__ __forceinline__ void tile_fma(const uint4 (&raw)[TILE / TileT<PREC>::EPC], const TileSetDev &ts, long long g,
                                         const typename TileT<PREC>::Acc *xs, typename TileT<PREC>::Acc *ys, int lane,
                                         int &curI, typename TileT<PREC>::Acc &racc) {
    using Acc = typename TileT<PREC>::Acc;
    constexpr int EPC = TileT<PREC>::EPC;
    constexpr int CPR = TILE / EPC;
    constexpr int LOG_CPR = (CPR == 16) ? 4 : (CPR == 8) ? 3 : 2;
    const int cq = lane % CPR, h = lane / CPR;
    const int idx = EPC * cq + h;
    const unsigned ij = ts.tile_ij[g];
    const int I = ij >> 16, J = ij & 0xffff;
    const float sc = (PREC == SCHUR_BF16) ? ts.scale[g] : 1.0f;
    Acc xc[EPC], xr[CPR], rs[CPR], cs[EPC];
#pragma unroll
    for (int j = 0; j < EPC; ++j) { xc[j] = xs[TILE * J + EPC * cq + j]; cs[j] = 0; }
#pragma unroll
    for (int q = 0; q < CPR; ++q) { xr[q] = xs[TILE * I + EPC * q + h]; rs[q] = 0; }
#pragma unroll
    for (int q = 0; q < CPR; ++q) {
        Acc e[EPC];
        unpack<PREC>(raw[q], e, sc);
#pragma unroll
        for (int j = 0; j < EPC; ++j) {
            rs[q] += e[j] * xc[j];
            cs[j] += e[j] * xr[q];
        }
    }
    Acc rsum = reduce_scatter<CPR, 0>(rs, lane);
    if (I != curI) {
        if (curI >= 0) atomicAdd(&ys[TILE * curI + idx], racc);
        curI = I;
        racc = 0;
    }
    racc += rsum;
    if (I != J) {
        Acc csum = reduce_scatter<EPC, LOG_CPR>(cs, lane);
        atomicAdd(&ys[TILE * J + idx], csum);
    }
}

// MODE 0: x = src (outside the PCG loop)
// MODE 1: x = src + beta * src2 with beta = rho_k / rho_{k-1} (PCG direction p = y + beta p)
// MODE 2: x = src inside the PCG loop (skipped after convergence)
// MODE 3: x = src, only when a residual replacement is pending (mixed precision)
template <int PREC, int MODE>
__global__ void __launch_bounds__(256, 2)
tile_symv_kernel(TileSetDev ts, DevProblem P, const double *src, const double *src2, double *out, int slot) {
    pdl_enter();
    using Acc = typename TileT<PREC>::Acc;
    constexpr int EPC = TileT<PREC>::EPC;
    constexpr int CPR = TILE / EPC;          // 16-byte chunks per tile row (= loads per lane)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32];
    __shared__ int s_item;
    __shared__ double s_beta;

    if (MODE != 0) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
        if (MODE == 3 && P.st->replace_iter != iter) return;
        if (MODE == 1) {
            if (threadIdx.x == 0) s_beta = (iter == 0) ? 0.0 : P.scal[SC_RHO] / P.rho_hist[iter - 1];
            __syncthreads();
        }
    }
    const double beta = (MODE == 1) ? s_beta : 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int idx = EPC * (lane % CPR) + lane / CPR;   // row/column of this lane after the reductions

    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(&ts.queue[0], 1);
        __syncthreads();
        const int item = s_item;
        if (item >= ts.nitems) break;
        const int4 it = ts.items[item];
        const int m = it.x, k0 = it.y, k1 = it.z;
        const int n = ts.mat_n[m], voff = ts.mat_voff[m], tn = ts.mat_tn[m];
        const int np = tn * TILE;
        Acc *xs = reinterpret_cast<Acc *>(smem_raw);
        Acc *ys = xs + np;
        for (int i = threadIdx.x; i < np; i += blockDim.x) {
            double v = 0.0;
            if (i < n) v = (MODE == 1) ? src[voff + i] + beta * src2[voff + i] : src[voff + i];
            xs[i] = (Acc)v;
            ys[i] = (Acc)0;
        }
        __syncthreads();

        const long long tbase = ts.mat_tile0[m];
        const uint4 *tiles = reinterpret_cast<const uint4 *>(ts.tiles);
        int curI = -1;
        Acc racc = 0;
        int k = k0 + warp;
        if (PREC == SCHUR_FP64) {
            // 8 KB per tile and warp already keep enough bytes in flight
            for (; k < k1; k += nw) {
                uint4 raw[CPR];
                load_tile<CPR>(raw, tiles, tbase + k, lane);
                tile_fma<PREC>(raw, ts, tbase + k, xs, ys, lane, curI, racc);
            }
        } else {
            // software pipeline: the next tile of this warp is in flight while one is reduced
            uint4 ra[CPR], rb[CPR];
            if (k < k1) load_tile<CPR>(ra, tiles, tbase + k, lane);
            for (;;) {
                if (k >= k1) break;
                if (k + nw < k1) load_tile<CPR>(rb, tiles, tbase + k + nw, lane);
                tile_fma<PREC>(ra, ts, tbase + k, xs, ys, lane, curI, racc);
                k += nw;
                if (k >= k1) break;
                if (k + nw < k1) load_tile<CPR>(ra, tiles, tbase + k + nw, lane);
                tile_fma<PREC>(rb, ts, tbase + k, xs, ys, lane, curI, racc);
                k += nw;
            }
        }
        if (curI >= 0) atomicAdd(&ys[TILE * curI + idx], racc);
        __syncthreads();

        // item output: partial y and its dot with x
        const bool whole = (k0 == 0) && (k1 == tn * (tn + 1) / 2);
        double dot = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double yv = (double)ys[i];
            dot += (double)xs[i] * yv;
            if (whole) out[voff + i] = yv;
            else atomicAdd(&out[voff + i], yv);
        }
        dot = block_sum(dot, red);
        if (threadIdx.x == 0 && ts.item_dot) ts.item_dot[item] = dot;
        __syncthreads();
    }
    // the last CTA to finish resets the work queue for the next launch and, in
    // the PCG loop, adds the item dot products p.Ap in item order
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&ts.queue[1], 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        if (MODE == 1) {
            __threadfence();
            double t = 0.0;
            for (int i = threadIdx.x; i < ts.nitems; i += blockDim.x) t += __ldcg(&ts.item_dot[i]);
            t = block_sum(t, red);
            if (threadIdx.x == 0) P.scal[SC_PAP] = t;
        }
        if (threadIdx.x == 0) {
            ts.queue[0] = 0;
            ts.queue[1] = 0;
            __threadfence();
        }
    }
}


// ---------------------------------------------------------------------------------------------
// TMA-staged tile SYMV.  One producer warp streams the tiles of the work queue
// into a ring of shared-memory stages with 1D bulk copies
// (cp.async.bulk ... mbarrier::complete_tx, L2 evict-first); eight consumer
// warps reduce them (one tile per warp per stage) as in tile_symv_kernel.
// Full/empty mbarriers hand the stages over; every wait is bounded: on time-out
// the kernel records DevState::error, the producer drains its copies in flight
// and the CTA returns.
constexpr int TMA_CONSUMERS = 8;
constexpr int TMA_MAX_STAGES = 16;
constexpr long long WAIT_LIMIT = 1ll << 24;   // polls (with back-off) before a wait gives up

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase of `parity`; false if the limit ran out
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
    for (long long i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try(bar, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar,
                                         unsigned long long pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(TMA_CONSUMERS * 32) : "memory"); }

__device__ double consumer_sum(double v, double *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    consumer_sync();
    if (lane == 0) sh[wid] = v;
    consumer_sync();
    double s = 0.0;
    for (int i = 0; i < TMA_CONSUMERS; ++i) s += sh[i];
    consumer_sync();
    return s;
}

struct StageMeta {
    int item, k, cnt, flags;  // flags: 1 first chunk of the item, 2 last chunk
};

template <int PREC, int MODE>
__global__ void __launch_bounds__((TMA_CONSUMERS + 1) * 32, 1)
tile_symv_tma_kernel(TileSetDev ts, DevProblem P, const double *src, const double *src2, double *out, int slot,
                     int nstages, int xs_elems) {
    pdl_enter();
    using Acc = typename TileT<PREC>::Acc;
    constexpr int EPC = TileT<PREC>::EPC;
    constexpr int CPR = TILE / EPC;
    constexpr unsigned TILE_BYTES = TILE * TILE * (PREC == SCHUR_FP64 ? 8 : PREC == SCHUR_FP32 ? 4 : 2);
    constexpr unsigned STAGE_BYTES = TMA_CONSUMERS * TILE_BYTES;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long full_bar[TMA_MAX_STAGES], empty_bar[TMA_MAX_STAGES];
    __shared__ StageMeta meta[TMA_MAX_STAGES];
    __shared__ double red[32];
    __shared__ double s_beta;
    __shared__ int s_last;

    if (MODE != 0) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
        if (MODE == 3 && P.st->replace_iter != iter) return;
        if (MODE == 1) {
            if (threadIdx.x == 0) s_beta = (iter == 0) ? 0.0 : P.scal[SC_RHO] / P.rho_hist[iter - 1];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *ring = smem_raw;
    Acc *xs = reinterpret_cast<Acc *>(smem_raw + (size_t)nstages * STAGE_BYTES);
    Acc *ys = xs + xs_elems;
    if (threadIdx.x == 0) {
        for (int i = 0; i < nstages; ++i) {
            mbar_init(&full_bar[i], 1);
            mbar_init(&empty_bar[i], TMA_CONSUMERS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const double beta = (MODE == 1) ? s_beta : 0.0;

    if (warp == TMA_CONSUMERS) {
        // ---------------- producer: one lane issues the bulk copies
        if (lane == 0) {
            const unsigned long long pol = policy_evict_first();
            const unsigned char *tiles = reinterpret_cast<const unsigned char *>(ts.tiles);
            long long c = 0;          // chunk counter
            long long last_c[TMA_MAX_STAGES];
            for (int i = 0; i < TMA_MAX_STAGES; ++i) last_c[i] = -1;
            bool ok = true;
            for (;;) {
                int item = atomicAdd(&ts.queue[0], 1);
                int4 it = make_int4(0, 0, 0, 0);
                if (item < ts.nitems) it = ts.items[item];
                const int k0 = it.y, k1 = it.z;
                const long long tbase = item < ts.nitems ? ts.mat_tile0[it.x] : 0;
                int k = k0;
                do {
                    const int st = (int)(c % nstages);
                    const long long round = c / nstages;
                    if (round > 0 && !mbar_wait(&empty_bar[st], (unsigned)((round - 1) & 1))) { ok = false; break; }
                    if (item >= ts.nitems) {
                        meta[st] = StageMeta{-1, 0, 0, 0};
                        mbar_arrive(&full_bar[st]);
                        ++c;
                        break;
                    }
                    const int cnt = min(TMA_CONSUMERS, k1 - k);
                    meta[st] = StageMeta{item, k, cnt, (k == k0 ? 1 : 0) | (k + cnt == k1 ? 2 : 0)};
                    mbar_arrive_tx(&full_bar[st], (unsigned)cnt * TILE_BYTES);
                    bulk_g2s(ring + (size_t)st * STAGE_BYTES, tiles + (size_t)(tbase + k) * TILE_BYTES,
                             (unsigned)cnt * TILE_BYTES, &full_bar[st], pol);
                    last_c[st] = c;
                    ++c;
                    k += cnt;
                } while (k < k1);
                if (!ok || item >= ts.nitems) break;
            }
            if (!ok) {
                atomicExch(&P.st->error, 1);
                // drain: wait (bounded) for the copies this thread issued
                for (int st = 0; st < nstages; ++st)
                    if (last_c[st] >= 0) mbar_wait(&full_bar[st], (unsigned)((last_c[st] / nstages) & 1));
            }
        }
    } else {
        // ---------------- consumers
        const int idx = EPC * (lane % CPR) + lane / CPR;
        long long c = 0;
        int curI = -1, item = -1, n = 0, voff = 0, whole = 0;
        Acc racc = 0;
        for (;;) {
            const int st = (int)(c % nstages);
            if (!mbar_wait(&full_bar[st], (unsigned)((c / nstages) & 1))) {
                atomicExch(&P.st->error, 1);
                break;
            }
            const StageMeta m = meta[st];
            if (m.item < 0) break;
            if (m.flags & 1) {
                // new item: stage x, clear y (the previous item's epilogue ended with a barrier)
                item = m.item;
                const int4 it = ts.items[item];
                n = ts.mat_n[it.x];
                voff = ts.mat_voff[it.x];
                const int tn = ts.mat_tn[it.x];
                whole = (it.y == 0) && (it.z == tn * (tn + 1) / 2);
                for (int i = threadIdx.x; i < TILE * tn; i += TMA_CONSUMERS * 32) {
                    double v = 0.0;
                    if (i < n) v = (MODE == 1) ? src[voff + i] + beta * src2[voff + i] : src[voff + i];
                    xs[i] = (Acc)v;
                    ys[i] = (Acc)0;
                }
                consumer_sync();
                curI = -1;
                racc = 0;
            }
            if (warp < m.cnt) {
                const uint4 *tp = reinterpret_cast<const uint4 *>(ring + (size_t)st * STAGE_BYTES + (size_t)warp * TILE_BYTES);
                uint4 raw[CPR];
#pragma unroll
                for (int q = 0; q < CPR; ++q) raw[q] = tp[q * 32 + lane];
                tile_fma<PREC>(raw, ts, ts.mat_tile0[ts.items[item].x] + m.k + warp, xs, ys, lane, curI, racc);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty_bar[st]);
            ++c;
            if (m.flags & 2) {
                if (curI >= 0) atomicAdd(&ys[TILE * curI + idx], racc);
                curI = -1;
                racc = 0;
                consumer_sync();
                double dot = 0.0;
                for (int i = threadIdx.x; i < n; i += TMA_CONSUMERS * 32) {
                    const double yv = (double)ys[i];
                    dot += (double)xs[i] * yv;
                    if (whole) out[voff + i] = yv;
                    else atomicAdd(&out[voff + i], yv);
                }
                dot = consumer_sum(dot, red);
                if (threadIdx.x == 0 && ts.item_dot) ts.item_dot[item] = dot;
            }
        }
    }
    // the last CTA resets the work queue and (PCG loop) adds the item dot products in order
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&ts.queue[1], 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        if (MODE == 1) {
            __threadfence();
            double t = 0.0;
            for (int i = threadIdx.x; i < ts.nitems; i += blockDim.x) t += __ldcg(&ts.item_dot[i]);
            t = block_sum(t, red);
            if (threadIdx.x == 0) P.scal[SC_PAP] = t;
        }
        if (threadIdx.x == 0) {
            ts.queue[0] = 0;
            ts.queue[1] = 0;
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// coarse problem: out = (GG^T)^-1 in   (dense symmetric, one warp per row)
__global__ void coarse_kernel(DevProblem P, const double *in, double *out, int slot, int looped) {
    pdl_enter();
    if (looped) {
        int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
    }
    int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (row >= P.nK) return;
    const double *col = P.GGtinv + (size_t)row * P.nP;
    // four independent partial sums: the loads of four steps are in flight together
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int b = lane;
    for (; b + 96 < P.nP; b += 128) {
        s0 += __ldg(col + b) * __ldg(in + b);
        s1 += __ldg(col + b + 32) * __ldg(in + b + 32);
        s2 += __ldg(col + b + 64) * __ldg(in + b + 64);
        s3 += __ldg(col + b + 96) * __ldg(in + b + 96);
    }
    for (; b < P.nP; b += 32) s0 += __ldg(col + b) * __ldg(in + b);
    double s = warp_sum((s0 + s1) + (s2 + s3));
    if (lane == 0) out[row] = s;
}

// x = G^T alpha (initial lambda_0 = G^T (GG^T)^-1 e)
__global__ void gt_kernel(DevProblem P, const double *a, double *xout) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < P.NL) xout[e] = gt_alpha(P, e, a);
}

__global__ void zero_kernel(double *v, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = 0.0;
}

__global__ void zero2_kernel(double *a, double *b, int n) {
    pdl_enter();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { a[i] = 0.0; b[i] = 0.0; }
}

// r = b - assemble(Ax); d = G r per subdomain; ||b||^2 total (initial call).  One CTA per subdomain.
__global__ void __launch_bounds__(1024) r0_kernel(DevProblem P, double *Ax, int replace_mode, int slot) {
    pdl_enter();
    extern __shared__ double rv_s[];
    __shared__ double sh[32 * KMAX];
    if (replace_mode) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter) || P.st->replace_iter != iter) return;
    }
    const int dsub = blockIdx.x;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    double bb = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int q = P.partner[e];
        const double a = Ax[e] + (q >= 0 ? Ax[q] : 0.0);
        const double rv = P.bL[e] - a;
        P.r[e] = rv;
        rv_s[e - e0] = rv;
        bb += P.bL[e] * P.bL[e] * P.minv[e];
    }
    __syncthreads();
    g_dot(P, dsub, rv_s, sh);
    if (!replace_mode) grid_total(block_sum(bb, sh), P.part_b, P.done + DONE_B, P.scal + SC_BN2, sh);
}

// ||P r||^2 with alpha = (GG^T)^-1 G r (initial stop tolerance)
__global__ void pnorm_kernel(DevProblem P) {
    __shared__ double sh[32];
    const int dsub = blockIdx.x;
    double s = 0.0;
    for (int e = P.loff[dsub] + threadIdx.x; e < P.loff[dsub + 1]; e += blockDim.x) {
        double u = P.r[e] - gt_alpha(P, e, P.alpha);
        s += u * u * P.minv[e];
    }
    grid_total(block_sum(s, sh), P.part_w, P.done + DONE_PN, P.scal + SC_PN2, sh);
}

__global__ void tol_kernel(DevProblem P) {
    if (threadIdx.x == 0) {
        const double un = sqrt(P.scal[SC_PN2]), bn = sqrt(P.scal[SC_BN2]);
        P.st->tol = P.st->precision * fmin(un, bn);
        P.st->rmax = un;
    }
}

// w = r - G^T alpha (||w||^2 total), u_T = B^T (W w) and, for the lumped
// preconditioner, v_T = K_TT u_T (sliced ELL).  With no preconditioner y = w
// and rho = y.w is taken here.  One CTA per subdomain.
template <int PRECOND>
__global__ void __launch_bounds__(TPB1) w_prec_kernel(DevProblem P, int slot) {
    pdl_enter();
    extern __shared__ double sm[];
    __shared__ double sh[32];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int dsub = blockIdx.x;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    const int t0 = P.toff[dsub], t1 = P.toff[dsub + 1], nt = t1 - t0;
    double *wsm = sm;              // w of the subdomain rows
    double *u = sm + (e1 - e0);    // B^T W w on the touched DOFs
    double ww = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const double wv = __ldg(P.r + e) - gt_alpha(P, e, P.alpha);
        P.w[e] = wv;
        wsm[e - e0] = wv;
        if (PRECOND == PREC_NONE) P.y[e] = wv;
        ww += wv * wv * __ldg(P.minv + e);
    }
    ww = block_sum(ww, sh);  // also a barrier for wsm
    grid_total(ww, P.part_w, P.done + DONE_W, P.scal + SC_WN2, sh);
    if (PRECOND == PREC_NONE) {
        grid_total(ww, P.part_rho, P.done + DONE_RHO, P.scal + SC_RHO, sh);
        return;
    }
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        double s = 0.0;
        for (int j = __ldg(P.trow_ptr + t0 + t); j < __ldg(P.trow_ptr + t0 + t + 1); ++j) {
            const int e = __ldg(P.trow_idx + j);
            s += __ldg(P.ws + e) * wsm[e - e0];
        }
        if (PRECOND == PREC_LUMPED) u[t] = s;
        else P.uT[t0 + t] = s;
        if (PRECOND == PREC_WEIGHT) P.vT[t0 + t] = s;
    }
    if (PRECOND != PREC_LUMPED) return;
    __syncthreads();
    const int sl0 = P.slice0[dsub];
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        const int sl = sl0 + (t >> 5), ln = t & 31;
        const int base = __ldg(P.ell_ptr + sl), wd = __ldg(P.ell_w + sl);
        // four independent entries per step: their loads are in flight together
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int j = 0;
        for (; j + 3 < wd; j += 4) {
            const int o = base + j * 32 + ln;
            const double v0 = __ldg(P.ell_val + o), v1 = __ldg(P.ell_val + o + 32), v2 = __ldg(P.ell_val + o + 64),
                         v3 = __ldg(P.ell_val + o + 96);
            const int c0 = __ldg(P.ell_col + o), c1 = __ldg(P.ell_col + o + 32), c2 = __ldg(P.ell_col + o + 64),
                      c3 = __ldg(P.ell_col + o + 96);
            s0 += v0 * u[c0];
            s1 += v1 * u[c1];
            s2 += v2 * u[c2];
            s3 += v3 * u[c3];
        }
        for (; j < wd; ++j) {
            const int o = base + j * 32 + ln;
            s0 += __ldg(P.ell_val + o) * u[__ldg(P.ell_col + o)];
        }
        P.vT[t0 + t] = (s0 + s1) + (s2 + s3);
    }
}

// z = assemble(W B v_T); d = G z.  One CTA per subdomain.
__global__ void __launch_bounds__(1024) z_kernel(DevProblem P, int slot) {
    pdl_enter();
    extern __shared__ double zs[];
    __shared__ double sh[32 * KMAX];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int dsub = blockIdx.x;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int pt = __ldg(P.ptidx + e);
        double zv = __ldg(P.ws + e) * __ldg(P.vT + __ldg(P.tidx + e));
        if (pt >= 0) zv += __ldg(P.pws + e) * __ldg(P.vT + pt);
        P.z[e] = zv;
        zs[e - e0] = zv;
    }
    __syncthreads();
    g_dot(P, dsub, zs, sh);
}

// y = z - G^T alpha, rho = y.w total; clear the F apply accumulators.
__global__ void __launch_bounds__(1024) y_kernel(DevProblem P, double *Ax64, int slot) {
    pdl_enter();
    __shared__ double sh[32];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int dsub = blockIdx.x;
    double s = 0.0;
    for (int e = P.loff[dsub] + threadIdx.x; e < P.loff[dsub + 1]; e += blockDim.x) {
        const double yv = __ldg(P.z + e) - gt_alpha(P, e, P.alpha);
        P.y[e] = yv;
        s += yv * __ldg(P.w + e) * __ldg(P.minv + e);
        P.Ap[e] = 0.0;
        Ax64[e] = 0.0;
    }
    grid_total(block_sum(s, sh), P.part_rho, P.done + DONE_RHO, P.scal + SC_RHO, sh);
}

__global__ void zero_vT_kernel(DevProblem P, int slot) {
    pdl_enter();
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P.NT; t += gridDim.x * blockDim.x) P.vT[t] = 0.0;
}

// p = y + beta p, x += alpha p, r -= alpha assemble(Ap), d = G r, convergence check.
// Device-side loop control (graph_loop): the WHILE node repeats the iteration while h_loop is
// non-zero, the IF node at the top of an iteration runs the residual replacement when h_repl is.
struct LoopCtl {
    int on;                              // 0: launched outside the conditional graph
    cudaGraphConditionalHandle h_loop, h_repl;
};

__global__ void __launch_bounds__(1024) update_kernel(DevProblem P, int slot) {
    pdl_enter();
    extern __shared__ double rs_s[];
    __shared__ double sh[32 * KMAX];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const double rho = P.scal[SC_RHO];
    const double pAp = P.scal[SC_PAP];
    const double wn2 = P.scal[SC_WN2];
    const double beta = (iter == 0) ? 0.0 : rho / P.rho_hist[iter - 1];
    const double alpha = rho / pAp;
    const int dsub = blockIdx.x;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int q = __ldg(P.partner + e);
        const double ap = __ldg(P.Ap + e) + (q >= 0 ? __ldg(P.Ap + q) : 0.0);
        const double pv = __ldg(P.y + e) + beta * P.p[e];
        P.p[e] = pv;
        P.x[e] += alpha * pv;
        const double rv = P.r[e] - alpha * ap;
        P.r[e] = rv;
        rs_s[e - e0] = rv;
    }
    __syncthreads();
    g_dot(P, dsub, rs_s, sh);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        DevState *st = P.st;
        P.rho_hist[iter] = rho;
        const double wn = sqrt(wn2);
        st->last_norm = wn;
        if (!st->mixed) {
            if (wn < st->tol && st->conv_iter < 0) st->conv_iter = iter;
        } else {
            // reliable updates (residual replacement): converge only on a residual
            // recomputed in FP64, replace the iterated residual once it dropped by
            // `delta` below the largest norm seen since the last replacement
            const bool fresh = st->true_iter == iter;
            st->rmax = fresh ? wn : fmax(st->rmax, wn);
            bool replace = false;
            if (wn < st->tol) {
                if (fresh) {
                    if (st->conv_iter < 0) st->conv_iter = iter;
                } else {
                    replace = true;
                }
            } else if (wn < st->delta * st->rmax) {
                replace = true;
            }
            if (replace) {
                st->replace_iter = iter + 1;
                st->true_iter = iter + 1;
                st->replacements += 1;
            }
        }
    }
}

__global__ void chunk_end_kernel(DevProblem P, int chunk) {
    pdl_enter();
    if (threadIdx.x == 0 && blockIdx.x == 0) P.st->iter_base += chunk;
}

// End of one pass of the loop graph: always runs (no skip test), advances the iteration, asks for the
// residual replacement that the update requested for the next iteration, and keeps the WHILE node
// going only while the solve has neither converged, nor reached max_iterations, nor recorded a
// pipeline error, so the loop ends after at most max_iterations passes.  (A separate kernel, so that
// the kernels of the chunked graphs make no device-runtime call.)
__global__ void loop_end_kernel(DevProblem P, LoopCtl lc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        DevState *st = P.st;
        const int done = ++st->iter_base;
        const bool more = st->conv_iter < 0 && done < st->max_it && st->error == 0;
        cudaGraphSetConditional(lc.h_repl, (more && st->replace_iter == done) ? 1u : 0u);
        cudaGraphSetConditional(lc.h_loop, more ? 1u : 0u);
    }
}



// ---------------------------------------------------------------------------------------------
// Partitioned dual problem: operators between caller vectors in the whole problem's multiplier
// numbering and this instance's local rows.
__global__ void gather_lambda_kernel(const int *lam, const double *x, double *xl, int NL) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < NL) xl[e] = x[lam[e]];
}
// y[lambda] += yl (two local rows of one multiplier add both), yl cleared for the next accumulation
__global__ void scatter_lambda_kernel(const int *lam, double *yl, double *y, int NL) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < NL) {
        atomicAdd(&y[lam[e]], yl[e]);
        yl[e] = 0.0;
    }
}
// u_T = B^T W x on the touched DOFs (x in the whole numbering); WEIGHT also v_T = u_T
template <int PRECOND>
__global__ void prec_gather_kernel(DevProblem P, const int *lam, const double *x) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.NT) return;
    double s = 0.0;
    for (int q = P.trow_ptr[t]; q < P.trow_ptr[t + 1]; ++q) {
        const int e = P.trow_idx[q];
        s += P.ws[e] * x[lam[e]];
    }
    P.uT[t] = s;
    if (PRECOND == PREC_WEIGHT) P.vT[t] = s;
}
// v_T = K_TT u_T (sliced ELL; LUMPED, MAGIC and SUPER_DIRICHLET matrices)
__global__ void prec_ell_kernel(DevProblem P) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.NT) return;
    const int t0 = P.tbase[t], ts = P.tslot[t];
    const int sl = ts >> 5, ln = ts & 31;
    const int base = P.ell_ptr[sl], wd = P.ell_w[sl];
    double s = 0.0;
    for (int q = 0; q < wd; ++q) {
        const int o = base + q * 32 + ln;
        s += P.ell_val[o] * P.uT[t0 + P.ell_col[o]];
    }
    P.vT[t] = s;
}
// y[lambda] += W B v_T
__global__ void prec_scatter_kernel(DevProblem P, const int *lam, double *y) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < P.NL) atomicAdd(&y[lam[e]], P.ws[e] * P.vT[P.tidx[e]]);
}

// ---------------------------------------------------------------------------------------------
// K^+ on the device: forward/backward substitution with the Cholesky factor of
// K_reg (factor order), stored as 32x32 lower tiles (I >= J), block column by
// block column; the diagonal tiles hold the inverse of their 32x32 triangular block,
// so a diagonal step is a 32-term product per lane instead of a chain of 32 dependent
// divisions.  One CTA per subdomain; diagonal blocks are applied by warp 0 with
// shuffles, off-diagonal blocks by all warps.
struct KplusDev {
    int nd;
    const int *n;            // DOFs per subdomain
    const int *tn;           // 32-blocks per subdomain
    const int *doff;         // local-DOF offsets (nd+1)
    const long long *tile0;  // first tile of each subdomain
    const int *pos;          // local DOF -> factor position (concatenated)
    const double *L;         // tiles
    const int *jt;           // first 32-block holding a touched DOF (factor order: untouched DOFs first)
    double *z;               // forward results L^-1 f kept by mode 1 (factor order, concatenated)
    // tiles of block column J that are not all zero (the factor keeps the envelope of K_reg, so
    // whole tiles left of a row's first coupling are exactly zero): rows[cptr[cbase[d] + J] ..
    // cptr[cbase[d] + J + 1]) in ascending order, the diagonal tile first
    const int *cbase;
    const int *cptr;
    const int *rows;
    const long long *tpre;   // 32-blocks of the subdomains before d (vectors of kplus_mma_kernel in global memory)
};

// nz[t] = 1 when tile t holds a nonzero (one warp per tile)
__global__ void tile_nz_kernel(const double *L, long long ntiles, unsigned char *nz) {
    const int lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long t = w0; t < ntiles; t += nw) {
        const double *tp = L + (size_t)t * TILE * TILE;
        bool any = false;
        for (int k = lane; k < TILE * TILE; k += 32) any |= tp[k] != 0.0;
        any = __any_sync(FULL, any);
        if (lane == 0) nz[t] = any ? 1 : 0;
    }
}

// K^+ modes of kplus_kernel:
//   0  out = K^+ in;
//   1  (b = B K^+ f needs K^+ f at the touched DOFs only) forward pass over every block, kept in z;
//      backward pass over the blocks from jt on: out is K^+ in at the touched DOFs, not elsewhere;
//   2  (primal, in = -B^T lambda is zero at the untouched DOFs) forward pass from block jt on, plus
//      the kept z = L^-1 f, then the whole backward pass: out = K^+ (f - B^T lambda).
enum { KPLUS_FULL = 0, KPLUS_TOUCHED = 1, KPLUS_PRIMAL = 2 };

__device__ __forceinline__ long long ltile(int T, int I, int J) {
    return (long long)J * T - (long long)J * (J - 1) / 2 + (I - J);
}

__global__ void __launch_bounds__(256) kplus_kernel(KplusDev K, const double *in, double *out, int mode) {
    extern __shared__ double v[];
    __shared__ double part[8][32];
    const int d = blockIdx.x;
    const int n = K.n[d], T = K.tn[d], o = K.doff[d];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int *pos = K.pos + o;
    const uint4 *tiles = reinterpret_cast<const uint4 *>(K.L) + (size_t)K.tile0[d] * (TILE * 16);
    const double *dtiles = K.L + (size_t)K.tile0[d] * TILE * TILE;
    const int *cp = K.cptr + K.cbase[d];
    for (int i = threadIdx.x; i < TILE * T; i += blockDim.x) v[i] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) v[pos[i]] = in[o + i];
    __syncthreads();
    const int cq = lane % 16, h = lane / 16, idx = 2 * cq + h;
    const int jt = mode == KPLUS_FULL ? 0 : K.jt[d];
    double *zs = K.z + o;
    // forward: L y = f (rows before block jt are zero in mode 2, so their steps are skipped)
    for (int J = (mode == KPLUS_PRIMAL ? jt : 0); J < T; ++J) {
        if (warp == 0) {
            // y_J = inv(L_JJ) v_J: lane r forms row r (zero above the diagonal)
            const double *row = dtiles + (size_t)ltile(T, J, J) * TILE * TILE + lane * TILE;
            const double vr = v[TILE * J + lane];
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int k = 0; k < TILE; k += 2) {
                s0 += row[k] * __shfl_sync(FULL, vr, k);
                s1 += row[k + 1] * __shfl_sync(FULL, vr, k + 1);
            }
            v[TILE * J + lane] = s0 + s1;
        }
        __syncthreads();
        for (int q = cp[J] + 1 + warp; q < cp[J + 1]; q += nw) {
            const int I = K.rows[q];
            const uint4 *tp = tiles + (size_t)ltile(T, I, J) * (TILE * 16);
            double rs[16];
            const double x0 = v[TILE * J + 2 * cq], x1 = v[TILE * J + 2 * cq + 1];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                uint4 u = ld_stream(tp + q * 32 + lane);
                rs[q] = __hiloint2double(u.y, u.x) * x0 + __hiloint2double(u.w, u.z) * x1;
            }
            double r = reduce_scatter<16, 0>(rs, lane);
            v[TILE * I + idx] -= r;
        }
        __syncthreads();
    }
    if (mode == KPLUS_TOUCHED) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) zs[i] = v[i];
        __syncthreads();
    } else if (mode == KPLUS_PRIMAL) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) v[i] += zs[i];
        __syncthreads();
    }
    // backward: L^T x = y (in mode 1 only down to block jt)
    for (int J = T - 1; J >= (mode == KPLUS_TOUCHED ? jt : 0); --J) {
        double cpart = 0.0;
        for (int q = cp[J] + 1 + warp; q < cp[J + 1]; q += nw) {
            const int I = K.rows[q];
            const uint4 *tp = tiles + (size_t)ltile(T, I, J) * (TILE * 16);
            double cs[2] = {0.0, 0.0};
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                uint4 u = ld_stream(tp + q * 32 + lane);
                double xr = v[TILE * I + 2 * q + h];
                cs[0] += __hiloint2double(u.y, u.x) * xr;
                cs[1] += __hiloint2double(u.w, u.z) * xr;
            }
            cpart += reduce_scatter<2, 4>(cs, lane);
        }
        part[warp][idx] = cpart;
        __syncthreads();
        if (warp == 0) {
            double vc = v[TILE * J + lane];
            for (int w = 0; w < nw; ++w) vc -= part[w][lane];
            // x_J = inv(L_JJ)^T v_J: lane c forms column c of inv(L_JJ)
            const double *tile = dtiles + (size_t)ltile(T, J, J) * TILE * TILE;
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int k = 0; k < TILE; k += 2) {
                s0 += tile[k * TILE + lane] * __shfl_sync(FULL, vc, k);
                s1 += tile[(k + 1) * TILE + lane] * __shfl_sync(FULL, vc, k + 1);
            }
            v[TILE * J + lane] = s0 + s1;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) out[o + i] = v[pos[i]];
}

// Implicit F apply (the reference's default without explicit Schur complements,
// src/solver/specific/cpu/itersolvercpu.cpp:73-106 with Domain::multKplusLocal, Domain.cpp:271-338):
// (S_i x)_r = s_r (K_i^+ B_i^T x)[dof_r] through the device Cholesky factor instead of stored S_i.
// B_i^T x is zero at the untouched DOFs, which the factor order puts first, and only the touched
// DOFs are read back, so the forward pass starts and the backward pass stops at the first touched
// 32-block: both passes read only the factor's trailing touched part L_TT (its tiles that are not
// all zero).  One CTA per subdomain writes the unassembled local product, as the tile SYMV does.
// MODE 0: x = src, out += S x.  MODE 1 (PCG loop): x = src + beta src2 (direction p = y + beta p),
// out = S x and p.Ap into SC_PAP.
template <int MODE>
__global__ void __launch_bounds__(256) kplus_dual_kernel(KplusDev K, DevProblem P, const int *rdof,
                                                         const double *rsign, const double *src, const double *src2,
                                                         double *out, int slot) {
    pdl_enter();
    extern __shared__ double v[];
    __shared__ double part[8][32];
    __shared__ double sh[32];
    double beta = 0.0;
    if (MODE == 1) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
        beta = (iter == 0) ? 0.0 : P.scal[SC_RHO] / P.rho_hist[iter - 1];
    }
    const int d = blockIdx.x;
    const int T = K.tn[d], o = K.doff[d];
    const int e0 = P.loff[d], e1 = P.loff[d + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int *pos = K.pos + o;
    const uint4 *tiles = reinterpret_cast<const uint4 *>(K.L) + (size_t)K.tile0[d] * (TILE * 16);
    const double *dtiles = K.L + (size_t)K.tile0[d] * TILE * TILE;
    const int *cp = K.cptr + K.cbase[d];
    const int jt = K.jt[d];
    for (int i = TILE * jt + threadIdx.x; i < TILE * T; i += blockDim.x) v[i] = 0.0;
    __syncthreads();
    // B^T x: several multipliers (Dirichlet and gluing rows) may share a DOF
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const double xv = (MODE == 1) ? src[e] + beta * src2[e] : src[e];
        atomicAdd(&v[pos[rdof[e] - o]], rsign[e] * xv);
    }
    __syncthreads();
    const int cq = lane % 16, h = lane / 16, idx = 2 * cq + h;
    for (int J = jt; J < T; ++J) {   // forward: L y = B^T x
        if (warp == 0) {
            const double *row = dtiles + (size_t)ltile(T, J, J) * TILE * TILE + lane * TILE;
            const double vr = v[TILE * J + lane];
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int k = 0; k < TILE; k += 2) {
                s0 += row[k] * __shfl_sync(FULL, vr, k);
                s1 += row[k + 1] * __shfl_sync(FULL, vr, k + 1);
            }
            v[TILE * J + lane] = s0 + s1;
        }
        __syncthreads();
        for (int q = cp[J] + 1 + warp; q < cp[J + 1]; q += nw) {
            const int I = K.rows[q];
            const uint4 *tp = tiles + (size_t)ltile(T, I, J) * (TILE * 16);
            double rs[16];
            const double x0 = v[TILE * J + 2 * cq], x1 = v[TILE * J + 2 * cq + 1];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const uint4 u = ld_stream(tp + k * 32 + lane);
                rs[k] = __hiloint2double(u.y, u.x) * x0 + __hiloint2double(u.w, u.z) * x1;
            }
            v[TILE * I + idx] -= reduce_scatter<16, 0>(rs, lane);
        }
        __syncthreads();
    }
    for (int J = T - 1; J >= jt; --J) {   // backward: L^T z = y, down to the first touched block
        double cpart = 0.0;
        for (int q = cp[J] + 1 + warp; q < cp[J + 1]; q += nw) {
            const int I = K.rows[q];
            const uint4 *tp = tiles + (size_t)ltile(T, I, J) * (TILE * 16);
            double cs[2] = {0.0, 0.0};
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const uint4 u = ld_stream(tp + k * 32 + lane);
                const double xr = v[TILE * I + 2 * k + h];
                cs[0] += __hiloint2double(u.y, u.x) * xr;
                cs[1] += __hiloint2double(u.w, u.z) * xr;
            }
            cpart += reduce_scatter<2, 4>(cs, lane);
        }
        part[warp][idx] = cpart;
        __syncthreads();
        if (warp == 0) {
            double vc = v[TILE * J + lane];
            for (int w = 0; w < nw; ++w) vc -= part[w][lane];
            const double *tile = dtiles + (size_t)ltile(T, J, J) * TILE * TILE;
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int k = 0; k < TILE; k += 2) {
                s0 += tile[k * TILE + lane] * __shfl_sync(FULL, vc, k);
                s1 += tile[(k + 1) * TILE + lane] * __shfl_sync(FULL, vc, k + 1);
            }
            v[TILE * J + lane] = s0 + s1;
        }
        __syncthreads();
    }
    double dot = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const double yv = rsign[e] * v[pos[rdof[e] - o]];
        if (MODE == 1) {
            out[e] = yv;
            dot += (src[e] + beta * src2[e]) * yv;
        } else {
            out[e] += yv;
        }
    }
    if (MODE == 1) grid_total(block_sum(dot, sh), P.part_w + P.nd, P.done + DONE_PAP_IMPLICIT, P.scal + SC_PAP, sh);
}

// K^+ on NC right-hand sides at once (columns j0 .. j0+NC-1 of in/out, `stride` doubles apart):
// every factor tile is loaded once per pass and applied to all NC columns, so the factor is read
// once for NC load cases.  Same tile walk and modes as kplus_kernel; z (mode 1/2) holds the
// forward results of every column at the same stride.  Warps take off-diagonal tiles; warp w
// handles the diagonal blocks of columns w, w + 8, ...
template <int NC>
__global__ void __launch_bounds__(256) kplus_multi_kernel(KplusDev K, const double *in, double *out, int mode,
                                                          int j0, long long stride, double *z) {
    extern __shared__ double vm[];              // [NC][TILE * T]
    __shared__ double part[8][NC][TILE];
    const int d = blockIdx.x;
    const int n = K.n[d], T = K.tn[d], o = K.doff[d];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int NP = TILE * T;
    const int *pos = K.pos + o;
    const uint4 *tiles = reinterpret_cast<const uint4 *>(K.L) + (size_t)K.tile0[d] * (TILE * 16);
    const double *dtiles = K.L + (size_t)K.tile0[d] * TILE * TILE;
    const int *cp = K.cptr + K.cbase[d];
    const int jt = mode == KPLUS_FULL ? 0 : K.jt[d];
    for (int i = threadIdx.x; i < NC * NP; i += blockDim.x) vm[i] = 0.0;
    __syncthreads();
    for (int c = 0; c < NC; ++c)
        for (int i = threadIdx.x; i < n; i += blockDim.x) vm[c * NP + pos[i]] = in[(size_t)(j0 + c) * stride + o + i];
    __syncthreads();
    const int cq = lane % 16, h = lane / 16, idx = 2 * cq + h;
    for (int J = (mode == KPLUS_PRIMAL ? jt : 0); J < T; ++J) {
        {
            const double *row = dtiles + (size_t)ltile(T, J, J) * TILE * TILE + lane * TILE;
            for (int c = warp; c < NC; c += nw) {
                double *vc = vm + c * NP;
                const double vr = vc[TILE * J + lane];
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int k = 0; k < TILE; k += 2) {
                    s0 += row[k] * __shfl_sync(FULL, vr, k);
                    s1 += row[k + 1] * __shfl_sync(FULL, vr, k + 1);
                }
                vc[TILE * J + lane] = s0 + s1;
            }
        }
        __syncthreads();
        for (int qi = cp[J] + 1 + warp; qi < cp[J + 1]; qi += nw) {
            const int I = K.rows[qi];
            const uint4 *tp = tiles + (size_t)ltile(T, I, J) * (TILE * 16);
            uint4 t[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) t[q] = ld_stream(tp + q * 32 + lane);
            for (int c = 0; c < NC; ++c) {
                double *vc = vm + c * NP;
                const double x0 = vc[TILE * J + 2 * cq], x1 = vc[TILE * J + 2 * cq + 1];
                double rs[16];
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    rs[q] = __hiloint2double(t[q].y, t[q].x) * x0 + __hiloint2double(t[q].w, t[q].z) * x1;
                const double r = reduce_scatter<16, 0>(rs, lane);
                vc[TILE * I + idx] -= r;
            }
        }
        __syncthreads();
    }
    if (mode == KPLUS_TOUCHED) {
        for (int c = 0; c < NC; ++c)
            for (int i = threadIdx.x; i < n; i += blockDim.x) z[(size_t)(j0 + c) * stride + o + i] = vm[c * NP + i];
        __syncthreads();
    } else if (mode == KPLUS_PRIMAL) {
        for (int c = 0; c < NC; ++c)
            for (int i = threadIdx.x; i < n; i += blockDim.x) vm[c * NP + i] += z[(size_t)(j0 + c) * stride + o + i];
        __syncthreads();
    }
    for (int J = T - 1; J >= (mode == KPLUS_TOUCHED ? jt : 0); --J) {
        double cpart[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) cpart[c] = 0.0;
        for (int qi = cp[J] + 1 + warp; qi < cp[J + 1]; qi += nw) {
            const int I = K.rows[qi];
            const uint4 *tp = tiles + (size_t)ltile(T, I, J) * (TILE * 16);
            uint4 t[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) t[q] = ld_stream(tp + q * 32 + lane);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const double *vc = vm + c * NP;
                double cs[2] = {0.0, 0.0};
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const double xr = vc[TILE * I + 2 * q + h];
                    cs[0] += __hiloint2double(t[q].y, t[q].x) * xr;
                    cs[1] += __hiloint2double(t[q].w, t[q].z) * xr;
                }
                cpart[c] += reduce_scatter<2, 4>(cs, lane);
            }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) part[warp][c][idx] = cpart[c];
        __syncthreads();
        {
            const double *tile = dtiles + (size_t)ltile(T, J, J) * TILE * TILE;
            for (int c = warp; c < NC; c += nw) {
                double *vc = vm + c * NP;
                double v0 = vc[TILE * J + lane];
                for (int w = 0; w < nw; ++w) v0 -= part[w][c][lane];
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int k = 0; k < TILE; k += 2) {
                    s0 += tile[k * TILE + lane] * __shfl_sync(FULL, v0, k);
                    s1 += tile[(k + 1) * TILE + lane] * __shfl_sync(FULL, v0, k + 1);
                }
                vc[TILE * J + lane] = s0 + s1;
            }
        }
        __syncthreads();
    }
    for (int c = 0; c < NC; ++c)
        for (int i = threadIdx.x; i < n; i += blockDim.x) out[(size_t)(j0 + c) * stride + o + i] = vm[c * NP + pos[i]];
}

// K^+ on NC = 8 or 16 right-hand sides with FP64 tensor-core MMAs (mma.m8n8k4.f64).  Same tile
// walk, nonzero-tile lists and modes as kplus_multi_kernel.  Every 32 x 32 step is
// C(32 x NC) += A(32 x 32) B(32 x NC) as 4 x NC/8 blocks of 8 x 8 over 8 k-steps of 4: A is the
// factor tile read straight from global memory in fragment order (the tile in the forward pass, its
// transpose in the backward pass; every 32-byte sector is read once), B the column block of the
// vectors in shared memory.  The vectors are kept in factor order, NP + KPM_PAD doubles apart, so
// that the fragment loads and stores take the minimum two wavefronts.  Warps take the off-diagonal
// tiles of a block column in turn; the diagonal step (inverse diagonal tile) is split over 4 x NC/8
// warps.  The backward partial sums of the warps meet in shared memory.
constexpr int KPM_PAD = 4;

__device__ __forceinline__ void dmma84(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

template <int NC, bool GL>
__global__ void __launch_bounds__(256, 1) kplus_mma_kernel(KplusDev K, const double *in, double *out, int mode,
                                                           int j0, long long stride, double *z, double *gvec) {
    static_assert(NC == 8 || NC == 16, "K+ MMA kernel: 8 or 16 columns");
    constexpr int NB = NC / 8;
    extern __shared__ double vm_s[];               // [NC][NP + KPM_PAD]
    __shared__ double part[8][4 * NB * 2 * 32];    // backward partials per warp, fragment order
    const int d = blockIdx.x;
    const int n = K.n[d], T = K.tn[d], o = K.doff[d];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gr = lane >> 2, gc = lane & 3;       // fragment row (group) and column in the group
    const int NP = TILE * T, NPp = NP + KPM_PAD;
    const int *pos = K.pos + o;
    const double *L = K.L + (size_t)K.tile0[d] * TILE * TILE;
    const int *cp = K.cptr + K.cbase[d];
    const int jt = mode == KPLUS_FULL ? 0 : K.jt[d];
    // GL: the vectors of subdomains too large for shared memory live in a global (L2-resident)
    // scratch, NC (32 T_d + KPM_PAD) doubles per subdomain; the block barriers order them as well
    double *vm = GL ? gvec + (size_t)NC * ((size_t)TILE * K.tpre[d] + (size_t)KPM_PAD * d) : vm_s;
    for (int i = threadIdx.x; i < NC * NPp; i += blockDim.x) vm[i] = 0.0;
    __syncthreads();
    for (int c = 0; c < NC; ++c)
        for (int i = threadIdx.x; i < n; i += blockDim.x) vm[c * NPp + pos[i]] = in[(size_t)(j0 + c) * stride + o + i];
    __syncthreads();

    // block J := inv(L_JJ) block J (trans: inv(L_JJ)^T), warps 0 .. 4 NB - 1, one 8 x 8 block each
    auto diag = [&](int J, bool trans) {
        const bool act = warp < 4 * NB;
        const int mb = warp & 3, nb = warp >> 2;
        double acc[2] = {0.0, 0.0};
        if (act) {
            const double *tile = L + (size_t)ltile(T, J, J) * TILE * TILE;
            const double *bcol = vm + (size_t)(8 * nb + gr) * NPp + TILE * J;
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const int k = 4 * ks + gc;
                const double a = trans ? __ldg(tile + k * TILE + 8 * mb + gr) : __ldg(tile + (8 * mb + gr) * TILE + k);
                dmma84(acc, a, bcol[k]);
            }
        }
        __syncthreads();   // block J read by every active warp before it is overwritten
        if (act) {
            double *cc = vm + (size_t)(8 * nb + 2 * gc) * NPp + TILE * J + 8 * mb + gr;
            cc[0] = acc[0];
            cc[NPp] = acc[1];
        }
        __syncthreads();
    };

    // Factor fragments come straight from global memory in fragment order; a warp's next tile is
    // loaded while the MMAs of its current one run, and its first tile of the next block column
    // before the barriers and the diagonal step of that column.
    auto fload = [&](int J, int qx, double (&a)[4][8]) {
        const double *tile = L + (size_t)ltile(T, K.rows[qx], J) * TILE * TILE + gr * TILE + gc;
#pragma unroll
        for (int mb = 0; mb < 4; ++mb)
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) a[mb][ks] = __ldg(tile + 8 * mb * TILE + 4 * ks);
    };
    auto bload = [&](int J, int qx, double (&a)[4][8]) {   // A = L_IJ^T: A[m][k] = L_IJ[k][m]
        const double *tile = L + (size_t)ltile(T, K.rows[qx], J) * TILE * TILE + gc * TILE + gr;
#pragma unroll
        for (int mb = 0; mb < 4; ++mb)
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) a[mb][ks] = __ldg(tile + 4 * ks * TILE + 8 * mb);
    };
    double a0[4][8], a1[4][8];
    // forward: L y = f
    const int jf = mode == KPLUS_PRIMAL ? jt : 0;
    if (jf < T && cp[jf] + 1 + warp < cp[jf + 1]) fload(jf, cp[jf] + 1 + warp, a0);
    for (int J = jf; J < T; ++J) {
        diag(J, false);
        double bf[8][NB];
#pragma unroll
        for (int ks = 0; ks < 8; ++ks)
#pragma unroll
            for (int nb = 0; nb < NB; ++nb) bf[ks][nb] = vm[(size_t)(8 * nb + gr) * NPp + TILE * J + 4 * ks + gc];
        auto fproc = [&](int qx, const double (&af)[4][8]) {
            const int I = K.rows[qx];
            double acc[4][NB][2];
#pragma unroll
            for (int mb = 0; mb < 4; ++mb)
#pragma unroll
                for (int nb = 0; nb < NB; ++nb) {
                    acc[mb][nb][0] = 0.0;
                    acc[mb][nb][1] = 0.0;
#pragma unroll
                    for (int ks = 0; ks < 8; ++ks) dmma84(acc[mb][nb], af[mb][ks], bf[ks][nb]);
                }
#pragma unroll
            for (int mb = 0; mb < 4; ++mb)
#pragma unroll
                for (int nb = 0; nb < NB; ++nb) {
                    double *cc = vm + (size_t)(8 * nb + 2 * gc) * NPp + TILE * I + 8 * mb + gr;
                    cc[0] -= acc[mb][nb][0];
                    cc[NPp] -= acc[mb][nb][1];
                }
        };
        const int qe = cp[J + 1];
        for (int qi = cp[J] + 1 + warp; qi < qe; qi += 16) {
            if (qi + 8 < qe) fload(J, qi + 8, a1);
            fproc(qi, a0);
            if (qi + 8 >= qe) break;
            if (qi + 16 < qe) fload(J, qi + 16, a0);
            fproc(qi + 8, a1);
        }
        if (J + 1 < T && cp[J + 1] + 1 + warp < cp[J + 2]) fload(J + 1, cp[J + 1] + 1 + warp, a0);
        __syncthreads();
    }
    if (mode == KPLUS_TOUCHED) {
        for (int c = 0; c < NC; ++c)
            for (int i = threadIdx.x; i < n; i += blockDim.x) z[(size_t)(j0 + c) * stride + o + i] = vm[c * NPp + i];
        __syncthreads();
    } else if (mode == KPLUS_PRIMAL) {
        for (int c = 0; c < NC; ++c)
            for (int i = threadIdx.x; i < n; i += blockDim.x) vm[c * NPp + i] += z[(size_t)(j0 + c) * stride + o + i];
        __syncthreads();
    }
    // backward: L^T x = y (mode 1: down to block jt)
    const int jb = mode == KPLUS_TOUCHED ? jt : 0;
    if (T - 1 >= jb && cp[T - 1] + 1 + warp < cp[T]) bload(T - 1, cp[T - 1] + 1 + warp, a0);
    for (int J = T - 1; J >= jb; --J) {
        double acc[4][NB][2];
#pragma unroll
        for (int mb = 0; mb < 4; ++mb)
#pragma unroll
            for (int nb = 0; nb < NB; ++nb) acc[mb][nb][0] = acc[mb][nb][1] = 0.0;
        auto bproc = [&](int qx, const double (&af)[4][8]) {
            const int I = K.rows[qx];
            double bf[8][NB];
#pragma unroll
            for (int ks = 0; ks < 8; ++ks)
#pragma unroll
                for (int nb = 0; nb < NB; ++nb) bf[ks][nb] = vm[(size_t)(8 * nb + gr) * NPp + TILE * I + 4 * ks + gc];
#pragma unroll
            for (int mb = 0; mb < 4; ++mb)
#pragma unroll
                for (int nb = 0; nb < NB; ++nb)
#pragma unroll
                    for (int ks = 0; ks < 8; ++ks) dmma84(acc[mb][nb], af[mb][ks], bf[ks][nb]);
        };
        const int qe = cp[J + 1];
        for (int qi = cp[J] + 1 + warp; qi < qe; qi += 16) {
            if (qi + 8 < qe) bload(J, qi + 8, a1);
            bproc(qi, a0);
            if (qi + 8 >= qe) break;
            if (qi + 16 < qe) bload(J, qi + 16, a0);
            bproc(qi + 8, a1);
        }
        if (J - 1 >= jb && cp[J - 1] + 1 + warp < cp[J]) bload(J - 1, cp[J - 1] + 1 + warp, a0);
#pragma unroll
        for (int mb = 0; mb < 4; ++mb)
#pragma unroll
            for (int nb = 0; nb < NB; ++nb) {
                part[warp][((mb * NB + nb) * 2 + 0) * 32 + lane] = acc[mb][nb][0];
                part[warp][((mb * NB + nb) * 2 + 1) * 32 + lane] = acc[mb][nb][1];
            }
        __syncthreads();
        for (int q = threadIdx.x; q < 32 * NC; q += blockDim.x) {
            const int ln = q & 31, e = (q >> 5) & 1, blk = q >> 6, mb = blk / NB, nb = blk % NB;
            double sum = 0.0;
#pragma unroll
            for (int w = 0; w < 8; ++w) sum += part[w][q];
            vm[(size_t)(8 * nb + 2 * (ln & 3) + e) * NPp + TILE * J + 8 * mb + (ln >> 2)] -= sum;
        }
        __syncthreads();
        diag(J, true);
    }
    for (int c = 0; c < NC; ++c)
        for (int i = threadIdx.x; i < n; i += blockDim.x) out[(size_t)(j0 + c) * stride + o + i] = vm[c * NPp + pos[i]];
}

// subdomain loads f_i = rhs(caller DOF) / multiplicity
__global__ void split_rhs_kernel(const double *rhs, const int *gdof, const double *invm, double *f, int ntot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ntot) {
        int g = gdof[i];
        f[i] = g >= 0 ? rhs[g] * invm[i] : 0.0;
    }
}

// e = -R^T f per subdomain
__global__ void evec_kernel(DevProblem P, const int *doff, const int *rofs, const double *R, const double *f, double *e) {
    __shared__ double sh[32 * KMAX];
    const int d = blockIdx.x;
    const int n = doff[d + 1] - doff[d], nk = P.kof[d + 1] - P.kof[d];
    const double *Rd = R + rofs[d];
    double acc[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) acc[k] = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double fi = f[doff[d] + i];
        for (int k = 0; k < nk; ++k) acc[k] += Rd[(size_t)k * n + i] * fi;
    }
    block_sum_k(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < nk; ++k) e[P.kof[d] + k] = -acc[k];
}

// b at every local row: own (s K^+ f)[dof] - c plus the partner's
__global__ void bvec_kernel(DevProblem P, const int *rdof, const double *rsign, const double *rc, const double *kf,
                            double *bL) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.NL) return;
    double b = rsign[e] * kf[rdof[e]] - rc[e];
    int q = P.partner[e];
    if (q >= 0) b += rsign[q] * kf[rdof[q]] - rc[q];
    bL[e] = b;
}

// g = f - B^T lambda (local DOF space), gathered through the touched-DOF rows
__global__ void primal_rhs_kernel(DevProblem P, const int *tdof_g, const double *rsign, const double *f, double *g,
                                  int ntot) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) g[i] = f ? f[i] : 0.0;
}
__global__ void primal_bt_kernel(DevProblem P, const int *tdof_g, const double *rsign, double *g) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.NT) return;
    double s = 0.0;
    for (int j = P.trow_ptr[t]; j < P.trow_ptr[t + 1]; ++j) {
        int e = P.trow_idx[j];
        s += rsign[e] * P.x[e];
    }
    g[tdof_g[t]] -= s;
}

// u += R alpha (dual kernel basis and amplitudes), merged into the caller's DOF vector
// (average over subdomains)
__global__ void primal_merge_kernel(DevProblem P, const int *doff, const int *rofs, const double *R, const double *u,
                                    const int *gdof, const double *invm, double *sol) {
    const int d = blockIdx.x;
    const int n = doff[d + 1] - doff[d], nk = P.kof[d + 1] - P.kof[d];
    const double *Rd = R + rofs[d];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double val = u[doff[d] + i];
        for (int k = 0; k < nk; ++k) val += Rd[(size_t)k * n + i] * P.alpha[P.akof[d] + k];
        int g = gdof[doff[d] + i];
        if (g >= 0) atomicAdd(&sol[g], val * invm[doff[d] + i]);
    }
}


// ---------------------------------------------------------------------------------------------
// Hybrid Total FETI: the cluster correction of the dual operator and the cluster K^+.
// cond: 0 always, 1 inside the PCG loop, 3 inside the loop on a residual-replacement iteration.
__device__ __forceinline__ bool hyb_skip(const DevProblem &P, int slot, int cond) {
    if (cond == 0) return false;
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return true;
    return cond == 3 && P.st->replace_iter != iter;
}

// z_i = V_i^T x_i: one warp per column of V_i.  With x == null the PCG direction
// p = y + beta p is formed on the fly, as the tile SYMV does (update_kernel stores it later).
__global__ void hyb_vt_kernel(DevProblem P, HybDev H, const double *x, int slot, int cond) {
    pdl_enter();
    if (hyb_skip(P, slot, cond)) return;
    const int d = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int e0 = P.loff[d], ni = P.loff[d + 1] - e0;
    const int z0 = H.zof[d], m = H.zof[d + 1] - z0;
    const double *V = H.V + H.voff[d];
    double beta = 0.0;
    if (x == nullptr) {
        const int iter = P.st->iter_base + slot;
        beta = iter == 0 ? 0.0 : P.scal[SC_RHO] / P.rho_hist[iter - 1];
    }
    for (int c = wid; c < m; c += nw) {
        const double *col = V + (size_t)c * ni;
        double s = 0.0;
        if (x == nullptr)
            for (int r = lane; r < ni; r += 32) s += col[r] * (P.y[e0 + r] + beta * P.p[e0 + r]);
        else
            for (int r = lane; r < ni; r += 32) s += col[r] * x[e0 + r];
        s = warp_sum(s);
        if (lane == 0) H.z[z0 + c] = s;
    }
}

// w_c = M_c z_c for every cluster; z_c is gathered from the member slots in member order.
// grid (ncl, row blocks); with dot != null the last CTA subtracts sum_c z_c . w_c from *dot.
constexpr int HM_ROWS = 64;
__global__ void __launch_bounds__(256) hyb_m_kernel(DevProblem P, HybDev H, int slot, int cond, double *dot) {
    pdl_enter();
    if (hyb_skip(P, slot, cond)) return;
    extern __shared__ double hz[];
    __shared__ double sh[32];
    __shared__ int s_last;
    const int c = blockIdx.x;
    const int nc = H.cof[c + 1] - H.cof[c];
    for (int i = threadIdx.x; i < nc; i += blockDim.x) hz[i] = 0.0;
    __syncthreads();
    for (int q = H.mem_ptr[c]; q < H.mem_ptr[c + 1]; ++q) {
        const int d = H.mem[q];
        // the slots of one subdomain map to distinct entries of the cluster vector
        for (int j = H.zof[d] + threadIdx.x; j < H.zof[d + 1]; j += blockDim.x) hz[H.vmap[j]] += H.z[j];
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int r0 = blockIdx.y * HM_ROWS, r1 = min(nc, r0 + HM_ROWS);
    const double *M = H.M + H.mof[c];
    double zw = 0.0;
    for (int r = r0 + wid; r < r1; r += nw) {
        const double *col = M + (size_t)r * nc;    // symmetric: column r = row r
        double s = 0.0;
        for (int j = lane; j < nc; j += 32) s += col[j] * hz[j];
        s = warp_sum(s);
        if (lane == 0) {
            H.w[H.cof[c] + r] = s;
            zw += s * hz[r];
        }
    }
    if (dot == nullptr) return;
    zw = block_sum(zw, sh);
    const int cta = blockIdx.y * gridDim.x + blockIdx.x, ncta = gridDim.x * gridDim.y;
    if (threadIdx.x == 0) {
        H.part[cta] = zw;
        __threadfence();
        s_last = (atomicAdd(H.done, 1) == ncta - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double t = 0.0;
        for (int i = threadIdx.x; i < ncta; i += blockDim.x) t += __ldcg(&H.part[i]);
        t = block_sum(t, sh);
        if (threadIdx.x == 0) {
            *dot -= t;
            *H.done = 0;
        }
    }
}

// y_i -= V_i w_{c(i)}: one thread per row
__global__ void hyb_v_kernel(DevProblem P, HybDev H, double *y, int slot, int cond) {
    pdl_enter();
    if (hyb_skip(P, slot, cond)) return;
    extern __shared__ double wl[];
    const int d = blockIdx.x;
    const int e0 = P.loff[d], ni = P.loff[d + 1] - e0;
    const int z0 = H.zof[d], m = H.zof[d + 1] - z0;
    const double *wc = H.w + H.cof[H.sub_cl[d]];
    for (int j = threadIdx.x; j < m; j += blockDim.x) wl[j] = wc[H.vmap[z0 + j]];
    __syncthreads();
    const double *V = H.V + H.voff[d];
    for (int r = threadIdx.x; r < ni; r += blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < m; ++c) s += V[(size_t)c * ni + r] * wl[c];
        y[e0 + r] -= s;
    }
}

// cluster K^+ on primal vectors, step 1: z_i = [B0_i (K_i^+ x_i); -R_i^T x_i]
__global__ void hyb_kz_kernel(DevProblem P, HybDev H, const int *doff, const int *rofs, const double *R,
                              const double *kx, const double *x) {
    __shared__ double sh[32 * KMAX];
    const int d = blockIdx.x;
    const int n = doff[d + 1] - doff[d], z0 = H.zof[d], m0 = H.m0[d], nk = H.zof[d + 1] - z0 - m0;
    for (int j = threadIdx.x; j < m0; j += blockDim.x) H.z[z0 + j] = H.b0sign[z0 + j] * kx[doff[d] + H.b0dof[z0 + j]];
    const double *Rd = R + rofs[d];
    double acc[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) acc[k] = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double xi = x[doff[d] + i];
        for (int k = 0; k < nk; ++k) acc[k] += Rd[(size_t)k * n + i] * xi;
    }
    block_sum_k(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < nk; ++k) H.z[z0 + m0 + k] = -acc[k];
}

// step 2: g_i = x_i - B0_i^T lambda0 (one thread walks a subdomain's corner entries: a corner DOF
// can appear in several rows of one subdomain)
__global__ void hyb_copy_kernel(const double *x, double *g, int ntot) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) g[i] = x[i];
}
__global__ void hyb_kb0_kernel(DevProblem P, HybDev H, const int *doff, double *g) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= P.nd) return;
    const int z0 = H.zof[d], m0 = H.m0[d];
    const double *wc = H.w + H.cof[H.sub_cl[d]];
    for (int j = 0; j < m0; ++j) g[doff[d] + H.b0dof[z0 + j]] -= H.b0sign[z0 + j] * wc[H.vmap[z0 + j]];
}

// step 3: out_i += R_i alpha_i
__global__ void hyb_kr_kernel(DevProblem P, HybDev H, const int *doff, const int *rofs, const double *R, double *out) {
    const int d = blockIdx.x;
    const int n = doff[d + 1] - doff[d], z0 = H.zof[d], m0 = H.m0[d], nk = H.zof[d + 1] - z0 - m0;
    const double *wc = H.w + H.cof[H.sub_cl[d]];
    const double *Rd = R + rofs[d];
    double a[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) a[k] = k < nk ? wc[H.vmap[z0 + m0 + k]] : 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < nk; ++k) s += Rd[(size_t)k * n + i] * a[k];
        out[doff[d] + i] += s;
    }
}

}  // namespace

// =============================================================================================
constexpr int kSizeClasses = 5;

struct TileSetHost {
    int prec = -1;
    int nitems = 0;
    size_t bytes = 0;          // stored bytes
    double alg_bytes = 0.0;    // algorithmic bytes of one apply (triangle + vectors)
    int4 *items = nullptr;
    int *mat_n = nullptr, *mat_voff = nullptr, *mat_tn = nullptr;
    long long *mat_tile0 = nullptr;
    unsigned *tile_ij = nullptr;
    void *tiles = nullptr;
    float *scale = nullptr;
    double *item_dot = nullptr;
    int *queue = nullptr;
    int kernel = 0;                 // 0 register prefetch, 1 TMA pipeline (autotuned)
    std::vector<int> h_tn;          // tile rows per matrix (host copy for re-itemising)
    long long total_tiles = 0;
    std::vector<int> class_tpi;     // chosen tiles per item of each size class
    TileSetDev dev() const {
        TileSetDev t;
        t.nitems = nitems; t.prec = prec; t.items = items; t.mat_n = mat_n; t.mat_voff = mat_voff; t.mat_tn = mat_tn;
        t.mat_tile0 = mat_tile0; t.tile_ij = tile_ij; t.tiles = tiles; t.scale = scale; t.item_dot = item_dot;
        t.queue = queue;
        return t;
    }
};

struct GpuSolver::Impl {
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    SolveOptions opt;
    std::vector<void *> allocs;
    size_t bytes = 0;
    DevProblem P{};
    DevState *st = nullptr;
    TileSetHost F64, Flow, Dir;
    bool implicit = false;        // F64 applies run through the K^+ factor (kplus_dual_kernel), no S_i tiles
    long long implicit_tiles = 0; // factor tiles one implicit pass applies (touched block columns, not all zero)
    void launch_implicit(int mode, const double *src, const double *src2, double *out, int slot);
    void release(void *p);        // frees one allocation of `allocs` before the solver goes
    int max_tn = 0, max_tn_dir = 0, max_nt = 0, max_ni = 0;
    // threads of the per-subdomain vector kernels of the PCG loop: as many as keep every subdomain's
    // CTA resident in one wave (2048 threads per SM), so that each thread has about one row
    int tpbv = 256;
    std::vector<int> h_lam;       // L row -> lambda
    int *d_lam = nullptr;         // the same on the device
    std::vector<int> h_loff;
    std::vector<int> h_doff;      // local-DOF offsets of the subdomains (K^+ vectors)
    int n_lambda = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_chunk = 0, graph_prec = -1, graph_precond = -1;
    double *Ax64 = nullptr;   // F apply output outside the iteration operator (initial, replacement, tests)
    // device K^+ and the right-hand-side / primal vectors
    KplusDev KP{};
    long long kplus_tiles_kept = 0, kplus_tiles_total = 0;   // factor tiles applied / stored
    long long kp_tsum = 0;                                    // 32-blocks of all subdomains
    double *kp_gvec = nullptr;                                // kplus_mma_kernel<NC, true> vectors
    size_t kp_gvec_n = 0;
    int max_T = 0, ntot = 0, n_caller = 0;
    int *d_doff = nullptr, *d_rofs = nullptr, *d_gdof = nullptr, *d_rdof = nullptr, *d_tdof_g = nullptr;
    double *d_invm = nullptr, *d_R = nullptr, *d_rsign = nullptr, *d_rc = nullptr;
    // dual kernel basis per subdomain (the subdomain kernel, or the cluster kernel R_i H_i)
    double *d_Rd = nullptr;
    int *d_rdofs = nullptr;
    std::vector<int> dual_to_partial;   // dual kernel index -> one partial slot holding it
    // Hybrid Total FETI
    bool hybrid = false;
    HybDev H{};
    int hyb_max_m = 0, hyb_rows = 1;
    double *d_h = nullptr;              // primal scratch of the cluster K^+
    void upload_hybrid(const Decomposition &dec, const Prep &prep);
    // y -= V M V^T x (cond as hyb_skip; x null: the PCG direction y + beta p; dot: p.Ap to correct)
    void launch_hybrid_F(const double *x, double *y, int slot, int cond, double *dot);
    // out = K_c^+ in on the concatenated local primal vectors (Total FETI: K^+ in)
    void launch_kplus_dual(const double *in, double *out);
    void launch_kplus_dual_multi(const double *in, double *out, int ncol);
    int hyb_w_size = 0;                       // cluster vector length (sum over clusters)
    double *hyb_wsave = nullptr, *hyb_hm = nullptr;   // per-column cluster vectors / second K^+ inputs
    size_t hyb_wsave_n = 0, hyb_hm_n = 0;
    double *d_f = nullptr, *d_kf = nullptr, *d_g = nullptr, *d_rhs = nullptr, *d_sol = nullptr;
    double *h_pinned = nullptr;
    size_t h_pinned_n = 0;
    std::vector<cudaEvent_t> stage_ev;
    void ensure_pinned(size_t n);
    void h2d_columns(double *dev, size_t dev_pitch, const double *host, size_t host_pitch, size_t count, int ncols);
    void d2h_columns(double *host, size_t host_pitch, const double *dev, size_t dev_pitch, size_t count, int ncols);
    // block (multi right-hand-side) solver
    struct Block {
        int nr = 0;
        BlockDev B{};
        int2 *units = nullptr;
        int nunits = 0;
        cudaGraphExec_t graph = nullptr;
        int graph_chunk = 0, graph_prec = -1, graph_precond = -1;
        double *rhs = nullptr, *sol = nullptr, *f = nullptr, *kf = nullptr, *g = nullptr;
        double *zk = nullptr;   // forward results L^-1 f of every column (K^+ modes 1 and 2)
        int flat_grid = 1;
        int2 *units4 = nullptr;
        int nunits4 = 0;
        float *pan = nullptr;          // K-major panels of the mixed blocks (asynchronous tensor-core SYMM)
        int2 *dunits = nullptr;   // SYMM units of the Dirichlet blocks (Dirichlet preconditioner)
        int ndunits = 0;
    } blk;
    void ensure_block(int nr);
    void prepare_symm_panels();
    void launch_symm(const TileSetHost &T, bool src32, const double *x64, const float *x32, double *out, int slot,
                     int mode);
    void launch_block_iteration(int slot);
    // block cluster correction y -= V M V^T x for nr columns
    double *bh_z = nullptr, *bh_w = nullptr, *bh_part = nullptr;
    int *bh_done = nullptr;
    void launch_block_hybrid(const double *x, double *y, int slot, int cond, double *dot);
    // element data for the adjoint sensitivities
    int *el_dofs = nullptr;
    double *el_K = nullptr, *el_out = nullptr, *el_u = nullptr, *el_v = nullptr;
    size_t el_count = 0;
    int el_nd = 0, el_n = 0;
    double *e_dev = nullptr;
    int rho_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    template <typename T>
    T *alloc(size_t n) {
        void *p = nullptr;
        if (n == 0) n = 1;
        CUDA_CHECK(cudaMalloc(&p, n * sizeof(T)));
        allocs.push_back(p);
        alloc_sizes.push_back(n * sizeof(T));
        bytes += n * sizeof(T);
        return (T *)p;
    }
    size_t alloc_bytes_of(void *p) const {
        for (size_t i = 0; i < allocs.size(); ++i)
            if (allocs[i] == p) return alloc_sizes[i];
        return 0;
    }
    std::vector<size_t> alloc_sizes;
    template <typename T>
    T *upload(const std::vector<T> &v) {
        T *p = alloc<T>(v.size());
        if (!v.empty()) CUDA_CHECK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        return p;
    }
    ~Impl() {
        if (blk.graph) cudaGraphExecDestroy(blk.graph);
        if (graph_loop) cudaGraphExecDestroy(graph_loop);
        if (h_pinned) cudaFreeHost(h_pinned);
        for (cudaEvent_t e : stage_ev) cudaEventDestroy(e);
        if (graph) cudaGraphExecDestroy(graph);
        for (void *p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }

    void build_tiles(TileSetHost &T, int prec, const std::vector<const double *> &mats, const std::vector<int> &ns,
                     const std::vector<int> &voffs, int tiles_per_item, double *dev64 = nullptr);
    // takes over a device buffer allocated elsewhere (freed with the solver)
    template <typename T>
    T *adopt(T *&p, size_t n) {
        T *q = p;
        p = nullptr;
        allocs.push_back(q);
        alloc_sizes.push_back(n * sizeof(T));
        bytes += n * sizeof(T);
        return q;
    }
    void itemize(TileSetHost &T, const std::vector<int> &tpi, int only_class);
    void autotune(TileSetHost &T, double *x, double *y, int ny);
    void launch_tiles(const TileSetHost &T, int mode, const double *src, const double *src2, double *out, int slot);
    void capture_chunk(int chunk);
    bool capture_loop();
    cudaGraphExec_t graph_loop = nullptr;
    int graph_loop_key = -1;
    bool loop_refused = false;
    void launch_replacement(int slot);
    void launch_iteration(int slot, bool with_replacement = true, LoopCtl lc = LoopCtl{0, 0, 0});
    int kernels_per_iteration() const;
    void upload_kplus(const Decomposition &dec, const Prep &prep, const std::vector<int> &loff,
                      const std::vector<int> &toff);
    void launch_kplus(const double *in, double *out, int mode = KPLUS_FULL);
    void launch_kplus_multi(const double *in, double *out, int ncol, int mode, double *z);
};

// dynamic shared memory available to kplus_multi_kernel<NC> next to its static partial sums
static size_t kplus_multi_smem(int nc) { return (size_t)220 * 1024 - (size_t)nc * 8 * TILE * sizeof(double); }
// dynamic shared memory available to kplus_mma_kernel<NC> next to its 16 KB per 8 columns of partials
static size_t kplus_mma_smem(int nc) { return (size_t)226 * 1024 - (size_t)(nc / 8) * 16 * 1024; }
static bool kplus_mma_enabled() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_KPLUS_MMA");
        return !(e && e[0] == '0');
    }();
    return on;
}

// K^+ on ncol columns (stride ntot): groups of NC columns per pass, NC as large as shared memory allows.
void GpuSolver::Impl::launch_kplus_multi(const double *in, double *out, int ncol, int mode, double *z) {
    const size_t per_col = sizeof(double) * TILE * (size_t)max_T;
    int j0 = 0;
    while (j0 < ncol) {
        const int left = ncol - j0;
        // (groups of 16, 8, 4 and 2 gave 120, 128, 120 and 133 ms of batched e2e on c2)
        int nc = 16;
        while (nc > 1 && (nc > left || (size_t)nc * per_col > kplus_multi_smem(nc))) nc /= 2;
        const size_t sm = (size_t)nc * per_col;
        // FP64 tensor-core variant for 8 or 16 columns when the padded vectors fit next to its
        // partial sums
        const size_t sm_mma = sizeof(double) * (size_t)nc * ((size_t)TILE * max_T + KPM_PAD);
        if (kplus_mma_enabled() && (nc == 16 || nc == 8) && sm_mma <= kplus_mma_smem(nc)) {
            if (nc == 16) kplus_mma_kernel<16, false><<<P.nd, 256, sm_mma, stream>>>(KP, in, out, mode, j0, ntot, z, nullptr);
            else kplus_mma_kernel<8, false><<<P.nd, 256, sm_mma, stream>>>(KP, in, out, mode, j0, ntot, z, nullptr);
            CUDA_CHECK(cudaGetLastError());
            j0 += nc;
            continue;
        }
        if (kplus_mma_enabled() && left >= 8) {
            // subdomains too large for the vectors in shared memory: 16 (or 8) columns with the
            // vectors in a global scratch instead of 2-4 columns per pass
            const int ncg = left >= 16 ? 16 : 8;
            const size_t need = (size_t)ncg * ((size_t)TILE * kp_tsum + (size_t)KPM_PAD * P.nd);
            if (kp_gvec_n < need) {
                kp_gvec = alloc<double>(need);
                kp_gvec_n = need;
            }
            if (ncg == 16) kplus_mma_kernel<16, true><<<P.nd, 256, 0, stream>>>(KP, in, out, mode, j0, ntot, z, kp_gvec);
            else kplus_mma_kernel<8, true><<<P.nd, 256, 0, stream>>>(KP, in, out, mode, j0, ntot, z, kp_gvec);
            CUDA_CHECK(cudaGetLastError());
            j0 += ncg;
            continue;
        }
        switch (nc) {
        case 16: kplus_multi_kernel<16><<<P.nd, 256, sm, stream>>>(KP, in, out, mode, j0, ntot, z); break;
        case 8: kplus_multi_kernel<8><<<P.nd, 256, sm, stream>>>(KP, in, out, mode, j0, ntot, z); break;
        case 4: kplus_multi_kernel<4><<<P.nd, 256, sm, stream>>>(KP, in, out, mode, j0, ntot, z); break;
        case 2: kplus_multi_kernel<2><<<P.nd, 256, sm, stream>>>(KP, in, out, mode, j0, ntot, z); break;
        default: kplus_multi_kernel<1><<<P.nd, 256, sm, stream>>>(KP, in, out, mode, j0, ntot, z); break;
        }
        CUDA_CHECK(cudaGetLastError());
        j0 += nc;
    }
}

void GpuSolver::Impl::launch_kplus(const double *in, double *out, int mode) {
    size_t sm = sizeof(double) * TILE * (size_t)max_T;
    kplus_kernel<<<P.nd, 256, sm, stream>>>(KP, in, out, mode);
    CUDA_CHECK(cudaGetLastError());
}

void GpuSolver::Impl::upload_kplus(const Decomposition &dec, const Prep &prep, const std::vector<int> &loff,
                                   const std::vector<int> &toff) {
    const int nd = dec.ndom;
    const int dpn = dec.dpn;
    std::vector<int> n(nd), tn(nd), doff(nd + 1, 0), rofs(nd + 1, 0), rdofs(nd + 1, 0);
    std::vector<long long> tile0(nd + 1, 0);
    max_T = 0;
    for (int d = 0; d < nd; ++d) {
        n[d] = prep.sub[d].n;
        tn[d] = (n[d] + TILE - 1) / TILE;
        max_T = std::max(max_T, tn[d]);
        doff[d + 1] = doff[d] + n[d];
        rofs[d + 1] = rofs[d] + n[d] * prep.sub[d].nk;
        rdofs[d + 1] = rdofs[d] + n[d] * prep.sub[d].dnk;
        tile0[d + 1] = tile0[d] + (long long)tn[d] * (tn[d] + 1) / 2;
    }
    FETI_CHECK(sizeof(double) * TILE * (size_t)max_T <= 200 * 1024, "FETI4I: subdomain too large for the device K+ kernel");
    ntot = doff[nd];
    std::vector<int> pos(ntot), gdof(ntot), tdof_g(toff[nd]);
    std::vector<double> invm(ntot), R(rofs[nd]), Rd(prep.method == 1 ? rdofs[nd] : 0);
    DevPrepStore *ds = prep.dstore.get();
    if (ds) FETI_CHECK(ds->kp_tiles && ds->kp_tile0 == tile0, "FETI4I: device K+ tiles do not match the subdomains");
    std::vector<double> L(ds ? 0 : (size_t)tile0[nd] * TILE * TILE, 0.0);
    n_caller = 0;
    for (int d = 0; d < nd; ++d) {
        const SubPrep &S = prep.sub[d];
        const DomainRows &D = dec.dom[d];
        for (int i = 0; i < n[d]; ++i) pos[doff[d] + i] = S.pos[i];
        for (int a = 0; a < (int)D.nodes.size(); ++a)
            for (int c = 0; c < dpn; ++c) {
                int g = dec.node_dof[(size_t)D.nodes[a] * dpn + c];
                gdof[doff[d] + dpn * a + c] = g;
                invm[doff[d] + dpn * a + c] = 1.0 / dec.node_ndom[D.nodes[a]];
                n_caller = std::max(n_caller, g + 1);
            }
        std::copy(S.R.begin(), S.R.end(), R.begin() + rofs[d]);
        if (prep.method == 1) std::copy(S.Rd.begin(), S.Rd.end(), Rd.begin() + rdofs[d]);
        for (int t = 0; t < S.t; ++t) tdof_g[toff[d] + t] = doff[d] + S.tdof[t];
        if (ds) continue;   // factor tiles written by the device preprocessing
        const int T = tn[d], nn = n[d];
        for (int J = 0; J < T; ++J)
            for (int I = J; I < T; ++I) {
                double *tile = L.data() + (size_t)(tile0[d] + (long long)J * T - (long long)J * (J - 1) / 2 + (I - J)) * TILE * TILE;
                for (int r = 0; r < TILE; ++r)
                    for (int c = 0; c < TILE; ++c) {
                        int gr = TILE * I + r, gc = TILE * J + c;
                        double v = 0.0;
                        if (gr < nn && gc < nn) { if (gr >= gc) v = S.Lp[dense::packed_index(nn, gr, gc)]; }
                        else if (gr == gc) v = 1.0;
                        tile[r * TILE + c] = v;
                    }
                if (I == J) {
                    // diagonal tile: inverse of its lower-triangular block, column by column
                    double inv[TILE * TILE] = {};
                    for (int c = 0; c < TILE; ++c) {
                        for (int r = c; r < TILE; ++r) {
                            double sum = (r == c) ? 1.0 : 0.0;
                            for (int k = c; k < r; ++k) sum -= tile[r * TILE + k] * inv[k * TILE + c];
                            inv[r * TILE + c] = sum / tile[r * TILE + r];
                        }
                    }
                    std::copy(inv, inv + TILE * TILE, tile);
                }
            }
    }
    // per local multiplier row: DOF in the concatenated local space, sign, Dirichlet value
    const int NL = loff[nd];
    std::vector<int> rdof(NL);
    std::vector<double> rsign(NL), rc(NL);
    for (int d = 0; d < nd; ++d) {
        const DomainRows &D = dec.dom[d];
        for (size_t r = 0; r < D.lam.size(); ++r) {
            rdof[loff[d] + r] = doff[d] + D.dof[r];
            rsign[loff[d] + r] = D.sign[r];
            rc[loff[d] + r] = D.c[r];
        }
    }
    KP.nd = nd;
    KP.n = upload(n);
    KP.tn = upload(tn);
    d_doff = upload(doff);
    h_doff = doff;
    KP.doff = d_doff;
    KP.tile0 = upload(tile0);
    KP.pos = upload(pos);
    {
        std::vector<int> jt(nd);
        for (int d = 0; d < nd; ++d) jt[d] = (prep.sub[d].n - prep.sub[d].t) / TILE;
        KP.jt = upload(jt);
        KP.z = alloc<double>(std::max(1, ntot));
    }
    KP.L = ds ? adopt(ds->kp_tiles, (size_t)tile0[nd] * TILE * TILE) : upload(L);
    {
        // nonzero tiles per block column, found on the device factor
        const long long ntiles = tile0[nd];
        unsigned char *d_nz = nullptr;
        CUDA_CHECK(cudaMalloc(&d_nz, (size_t)std::max<long long>(1, ntiles)));
        tile_nz_kernel<<<nsm * 8, 256, 0, stream>>>(KP.L, ntiles, d_nz);
        CUDA_CHECK(cudaGetLastError());
        std::vector<unsigned char> nz((size_t)ntiles);
        CUDA_CHECK(cudaMemcpyAsync(nz.data(), d_nz, (size_t)ntiles, cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
        CUDA_CHECK(cudaFree(d_nz));
        std::vector<int> cbase(nd + 1, 0), cptr, rows;
        long long kept = 0;
        for (int d = 0; d < nd; ++d) {
            const int T = tn[d];
            cbase[d] = (int)cptr.size();
            for (int J = 0; J < T; ++J) {
                cptr.push_back((int)rows.size());
                const long long c0 = tile0[d] + (long long)J * T - (long long)J * (J - 1) / 2;
                rows.push_back(J);   // the diagonal tile (its inverse) is always applied
                for (int I = J + 1; I < T; ++I)
                    if (nz[(size_t)(c0 + I - J)]) rows.push_back(I);
            }
            cptr.push_back((int)rows.size());
        }
        kept = (long long)rows.size();
        cbase[nd] = (int)cptr.size();
        implicit_tiles = 0;
        for (int d = 0; d < nd; ++d) {
            const int jt_d = (prep.sub[d].n - prep.sub[d].t) / TILE;
            implicit_tiles += cptr[cbase[d] + tn[d]] - cptr[cbase[d] + jt_d];
        }
        FETI_CHECK(kept < (1LL << 31), "FETI4I: too many factor tiles");
        KP.cbase = upload(cbase);
        KP.cptr = upload(cptr);
        KP.rows = upload(rows);
        std::vector<long long> tpre(nd + 1, 0);
        for (int d = 0; d < nd; ++d) tpre[d + 1] = tpre[d] + tn[d];
        KP.tpre = upload(tpre);
        kp_tsum = tpre[nd];
        kplus_tiles_kept = kept;
        kplus_tiles_total = ntiles;
    }
    d_rofs = upload(rofs);
    d_gdof = upload(gdof);
    d_invm = upload(invm);
    d_R = upload(R);
    if (prep.method == 1) {
        d_Rd = upload(Rd);
        d_rdofs = upload(rdofs);
        d_h = alloc<double>(ntot);
    } else {
        d_Rd = d_R;
        d_rdofs = d_rofs;
    }
    d_rdof = upload(rdof);
    d_rsign = upload(rsign);
    d_rc = upload(rc);
    d_tdof_g = upload(tdof_g);
    d_f = alloc<double>(ntot);
    d_kf = alloc<double>(ntot);
    d_g = alloc<double>(ntot);
    d_rhs = alloc<double>(std::max(1, n_caller));
    d_sol = alloc<double>(std::max(1, n_caller));
    cudaFuncSetAttribute(kplus_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(kplus_dual_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(kplus_dual_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    CUDA_CHECK(cudaFuncSetAttribute(kplus_multi_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kplus_multi_smem(16)));
    CUDA_CHECK(cudaFuncSetAttribute(kplus_multi_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kplus_multi_smem(8)));
    CUDA_CHECK(cudaFuncSetAttribute(kplus_multi_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kplus_multi_smem(4)));
    CUDA_CHECK(cudaFuncSetAttribute(kplus_multi_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kplus_multi_smem(2)));
    CUDA_CHECK(cudaFuncSetAttribute(kplus_multi_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kplus_multi_smem(1)));
    CUDA_CHECK(cudaFuncSetAttribute(kplus_mma_kernel<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kplus_mma_smem(16)));
    CUDA_CHECK(cudaFuncSetAttribute(kplus_mma_kernel<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kplus_mma_smem(8)));
}

void GpuSolver::Impl::upload_hybrid(const Decomposition &dec, const Prep &prep) {
    hybrid = prep.method == 1;
    if (!hybrid) return;
    const int nd = dec.ndom, ncl = (int)prep.clusters.size();
    std::vector<long long> voff(nd), mof(ncl);
    std::vector<int> zof(nd + 1, 0), m0(nd), sub_cl(nd), cof(ncl + 1, 0), mem_ptr(ncl + 1, 0), mem, member_idx(nd, -1);
    long long mtot = 0;
    int max_nc = 1;
    for (int c = 0; c < ncl; ++c) {
        const ClusterPrep &C = prep.clusters[c];
        const int nc = C.n0 + C.ka;
        cof[c + 1] = cof[c] + nc;
        mof[c] = mtot;
        mtot += (long long)nc * nc;
        max_nc = std::max(max_nc, nc);
        for (size_t i = 0; i < C.members.size(); ++i) {
            mem.push_back(C.members[i]);
            member_idx[C.members[i]] = (int)i;
        }
        mem_ptr[c + 1] = (int)mem.size();
    }
    size_t vtot = 0;
    int max_m = 1;
    for (int d = 0; d < nd; ++d) {
        const SubPrep &S = prep.sub[d];
        const int m = (int)S.b0_row.size() + S.nk;
        zof[d + 1] = zof[d] + m;
        m0[d] = (int)S.b0_row.size();
        voff[d] = (long long)vtot;
        vtot += (size_t)S.ni * m;
        sub_cl[d] = prep.sub_cluster[d];
        max_m = std::max(max_m, m);
        FETI_CHECK(S.V.size() == (size_t)S.ni * m, "internal: cluster correction block of a subdomain has the wrong size");
    }
    FETI_CHECK(sizeof(double) * (size_t)max_nc <= 200 * 1024 && sizeof(double) * (size_t)max_m <= 200 * 1024,
               "FETI4I: a cluster's corner problem is too large for the device; use more clusters");
    std::vector<int> vmap(zof[nd]), b0dof(zof[nd], 0);
    std::vector<double> b0sign(zof[nd], 0.0), V(vtot), M(mtot);
    for (int d = 0; d < nd; ++d) {
        const SubPrep &S = prep.sub[d];
        const ClusterPrep &C = prep.clusters[sub_cl[d]];
        const int z0 = zof[d];
        for (int j = 0; j < m0[d]; ++j) {
            vmap[z0 + j] = S.b0_row[j];
            b0dof[z0 + j] = S.b0_dof[j];
            b0sign[z0 + j] = S.b0_sign[j];
        }
        for (int k = 0; k < S.nk; ++k) vmap[z0 + m0[d] + k] = C.n0 + C.akofs[member_idx[d]] + k;
        std::copy(S.V.begin(), S.V.end(), V.begin() + voff[d]);
    }
    for (int c = 0; c < ncl; ++c) std::copy(prep.clusters[c].M.begin(), prep.clusters[c].M.end(), M.begin() + mof[c]);
    H.ncl = ncl;
    H.max_nc = max_nc;
    H.voff = upload(voff);
    H.zof = upload(zof);
    H.m0 = upload(m0);
    H.vmap = upload(vmap);
    H.sub_cl = upload(sub_cl);
    H.cof = upload(cof);
    H.mof = upload(mof);
    H.M = upload(M);
    H.V = upload(V);
    H.mem_ptr = upload(mem_ptr);
    H.mem = upload(mem);
    H.b0dof = upload(b0dof);
    H.b0sign = upload(b0sign);
    H.z = alloc<double>(zof[nd]);
    H.w = alloc<double>(cof[ncl]);
    hyb_w_size = cof[ncl];
    hyb_rows = (max_nc + HM_ROWS - 1) / HM_ROWS;
    H.part = alloc<double>((size_t)ncl * hyb_rows);
    H.done = alloc<int>(1);
    CUDA_CHECK(cudaMemset(H.done, 0, sizeof(int)));
    hyb_max_m = max_m;
    cudaFuncSetAttribute(hyb_m_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(hyb_v_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

void GpuSolver::Impl::launch_hybrid_F(const double *x, double *y, int slot, int cond, double *dot) {
    if (!hybrid) return;
    launch_pdl(hyb_vt_kernel, dim3(P.nd), dim3(256), 0, stream, P, H, x, slot, cond);
    launch_pdl(hyb_m_kernel, dim3(H.ncl, hyb_rows), dim3(256), sizeof(double) * H.max_nc, stream, P, H, slot, cond, dot);
    launch_pdl(hyb_v_kernel, dim3(P.nd), dim3(256), sizeof(double) * hyb_max_m, stream, P, H, y, slot, cond);
}

// K_c^+ (or K^+) on ncol columns (stride ntot): both K^+ passes of the cluster solve on all columns
// at once (kplus_multi_kernel); the small cluster steps run column by column, with each column's
// cluster vector kept for its final R alpha step.
void GpuSolver::Impl::launch_kplus_dual_multi(const double *in, double *out, int ncol) {
    launch_kplus_multi(in, out, ncol, KPLUS_FULL, nullptr);
    if (!hybrid) return;
    const int wn = hyb_w_size;
    if (hyb_wsave_n < (size_t)ncol * wn) {
        hyb_wsave = alloc<double>((size_t)ncol * wn);
        hyb_wsave_n = (size_t)ncol * wn;
    }
    if (hyb_hm_n < (size_t)ncol * ntot) {
        hyb_hm = alloc<double>((size_t)ncol * ntot);
        hyb_hm_n = (size_t)ncol * ntot;
    }
    for (int j = 0; j < ncol; ++j) {
        const double *inj = in + (size_t)j * ntot;
        double *outj = out + (size_t)j * ntot, *hj = hyb_hm + (size_t)j * ntot;
        hyb_kz_kernel<<<P.nd, 256, 0, stream>>>(P, H, d_doff, d_rofs, d_R, outj, inj);
        hyb_m_kernel<<<dim3(H.ncl, hyb_rows), 256, sizeof(double) * H.max_nc, stream>>>(P, H, 0, 0, nullptr);
        hyb_copy_kernel<<<std::max(1, std::min(4096, (ntot + 255) / 256)), 256, 0, stream>>>(inj, hj, ntot);
        hyb_kb0_kernel<<<(P.nd + 127) / 128, 128, 0, stream>>>(P, H, d_doff, hj);
        CUDA_CHECK(cudaMemcpyAsync(hyb_wsave + (size_t)j * wn, H.w, sizeof(double) * wn, cudaMemcpyDeviceToDevice,
                                   stream));
    }
    launch_kplus_multi(hyb_hm, out, ncol, KPLUS_FULL, nullptr);
    for (int j = 0; j < ncol; ++j) {
        HybDev Hj = H;
        Hj.w = hyb_wsave + (size_t)j * wn;
        hyb_kr_kernel<<<P.nd, 256, 0, stream>>>(P, Hj, d_doff, d_rofs, d_R, out + (size_t)j * ntot);
    }
    CUDA_CHECK(cudaGetLastError());
}

void GpuSolver::Impl::launch_kplus_dual(const double *in, double *out) {
    launch_kplus(in, out);
    if (!hybrid) return;
    hyb_kz_kernel<<<P.nd, 256, 0, stream>>>(P, H, d_doff, d_rofs, d_R, out, in);
    hyb_m_kernel<<<dim3(H.ncl, hyb_rows), 256, sizeof(double) * H.max_nc, stream>>>(P, H, 0, 0, nullptr);
    hyb_copy_kernel<<<std::max(1, std::min(4096, (ntot + 255) / 256)), 256, 0, stream>>>(in, d_h, ntot);
    hyb_kb0_kernel<<<(P.nd + 127) / 128, 128, 0, stream>>>(P, H, d_doff, d_h);
    launch_kplus(d_h, out);
    hyb_kr_kernel<<<P.nd, 256, 0, stream>>>(P, H, d_doff, d_rofs, d_R, out);
    CUDA_CHECK(cudaGetLastError());
}

// FP64 Schur tiles already on the device -> FP32 or BF16 (per-tile scale) tiles.
__global__ void __launch_bounds__(256) convert_tiles_kernel(const double *src, void *dst, float *scale, int prec,
                                                            long long ntiles) {
    __shared__ float s_red[8];
    for (long long g = blockIdx.x; g < ntiles; g += gridDim.x) {
        const double *t = src + (size_t)g * TILE * TILE;
        float s = 1.0f;
        if (prec == SCHUR_BF16) {
            double amax = 0.0;
            for (int q = threadIdx.x; q < TILE * TILE; q += 256) amax = fmax(amax, fabs(t[q]));
            float a = (float)amax;
            for (int o = 16; o; o >>= 1) a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
            if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = a;
            __syncthreads();
            a = 0.0f;
            for (int w = 0; w < 8; ++w) a = fmaxf(a, s_red[w]);
            s = a > 0.0f ? a : 1.0f;
            if (threadIdx.x == 0) scale[g] = s;
            __syncthreads();
        }
        for (int q = threadIdx.x; q < TILE * TILE; q += 256) {
            const size_t o = (size_t)g * TILE * TILE + q;
            if (prec == SCHUR_FP32) ((float *)dst)[o] = (float)t[q];
            else ((__nv_bfloat16 *)dst)[o] = __float2bfloat16_rn((float)(t[q] / s));
        }
    }
}

void GpuSolver::Impl::build_tiles(TileSetHost &T, int prec, const std::vector<const double *> &mats,
                                  const std::vector<int> &ns, const std::vector<int> &voffs, int tiles_per_item,
                                  double *dev64) {
    const int nm = (int)mats.size();
    const size_t esz = prec == SCHUR_FP64 ? 8 : prec == SCHUR_FP32 ? 4 : 2;
    const size_t tbytes = (size_t)TILE * TILE * esz;
    std::vector<int> mn(nm), mv(nm), mt(nm);
    std::vector<long long> m0(nm);
    long long total = 0;
    double alg = 0.0;
    for (int m = 0; m < nm; ++m) {
        mn[m] = ns[m];
        mv[m] = voffs[m];
        mt[m] = (ns[m] + TILE - 1) / TILE;
        m0[m] = total;
        total += (long long)mt[m] * (mt[m] + 1) / 2;
        alg += (double)ns[m] * (ns[m] + 1) / 2 * (double)esz + (double)ns[m] * (4 + 8 + 8);
    }
    std::vector<unsigned> ij(total);
    if (dev64) {
        // tiles already on the device (device preprocessing): FP64 taken over, others converted
        for (int m = 0; m < nm; ++m) {
            long long g = m0[m];
            for (int I = 0; I < mt[m]; ++I)
                for (int J = I; J < mt[m]; ++J, ++g) ij[g] = ((unsigned)I << 16) | (unsigned)J;
        }
        T.prec = prec;
        T.bytes = (size_t)total * tbytes;
        T.alg_bytes = alg;
        T.mat_n = upload(mn);
        T.mat_voff = upload(mv);
        T.mat_tn = upload(mt);
        T.mat_tile0 = upload(m0);
        T.tile_ij = upload(ij);
        T.scale = nullptr;
        if (prec == SCHUR_FP64) {
            T.tiles = dev64;
        } else {
            T.tiles = alloc<unsigned char>((size_t)std::max<long long>(total, 1) * tbytes);
            if (prec == SCHUR_BF16) T.scale = alloc<float>((size_t)std::max<long long>(total, 1));
            if (total > 0)
                convert_tiles_kernel<<<(unsigned)std::min<long long>(total, 65535), 256>>>(dev64, T.tiles, T.scale,
                                                                                          prec, total);
            CUDA_CHECK(cudaGetLastError());
        }
        T.h_tn = mt;
        T.total_tiles = total;
        T.items = alloc<int4>((size_t)total);
        T.item_dot = alloc<double>((size_t)total);
        T.queue = alloc<int>(2);
        CUDA_CHECK(cudaMemset(T.queue, 0, 2 * sizeof(int)));
        T.kernel = opt.tile_kernel;
        T.class_tpi.assign(kSizeClasses, tiles_per_item);
        itemize(T, T.class_tpi, -1);
        return;
    }
    std::vector<unsigned char> data((size_t)total * tbytes);
    std::vector<float> sc(prec == SCHUR_BF16 ? total : 0);
    for (int m = 0; m < nm; ++m) {
        const double *S = mats[m];
        const int n = ns[m], tn = mt[m];
        long long g = m0[m];
        for (int I = 0; I < tn; ++I)
            for (int J = I; J < tn; ++J, ++g) {
                ij[g] = ((unsigned)I << 16) | (unsigned)J;
                unsigned char *dst = data.data() + (size_t)g * tbytes;
                double amax = 0.0;
                if (prec == SCHUR_BF16)
                    for (int r = 0; r < TILE; ++r)
                        for (int c = 0; c < TILE; ++c) {
                            int gr = TILE * I + r, gc = TILE * J + c;
                            if (gr < n && gc < n) amax = std::max(amax, std::fabs(S[(size_t)gc * n + gr]));
                        }
                float s = (amax > 0) ? (float)amax : 1.0f;
                if (prec == SCHUR_BF16) sc[g] = s;
                for (int r = 0; r < TILE; ++r)
                    for (int c = 0; c < TILE; ++c) {
                        int gr = TILE * I + r, gc = TILE * J + c;
                        double v = (gr < n && gc < n) ? S[(size_t)gc * n + gr] : 0.0;
                        size_t o = (size_t)r * TILE + c;
                        if (prec == SCHUR_FP64) ((double *)dst)[o] = v;
                        else if (prec == SCHUR_FP32) ((float *)dst)[o] = (float)v;
                        else ((__nv_bfloat16 *)dst)[o] = __float2bfloat16_rn((float)(v / s));
                    }
            }
    }
    T.prec = prec;
    T.bytes = data.size();
    T.alg_bytes = alg;
    T.mat_n = upload(mn);
    T.mat_voff = upload(mv);
    T.mat_tn = upload(mt);
    T.mat_tile0 = upload(m0);
    T.tile_ij = upload(ij);
    T.tiles = upload(data);
    T.scale = prec == SCHUR_BF16 ? upload(sc) : nullptr;
    T.h_tn = mt;
    T.total_tiles = total;
    // item buffers sized for the finest granularity (one tile per item)
    T.items = alloc<int4>((size_t)total);
    T.item_dot = alloc<double>((size_t)total);
    T.queue = alloc<int>(2);
    CUDA_CHECK(cudaMemset(T.queue, 0, 2 * sizeof(int)));
    T.kernel = opt.tile_kernel;
    T.class_tpi.assign(kSizeClasses, tiles_per_item);
    itemize(T, T.class_tpi, -1);
}

// Size class of a matrix with tn tile rows (autotuning granularity).
static int size_class(int tn) { return tn <= 8 ? 0 : tn <= 16 ? 1 : tn <= 32 ? 2 : tn <= 64 ? 3 : 4; }

// Work items: per matrix, pieces of about tpi[class] tiles; largest matrices first.
// only_class >= 0 restricts the list to one size class (autotuning).
void GpuSolver::Impl::itemize(TileSetHost &T, const std::vector<int> &tpi, int only_class) {
    const int nm = (int)T.h_tn.size();
    std::vector<int> order(nm);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return T.h_tn[a] > T.h_tn[b]; });
    std::vector<int4> items;
    for (int m : order) {
        const int cls = size_class(T.h_tn[m]);
        if (only_class >= 0 && cls != only_class) continue;
        const int nt = T.h_tn[m] * (T.h_tn[m] + 1) / 2;
        const int per = std::max(1, tpi[cls]);
        const int pieces = std::max(1, (nt + per - 1) / per);
        for (int k = 0; k < pieces; ++k) {
            int a = (int)((long long)nt * k / pieces), b = (int)((long long)nt * (k + 1) / pieces);
            items.push_back(make_int4(m, a, b, 0));
        }
    }
    T.nitems = (int)items.size();
    if (!items.empty())
        CUDA_CHECK(cudaMemcpy(T.items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
}

// Autotuner: for each kernel variant and size class, time class-only applies over
// candidate item granularities; keep the fastest (variant, per-class granularity).
void GpuSolver::Impl::autotune(TileSetHost &T, double *x, double *y, int ny) {
    const int cands[] = {16, 48, 128, 384, 1 << 20};
    std::vector<int> present(kSizeClasses, 0);
    for (int tn : T.h_tn) present[size_class(tn)] = 1;
    cudaEvent_t a, b;
    CUDA_CHECK(cudaEventCreate(&a));
    CUDA_CHECK(cudaEventCreate(&b));
    auto time_launch = [&](int reps) {
        for (int i = 0; i < 2; ++i) launch_tiles(T, 0, x, nullptr, y, 0);
        CUDA_CHECK(cudaEventRecord(a, stream));
        for (int i = 0; i < reps; ++i) launch_tiles(T, 0, x, nullptr, y, 0);
        CUDA_CHECK(cudaEventRecord(b, stream));
        CUDA_CHECK(cudaEventSynchronize(b));
        float ms = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
        return ms / reps;
    };
    double best_total = 1e30;
    int best_kernel = T.kernel;
    std::vector<int> best_tpi = T.class_tpi;
    for (int kern = 0; kern < 2; ++kern) {
        T.kernel = kern;
        std::vector<int> tpi = T.class_tpi;
        double total = 0.0;
        for (int c = 0; c < kSizeClasses; ++c) {
            if (!present[c]) continue;
            double bt = 1e30;
            for (int cand : cands) {
                std::vector<int> t = tpi;
                t[c] = cand;
                itemize(T, t, c);
                double ms = time_launch(5);
                if (ms < bt) { bt = ms; tpi[c] = cand; }
            }
            total += bt;
        }
        if (total < best_total) { best_total = total; best_kernel = kern; best_tpi = tpi; }
    }
    T.kernel = best_kernel;
    T.class_tpi = best_tpi;
    itemize(T, T.class_tpi, -1);
    CUDA_CHECK(cudaMemsetAsync(y, 0, sizeof(double) * ny, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}

static size_t tile_smem(int prec, int max_tn) {
    size_t acc = prec == SCHUR_FP64 ? 8 : 4;
    return 2 * acc * (size_t)max_tn * TILE;
}

void GpuSolver::Impl::release(void *p) {
    for (size_t i = 0; i < allocs.size(); ++i)
        if (allocs[i] == p) {
            CUDA_CHECK(cudaFree(p));
            bytes -= alloc_sizes[i];
            allocs.erase(allocs.begin() + i);
            alloc_sizes.erase(alloc_sizes.begin() + i);
            return;
        }
}

void GpuSolver::Impl::launch_implicit(int mode, const double *src, const double *src2, double *out, int slot) {
    FETI_CHECK(mode == 0 || mode == 1, "internal: implicit F apply in an unsupported mode");
    const size_t sm = sizeof(double) * TILE * (size_t)max_T;
    if (mode == 0)
        launch_pdl(kplus_dual_kernel<0>, dim3(P.nd), dim3(256), sm, stream, KP, P, (const int *)d_rdof,
                   (const double *)d_rsign, src, src2, out, slot);
    else
        launch_pdl(kplus_dual_kernel<1>, dim3(P.nd), dim3(256), sm, stream, KP, P, (const int *)d_rdof,
                   (const double *)d_rsign, src, src2, out, slot);
    CUDA_CHECK(cudaGetLastError());
}

void GpuSolver::Impl::launch_tiles(const TileSetHost &T, int mode, const double *src, const double *src2, double *out,
                                   int slot) {
    if (implicit && &T == &F64) {
        launch_implicit(mode, src, src2, out, slot);
        return;
    }
    int mtn = (&T == &Dir) ? max_tn_dir : max_tn;
    TileSetDev td = T.dev();
    FETI_CHECK(mode != 1 || src2 != nullptr, "internal: PCG direction update without a previous direction");
    if (T.kernel == 1) {
        const size_t acc = T.prec == SCHUR_FP64 ? 8 : 4;
        const size_t tile_bytes = (size_t)TILE * TILE * (T.prec == SCHUR_FP64 ? 8 : T.prec == SCHUR_FP32 ? 4 : 2);
        const size_t stage = (size_t)TMA_CONSUMERS * tile_bytes;
        const int xs_elems = TILE * mtn;
        const size_t xbytes = 2 * acc * (size_t)xs_elems;
        const size_t budget = 220 * 1024;
        int nst = (int)std::min<size_t>(TMA_MAX_STAGES, (budget - std::min(budget, xbytes)) / stage);
        FETI_CHECK(nst >= 2, "FETI4I: subdomain too large for the TMA tile pipeline");
        const size_t sm = (size_t)nst * stage + xbytes;
        const int grid = std::max(1, std::min(T.nitems, nsm));
#define LAUNCHT(PR, MD)                                                                                 \
    launch_pdl(tile_symv_tma_kernel<PR, MD>, dim3(grid), dim3((TMA_CONSUMERS + 1) * 32), sm, stream, td, P, src, src2, \
               out, slot, nst, xs_elems)
#define LAUNCHT_MODES(PR)                                  \
    switch (mode) {                                        \
    case 0: LAUNCHT(PR, 0); break;                         \
    case 1: LAUNCHT(PR, 1); break;                         \
    case 2: LAUNCHT(PR, 2); break;                         \
    default: LAUNCHT(PR, 3); break;                        \
    }
        if (T.prec == SCHUR_FP64) { LAUNCHT_MODES(SCHUR_FP64) }
        else if (T.prec == SCHUR_FP32) { LAUNCHT_MODES(SCHUR_FP32) }
        else { LAUNCHT_MODES(SCHUR_BF16) }
#undef LAUNCHT_MODES
#undef LAUNCHT
        CUDA_CHECK(cudaGetLastError());
        return;
    }
    size_t sm = tile_smem(T.prec, mtn);
    int grid = std::max(1, std::min(T.nitems, nsm * 2));
#define LAUNCH(PR, MD) launch_pdl(tile_symv_kernel<PR, MD>, dim3(grid), dim3(256), sm, stream, td, P, src, src2, out, slot)
#define LAUNCH_MODES(PR)                                   \
    switch (mode) {                                        \
    case 0: LAUNCH(PR, 0); break;                          \
    case 1: LAUNCH(PR, 1); break;                          \
    case 2: LAUNCH(PR, 2); break;                          \
    default: LAUNCH(PR, 3); break;                         \
    }
    if (T.prec == SCHUR_FP64) { LAUNCH_MODES(SCHUR_FP64) }
    else if (T.prec == SCHUR_FP32) { LAUNCH_MODES(SCHUR_FP32) }
    else { LAUNCH_MODES(SCHUR_BF16) }
#undef LAUNCH_MODES
#undef LAUNCH
    CUDA_CHECK(cudaGetLastError());
}

template <int PR>
static void set_tile_limits(int v) {
    cudaFuncSetAttribute(tile_symv_kernel<PR, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(tile_symv_kernel<PR, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(tile_symv_kernel<PR, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(tile_symv_kernel<PR, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    const int t = 225 * 1024;
    cudaFuncSetAttribute(tile_symv_tma_kernel<PR, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, t);
    cudaFuncSetAttribute(tile_symv_tma_kernel<PR, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, t);
    cudaFuncSetAttribute(tile_symv_tma_kernel<PR, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, t);
    cudaFuncSetAttribute(tile_symv_tma_kernel<PR, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, t);
}

static void set_smem_limits() {
    static bool done = false;
    if (done) return;
    const int v = 200 * 1024;
    set_tile_limits<SCHUR_FP64>(v);
    set_tile_limits<SCHUR_FP32>(v);
    set_tile_limits<SCHUR_BF16>(v);
    cudaFuncSetAttribute(w_prec_kernel<PREC_NONE>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(w_prec_kernel<PREC_LUMPED>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(w_prec_kernel<PREC_WEIGHT>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(w_prec_kernel<PREC_DIRICHLET>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(r0_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    cudaFuncSetAttribute(update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    done = true;
}

// One PCG iteration (reference order: w = P r, z = M w, y = P z, p, F p, update).
void GpuSolver::Impl::launch_replacement(int slot) {
    const int nd = P.nd;
    launch_tiles(F64, 3, P.x, nullptr, Ax64, slot);
    launch_hybrid_F(P.x, Ax64, slot, 3, nullptr);
    launch_pdl(r0_kernel, dim3(nd), dim3(tpbv), sizeof(double) * max_ni, stream, P, Ax64, 1, slot);
}

void GpuSolver::Impl::launch_iteration(int slot, bool with_replacement, LoopCtl lc) {
    const int nd = P.nd;
    const int cgrid = (P.nK + 7) / 8;
    const bool mixed = opt.schur_precision != SCHUR_FP64;
    const TileSetHost &Fop = mixed ? Flow : F64;
    if (mixed && with_replacement) {
        // residual replacement r = b - F64 x when the previous update asked for it
        launch_tiles(F64, 3, P.x, nullptr, Ax64, slot);
        launch_hybrid_F(P.x, Ax64, slot, 3, nullptr);
        launch_pdl(r0_kernel, dim3(nd), dim3(tpbv), sizeof(double) * max_ni, stream, P, Ax64, 1, slot);
    }
    launch_pdl(coarse_kernel, dim3(cgrid), dim3(256), 0, stream, P, P.d, P.alpha, slot, 1);
    const size_t tsm = sizeof(double) * (size_t)(max_ni + max_nt);
    switch (opt.precond) {
    case PREC_NONE: launch_pdl(w_prec_kernel<PREC_NONE>, dim3(nd), dim3(TPB1), tsm, stream, P, slot); break;
    case PREC_LUMPED: launch_pdl(w_prec_kernel<PREC_LUMPED>, dim3(nd), dim3(TPB1), tsm, stream, P, slot); break;
    case PREC_WEIGHT: launch_pdl(w_prec_kernel<PREC_WEIGHT>, dim3(nd), dim3(TPB1), tsm, stream, P, slot); break;
    default: launch_pdl(w_prec_kernel<PREC_DIRICHLET>, dim3(nd), dim3(TPB1), tsm, stream, P, slot); break;
    }
    if (opt.precond != PREC_NONE) {
        if (opt.precond == PREC_DIRICHLET) {
            launch_pdl(zero_vT_kernel, dim3(std::max(1, std::min(1024, (P.NT + 255) / 256))), dim3(256), 0, stream, P,
                       slot);
            launch_tiles(Dir, 2, P.uT, nullptr, P.vT, slot);
        }
        launch_pdl(z_kernel, dim3(nd), dim3(tpbv), sizeof(double) * max_ni, stream, P, slot);
        launch_pdl(coarse_kernel, dim3(cgrid), dim3(256), 0, stream, P, P.d, P.alpha, slot, 1);
        launch_pdl(y_kernel, dim3(nd), dim3(tpbv), 0, stream, P, Ax64, slot);
    } else {
        launch_pdl(zero2_kernel, dim3((P.NL + 255) / 256), dim3(256), 0, stream, P.Ap, Ax64, P.NL);
    }
    launch_tiles(Fop, 1, P.y, P.p, P.Ap, slot);
    launch_hybrid_F(nullptr, P.Ap, slot, 1, P.scal + SC_PAP);   // p = y + beta p formed on the fly
    launch_pdl(update_kernel, dim3(nd), dim3(tpbv), sizeof(double) * max_ni, stream, P, slot);
    (void)lc;
}

int GpuSolver::Impl::kernels_per_iteration() const {
    const bool mixed = opt.schur_precision != SCHUR_FP64;
    int k = 3;  // coarse, w/prec, update
    k += 1;     // F apply
    if (mixed) k += 2;
    if (opt.precond != PREC_NONE) k += 3 + (opt.precond == PREC_DIRICHLET ? 2 : 0);
    else k += 1;
    if (hybrid) k += mixed ? 6 : 3;
    return k;
}

void GpuSolver::Impl::capture_chunk(int chunk) {
    if (graph && graph_chunk == chunk && graph_prec == opt.schur_precision && graph_precond == opt.precond) return;
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    cudaGraph_t g;
    CUDA_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    for (int j = 0; j < chunk; ++j) launch_iteration(j);
    launch_pdl(chunk_end_kernel, dim3(1), dim3(32), 0, stream, P, chunk);
    CUDA_CHECK(cudaStreamEndCapture(stream, &g));
    CUDA_CHECK(cudaGraphInstantiate(&graph, g, 0));
    cudaGraphDestroy(g);
    graph_chunk = chunk;
    graph_prec = opt.schur_precision;
    graph_precond = opt.precond;
}

// The whole dual PCG as one graph: a WHILE node around one iteration (its slot 0, iter_base advanced
// by one per pass) and, in mixed precision, an IF node at its top for the residual replacement.
// update_kernel sets the IF condition and loop_end_kernel the WHILE condition, so the loop stops at
// the converged iteration and no replacement kernels are launched in the iterations that do not
// replace.  Returns false when the runtime refuses conditional nodes (graph chunks are used then).
bool GpuSolver::Impl::capture_loop() {
    const int key = opt.schur_precision * 16 + opt.precond;
    if (graph_loop && graph_loop_key == key) return true;
    if (graph_loop) { cudaGraphExecDestroy(graph_loop); graph_loop = nullptr; }
    if (pdl_enabled() || loop_refused || !loop_graph_enabled()) return false;
    const bool mixed = opt.schur_precision != SCHUR_FP64;
    cudaGraph_t g = nullptr, tmp = nullptr;
    LoopCtl lc{1, 0, 0};
    auto fail = [&](cudaError_t e) {
        FETI_LOG(1, "FETI4I: conditional graph nodes unavailable (%s); using graph chunks\n", cudaGetErrorString(e));
        cudaStreamCaptureStatus cs;
        if (cudaStreamIsCapturing(stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
            cudaStreamEndCapture(stream, &tmp);
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        loop_refused = true;
        return false;
    };
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaGraphConditionalHandleCreate(&lc.h_loop, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return fail(e);
    if ((e = cudaGraphConditionalHandleCreate(&lc.h_repl, g, 0, cudaGraphCondAssignDefault)) != cudaSuccess) return fail(e);
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = lc.h_loop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    if ((e = cudaGraphAddNode(&wnode, g, nullptr, 0, &wp)) != cudaSuccess) return fail(e);
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    cudaGraphNode_t top = nullptr;
    if (mixed) {
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = lc.h_repl;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        if ((e = cudaGraphAddNode(&top, body, nullptr, 0, &ip)) != cudaSuccess) return fail(e);
        if ((e = cudaStreamBeginCaptureToGraph(stream, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return fail(e);
        launch_replacement(0);
        if ((e = cudaStreamEndCapture(stream, &tmp)) != cudaSuccess) return fail(e);
    }
    if ((e = cudaStreamBeginCaptureToGraph(stream, body, top ? &top : nullptr, nullptr, top ? 1 : 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return fail(e);
    launch_iteration(0, false, lc);
    loop_end_kernel<<<1, 32, 0, stream>>>(P, lc);
    if ((e = cudaStreamEndCapture(stream, &tmp)) != cudaSuccess) return fail(e);
    if ((e = cudaGraphInstantiate(&graph_loop, g, 0)) != cudaSuccess) return fail(e);
    cudaGraphDestroy(g);
    graph_loop_key = key;
    return true;
}

GpuSolver::GpuSolver() : impl(new Impl) {}
GpuSolver::~GpuSolver() { delete impl; }
size_t GpuSolver::device_bytes() const { return impl->bytes; }
double GpuSolver::kplus_tile_fraction() const {
    return impl->kplus_tiles_total ? (double)impl->kplus_tiles_kept / (double)impl->kplus_tiles_total : 0.0;
}
int GpuSolver::device_id() const { return impl->device; }
void GpuSolver::set_options(const SolveOptions &opt) {
    FETI_CHECK(opt.schur_explicit == impl->opt.schur_explicit,
               "FETI4I: explicit or implicit F apply is fixed at instance creation");
    FETI_CHECK(opt.schur_precision == SCHUR_FP64 || impl->Flow.prec == opt.schur_precision,
               "FETI4I: the requested Schur precision was not prepared on the device");
    FETI_CHECK(opt.precond == impl->opt.precond, "FETI4I: the preconditioner is fixed at instance creation");
    int tpi = impl->opt.tiles_per_item;
    impl->opt = opt;
    impl->opt.tiles_per_item = tpi;
}

bool cuda_available(std::string &why) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        why = (e != cudaSuccess) ? cudaGetErrorString(e) : "no CUDA device";
        return false;
    }
    return true;
}

void GpuSolver::upload(const Decomposition &dec, const Prep &prep, const SolveOptions &opt) {
    const double tu0 = now_s();
    Impl &I = *impl;
    I.opt = opt;
    std::string why;
    FETI_CHECK(cuda_available(why), "FETI4I: no usable CUDA device (" + why + "); the dual solver runs on the GPU only");
    CUDA_CHECK(cudaGetDevice(&I.device));
    cudaDeviceProp prop;
    CUDA_CHECK(cudaGetDeviceProperties(&prop, I.device));
    FETI_CHECK(prop.major == 10, "FETI4I: this build targets sm_100a (B200); found compute capability " +
                                     std::to_string(prop.major) + "." + std::to_string(prop.minor));
    I.nsm = prop.multiProcessorCount;
    CUDA_CHECK(cudaStreamCreateWithFlags(&I.stream, cudaStreamNonBlocking));
    CUDA_CHECK(cudaEventCreate(&I.ev0));
    CUDA_CHECK(cudaEventCreate(&I.ev1));
    set_smem_limits();

    const int nd = dec.ndom;
    // kof: partial G-product blocks (one per subdomain, dual kernel columns of the subdomain)
    std::vector<int> loff(nd + 1, 0), kof(nd + 1, 0), toff(nd + 1, 0), akof(nd, 0);
    for (int d = 0; d < nd; ++d) {
        loff[d + 1] = loff[d] + prep.sub[d].ni;
        kof[d + 1] = kof[d] + prep.sub[d].dnk;
        akof[d] = prep.kofs[d];
        toff[d + 1] = toff[d] + prep.sub[d].t;
        FETI_CHECK(prep.sub[d].nk <= KMAX && prep.sub[d].dnk <= KMAX, "FETI4I: kernel dimension above the supported bound");
    }
    const int NL = loff[nd], NT = toff[nd];
    I.n_lambda = dec.n_lambda;
    I.h_loff = loff;
    {
        const int per_sm = std::max(1, (nd + I.nsm - 1) / I.nsm);
        I.tpbv = std::max(128, std::min(1024, (2048 / per_sm) / 32 * 32));
    }
    I.h_lam.resize(NL);
    int KS = 1;
    for (int d = 0; d < nd; ++d) KS = std::max(KS, prep.sub[d].dnk);
    std::vector<int> partner(NL, -1), tidx(NL), rkof(NL), rnk(NL);
    std::vector<double> ws(NL), minv(NL), Gl((size_t)NL * KS, 0.0);
    I.max_ni = 0;
    for (int d = 0; d < nd; ++d) {
        const DomainRows &D = dec.dom[d];
        const SubPrep &S = prep.sub[d];
        I.max_ni = std::max(I.max_ni, S.ni);
        for (int r = 0; r < S.ni; ++r) {
            int e = loff[d] + r;
            int l = D.lam[r];
            I.h_lam[e] = l;
            int d0 = prep.own_dom[2 * (size_t)l], d1 = prep.own_dom[2 * (size_t)l + 1];
            int r0 = prep.own_row[2 * (size_t)l], r1 = prep.own_row[2 * (size_t)l + 1];
            if (d1 >= 0) partner[e] = (d0 == d && r0 == r) ? loff[d1] + r1 : loff[d0] + r0;
            tidx[e] = toff[d] + S.trow[r];
            ws[e] = D.w[r] * D.sign[r];
            minv[e] = d1 >= 0 ? 0.5 : 1.0;
            rkof[e] = akof[d];
            rnk[e] = S.dnk;
            for (int k = 0; k < S.dnk; ++k) Gl[(size_t)e * KS + k] = S.Gd[(size_t)k * S.ni + r];
        }
    }
    I.d_lam = I.upload(I.h_lam);
    // partner data of every row (shortens the dependent-load chains of the assembly)
    std::vector<int> ptidx(NL, -1), pkof(NL, 0), pnk(NL, 0);
    std::vector<double> pws(NL, 0.0), Gp((size_t)NL * KS, 0.0);
    for (int e = 0; e < NL; ++e) {
        int q = partner[e];
        if (q < 0) continue;
        ptidx[e] = tidx[q];
        pws[e] = ws[q];
        pkof[e] = rkof[q];
        pnk[e] = rnk[q];
        for (int k = 0; k < KS; ++k) Gp[(size_t)e * KS + k] = Gl[(size_t)q * KS + k];
    }
    // T space: rows of each touched DOF
    std::vector<int> trow_ptr(NT + 1, 0), trow_idx(NL);
    for (int e = 0; e < NL; ++e) trow_ptr[tidx[e] + 1]++;
    for (int t = 0; t < NT; ++t) trow_ptr[t + 1] += trow_ptr[t];
    {
        std::vector<int> fill(trow_ptr.begin(), trow_ptr.end() - 1);
        for (int e = 0; e < NL; ++e) trow_idx[fill[tidx[e]]++] = e;
    }
    // lumped preconditioner: K_TT of each subdomain in sliced ELL (32 rows, column-major)
    std::vector<int> slice0(nd + 1, 0), ell_ptr, ell_w;
    std::vector<unsigned short> ell_col;
    std::vector<double> ell_val;
    I.max_nt = 0;
    for (int d = 0; d < nd; ++d) {
        const SubPrep &S = prep.sub[d];
        I.max_nt = std::max(I.max_nt, S.t);
        slice0[d + 1] = slice0[d];
        if (opt.precond != PREC_LUMPED) continue;
        FETI_CHECK(S.t < 65536, "FETI4I: too many interface DOFs in one subdomain for the lumped kernel");
        for (int t0 = 0; t0 < S.t; t0 += 32) {
            int w = 0;
            for (int t = t0; t < std::min(S.t, t0 + 32); ++t) w = std::max(w, S.KT_ptr[t + 1] - S.KT_ptr[t]);
            ell_ptr.push_back((int)ell_val.size());
            ell_w.push_back(w);
            size_t base = ell_val.size();
            ell_val.resize(base + (size_t)32 * w, 0.0);
            ell_col.resize(base + (size_t)32 * w, 0);
            for (int t = t0; t < std::min(S.t, t0 + 32); ++t)
                for (int j = S.KT_ptr[t]; j < S.KT_ptr[t + 1]; ++j) {
                    size_t o = base + (size_t)(j - S.KT_ptr[t]) * 32 + (t - t0);
                    ell_val[o] = S.KT_val[j];
                    ell_col[o] = (unsigned short)S.KT_col[j];
                }
            slice0[d + 1]++;
        }
    }
    std::vector<int> tbase(NT), tslot(NT);
    for (int d = 0; d < nd; ++d)
        for (int t = toff[d]; t < toff[d + 1]; ++t) {
            tbase[t] = toff[d];
            tslot[t] = ((slice0[d] + ((t - toff[d]) >> 5)) << 5) | ((t - toff[d]) & 31);
        }
    FETI_CHECK(sizeof(double) * (size_t)(I.max_nt + I.max_ni) <= 200 * 1024,
               "FETI4I: subdomain interface too large for the preconditioner kernel");

    DevProblem &P = I.P;
    P.nd = nd; P.NL = NL; P.nK = prep.n_kern; P.NT = NT; P.KS = KS; P.nP = kof[nd];
    P.loff = I.upload(loff); P.kof = I.upload(kof); P.toff = I.upload(toff); P.akof = I.upload(akof);
    P.partner = I.upload(partner); P.tidx = I.upload(tidx); P.ptidx = I.upload(ptidx);
    P.ws = I.upload(ws); P.pws = I.upload(pws); P.minv = I.upload(minv);
    P.Gl = I.upload(Gl); P.Gp = I.upload(Gp);
    P.rkof = I.upload(rkof); P.rnk = I.upload(rnk); P.pkof = I.upload(pkof); P.pnk = I.upload(pnk);
    P.trow_ptr = I.upload(trow_ptr); P.trow_idx = I.upload(trow_idx);
    P.slice0 = I.upload(slice0); P.ell_ptr = I.upload(ell_ptr); P.ell_w = I.upload(ell_w);
    P.ell_col = I.upload(ell_col); P.ell_val = I.upload(ell_val);
    P.tbase = I.upload(tbase); P.tslot = I.upload(tslot);
    P.scal = I.alloc<double>(SC_COUNT);
    P.done = I.alloc<int>(DONE_COUNT);
    CUDA_CHECK(cudaMemset(P.done, 0, sizeof(int) * DONE_COUNT));
    {
        // (GG^T)^-1 times the sum over the partial blocks: column b of partial block d, kernel k
        // is column akof[d] + k of (GG^T)^-1
        // ((GG^T)^-1 is symmetric: row r of it is read contiguously)
        const int nK = prep.n_kern, nP = kof[nd];
        std::vector<double> Gx((size_t)nK * nP);
        std::vector<int> bcol(nP);
        I.dual_to_partial.assign(nK, -1);
        for (int d = 0; d < nd; ++d)
            for (int k = 0; k < prep.sub[d].dnk; ++k) {
                const int b = kof[d] + k, col = akof[d] + k;
                bcol[b] = col;
                if (I.dual_to_partial[col] < 0) I.dual_to_partial[col] = b;
            }
#pragma omp parallel for schedule(static)
        for (int r = 0; r < nK; ++r) {
            const double *src = prep.GGt_inv.data() + (size_t)r * nK;
            double *dst = Gx.data() + (size_t)r * nP;
            for (int b = 0; b < nP; ++b) dst[b] = src[bcol[b]];
        }
        P.GGtinv = I.upload(Gx);
    }
    P.bL = I.alloc<double>(NL);
    P.x = I.alloc<double>(NL); P.r = I.alloc<double>(NL); P.w = I.alloc<double>(NL); P.z = I.alloc<double>(NL);
    P.y = I.alloc<double>(NL); P.p = I.alloc<double>(NL); P.Ap = I.alloc<double>(NL);
    I.Ax64 = I.alloc<double>(NL);
    P.uT = I.alloc<double>(NT); P.vT = I.alloc<double>(NT);
    P.d = I.alloc<double>(P.nP);
    P.alpha = I.alloc<double>(prep.n_kern + KS);
    CUDA_CHECK(cudaMemset(P.alpha, 0, sizeof(double) * (prep.n_kern + KS)));
    I.e_dev = I.alloc<double>(P.nP);
    P.part_w = I.alloc<double>(2 * nd); P.part_rho = I.alloc<double>(nd); P.part_b = I.alloc<double>(nd);
    P.rho_hist = I.alloc<double>((size_t)opt.max_iterations + 64);
    I.st = I.alloc<DevState>(1);
    P.st = I.st;
    CUDA_CHECK(cudaMemset(P.Ap, 0, sizeof(double) * NL));
    CUDA_CHECK(cudaMemset(I.Ax64, 0, sizeof(double) * NL));
    CUDA_CHECK(cudaMemset(P.p, 0, sizeof(double) * NL));
    I.rho_cap = opt.max_iterations + 64;

    const double tu1 = now_s();
    // Schur tiles: FP64 always (true residuals, FP64 path), low precision on request
    std::vector<const double *> mats(nd);
    std::vector<int> ns(nd), voffs(nd);
    I.max_tn = 0;
    for (int d = 0; d < nd; ++d) {
        mats[d] = prep.sub[d].S.data();
        ns[d] = prep.sub[d].ni;
        voffs[d] = loff[d];
        I.max_tn = std::max(I.max_tn, (ns[d] + TILE - 1) / TILE);
    }
    FETI_CHECK(tile_smem(SCHUR_FP64, I.max_tn) <= 200 * 1024, "FETI4I: a Schur complement is too large for the tile kernel");
    DevPrepStore *ds = prep.dstore.get();
    FETI_CHECK(!ds || (ds->nd == nd && ds->s_tiles && ds->kp_tiles), "FETI4I: device preprocessing store missing");
    I.implicit = !opt.schur_explicit;
    if (I.implicit) {
        // F through the K^+ factor: no S_i tiles on the device (those of the device preprocessing are freed)
        FETI_CHECK(prep.method == 0, "FETI4I: the implicit F apply (no explicit Schur complements) is Total FETI only");
        FETI_CHECK(opt.schur_precision == SCHUR_FP64,
                   "FETI4I: the implicit F apply runs in FP64 (the Schur precision applies to explicit S_i)");
        if (ds && ds->s_tiles) {
            CUDA_CHECK(cudaFree(ds->s_tiles));
            ds->s_tiles = nullptr;
        }
        I.F64.prec = SCHUR_FP64;
    } else {
        double *s64 = ds ? I.adopt(ds->s_tiles, (size_t)ds->s_tile0[nd] * TILE * TILE) : nullptr;
        I.build_tiles(I.F64, SCHUR_FP64, mats, ns, voffs, opt.tiles_per_item, s64);
        if (opt.schur_precision != SCHUR_FP64)
            I.build_tiles(I.Flow, opt.schur_precision, mats, ns, voffs, opt.tiles_per_item, s64);
    }
    if (opt.precond == PREC_DIRICHLET) {
        std::vector<const double *> dm(nd);
        std::vector<int> dn(nd), dv(nd);
        I.max_tn_dir = 0;
        for (int d = 0; d < nd; ++d) {
            dm[d] = prep.sub[d].Sdir.data();
            dn[d] = prep.sub[d].t;
            dv[d] = toff[d];
            I.max_tn_dir = std::max(I.max_tn_dir, (dn[d] + TILE - 1) / TILE);
        }
        FETI_CHECK(tile_smem(SCHUR_FP64, I.max_tn_dir) <= 200 * 1024, "FETI4I: a Dirichlet block is too large for the tile kernel");
        FETI_CHECK(!ds || ds->dir_tiles, "FETI4I: device preprocessing store has no Dirichlet blocks");
        double *d64 = ds ? I.adopt(ds->dir_tiles, (size_t)ds->dir_tile0[nd] * TILE * TILE) : nullptr;
        I.build_tiles(I.Dir, SCHUR_FP64, dm, dn, dv, opt.tiles_per_item, d64);
    }
    if (opt.autotune) {
        CUDA_CHECK(cudaMemset(P.w, 0, sizeof(double) * NL));
        if (!I.implicit) I.autotune(I.F64, P.w, I.Ax64, NL);
        if (opt.schur_precision != SCHUR_FP64) I.autotune(I.Flow, P.w, I.Ax64, NL);
        if (opt.precond == PREC_DIRICHLET) {
            CUDA_CHECK(cudaMemset(P.uT, 0, sizeof(double) * NT));
            I.autotune(I.Dir, P.uT, P.vT, NT);
        }
    }
    const double tu2 = now_s();
    I.upload_kplus(dec, prep, loff, toff);
    I.upload_hybrid(dec, prep);
    if (I.implicit) {
        // algorithmic bytes of one implicit apply: the touched factor tiles that are not all zero, read by the
        // forward and the backward pass, plus the vectors (index, sign, x in, y out per local multiplier)
        I.F64.alg_bytes = 2.0 * (double)I.implicit_tiles * TILE * TILE * sizeof(double) + (double)NL * (4 + 8 + 8 + 8);
    }
    CUDA_CHECK(cudaDeviceSynchronize());
    FETI_LOG(2, "FETI4I: upload: dual layout %.3f s, tiles and autotuning %.3f s, K+ and clusters %.3f s\n",
             tu1 - tu0, tu2 - tu1, now_s() - tu2);
}

std::string GpuSolver::tuning() const {
    auto one = [](const char *name, const TileSetHost &T) {
        std::string s = std::string(name) + ":" + (T.kernel ? "tma" : "ldg") + "[";
        for (size_t c = 0; c < T.class_tpi.size(); ++c) s += (c ? "," : "") + std::to_string(T.class_tpi[c]);
        return s + "]";
    };
    std::string s = one("f64", impl->F64);
    if (impl->Flow.prec >= 0) s += " " + one("low", impl->Flow);
    if (impl->Dir.prec >= 0) s += " " + one("dir", impl->Dir);
    return s;
}

// ---- caller arrays <-> device through the pinned staging buffer
// The arrays move in chunks of at least 1 MB: all host threads copy chunk k between the caller's
// (pageable) memory and the staging buffer while the copy engine moves chunk k - 1.
namespace {
constexpr size_t STAGE_MIN = (size_t)1 << 17;   // doubles per chunk, at least
constexpr int STAGE_EVENTS = 128;

void par_copy(double *dst, const double *src, size_t n) {
    const int nt = omp_get_max_threads();
    if (n < ((size_t)1 << 15) || nt <= 1) {
        std::memcpy(dst, src, n * sizeof(double));
        return;
    }
    const size_t per = (n + nt - 1) / nt;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int t = 0; t < nt; ++t) {
        const size_t b = (size_t)t * per;
        if (b < n) std::memcpy(dst + b, src + b, std::min(per, n - b) * sizeof(double));
    }
}
}  // namespace

void GpuSolver::Impl::ensure_pinned(size_t n) {
    n = std::max<size_t>(n, 1);
    if (h_pinned_n >= n) return;
    CUDA_CHECK(cudaStreamSynchronize(stream));   // no copy of the old buffer in flight
    if (h_pinned) CUDA_CHECK(cudaFreeHost(h_pinned));
    h_pinned = nullptr;
    h_pinned_n = 0;
    CUDA_CHECK(cudaMallocHost(&h_pinned, n * sizeof(double)));
    h_pinned_n = n;
}

// columns j < ncols: dev[j * dev_pitch + i] = host[j * host_pitch + i], i < count (enqueued on the
// stream; the caller's memory is free again on return)
void GpuSolver::Impl::h2d_columns(double *dev, size_t dev_pitch, const double *host, size_t host_pitch, size_t count,
                                  int ncols) {
    if (count == 0 || ncols <= 0) return;
    ensure_pinned(count * ncols);
    const size_t chunk = std::max(STAGE_MIN, count * ncols / STAGE_EVENTS + 1);
    for (int j = 0; j < ncols; ++j)
        for (size_t c0 = 0; c0 < count; c0 += chunk) {
            const size_t len = std::min(chunk, count - c0);
            double *stg = h_pinned + (size_t)j * count + c0;
            par_copy(stg, host + (size_t)j * host_pitch + c0, len);
            CUDA_CHECK(cudaMemcpyAsync(dev + (size_t)j * dev_pitch + c0, stg, len * sizeof(double),
                                       cudaMemcpyHostToDevice, stream));
        }
}

// columns j < ncols: host[j * host_pitch + i] = dev[j * dev_pitch + i], i < count (after the work
// enqueued before it; returns when the caller's memory holds the result)
void GpuSolver::Impl::d2h_columns(double *host, size_t host_pitch, const double *dev, size_t dev_pitch, size_t count,
                                  int ncols) {
    if (count == 0 || ncols <= 0) {
        CUDA_CHECK(cudaStreamSynchronize(stream));
        return;
    }
    ensure_pinned(count * ncols);
    const size_t chunk = std::max(STAGE_MIN, count * ncols / STAGE_EVENTS + 1);
    struct Piece { size_t stg, host, dev, len; };
    std::vector<Piece> pieces;
    for (int j = 0; j < ncols; ++j)
        for (size_t c0 = 0; c0 < count; c0 += chunk)
            pieces.push_back({(size_t)j * count + c0, (size_t)j * host_pitch + c0, (size_t)j * dev_pitch + c0,
                              std::min(chunk, count - c0)});
    while (stage_ev.size() < pieces.size()) {
        cudaEvent_t e;
        CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        stage_ev.push_back(e);
    }
    for (size_t k = 0; k < pieces.size(); ++k) {
        CUDA_CHECK(cudaMemcpyAsync(h_pinned + pieces[k].stg, dev + pieces[k].dev, pieces[k].len * sizeof(double),
                                   cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaEventRecord(stage_ev[k], stream));
    }
    for (size_t k = 0; k < pieces.size(); ++k) {
        CUDA_CHECK(cudaEventSynchronize(stage_ev[k]));
        par_copy(host + pieces[k].host, h_pinned + pieces[k].stg, pieces[k].len);
    }
}

void GpuSolver::solve_full(const double *rhs, int rhs_size, double *solution, int solution_size, SolveStats &stats,
                           bool upload_rhs) {
    Impl &I = *impl;
    DevProblem &P = I.P;
    const int nd = P.nd;
    if (upload_rhs) {
        CUDA_CHECK(cudaMemsetAsync(I.d_rhs, 0, sizeof(double) * std::max(1, I.n_caller), I.stream));
        const int ncp = std::min(rhs_size, I.n_caller);
        I.h2d_columns(I.d_rhs, 0, rhs, 0, (size_t)std::max(0, ncp), 1);
        split_rhs_kernel<<<(I.ntot + 255) / 256, 256, 0, I.stream>>>(I.d_rhs, I.d_gdof, I.d_invm, I.d_f, I.ntot);
        // Total FETI: b needs K^+ f at the touched DOFs only; the forward pass L^-1 f is kept for
        // the primal recovery
        if (I.hybrid) I.launch_kplus_dual(I.d_f, I.d_kf);
        else I.launch_kplus(I.d_f, I.d_kf, KPLUS_TOUCHED);
        evec_kernel<<<nd, TPB, 0, I.stream>>>(P, I.d_doff, I.d_rdofs, I.d_Rd, I.d_f, I.e_dev);
        bvec_kernel<<<(P.NL + 255) / 256, 256, 0, I.stream>>>(P, I.d_rdof, I.d_rsign, I.d_rc, I.d_kf, (double *)P.bL);
        CUDA_CHECK(cudaGetLastError());
    }
    solve(stats);
    // primal: u = K^+ (f - B^T lambda) + R alpha, averaged into the caller's DOFs; Total FETI
    // forms L^-1 (f - B^T lambda) from the kept L^-1 f and a forward pass over the touched blocks
    primal_rhs_kernel<<<std::max(1, std::min(4096, (I.ntot + 255) / 256)), 256, 0, I.stream>>>(
        P, I.d_tdof_g, I.d_rsign, I.hybrid ? I.d_f : nullptr, I.d_g, I.ntot);
    primal_bt_kernel<<<(P.NT + 255) / 256, 256, 0, I.stream>>>(P, I.d_tdof_g, I.d_rsign, I.d_g);
    if (I.hybrid) I.launch_kplus_dual(I.d_g, I.d_kf);
    else I.launch_kplus(I.d_g, I.d_kf, KPLUS_PRIMAL);
    CUDA_CHECK(cudaMemsetAsync(I.d_sol, 0, sizeof(double) * std::max(1, I.n_caller), I.stream));
    primal_merge_kernel<<<nd, TPB, 0, I.stream>>>(P, I.d_doff, I.d_rdofs, I.d_Rd, I.d_kf, I.d_gdof, I.d_invm, I.d_sol);
    CUDA_CHECK(cudaGetLastError());
    const int ncp = std::min(solution_size, I.n_caller);
    I.d2h_columns(solution, 0, I.d_sol, 0, (size_t)std::max(0, ncp), 1);
    for (int i = std::max(0, ncp); i < solution_size; ++i) solution[i] = 0.0;
    stats.kernel_launches += 10;
}

void GpuSolver::set_rhs(const std::vector<double> &b, const std::vector<double> &e) {
    Impl &I = *impl;
    std::vector<double> bL(I.h_lam.size());
    for (size_t i = 0; i < bL.size(); ++i) bL[i] = b[I.h_lam[i]];
    CUDA_CHECK(cudaMemcpyAsync((void *)I.P.bL, bL.data(), bL.size() * sizeof(double), cudaMemcpyHostToDevice, I.stream));
    std::vector<double> ep(I.P.nP, 0.0);
    for (size_t k = 0; k < e.size() && k < I.dual_to_partial.size(); ++k) ep[I.dual_to_partial[k]] = e[k];
    CUDA_CHECK(cudaMemcpyAsync(I.e_dev, ep.data(), ep.size() * sizeof(double), cudaMemcpyHostToDevice, I.stream));
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
}

void GpuSolver::solve(SolveStats &stats) {
    Impl &I = *impl;
    DevProblem &P = I.P;
    FETI_CHECK(I.opt.max_iterations + 64 <= I.rho_cap, "FETI4I: max_iterations grew after instance creation");
    const bool mixed = I.opt.schur_precision != SCHUR_FP64;
    DevState h{};
    h.conv_iter = -1;
    h.iter_base = 0;
    h.replace_iter = -1;
    h.true_iter = 0;
    h.replacements = 0;
    h.max_it = I.opt.max_iterations;
    h.mixed = mixed ? 1 : 0;
    h.error = 0;
    h.precision = I.opt.precision;
    h.delta = I.opt.reliable_delta;
    const int nd = P.nd;
    const int cgrid = (P.nK + 7) / 8;
    CUDA_CHECK(cudaEventRecord(I.ev0, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(I.st, &h, sizeof(h), cudaMemcpyHostToDevice, I.stream));
    // lambda_0 = G^T (GG^T)^-1 e ; r_0 = b - F lambda_0 ; tol = precision * min(|P r_0|, |b|)
    coarse_kernel<<<cgrid, 256, 0, I.stream>>>(P, I.e_dev, P.alpha, 0, 0);
    gt_kernel<<<(P.NL + 255) / 256, 256, 0, I.stream>>>(P, P.alpha, P.x);
    zero_kernel<<<(P.NL + 255) / 256, 256, 0, I.stream>>>(P.p, P.NL);
    I.launch_tiles(I.F64, 0, P.x, nullptr, I.Ax64, 0);
    I.launch_hybrid_F(P.x, I.Ax64, 0, 0, nullptr);
    r0_kernel<<<nd, TPB, sizeof(double) * I.max_ni, I.stream>>>(P, I.Ax64, 0, 0);
    zero_kernel<<<(P.NL + 255) / 256, 256, 0, I.stream>>>(I.Ax64, P.NL);
    coarse_kernel<<<cgrid, 256, 0, I.stream>>>(P, P.d, P.alpha, 0, 0);
    pnorm_kernel<<<nd, TPB, 0, I.stream>>>(P);
    tol_kernel<<<1, 256, 0, I.stream>>>(P);
    CUDA_CHECK(cudaGetLastError());
    int launches = 9;
    const int chunk = std::max(1, I.opt.chunk);
    const bool loop = I.opt.use_graph && I.capture_loop();
    if (I.opt.use_graph && !loop) I.capture_chunk(chunk);
    DevState hs{};
    if (loop) {
        CUDA_CHECK(cudaGraphLaunch(I.graph_loop, I.stream));
        CUDA_CHECK(cudaMemcpyAsync(&hs, I.st, sizeof(hs), cudaMemcpyDeviceToHost, I.stream));
        CUDA_CHECK(cudaStreamSynchronize(I.stream));
        const int its = std::max(1, hs.conv_iter >= 0 ? hs.conv_iter + 1 : std::min(hs.iter_base, I.opt.max_iterations));
        launches += its * (I.kernels_per_iteration() + 1) - (mixed ? 2 * (its - hs.replacements) : 0);
    }
    for (int done = 0; !loop && done < I.opt.max_iterations; done += chunk) {
        if (I.opt.use_graph) {
            CUDA_CHECK(cudaGraphLaunch(I.graph, I.stream));
        } else {
            for (int j = 0; j < chunk; ++j) I.launch_iteration(j);
            chunk_end_kernel<<<1, 32, 0, I.stream>>>(P, chunk);
        }
        launches += chunk * I.kernels_per_iteration() + 1;
        CUDA_CHECK(cudaMemcpyAsync(&hs, I.st, sizeof(hs), cudaMemcpyDeviceToHost, I.stream));
        CUDA_CHECK(cudaStreamSynchronize(I.stream));
        if (hs.conv_iter >= 0) break;
    }
    // amplitudes alpha = (GG^T)^-1 G r (d holds G r of the last update)
    coarse_kernel<<<cgrid, 256, 0, I.stream>>>(P, P.d, P.alpha, 0, 0);
    launches += 1;
    CUDA_CHECK(cudaEventRecord(I.ev1, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(&hs, I.st, sizeof(hs), cudaMemcpyDeviceToHost, I.stream));
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
    FETI_CHECK(hs.error == 0, "FETI4I: a device pipeline wait timed out (solve aborted)");
    float ms = 0.f;
    CUDA_CHECK(cudaEventElapsedTime(&ms, I.ev0, I.ev1));
    stats.t_solve_ms = ms;
    stats.converged = hs.conv_iter >= 0;
    stats.iterations = stats.converged ? hs.conv_iter + 1 : std::min(hs.iter_base, I.opt.max_iterations);
    stats.replacements = hs.replacements;
    stats.tol = hs.tol;
    stats.final_norm = hs.last_norm;
    stats.kernel_launches = launches;
    const TileSetHost &Fop = mixed ? I.Flow : I.F64;
    stats.fapply_bytes = Fop.alg_bytes;
}

void GpuSolver::get_solution(std::vector<double> &lambda, std::vector<double> &alpha) {
    Impl &I = *impl;
    std::vector<double> xL(I.h_lam.size());
    CUDA_CHECK(cudaMemcpy(xL.data(), I.P.x, xL.size() * sizeof(double), cudaMemcpyDeviceToHost));
    lambda.assign(I.n_lambda, 0.0);
    for (size_t e = 0; e < xL.size(); ++e) lambda[I.h_lam[e]] = xL[e];
    alpha.resize(I.P.nK);
    CUDA_CHECK(cudaMemcpy(alpha.data(), I.P.alpha, alpha.size() * sizeof(double), cudaMemcpyDeviceToHost));
}

void GpuSolver::subdomain_schur(int d, double *S) {
    FETI_CHECK(!impl->implicit, "FETI4I: no Schur complements are stored with the implicit F apply");
    Impl &I = *impl;
    const TileSetHost &T = I.F64;
    FETI_CHECK(d >= 0 && d < (int)T.h_tn.size(), "FETI4I: subdomain index out of range");
    long long t0 = 0;
    for (int m = 0; m < d; ++m) t0 += (long long)T.h_tn[m] * (T.h_tn[m] + 1) / 2;
    const int tn = T.h_tn[d], n = I.h_loff[d + 1] - I.h_loff[d];
    std::vector<double> tiles((size_t)tn * (tn + 1) / 2 * TILE * TILE);
    CUDA_CHECK(cudaMemcpy(tiles.data(), (const double *)T.tiles + (size_t)t0 * TILE * TILE,
                          tiles.size() * sizeof(double), cudaMemcpyDeviceToHost));
    long long g = 0;
    for (int Ib = 0; Ib < tn; ++Ib)
        for (int Jb = Ib; Jb < tn; ++Jb, ++g)
            for (int r = 0; r < TILE; ++r)
                for (int c = 0; c < TILE; ++c) {
                    const int i = TILE * Ib + r, j = TILE * Jb + c;
                    if (i >= n || j >= n) continue;
                    const double v = tiles[(size_t)g * TILE * TILE + r * TILE + c];
                    S[(size_t)j * n + i] = v;
                    S[(size_t)i * n + j] = v;
                }
}

void GpuSolver::subdomain_kplus(int d, double *x) {
    Impl &I = *impl;
    FETI_CHECK(d >= 0 && d + 1 < (int)I.h_doff.size(), "FETI4I: subdomain index out of range");
    const int o = I.h_doff[d], n = I.h_doff[d + 1] - I.h_doff[d];
    CUDA_CHECK(cudaMemsetAsync(I.d_f, 0, sizeof(double) * I.ntot, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(I.d_f + o, x, sizeof(double) * n, cudaMemcpyHostToDevice, I.stream));
    I.launch_kplus(I.d_f, I.d_kf);
    CUDA_CHECK(cudaMemcpyAsync(x, I.d_kf + o, sizeof(double) * n, cudaMemcpyDeviceToHost, I.stream));
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
}

void GpuSolver::dual_rhs(const double *rhs, int rhs_size, double *b, double *e, int n_lambda, int n_kern) {
    Impl &I = *impl;
    DevProblem &P = I.P;
    CUDA_CHECK(cudaMemsetAsync(I.d_rhs, 0, sizeof(double) * std::max(1, I.n_caller), I.stream));
    const int ncp = std::min(rhs_size, I.n_caller);
    CUDA_CHECK(cudaMemcpyAsync(I.d_rhs, rhs, sizeof(double) * std::max(0, ncp), cudaMemcpyHostToDevice, I.stream));
    split_rhs_kernel<<<(I.ntot + 255) / 256, 256, 0, I.stream>>>(I.d_rhs, I.d_gdof, I.d_invm, I.d_f, I.ntot);
    if (I.hybrid) I.launch_kplus_dual(I.d_f, I.d_kf);
    else I.launch_kplus(I.d_f, I.d_kf, KPLUS_TOUCHED);
    evec_kernel<<<P.nd, TPB, 0, I.stream>>>(P, I.d_doff, I.d_rdofs, I.d_Rd, I.d_f, I.e_dev);
    bvec_kernel<<<(P.NL + 255) / 256, 256, 0, I.stream>>>(P, I.d_rdof, I.d_rsign, I.d_rc, I.d_kf, (double *)P.bL);
    CUDA_CHECK(cudaGetLastError());
    std::vector<double> bL(P.NL), ep(P.nP);
    CUDA_CHECK(cudaMemcpyAsync(bL.data(), P.bL, sizeof(double) * P.NL, cudaMemcpyDeviceToHost, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(ep.data(), I.e_dev, sizeof(double) * P.nP, cudaMemcpyDeviceToHost, I.stream));
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
    for (int i = 0; i < n_lambda; ++i) b[i] = 0.0;
    for (size_t r = 0; r < bL.size(); ++r) b[I.h_lam[r]] = bL[r];
    for (int k = 0; k < n_kern && k < (int)I.dual_to_partial.size(); ++k) e[k] = ep[I.dual_to_partial[k]];
}

void GpuSolver::apply_F(const double *x_lambda, double *y_lambda, int precision) {
    Impl &I = *impl;
    const TileSetHost &T = precision == SCHUR_FP64 ? I.F64 : I.Flow;
    FETI_CHECK(T.prec == precision, "FETI4I: the requested Schur precision was not prepared on the device");
    const int NL = I.P.NL;
    std::vector<double> xL(NL), yL(NL);
    for (int e = 0; e < NL; ++e) xL[e] = x_lambda[I.h_lam[e]];
    CUDA_CHECK(cudaMemcpyAsync(I.P.w, xL.data(), NL * sizeof(double), cudaMemcpyHostToDevice, I.stream));
    zero_kernel<<<(NL + 255) / 256, 256, 0, I.stream>>>(I.Ax64, NL);
    I.launch_tiles(T, 0, I.P.w, nullptr, I.Ax64, 0);
    I.launch_hybrid_F(I.P.w, I.Ax64, 0, 0, nullptr);
    CUDA_CHECK(cudaMemcpyAsync(yL.data(), I.Ax64, NL * sizeof(double), cudaMemcpyDeviceToHost, I.stream));
    zero_kernel<<<(NL + 255) / 256, 256, 0, I.stream>>>(I.Ax64, NL);
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
    for (int l = 0; l < I.n_lambda; ++l) y_lambda[l] = 0.0;
    for (int e = 0; e < NL; ++e) y_lambda[I.h_lam[e]] += yL[e];
}

double GpuSolver::time_F(int precision, int reps) {
    Impl &I = *impl;
    const TileSetHost &T = precision == SCHUR_FP64 ? I.F64 : I.Flow;
    FETI_CHECK(T.prec == precision, "FETI4I: the requested Schur precision was not prepared on the device");
    const int NL = I.P.NL;
    for (int i = 0; i < 3; ++i) {
        zero_kernel<<<(NL + 255) / 256, 256, 0, I.stream>>>(I.Ax64, NL);
        I.launch_tiles(T, 0, I.P.w, nullptr, I.Ax64, 0);
    }
    float total = 0.f;
    for (int i = 0; i < reps; ++i) {
        zero_kernel<<<(NL + 255) / 256, 256, 0, I.stream>>>(I.Ax64, NL);
        CUDA_CHECK(cudaEventRecord(I.ev0, I.stream));
        I.launch_tiles(T, 0, I.P.w, nullptr, I.Ax64, 0);
        CUDA_CHECK(cudaEventRecord(I.ev1, I.stream));
        CUDA_CHECK(cudaEventSynchronize(I.ev1));
        float ms = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, I.ev0, I.ev1));
        total += ms;
    }
    zero_kernel<<<(NL + 255) / 256, 256, 0, I.stream>>>(I.Ax64, NL);
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
    return total / reps;
}

// caller stream -> library stream -> caller stream ordering of a device-operator call
namespace {
struct StreamJoin {
    cudaStream_t caller, lib;
    cudaEvent_t ev;
    StreamJoin(cudaStream_t c, cudaStream_t l) : caller(c), lib(l) {
        CUDA_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CUDA_CHECK(cudaEventRecord(ev, caller));
        CUDA_CHECK(cudaStreamWaitEvent(lib, ev, 0));
    }
    void done() {
        CUDA_CHECK(cudaEventRecord(ev, lib));
        CUDA_CHECK(cudaStreamWaitEvent(caller, ev, 0));
        CUDA_CHECK(cudaEventDestroy(ev));
    }
};
}  // namespace

void GpuSolver::apply_F_device(const double *x, double *y, int precision, void *stream) {
    Impl &I = *impl;
    const TileSetHost &T = precision == SCHUR_FP64 ? I.F64 : I.Flow;
    FETI_CHECK(T.prec == precision, "FETI4I: the requested Schur precision was not prepared on the device");
    FETI_CHECK(!I.hybrid, "FETI4I: the device-operator entry points are Total FETI only");
    const int NL = I.P.NL;
    StreamJoin j((cudaStream_t)stream, I.stream);
    if (NL > 0) {
        gather_lambda_kernel<<<(NL + 255) / 256, 256, 0, I.stream>>>(I.d_lam, x, I.P.w, NL);
        I.launch_tiles(T, 0, I.P.w, nullptr, I.Ax64, 0);
        scatter_lambda_kernel<<<(NL + 255) / 256, 256, 0, I.stream>>>(I.d_lam, I.Ax64, y, NL);
        CUDA_CHECK(cudaGetLastError());
    }
    j.done();
}

void GpuSolver::apply_prec_device(const double *x, double *y, void *stream) {
    Impl &I = *impl;
    DevProblem &P = I.P;
    FETI_CHECK(!I.hybrid, "FETI4I: the device-operator entry points are Total FETI only");
    FETI_CHECK(I.opt.precond != PREC_NONE, "FETI4I: the instance has no preconditioner (PRECONDITIONER 0)");
    StreamJoin j((cudaStream_t)stream, I.stream);
    const int tg = (P.NT + 255) / 256, rg = (P.NL + 255) / 256;
    if (P.NL > 0) {
        switch (I.opt.precond) {
        case PREC_WEIGHT:
            prec_gather_kernel<PREC_WEIGHT><<<tg, 256, 0, I.stream>>>(P, I.d_lam, x);
            prec_scatter_kernel<<<rg, 256, 0, I.stream>>>(P, I.d_lam, y);
            break;
        case PREC_LUMPED:
            prec_gather_kernel<PREC_LUMPED><<<tg, 256, 0, I.stream>>>(P, I.d_lam, x);
            prec_ell_kernel<<<tg, 256, 0, I.stream>>>(P);
            prec_scatter_kernel<<<rg, 256, 0, I.stream>>>(P, I.d_lam, y);
            break;
        default:   // DIRICHLET: S_dir tiles
            prec_gather_kernel<PREC_DIRICHLET><<<tg, 256, 0, I.stream>>>(P, I.d_lam, x);
            zero_kernel<<<tg, 256, 0, I.stream>>>(P.vT, P.NT);
            I.launch_tiles(I.Dir, 0, P.uT, nullptr, P.vT, 0);
            prec_scatter_kernel<<<rg, 256, 0, I.stream>>>(P, I.d_lam, y);
            break;
        }
        CUDA_CHECK(cudaGetLastError());
    }
    j.done();
}

void GpuSolver::primal_from_dual(const double *rhs, int rhs_size, const double *lambda, const double *alpha,
                                 double *solution, int solution_size) {
    Impl &I = *impl;
    DevProblem &P = I.P;
    FETI_CHECK(!I.hybrid, "FETI4I: the device-operator entry points are Total FETI only");
    // f_i, and the forward pass L^-1 f kept for the primal (as in solve_full)
    CUDA_CHECK(cudaMemsetAsync(I.d_rhs, 0, sizeof(double) * std::max(1, I.n_caller), I.stream));
    const int ncp = std::min(rhs_size, I.n_caller);
    I.h2d_columns(I.d_rhs, 0, rhs, 0, (size_t)std::max(0, ncp), 1);
    split_rhs_kernel<<<(I.ntot + 255) / 256, 256, 0, I.stream>>>(I.d_rhs, I.d_gdof, I.d_invm, I.d_f, I.ntot);
    I.launch_kplus(I.d_f, I.d_kf, KPLUS_TOUCHED);
    // lambda at the local rows, the amplitudes of the instance's kernels
    std::vector<double> xL(P.NL);
    for (int e = 0; e < P.NL; ++e) xL[e] = lambda[I.h_lam[e]];
    CUDA_CHECK(cudaMemcpyAsync(P.x, xL.data(), sizeof(double) * P.NL, cudaMemcpyHostToDevice, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(P.alpha, alpha, sizeof(double) * P.nK, cudaMemcpyHostToDevice, I.stream));
    primal_rhs_kernel<<<std::max(1, std::min(4096, (I.ntot + 255) / 256)), 256, 0, I.stream>>>(
        P, I.d_tdof_g, I.d_rsign, nullptr, I.d_g, I.ntot);
    primal_bt_kernel<<<(P.NT + 255) / 256, 256, 0, I.stream>>>(P, I.d_tdof_g, I.d_rsign, I.d_g);
    I.launch_kplus(I.d_g, I.d_kf, KPLUS_PRIMAL);
    CUDA_CHECK(cudaMemsetAsync(I.d_sol, 0, sizeof(double) * std::max(1, I.n_caller), I.stream));
    primal_merge_kernel<<<P.nd, TPB, 0, I.stream>>>(P, I.d_doff, I.d_rdofs, I.d_Rd, I.d_kf, I.d_gdof, I.d_invm, I.d_sol);
    CUDA_CHECK(cudaGetLastError());
    const int nco = std::min(solution_size, I.n_caller);
    I.d2h_columns(solution, 0, I.d_sol, 0, (size_t)std::max(0, nco), 1);
    for (int i = std::max(0, nco); i < solution_size; ++i) solution[i] = 0.0;
}

double GpuSolver::fapply_bytes(int precision) const {
    const TileSetHost &T = precision == SCHUR_FP64 ? impl->F64 : impl->Flow;
    return T.alg_bytes;
}

}  // namespace feti

// =============================================================================================
// Allocation-free batched tile SYMV (FETI4ITiledSymvNoAlloc).
//
// For callers that own every byte of device memory themselves (a finite-element
// code that reserves HBM in its own pool at start-up and must not allocate while
// it runs): the caller passes the tiles, descriptors, x and y; the only scratch
// the kernel needs (work-queue counters and one dot partial per matrix) lives in
// the file-scope array below, NOALLOC_MAX_MATRICES matrices at most.  Every GPU
// that loads the library holds this array until the process exits.  All calls
// share it and it keeps the last call's contents, so each call clears its
// counters first, and calls that overlap on the GPU (different streams) race.
namespace feti {
namespace {

constexpr int NOALLOC_MAX_MATRICES = 16384;
constexpr int NOALLOC_MAX_ORDER = 3200;   // 2 * 32 * ceil(order/32) doubles of shared memory per CTA

struct NoAllocScratch {
    int queue;      // next matrix to take
    int done;       // CTAs that finished
    int pad[62];
    double dots[NOALLOC_MAX_MATRICES];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// one 32x32 tile with known block coordinates (I, J), FP64
__device__ __forceinline__ void tile_fma_noalloc(const uint4 (&raw)[16], int I, int J, const double *xs, double *ys,
                                                 int lane) {
    const int cq = lane % 16, h = lane / 16, idx = 2 * cq + h;
    double xc[2], xr[16], rs[16], cs[2];
    xc[0] = xs[TILE * J + 2 * cq];
    xc[1] = xs[TILE * J + 2 * cq + 1];
    cs[0] = cs[1] = 0.0;
#pragma unroll
    for (int q = 0; q < 16; ++q) { xr[q] = xs[TILE * I + 2 * q + h]; rs[q] = 0.0; }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const double e0 = __hiloint2double(raw[q].y, raw[q].x), e1 = __hiloint2double(raw[q].w, raw[q].z);
        rs[q] += e0 * xc[0] + e1 * xc[1];
        cs[0] += e0 * xr[q];
        cs[1] += e1 * xr[q];
    }
    atomicAdd(&ys[TILE * I + idx], reduce_scatter<16, 0>(rs, lane));
    if (I != J) atomicAdd(&ys[TILE * J + idx], reduce_scatter<2, 4>(cs, lane));
}

__global__ void __launch_bounds__(256, 2)
tile_symv_noalloc_kernel(const double *tiles, const long long *tile0, const int *order, const int *voff, int nmat,
                         int max_order, const double *x, double *y, double *dot_out, NoAllocScratch *scr) {
    extern __shared__ __align__(16) double nsm[];
    __shared__ double red[32];
    __shared__ int s_m, s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint4 *tl = reinterpret_cast<const uint4 *>(tiles);
    for (;;) {
        if (threadIdx.x == 0) s_m = atomicAdd(&scr->queue, 1);
        __syncthreads();
        const int m = s_m;
        if (m >= nmat) break;
        const int n = order[m];
        if (n > max_order || n < 0) {
            // violates the caller's stated bound: no product is formed; its y range and the total
            // dot are set to NaN so that the caller cannot mistake the result for a valid one
            const int o = voff[m];
            for (int i = threadIdx.x; i < n; i += blockDim.x) y[o + i] = __longlong_as_double(0x7ff8000000000000LL);
            if (threadIdx.x == 0) scr->dots[m] = __longlong_as_double(0x7ff8000000000000LL);
            __syncthreads();
            continue;
        }
        const int T = (n + TILE - 1) / TILE, o = voff[m];
        double *xs = nsm, *ys = nsm + TILE * T;
        for (int i = threadIdx.x; i < TILE * T; i += blockDim.x) {
            xs[i] = i < n ? x[o + i] : 0.0;
            ys[i] = 0.0;
        }
        __syncthreads();
        const int ntiles = T * (T + 1) / 2;
        // tiles k = warp, warp + nw, ...; (I, J) followed incrementally along the upper triangle
        int I = 0, off = warp;
        while (I < T && off >= T - I) { off -= T - I; ++I; }
        for (int k = warp; k < ntiles; k += nw) {
            uint4 raw[16];
            const uint4 *tp = tl + (size_t)(tile0[m] + k) * (TILE * 16);
#pragma unroll
            for (int q = 0; q < 16; ++q) raw[q] = ld_stream(tp + q * 32 + lane);
            tile_fma_noalloc(raw, I, I + off, xs, ys, lane);
            off += nw;
            while (I < T && off >= T - I) { off -= T - I; ++I; }
        }
        __syncthreads();
        double dot = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            y[o + i] = ys[i];
            dot += xs[i] * ys[i];
        }
        dot = block_sum(dot, red);
        if (threadIdx.x == 0) scr->dots[m] = dot;
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&scr->done, 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double t = 0.0;
        for (int i = threadIdx.x; i < nmat; i += blockDim.x) t += __ldcg(&scr->dots[i]);
        t = block_sum(t, red);
        if (threadIdx.x == 0 && dot_out) *dot_out = t;
    }
}

// device address of the scratch array, looked up once per device
NoAllocScratch *g_noalloc_ptr[256];
bool g_noalloc_ready[256];

}  // namespace

int tiled_symv_noalloc(const double *tiles, const long long *tile_offset, const int *order, const int *vector_offset,
                       int nmatrices, int max_order, const double *x, double *y, double *dot, void *stream) {
    FETI_CHECK(nmatrices >= 0 && nmatrices <= NOALLOC_MAX_MATRICES,
               "FETI4ITiledSymvNoAlloc: nmatrices must be in [0, " + std::to_string(NOALLOC_MAX_MATRICES) +
                   "] (size of the static scratch array)");
    FETI_CHECK(max_order >= 0 && max_order <= NOALLOC_MAX_ORDER,
               "FETI4ITiledSymvNoAlloc: max_order must be in [0, " + std::to_string(NOALLOC_MAX_ORDER) + "]");
    FETI_CHECK(nmatrices == 0 || (tiles && tile_offset && order && vector_offset && x && y),
               "FETI4ITiledSymvNoAlloc: null device pointer");
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    FETI_CHECK(dev >= 0 && dev < 256, "FETI4ITiledSymvNoAlloc: device index out of range");
    {
        // first call on this device: resolve the device address of the scratch array (under a lock, so
        // that host threads making their first calls together do the set-up once)
        static std::mutex setup_mutex;
        std::lock_guard<std::mutex> lock(setup_mutex);
        if (!g_noalloc_ready[dev]) {
            NoAllocScratch *p = nullptr;
            cudaError_t rc = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
            FETI_CHECK(rc == cudaSuccess, std::string("FETI4ITiledSymvNoAlloc: cudaGetSymbolAddress failed: ") +
                                              cudaGetErrorString(rc));
            const int smem = (int)(2 * sizeof(double) * TILE * ((NOALLOC_MAX_ORDER + TILE - 1) / TILE));
            CUDA_CHECK(
                cudaFuncSetAttribute(tile_symv_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            g_noalloc_ptr[dev] = p;
            g_noalloc_ready[dev] = true;
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    NoAllocScratch *scr = g_noalloc_ptr[dev];
    CUDA_CHECK(cudaMemsetAsync(scr, 0, offsetof(NoAllocScratch, dots), s));  // counters start at zero
    int nsm = 148;
    CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int grid = std::max(1, std::min(std::max(1, nmatrices), 2 * nsm));
    const size_t smem = 2 * sizeof(double) * TILE * (size_t)((max_order + TILE - 1) / TILE);
    tile_symv_noalloc_kernel<<<grid, 256, smem, s>>>(tiles, tile_offset, order, vector_offset, nmatrices, max_order, x,
                                                     y, dot, scr);
    CUDA_CHECK(cudaGetLastError());
    return 0;
}

}  // namespace feti

// =============================================================================================
// Element energies v_e^T K_e u_e (adjoint sensitivities d/drho_e of v^T K u)
namespace feti {
namespace {

__global__ void element_energy_kernel(int ne, int nd, const int *dofs, const double *K, const double *u,
                                      const double *v, double *out) {
    const int lane = threadIdx.x & 31;
    const int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (e >= ne) return;
    const int *de = dofs + (size_t)e * nd;
    const double *Ke = K + (size_t)e * nd * nd;
    double acc = 0.0;
    for (int a = 0; a < nd; ++a) {
        // row a: lanes stride over the columns (coalesced), v_a * sum_b K_ab u_b
        double s = 0.0;
        for (int b = lane; b < nd; b += 32) s += Ke[(size_t)a * nd + b] * u[de[b]];
        acc += v[de[a]] * s;
    }
    acc = warp_sum(acc);
    if (lane == 0) out[e] = acc;
}

}  // namespace

void GpuSolver::element_energies(const ElementData &el, const double *u, const double *v, int n, double *out) {
    Impl &I = *impl;
    const size_t ne = el.nelem();
    FETI_CHECK(ne > 0, "FETI4I: no elements");
    const int nd = (int)(el.dof_ptr[1] - el.dof_ptr[0]);
    for (size_t e = 0; e < ne; ++e)
        FETI_CHECK(el.dof_ptr[e + 1] - el.dof_ptr[e] == nd, "FETI4I: element energies need elements of one size");
    if (I.el_dofs == nullptr || I.el_count != ne || I.el_nd != nd) {
        I.el_dofs = I.upload(el.dofs);
        I.el_K = I.upload(el.vals);
        I.el_out = I.alloc<double>(ne);
        I.el_count = ne;
        I.el_nd = nd;
        I.el_n = 0;
    }
    if (I.el_n < n) {
        I.el_u = I.alloc<double>(n);
        I.el_v = I.alloc<double>(n);
        I.el_n = n;
    }
    CUDA_CHECK(cudaMemcpyAsync(I.el_u, u, sizeof(double) * n, cudaMemcpyHostToDevice, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(I.el_v, v, sizeof(double) * n, cudaMemcpyHostToDevice, I.stream));
    int maxdof = 0;
    for (int d : el.dofs) maxdof = std::max(maxdof, d);
    FETI_CHECK(maxdof < n, "FETI4I: element DOF outside the given vectors");
    const int wpb = 8;
    element_energy_kernel<<<(unsigned)((ne + wpb - 1) / wpb), 32 * wpb, 0, I.stream>>>((int)ne, nd, I.el_dofs, I.el_K,
                                                                                      I.el_u, I.el_v, I.el_out);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaMemcpyAsync(out, I.el_out, sizeof(double) * ne, cudaMemcpyDeviceToHost, I.stream));
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
}

}  // namespace feti

// =============================================================================================
// Block (multi right-hand-side) dual PCG: nr load cases solved together.
// Vectors are [row][rhs] (nr consecutive values per local row); scalars and
// stop tests are per right-hand side; the F apply is a tile SYMM.
namespace feti {
namespace {



constexpr int UNR = 4;   // rows in flight per thread in the block vector kernels
// resident CTAs per SM of the flat block vector kernels: the register cap that keeps 4 x 256 threads
// per SM (the uncapped kernels took up to 94 registers, 2 CTAs per SM, and stalled on latency)
constexpr int FLAT_MIN_BLOCKS = 4;

// per-column sum over a CTA: threads with the same column (tid % nr) are combined
__device__ void block_sum_cols(double v, int nr, double *sh /* >= 8*32 */, double *out_col /* nr */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o >= nr; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    __syncthreads();
    if (lane < nr) sh[wid * 32 + lane] = v;
    __syncthreads();
    if (threadIdx.x < nr) {
        double s = 0.0;
        for (int i = 0; i < nw; ++i) s += sh[i * 32 + threadIdx.x];
        out_col[threadIdx.x] = s;
    }
    __syncthreads();
}

// last-CTA total of per-CTA column partials (partials[cta * nr + j]) into out[j]
__device__ void grid_total_cols(const double *mine /* nr, shared */, double *partials, int nr, int *counter,
                                double *out) {
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x < nr) partials[blockIdx.x * nr + threadIdx.x] = mine[threadIdx.x];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(counter, 1) == (int)gridDim.x - 1);
    __syncthreads();
    if (s_last) {
        // every thread of the last CTA sums a fixed subset of the CTA partials of one column,
        // then the subsets are combined in shared memory (fixed order: deterministic)
        __threadfence();
        __shared__ double s_cols[1024];
        const int j = threadIdx.x & (nr - 1), g = threadIdx.x / nr, ng = blockDim.x / nr;
        double t = 0.0;
        for (int c = g; c < (int)gridDim.x; c += ng) t += __ldcg(&partials[c * nr + j]);
        s_cols[threadIdx.x] = t;
        __syncthreads();
        if (threadIdx.x < nr) {
            double u = 0.0;
            for (int q = 0; q < ng; ++q) u += s_cols[q * nr + threadIdx.x];
            out[threadIdx.x] = u;
        }
        if (threadIdx.x == 0) *counter = 0;
    }
}

// G_i v per column, v[(e - e0) * nr + j] (rows of the subdomain, written by this CTA)
__device__ void g_dot_cols(const DevProblem &P, const BlockDev &B, int dsub, const double *v, double *sh) {
    const int nr = B.nr;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    const int nk = P.kof[dsub + 1] - P.kof[dsub];
    for (int k = 0; k < nk; ++k) {
        double s = 0.0;
        for (int i = threadIdx.x; i < (e1 - e0) * nr; i += blockDim.x) s += P.Gl[(size_t)(e0 + (i >> B.lg)) * P.KS + k] * v[i];
        __shared__ double cols[32];
        block_sum_cols(s, nr, sh, cols);
        if (threadIdx.x < nr) B.d[(size_t)(P.kof[dsub] + k) * nr + threadIdx.x] = cols[threadIdx.x];
        __syncthreads();
    }
}

// G_i v per column from per-thread partial sums gk[k] = sum over the thread's elements of
// G[e, k] v[e, j] (every thread of the CTA on one column j = threadIdx.x & (nr - 1)): one pass over
// the rows instead of one per kernel vector
template <int KC>
__device__ void g_cols_reduce(const DevProblem &P, const BlockDev &B, int dsub, double (&gk)[KC], double *sh) {
    __shared__ double cols[32];
    const int nk = P.kof[dsub + 1] - P.kof[dsub];
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        if (k < nk) {   // uniform over the CTA
            block_sum_cols(gk[k], B.nr, sh, cols);
            if (threadIdx.x < B.nr) B.d[(size_t)(P.kof[dsub] + k) * B.nr + threadIdx.x] = cols[threadIdx.x];
            __syncthreads();
        }
    }
}

__device__ __forceinline__ double gt_alpha_col(const DevProblem &P, int e, int j, int nr, const double *a) {
    double s = 0.0;
    const int nk = P.rnk[e], ko = P.rkof[e], pn = P.pnk[e], po = P.pkof[e];
    const double *g = P.Gl + (size_t)e * P.KS, *gp = P.Gp + (size_t)e * P.KS;
    for (int k = 0; k < nk; ++k) s += g[k] * a[(size_t)(ko + k) * nr + j];
    for (int k = 0; k < pn; ++k) s += gp[k] * a[(size_t)(po + k) * nr + j];
    return s;
}

// Same with a compile-time kernel width KC (every row's coefficients padded to KC with zeros,
// the amplitudes padded by KC zero rows): the loads of all k are independent, so the rows a
// thread keeps in flight overlap their latencies.  KC = 0 falls back to the per-row counts.
template <int KC>
__device__ __forceinline__ double gt_alpha_colk(const DevProblem &P, int e, int j, int nr, const double *a) {
    if (KC == 0) return gt_alpha_col(P, e, j, nr, a);
    const int ko = P.rkof[e], po = P.pkof[e];
    const double *g = P.Gl + (size_t)e * KC, *gp = P.Gp + (size_t)e * KC;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < KC; ++k) s += g[k] * a[(size_t)(ko + k) * nr + j] + gp[k] * a[(size_t)(po + k) * nr + j];
    return s;
}

// conv[j]: -1 running, -2 zero right-hand side (frozen from the start), >= 0 stop iteration
__device__ __forceinline__ bool col_frozen(const BlockDev &B, int j, int iter) {
    const int c = B.conv[j];
    return c == -2 || (c >= 0 && iter > c);
}

// out (nK x nr) = (GG^T)^-1 in: a CTA owns CR rows; warp w takes one eighth of the inner dimension
// for those rows (lane = column, independent loads in flight), and the eight partial sums meet
// in shared memory in warp order
constexpr int CR = 4;
__global__ void __launch_bounds__(256) bcoarse_kernel(DevProblem P, BlockDev B, const double *in, double *out, int slot,
                                                      int looped) {
    pdl_enter();
    if (looped && skip_iter(P.st, P.st->iter_base + slot)) return;
    __shared__ double red[8][CR][32];
    const int nr = B.nr, nK = P.nK, nP = P.nP;
    const int r0 = blockIdx.x * CR;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int per = (nP + 7) / 8, b_lo = w * per, b_hi = min(nP, b_lo + per);
    const bool col = lane < nr;
    double acc[CR];
#pragma unroll
    for (int r = 0; r < CR; ++r) acc[r] = 0.0;
    const double *g[CR];
#pragma unroll
    for (int r = 0; r < CR; ++r) g[r] = P.GGtinv + (size_t)min(r0 + r, nK - 1) * nP;
#pragma unroll 8
    for (int b = b_lo; b < b_hi; ++b) {
        const double x = col ? in[(size_t)b * nr + lane] : 0.0;
#pragma unroll
        for (int r = 0; r < CR; ++r) acc[r] += g[r][b] * x;
    }
#pragma unroll
    for (int r = 0; r < CR; ++r) red[w][r][lane] = acc[r];
    __syncthreads();
    if (threadIdx.x < CR * 32) {
        const int r = threadIdx.x >> 5;
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) sum += red[q][r][lane];
        if (r0 + r < nK && col) out[(size_t)(r0 + r) * nr + lane] = sum;
    }
}

__global__ void bgt_kernel(DevProblem P, BlockDev B, const double *a, double *xout) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P.NL * B.nr) xout[i] = gt_alpha_col(P, (i >> B.lg), (i & (B.nr - 1)), B.nr, a);
}

// r = b - assemble(Ax), d = G r, |b_j|^2 totals (initial) / replacement
__global__ void br0_kernel(DevProblem P, BlockDev B, int replace_mode, int slot) {
    pdl_enter();
    __shared__ double sh[8 * 32];
    __shared__ double cols[32];
    if (replace_mode) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter) || P.st->replace_iter != iter) return;
    }
    const int nr = B.nr, dsub = blockIdx.x;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    double bb = 0.0;
    for (int i = threadIdx.x; i < (e1 - e0) * nr; i += blockDim.x) {
        const int e = e0 + (i >> B.lg), j = (i & (nr - 1));
        const int q = P.partner[e];
        const size_t o = (size_t)e * nr + j;
        const double a = B.Ax[o] + (q >= 0 ? B.Ax[(size_t)q * nr + j] : 0.0);
        const double rv = B.bL[o] - a;
        B.r[o] = rv;
        bb += B.bL[o] * B.bL[o] * P.minv[e];
    }
    __syncthreads();
    g_dot_cols(P, B, dsub, B.r + (size_t)e0 * nr, sh);
    if (!replace_mode) {
        block_sum_cols(bb, nr, sh, cols);
        grid_total_cols(cols, B.part, nr, B.done + DONE_B, B.scal + SC_BN2 * nr);
    }
}

__global__ void bpnorm_kernel(DevProblem P, BlockDev B) {
    __shared__ double sh[8 * 32];
    __shared__ double cols[32];
    const int nr = B.nr, dsub = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < (P.loff[dsub + 1] - P.loff[dsub]) * nr; i += blockDim.x) {
        const int e = P.loff[dsub] + (i >> B.lg), j = (i & (nr - 1));
        const double u = B.r[(size_t)e * nr + j] - gt_alpha_col(P, e, j, nr, B.alpha);
        s += u * u * P.minv[e];
    }
    block_sum_cols(s, nr, sh, cols);
    grid_total_cols(cols, B.part, nr, B.done + DONE_PN, B.scal + SC_PN2 * nr);
}

__global__ void btol_kernel(DevProblem P, BlockDev B) {
    const int j = threadIdx.x;
    if (j < B.nr) {
        const double un = sqrt(B.scal[SC_PN2 * B.nr + j]), bn = sqrt(B.scal[SC_BN2 * B.nr + j]);
        B.tol[j] = P.st->precision * fmin(un, bn);
        B.rmax[j] = un;
        B.conv[j] = (bn == 0.0 || un == 0.0) ? -2 : -1;
    }
}

// KC: the kernel width (1, 6: G z accumulated in registers while z is formed; 0: per-row counts,
// a second pass over z)
template <int KC>
__global__ void __launch_bounds__(TPBB) bz_kernel(DevProblem P, BlockDev B, int slot) {
    pdl_enter();
    __shared__ double sh[32 * 32];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr, dsub = blockIdx.x;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    const int cnt = (e1 - e0) * nr;
    constexpr int NG = KC > 0 ? KC : 1;
    double gk[NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) gk[k] = 0.0;
    for (int i0 = threadIdx.x; i0 < cnt; i0 += UNR * blockDim.x) {
        double zv[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < cnt) {
                const int e = e0 + (i >> B.lg), j = i & (nr - 1);
                const int pt = P.ptidx[e];
                zv[u] = P.ws[e] * B.vT[(size_t)P.tidx[e] * nr + j];
                if (pt >= 0) zv[u] += P.pws[e] * B.vT[(size_t)pt * nr + j];
            }
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < cnt) {
                B.z[(size_t)e0 * nr + i] = zv[u];
                if (KC > 0) {
                    const double *g = P.Gl + (size_t)(e0 + (i >> B.lg)) * NG;
#pragma unroll
                    for (int k = 0; k < NG; ++k) gk[k] += __ldg(g + k) * zv[u];
                }
            }
        }
    }
    __syncthreads();
    if (KC > 0) g_cols_reduce<NG>(P, B, dsub, gk, sh);
    else g_dot_cols(P, B, dsub, B.z + (size_t)e0 * nr, sh);
}

// ---- flat block kernels: a persistent grid over all rows (no per-subdomain reduction needed)
// thread column: the grid stride is a multiple of 32 >= nr, so every thread stays on column
// threadIdx.x & (nr - 1) and block_sum_cols combines the right partial sums

// u_T = B^T W w over all touched DOFs (v_T = u_T for the weight-function preconditioner)
template <int PRECOND>
__global__ void __launch_bounds__(256) bu_flat_kernel(DevProblem P, BlockDev B, int slot) {
    pdl_enter();
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr;
    const long long cnt = (long long)P.NT * nr, stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += stride) {
        const int t = (int)(i >> B.lg), j = (int)(i & (nr - 1));
        const int q0 = P.trow_ptr[t], q1 = P.trow_ptr[t + 1];
        double s = 0.0;
        for (int q = q0; q < q1; ++q) {
            const int e = P.trow_idx[q];
            s += P.ws[e] * B.w[(size_t)e * nr + j];
        }
        B.uT[i] = s;
        if (PRECOND == PREC_WEIGHT) B.vT[i] = s;
    }
}

// lumped v_T = K_TT u_T (sliced ELL of every subdomain)
// Two columns per thread (16-byte loads and stores; the per-row index loads serve both).
// Per-column block sums when every thread holds columns 2 (lane % (nr/2)) and 2 (lane % (nr/2)) + 1.
__device__ void block_sum_cols2(double s0, double s1, int nr, double *sh /* >= 8*32 */, double *out_col) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5, hnr = nr >> 1;
    for (int o = 16; o >= hnr; o >>= 1) {
        s0 += __shfl_xor_sync(FULL, s0, o);
        s1 += __shfl_xor_sync(FULL, s1, o);
    }
    __syncthreads();
    if (lane < hnr) {
        sh[wid * 32 + 2 * lane] = s0;
        sh[wid * 32 + 2 * lane + 1] = s1;
    }
    __syncthreads();
    if (threadIdx.x < nr) {
        double t = 0.0;
        for (int i = 0; i < nw; ++i) t += sh[i * 32 + threadIdx.x];
        out_col[threadIdx.x] = t;
    }
    __syncthreads();
}

template <int KC>
__device__ __forceinline__ double2 gt_alpha_colk2(const DevProblem &P, int e, int j, int nr, const double *a) {
    double2 r = make_double2(0.0, 0.0);
    if (KC == 0) {
        r.x = gt_alpha_col(P, e, j, nr, a);
        r.y = gt_alpha_col(P, e, j + 1, nr, a);
        return r;
    }
    const int ko = P.rkof[e], po = P.pkof[e];
    const double *g = P.Gl + (size_t)e * KC, *gp = P.Gp + (size_t)e * KC;
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        const double2 x = *reinterpret_cast<const double2 *>(a + (size_t)(ko + k) * nr + j);
        const double2 y = *reinterpret_cast<const double2 *>(a + (size_t)(po + k) * nr + j);
        r.x += g[k] * x.x + gp[k] * y.x;
        r.y += g[k] * x.y + gp[k] * y.y;
    }
    return r;
}

__global__ void __launch_bounds__(256, FLAT_MIN_BLOCKS) bell_flat2_kernel(DevProblem P, BlockDev B, int slot) {
    pdl_enter();
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr, lh = B.lg - 1;
    const long long cnt = (long long)P.NT * (nr >> 1), stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += stride) {
        const int t = (int)(i >> lh), j = 2 * (int)(i & ((nr >> 1) - 1));
        const int t0 = __ldg(P.tbase + t), ts = __ldg(P.tslot + t);
        const int sl = ts >> 5, ln = ts & 31;
        const int base = __ldg(P.ell_ptr + sl), wd = __ldg(P.ell_w + sl);
        const double2 *uT = reinterpret_cast<const double2 *>(B.uT);
        const size_t hn = (size_t)(nr >> 1), jh = (size_t)(j >> 1);
        // four entries in flight: the gathered u_T rows come from L2, one latency per four entries
        double2 s0 = make_double2(0.0, 0.0), s1 = s0, s2 = s0, s3 = s0;
        int q = 0;
        for (; q + 3 < wd; q += 4) {
            const int o = base + q * 32 + ln;
            const double v0 = __ldg(P.ell_val + o), v1 = __ldg(P.ell_val + o + 32), v2 = __ldg(P.ell_val + o + 64),
                         v3 = __ldg(P.ell_val + o + 96);
            const double2 u0 = __ldg(uT + (size_t)(t0 + __ldg(P.ell_col + o)) * hn + jh);
            const double2 u1 = __ldg(uT + (size_t)(t0 + __ldg(P.ell_col + o + 32)) * hn + jh);
            const double2 u2 = __ldg(uT + (size_t)(t0 + __ldg(P.ell_col + o + 64)) * hn + jh);
            const double2 u3 = __ldg(uT + (size_t)(t0 + __ldg(P.ell_col + o + 96)) * hn + jh);
            s0.x += v0 * u0.x; s0.y += v0 * u0.y;
            s1.x += v1 * u1.x; s1.y += v1 * u1.y;
            s2.x += v2 * u2.x; s2.y += v2 * u2.y;
            s3.x += v3 * u3.x; s3.y += v3 * u3.y;
        }
        for (; q < wd; ++q) {
            const int o = base + q * 32 + ln;
            const double v0 = __ldg(P.ell_val + o);
            const double2 u0 = __ldg(uT + (size_t)(t0 + __ldg(P.ell_col + o)) * hn + jh);
            s0.x += v0 * u0.x; s0.y += v0 * u0.y;
        }
        *reinterpret_cast<double2 *>(B.vT + (size_t)t * nr + j) =
            make_double2((s0.x + s1.x) + (s2.x + s3.x), (s0.y + s1.y) + (s2.y + s3.y));
    }
}

// w = r - G^T alpha, |w_j|^2 (and y = w, rho_j = |w_j|^2 without a preconditioner); two columns
// per thread, as in bell_flat2_kernel
template <int PRECOND, int KC>
__global__ void __launch_bounds__(256, FLAT_MIN_BLOCKS) bw_flat2_kernel(DevProblem P, BlockDev B, int slot) {
    pdl_enter();
    __shared__ double sh[8 * 32];
    __shared__ double cols[32];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr, lh = B.lg - 1;
    const long long cnt = (long long)P.NL * (nr >> 1), stride = (long long)gridDim.x * blockDim.x;
    double s0 = 0.0, s1 = 0.0;
    for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < cnt; i0 += UNR * stride) {
        double2 rv[UNR], ga[UNR];
        double mv[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const long long i = i0 + u * stride;
            if (i < cnt) {
                const int e = (int)(i >> lh), j = 2 * (int)(i & ((nr >> 1) - 1));
                rv[u] = *reinterpret_cast<const double2 *>(B.r + (size_t)e * nr + j);
                ga[u] = gt_alpha_colk2<KC>(P, e, j, nr, B.alpha);
                mv[u] = P.minv[e];
            }
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const long long i = i0 + u * stride;
            if (i < cnt) {
                const int e = (int)(i >> lh), j = 2 * (int)(i & ((nr >> 1) - 1));
                const double2 wv = make_double2(rv[u].x - ga[u].x, rv[u].y - ga[u].y);
                *reinterpret_cast<double2 *>(B.w + (size_t)e * nr + j) = wv;
                if (PRECOND == PREC_NONE) *reinterpret_cast<double2 *>(B.y + (size_t)e * nr + j) = wv;
                s0 += wv.x * wv.x * mv[u];
                s1 += wv.y * wv.y * mv[u];
            }
        }
    }
    block_sum_cols2(s0, s1, nr, sh, cols);
    grid_total_cols(cols, B.part, nr, B.done + DONE_W, B.scal + SC_WN2 * nr);
    if (PRECOND == PREC_NONE)
        grid_total_cols(cols, B.part + (size_t)gridDim.x * nr, nr, B.done + DONE_RHO, B.scal + SC_RHO * nr);
}

// w = r - G^T alpha and u_T = B^T W w in one pass over the touched DOFs: a thread takes one T entry
// and two columns, forms w at the (one to three) rows of that DOF, writes them, and adds
// ws_e w_e into u_T; |w_j|^2 as in bw_flat2_kernel.  Every row carries exactly one T entry, so every
// w is formed once.  WEIGHT also writes v_T = u_T.  Replaces bw_flat2 + bu_flat: w is not read back.
template <int PRECOND, int KC>
__global__ void __launch_bounds__(256, FLAT_MIN_BLOCKS) bwu_flat2_kernel(DevProblem P, BlockDev B, int slot) {
    pdl_enter();
    __shared__ double sh[8 * 32];
    __shared__ double cols[32];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr, lh = B.lg - 1;
    const long long cnt = (long long)P.NT * (nr >> 1), stride = (long long)gridDim.x * blockDim.x;
    double s0 = 0.0, s1 = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += stride) {
        const int t = (int)(i >> lh), j = 2 * (int)(i & ((nr >> 1) - 1));
        const int q0 = __ldg(P.trow_ptr + t), q1 = __ldg(P.trow_ptr + t + 1);
        double2 u = make_double2(0.0, 0.0);
        for (int q = q0; q < q1; ++q) {
            const int e = __ldg(P.trow_idx + q);
            const size_t o = (size_t)e * nr + j;
            const double2 rv = *reinterpret_cast<const double2 *>(B.r + o);
            const double2 ga = gt_alpha_colk2<KC>(P, e, j, nr, B.alpha);
            const double2 wv = make_double2(rv.x - ga.x, rv.y - ga.y);
            *reinterpret_cast<double2 *>(B.w + o) = wv;
            const double mv = __ldg(P.minv + e), ws = __ldg(P.ws + e);
            s0 += wv.x * wv.x * mv;
            s1 += wv.y * wv.y * mv;
            u.x += ws * wv.x;
            u.y += ws * wv.y;
        }
        *reinterpret_cast<double2 *>(B.uT + (size_t)t * nr + j) = u;
        if (PRECOND == PREC_WEIGHT) *reinterpret_cast<double2 *>(B.vT + (size_t)t * nr + j) = u;
    }
    block_sum_cols2(s0, s1, nr, sh, cols);
    grid_total_cols(cols, B.part, nr, B.done + DONE_W, B.scal + SC_WN2 * nr);
}

template <int KC>
__global__ void __launch_bounds__(256, FLAT_MIN_BLOCKS) by_flat2_kernel(DevProblem P, BlockDev B, int slot) {
    pdl_enter();
    __shared__ double sh[8 * 32];
    __shared__ double cols[32];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr, lh = B.lg - 1;
    const long long cnt = (long long)P.NL * (nr >> 1), stride = (long long)gridDim.x * blockDim.x;
    double s0 = 0.0, s1 = 0.0;
    for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < cnt; i0 += UNR * stride) {
        double2 zv[UNR], ga[UNR], wv[UNR];
        double mv[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const long long i = i0 + u * stride;
            if (i < cnt) {
                const int e = (int)(i >> lh), j = 2 * (int)(i & ((nr >> 1) - 1));
                const size_t o = (size_t)e * nr + j;
                zv[u] = *reinterpret_cast<const double2 *>(B.z + o);
                wv[u] = *reinterpret_cast<const double2 *>(B.w + o);
                ga[u] = gt_alpha_colk2<KC>(P, e, j, nr, B.alpha);
                mv[u] = P.minv[e];
            }
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const long long i = i0 + u * stride;
            if (i < cnt) {
                const int e = (int)(i >> lh), j = 2 * (int)(i & ((nr >> 1) - 1));
                const double2 yv = make_double2(zv[u].x - ga[u].x, zv[u].y - ga[u].y);
                *reinterpret_cast<double2 *>(B.y + (size_t)e * nr + j) = yv;
                s0 += yv.x * wv[u].x * mv[u];
                s1 += yv.y * wv[u].y * mv[u];
            }
        }
    }
    block_sum_cols2(s0, s1, nr, sh, cols);
    grid_total_cols(cols, B.part + (size_t)gridDim.x * nr, nr, B.done + DONE_RHO, B.scal + SC_RHO * nr);
}


// y = z - G^T alpha, rho_j = y.w

// p = y + beta_j p (and its FP32 copy).  Two columns per thread (16-byte loads and stores), UNR
// rows in flight; the grid stride is a multiple of nr / 2, so every thread keeps its columns and
// computes their beta once.
__global__ void __launch_bounds__(256, FLAT_MIN_BLOCKS) bp_kernel(DevProblem P, BlockDev B, int slot) {
    pdl_enter();
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr, hn = nr >> 1;
    const long long cnt = (long long)P.NL * hn, stride = (long long)gridDim.x * blockDim.x;
    const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 2 * (int)(i0 & (hn - 1));
    const bool f0 = col_frozen(B, j, iter), f1 = col_frozen(B, j + 1, iter);
    const double b0 = (iter == 0) ? 0.0 : B.scal[SC_RHO * nr + j] / B.rho_hist[(size_t)(iter - 1) * nr + j];
    const double b1 = (iter == 0) ? 0.0 : B.scal[SC_RHO * nr + j + 1] / B.rho_hist[(size_t)(iter - 1) * nr + j + 1];
    const double2 *y = reinterpret_cast<const double2 *>(B.y);
    double2 *p = reinterpret_cast<double2 *>(B.p);
    float2 *p32 = reinterpret_cast<float2 *>(B.p32);
    for (long long i = i0; i < cnt; i += UNR * stride) {
        double2 yv[UNR], pv[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const long long k = i + u * stride;
            if (k < cnt) {
                yv[u] = __ldg(y + k);
                pv[u] = p[k];
            }
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const long long k = i + u * stride;
            if (k < cnt) {
                const double2 r = make_double2(f0 ? 0.0 : yv[u].x + b0 * pv[u].x, f1 ? 0.0 : yv[u].y + b1 * pv[u].y);
                p[k] = r;
                p32[k] = make_float2((float)r.x, (float)r.y);
            }
        }
    }
}

// Two CTAs of 1024 threads per SM (32 registers, two rows in flight per thread): with 60 registers
// only one fitted, and the 512 subdomains of the heat workload ran in four waves.
template <int KC>
__global__ void __launch_bounds__(TPBB, 2) bupdate_kernel(DevProblem P, BlockDev B, int slot) {
    constexpr int UNR = 2;
    constexpr int NG = KC > 0 ? KC : 1;
    double gk[NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) gk[k] = 0.0;
    pdl_enter();
    __shared__ double sh[32 * 32];
    const int iter = P.st->iter_base + slot;
    if (skip_iter(P.st, iter)) return;
    const int nr = B.nr, dsub = blockIdx.x;
    const int e0 = P.loff[dsub], e1 = P.loff[dsub + 1];
    // the stride keeps each thread on one column: alpha_j once per thread
    const int jt = threadIdx.x & (nr - 1);
    const bool frozen = col_frozen(B, jt, iter);
    const double alpha = frozen ? 0.0 : B.scal[SC_RHO * nr + jt] / B.scal[SC_PAP * nr + jt];
    const int cnt = (e1 - e0) * nr;
    if (!frozen)
        for (int i0 = threadIdx.x; i0 < cnt; i0 += UNR * blockDim.x) {
            double xv[UNR], pv[UNR], rv[UNR], av[UNR];
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const int i = i0 + u * blockDim.x;
                if (i < cnt) {
                    const int e = e0 + (i >> B.lg);
                    const size_t o = (size_t)e0 * nr + i;
                    const int q = P.partner[e];
                    xv[u] = B.x[o];
                    pv[u] = B.p[o];
                    rv[u] = B.r[o];
                    av[u] = B.Ap[o] + (q >= 0 ? B.Ap[(size_t)q * nr + jt] : 0.0);
                }
            }
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const int i = i0 + u * blockDim.x;
                if (i < cnt) {
                    const size_t o = (size_t)e0 * nr + i;
                    B.x[o] = xv[u] + alpha * pv[u];
                    const double rn = rv[u] - alpha * av[u];
                    B.r[o] = rn;
                    if (KC > 0) {
                        const double *g = P.Gl + (size_t)(e0 + (i >> B.lg)) * NG;
#pragma unroll
                        for (int k = 0; k < NG; ++k) gk[k] += __ldg(g + k) * rn;
                    }
                }
            }
        }
    else if (KC > 0)
        // a converged column keeps its r: its G r is still the coarse input of the next iteration
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
            const double *g = P.Gl + (size_t)(e0 + (i >> B.lg)) * NG;
            const double rv = B.r[(size_t)e0 * nr + i];
#pragma unroll
            for (int k = 0; k < NG; ++k) gk[k] += __ldg(g + k) * rv;
        }
    __syncthreads();
    if (KC > 0) g_cols_reduce<NG>(P, B, dsub, gk, sh);
    else g_dot_cols(P, B, dsub, B.r + (size_t)e0 * nr, sh);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        DevState *st = P.st;
        bool replace = false;
        int nconv = 0;
        double worst = 0.0;
        const bool fresh = st->true_iter == iter;
        for (int j = 0; j < nr; ++j) {
            const double rho = B.scal[SC_RHO * nr + j];
            B.rho_hist[(size_t)iter * nr + j] = rho;
            if (B.conv[j] != -1) { ++nconv; continue; }
            const double wn = sqrt(B.scal[SC_WN2 * nr + j]);
            B.last_norm[j] = wn;
            worst = fmax(worst, wn / fmax(B.tol[j], 1e-300));
            if (!st->mixed) {
                if (wn < B.tol[j]) { B.conv[j] = iter; ++nconv; }
            } else {
                B.rmax[j] = fresh ? wn : fmax(B.rmax[j], wn);
                if (wn < B.tol[j]) {
                    if (fresh) { B.conv[j] = iter; ++nconv; }
                    else replace = true;
                } else if (wn < st->delta * B.rmax[j]) {
                    replace = true;
                }
            }
        }
        st->last_norm = worst;
        if (nconv == nr && st->conv_iter < 0) st->conv_iter = iter;
        if (replace && st->conv_iter < 0) {
            st->replace_iter = iter + 1;
            st->true_iter = iter + 1;
            st->replacements += 1;
        }
    }
}

// Tile SYMM, full read: a warp owns one 32-row tile row of one subdomain and
// accumulates Y_I = sum_J S_IJ X_J for all nr columns in registers, using the
// stored upper tile (I,J) for J >= I and the stored tile (J,I) transposed for J < I.
// Lane = (row group g, column j): NR columns, 32/NR row groups of NR rows each.
template <int PREC, int NR, int SRC>  // SRC 0: FP64 x (replacement/initial/FP64 path), 1: FP32 p copy
__global__ void __launch_bounds__(256, PREC == SCHUR_FP64 ? 2 : 3)
tile_symm_kernel(TileSetDev ts, DevProblem P, BlockDev B, const double *x64, const float *x32, double *out,
                 const int2 *units, int nunits, int slot, int mode) {
    pdl_enter();
    using Acc = typename TileT<PREC>::Acc;
    constexpr int EPC = TileT<PREC>::EPC;
    constexpr int G = 32 / NR;          // row groups
    constexpr unsigned TB = TILE * TILE * (PREC == SCHUR_FP64 ? 8 : 4);
    extern __shared__ __align__(16) unsigned char symm_smem[];
    __shared__ int s_last;
    if (mode != 0) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
        if (mode == 3 && P.st->replace_iter != iter) return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = lane % NR, g = lane / NR;
    unsigned char *wbuf = symm_smem + (size_t)warp * TB;
    Acc *tile = reinterpret_cast<Acc *>(wbuf);
    for (;;) {
        int u = 0;
        if (lane == 0) u = atomicAdd(&B.queue[0], 1);
        u = __shfl_sync(FULL, u, 0);
        if (u >= nunits) break;
        const int m = units[u].x, I = units[u].y;
        const int n = ts.mat_n[m], voff = ts.mat_voff[m], tn = ts.mat_tn[m];
        const long long t0 = ts.mat_tile0[m];
        Acc acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = 0;
        for (int J = 0; J < tn; ++J) {
            const bool upper = J >= I;
            const int a = upper ? I : J, b = upper ? J : I;
            const long long tid = t0 + (long long)a * tn - (long long)a * (a - 1) / 2 + (b - a);
            // tile -> shared memory (each lane copies 16-byte chunks)
            const uint4 *src = reinterpret_cast<const uint4 *>(ts.tiles) + (size_t)tid * (TB / 16);
            uint4 *dst = reinterpret_cast<uint4 *>(wbuf);
#pragma unroll
            for (int q = 0; q < (int)(TB / 16 / 32); ++q) dst[q * 32 + lane] = ld_stream(src + q * 32 + lane);
            __syncwarp();
            // x column j of block J, row c (zero past the subdomain's rows)
            const int rb = TILE * J;
            auto xval = [&](int c) -> Acc {
                const int row = rb + c;
                if (row >= n) return (Acc)0;
                return SRC ? (Acc)x32[(size_t)(voff + row) * NR + j] : (Acc)x64[(size_t)(voff + row) * NR + j];
            };
            if (upper) {
                // Y[r] += sum_c S[r][c] x[c], my rows r = g*NR + t; eight columns per step keep the
                // x values in few registers and NR independent accumulation chains in flight
#pragma unroll
                for (int c0 = 0; c0 < TILE; c0 += 8) {
                    Acc xc[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) xc[q] = xval(c0 + q);
#pragma unroll
                    for (int t = 0; t < NR; ++t) {
                        const Acc *srow = tile + (g * NR + t) * TILE + c0;
                        acc[t] += ((srow[0] * xc[0] + srow[1] * xc[1]) + (srow[2] * xc[2] + srow[3] * xc[3])) +
                                  ((srow[4] * xc[4] + srow[5] * xc[5]) + (srow[6] * xc[6] + srow[7] * xc[7]));
                    }
                }
            } else {
                // Y[r] += sum_c S_JI[c][r] x[c]
#pragma unroll 4
                for (int c = 0; c < TILE; ++c) {
                    const Acc *srow = tile + c * TILE + g * NR;
                    const Acc xv = xval(c);
#pragma unroll
                    for (int t = 0; t < NR; ++t) acc[t] += srow[t] * xv;
                }
            }
            __syncwarp();
        }
        // write the tile row and its dot with x (per column)
        double dot = 0.0;
#pragma unroll
        for (int t = 0; t < NR; ++t) {
            const int row = TILE * I + g * NR + t;
            if (row < n) {
                const size_t o = (size_t)(voff + row) * NR + j;
                out[o] = (double)acc[t];
                const double xv = SRC ? (double)x32[o] : x64[o];
                dot += xv * (double)acc[t];
            }
        }
#pragma unroll
        for (int o = 16; o >= NR; o >>= 1) dot += __shfl_xor_sync(FULL, dot, o);
        if (lane < NR) B.unit_dot[(size_t)u * NR + lane] = dot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&B.queue[1], 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        if (mode == 1) {
            __threadfence();
            if (threadIdx.x < NR) {
                double t = 0.0;
                for (int q = 0; q < nunits; ++q) t += __ldcg(&B.unit_dot[(size_t)q * NR + threadIdx.x]);
                B.scal[SC_PAP * NR + threadIdx.x] = t;
            }
        }
        if (threadIdx.x == 0) {
            B.queue[0] = 0;
            B.queue[1] = 0;
            __threadfence();
        }
    }
}

// Tile SYMM of FP64 tiles on the FP64 tensor cores (mma.m8n8k4.f64), with the units and results of
// tile_symm_kernel<SCHUR_FP64, NR, 0>.  A warp owns one 32-row tile row I of one subdomain and
// forms, for every block column J, C(32 x NR) += A(32 x 32) X_J(32 x NR): A is the stored tile
// (I, J) for J >= I and the transpose of the stored tile (J, I) for J < I, read straight from
// global memory in fragment order (every 32-byte sector once), as 4 x NR/8 blocks of 8 x 8 over
// 8 k-steps of 4.  x rows past the subdomain read as zero.
template <int NR>
__global__ void __launch_bounds__(256, 1)
tile_symm_mma_kernel(TileSetDev ts, DevProblem P, BlockDev B, const double *x64, double *out, const int2 *units,
                     int nunits, int slot, int mode) {
    pdl_enter();
    static_assert(NR == 8 || NR == 16 || NR == 32, "FP64 MMA SYMM: 8, 16 or 32 right-hand sides");
    constexpr int NB = NR / 8;
    __shared__ int s_last;
    if (mode != 0) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
        if (mode == 3 && P.st->replace_iter != iter) return;
    }
    const int lane = threadIdx.x & 31;
    const int gr = lane >> 2, gc = lane & 3;
    const double *tiles = reinterpret_cast<const double *>(ts.tiles);
    for (;;) {
        int u = 0;
        if (lane == 0) u = atomicAdd(&B.queue[0], 1);
        u = __shfl_sync(FULL, u, 0);
        if (u >= nunits) break;
        const int m = units[u].x, I = units[u].y;
        const int n = ts.mat_n[m], voff = ts.mat_voff[m], tn = ts.mat_tn[m];
        const long long t0 = ts.mat_tile0[m];
        double acc[4][NB][2];
#pragma unroll
        for (int mb = 0; mb < 4; ++mb)
#pragma unroll
            for (int nb = 0; nb < NB; ++nb) acc[mb][nb][0] = acc[mb][nb][1] = 0.0;
        for (int J = 0; J < tn; ++J) {
            const bool upper = J >= I;
            const int a = upper ? I : J, b = upper ? J : I;
            const double *tile = tiles + (size_t)(t0 + (long long)a * tn - (long long)a * (a - 1) / 2 + (b - a)) * (TILE * TILE);
            // A[r][k] = tile[r][k] (upper) or tile[k][r] (lower)
            const double *ab = upper ? tile + gr * TILE + gc : tile + gc * TILE + gr;
            const int s_m = upper ? 8 * TILE : 8, s_k = upper ? 4 : 4 * TILE;
            double bf[8][NB];
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const int row = TILE * J + 4 * ks + gc;
#pragma unroll
                for (int nb = 0; nb < NB; ++nb)
                    bf[ks][nb] = row < n ? __ldg(x64 + (size_t)(voff + row) * NR + 8 * nb + gr) : 0.0;
            }
#pragma unroll
            for (int mb = 0; mb < 4; ++mb) {
                double af[8];
#pragma unroll
                for (int ks = 0; ks < 8; ++ks) af[ks] = __ldg(ab + mb * s_m + ks * s_k);
#pragma unroll
                for (int nb = 0; nb < NB; ++nb)
#pragma unroll
                    for (int ks = 0; ks < 8; ++ks) dmma84(acc[mb][nb], af[ks], bf[ks][nb]);
            }
        }
        // rows of the tile row and their dot with x, per column
        double dot[NB][2];
#pragma unroll
        for (int nb = 0; nb < NB; ++nb) dot[nb][0] = dot[nb][1] = 0.0;
#pragma unroll
        for (int mb = 0; mb < 4; ++mb) {
            const int row = TILE * I + 8 * mb + gr;
            if (row < n) {
#pragma unroll
                for (int nb = 0; nb < NB; ++nb)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const size_t o = (size_t)(voff + row) * NR + 8 * nb + 2 * gc + e;
                        out[o] = acc[mb][nb][e];
                        dot[nb][e] += x64[o] * acc[mb][nb][e];
                    }
            }
        }
#pragma unroll
        for (int nb = 0; nb < NB; ++nb)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                double v = dot[nb][e];
                v += __shfl_xor_sync(FULL, v, 4);
                v += __shfl_xor_sync(FULL, v, 8);
                v += __shfl_xor_sync(FULL, v, 16);
                if (gr == 0) B.unit_dot[(size_t)u * NR + 8 * nb + 2 * gc + e] = v;
            }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&B.queue[1], 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        if (mode == 1) {
            __threadfence();
            if (threadIdx.x < NR) {
                double t = 0.0;
                for (int q = 0; q < nunits; ++q) t += __ldcg(&B.unit_dot[(size_t)q * NR + threadIdx.x]);
                B.scal[SC_PAP * NR + threadIdx.x] = t;
            }
        }
        if (threadIdx.x == 0) {
            B.queue[0] = 0;
            B.queue[1] = 0;
            __threadfence();
        }
    }
}

// ---- Tile SYMM on the 5th-generation tensor cores (FP32 tiles, 3xTF32 split)
// A unit is four consecutive 32-row tile rows of one subdomain (M = 128 rows of S).  For
// every 32-column block J the CTA stages A = S[128 rows, 32 columns] (upper tiles as stored,
// lower tiles transposed) and B = X_J^T (NR x 32) in shared memory, in the 128-byte swizzled
// K-major layout of the UMMA descriptors, each split into TF32 parts x = hi + lo.  One thread
// issues hi*hi + hi*lo + lo*hi as tcgen05.mma kind::tf32 (M=128, N=NR, K=8, four K steps)
// into an FP32 accumulator in tensor memory; the dropped lo*lo term and the TF32 rounding of
// lo leave about 2^-21 relative error per product, the order of FP32 accumulation.
// Two stages: staging block J+1 overlaps the MMAs of block J; tcgen05.commit arrives on the
// stage's mbarrier when its MMAs are done.  Every wait is bounded: on time-out the kernel
// records an error, waits (bounded) for its MMAs, frees its tensor memory and returns.
namespace tc {
constexpr int M = 128;
constexpr unsigned A_BYTES = M * 128;   // 128 rows x 32 FP32
constexpr int THREADS = 256;
// K-major operand, 128-byte swizzle: 8-row atoms of 1024 bytes (SBO), version 1
__device__ __forceinline__ uint64_t sdesc(unsigned addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)2 << 61);
}
// kind::tf32: D FP32, A and B TF32, both K-major, N = NR, M = 128
template <int N>
__host__ __device__ constexpr uint32_t idesc() {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// byte offset of FP32 element (row, k) inside a swizzled K-major operand (32 k per row)
__device__ __forceinline__ unsigned swz(int row, int chunk) {
    return (unsigned)((row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4));
}
__device__ __forceinline__ float tf32_hi(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
__device__ __forceinline__ void split_store(unsigned char *hi, unsigned char *lo, unsigned off, float4 v) {
    float4 h, l;
    h.x = tf32_hi(v.x); l.x = v.x - h.x;
    h.y = tf32_hi(v.y); l.y = v.y - h.y;
    h.z = tf32_hi(v.z); l.z = v.z - h.z;
    h.w = tf32_hi(v.w); l.w = v.w - h.w;
    *reinterpret_cast<float4 *>(hi + off) = h;
    *reinterpret_cast<float4 *>(lo + off) = l;
}
__device__ __forceinline__ void mma(unsigned tmem, uint64_t a, uint64_t b, uint32_t id, unsigned acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void commit(unsigned long long *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 16 columns of 32 lanes: lane i of warp w (w % 4 = q) gets TMEM lane 32q + i
__device__ __forceinline__ void ld16(unsigned taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void ld4(unsigned taddr, uint32_t (&r)[16]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void ld8(unsigned taddr, uint32_t (&r)[16]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
}  // namespace tc

template <int NR>
__global__ void __launch_bounds__(tc::THREADS, 2)
tile_symm_tc_kernel(TileSetDev ts, DevProblem P, BlockDev B, const float *x32, double *out, const int2 *units,
                    int nunits, int slot, int mode) {
    pdl_enter();
    static_assert(NR == 8 || NR == 16 || NR == 32, "tensor-core SYMM: 8, 16 or 32 right-hand sides");
    constexpr unsigned B_BYTES = NR * 128;
    constexpr unsigned STAGE = 2 * tc::A_BYTES + 2 * B_BYTES;
    constexpr int HALF = NR / 2;                 // columns read back by each warp half
    extern __shared__ unsigned char tc_smem[];
    __shared__ unsigned long long bar[2];
    __shared__ unsigned s_tmem;
    __shared__ int s_unit, s_last, s_err;
    __shared__ double s_dot[tc::THREADS / 32][NR];
    if (mode != 0) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned base = smem_u32(tc_smem);
    unsigned char *buf = tc_smem + ((1024u - (base & 1023u)) & 1023u);   // 1024-byte aligned stages
    const unsigned ncols = 32;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_err = 0;
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const unsigned tmem = s_tmem;
    constexpr uint32_t ID = tc::idesc<NR>();
    unsigned phase[2] = {0u, 0u};
    bool pending[2] = {false, false};
    unsigned seq = 0;
    bool ok = true;
    for (;;) {
        if (tid == 0) s_unit = atomicAdd(&B.queue[0], 1);
        const bool all_ok = __syncthreads_and(ok);   // a timed-out wait stops every thread together
        const int u = s_unit;
        if (u >= nunits || !all_ok) break;
        ok = true;
        const int m = units[u].x, I0 = 4 * units[u].y;
        const int n = ts.mat_n[m], voff = ts.mat_voff[m], tn = ts.mat_tn[m];
        const long long t0 = ts.mat_tile0[m];
        const float *tiles = reinterpret_cast<const float *>(ts.tiles);
        // block J of the unit into registers: four 16-byte A chunks and one B chunk per thread;
        // two register sets keep blocks J+1 and J+2 in flight while block J is staged
        constexpr int AIT = (tc::M * 8) / tc::THREADS;
        float4 ra0[AIT], ra1[AIT], rb0 = make_float4(0.f, 0.f, 0.f, 0.f), rb1 = rb0;
        auto load_block = [&](int J, float4 (&ra)[AIT], float4 &rb) {
#pragma unroll
            for (int it = 0; it < AIT; ++it) {
                const int q = tid + it * tc::THREADS;
                const int qq = q >> 8, I = I0 + qq;       // warp-uniform
                ra[it] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (I < tn && J >= I) {
                    const int rr = (q >> 3) & 31, c = q & 7;
                    const long long tid_ = t0 + (long long)I * tn - (long long)I * (I - 1) / 2 + (J - I);
                    const uint4 u4 =
                        ld_stream(reinterpret_cast<const uint4 *>(tiles + (size_t)tid_ * (TILE * TILE) + rr * TILE + 4 * c));
                    ra[it] = make_float4(__uint_as_float(u4.x), __uint_as_float(u4.y), __uint_as_float(u4.z),
                                         __uint_as_float(u4.w));
                } else if (I < tn) {
                    const int rr = q & 31, c = (q >> 5) & 7;
                    const long long tid_ = t0 + (long long)J * tn - (long long)J * (J - 1) / 2 + (I - J);
                    const float *tp = tiles + (size_t)tid_ * (TILE * TILE) + rr;
                    ra[it].x = tp[(4 * c + 0) * TILE];
                    ra[it].y = tp[(4 * c + 1) * TILE];
                    ra[it].z = tp[(4 * c + 2) * TILE];
                    ra[it].w = tp[(4 * c + 3) * TILE];
                }
            }
            if (tid < NR * 8) {
                const int nn = tid % NR, c = tid / NR;
                const int r0 = TILE * J + 4 * c;
                rb.x = (r0 + 0 < n) ? x32[(size_t)(voff + r0 + 0) * NR + nn] : 0.f;
                rb.y = (r0 + 1 < n) ? x32[(size_t)(voff + r0 + 1) * NR + nn] : 0.f;
                rb.z = (r0 + 2 < n) ? x32[(size_t)(voff + r0 + 2) * NR + nn] : 0.f;
                rb.w = (r0 + 3 < n) ? x32[(size_t)(voff + r0 + 3) * NR + nn] : 0.f;
            }
        };
        auto step = [&](int J, float4 (&ra)[AIT], float4 &rb) {
            const int st = seq & 1;
            if (pending[st]) {
                if (!mbar_wait(&bar[st], phase[st])) ok = false;
                phase[st] ^= 1u;
                pending[st] = false;
            }
            unsigned char *ahi = buf + st * STAGE, *alo = ahi + tc::A_BYTES, *bhi = alo + tc::A_BYTES,
                          *blo = bhi + B_BYTES;
#pragma unroll
            for (int it = 0; it < AIT; ++it) {
                const int q = tid + it * tc::THREADS;
                const int qq = q >> 8, I = I0 + qq;
                const bool up = (I < tn && J >= I);
                const int rr = up ? ((q >> 3) & 31) : (q & 31), c = up ? (q & 7) : ((q >> 5) & 7);
                tc::split_store(ahi, alo, tc::swz(qq * 32 + rr, c), ra[it]);
            }
            if (tid < NR * 8) tc::split_store(bhi, blo, tc::swz(tid % NR, tid / NR), rb);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                tc::fence_after();
                const unsigned a_hi = smem_u32(ahi), a_lo = smem_u32(alo), b_hi = smem_u32(bhi), b_lo = smem_u32(blo);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const unsigned off = 32u * kk;
                    tc::mma(tmem, tc::sdesc(a_hi + off), tc::sdesc(b_hi + off), ID, (J > 0 || kk > 0) ? 1u : 0u);
                    tc::mma(tmem, tc::sdesc(a_hi + off), tc::sdesc(b_lo + off), ID, 1u);
                    tc::mma(tmem, tc::sdesc(a_lo + off), tc::sdesc(b_hi + off), ID, 1u);
                }
                tc::commit(&bar[st]);
            }
            pending[st] = true;
            ++seq;
            if (J + 2 < tn) load_block(J + 2, ra, rb);   // in flight while blocks J and J+1 are processed
        };
        load_block(0, ra0, rb0);
        if (tn > 1) load_block(1, ra1, rb1);
        for (int J = 0; J < tn; J += 2) {
            step(J, ra0, rb0);
            if (J + 1 < tn) step(J + 1, ra1, rb1);
        }
        // the last commit tracks every MMA issued before it: the accumulator is complete
        {
            const int lst = (seq - 1) & 1;
            if (!mbar_wait(&bar[lst], phase[lst])) ok = false;
            phase[lst] ^= 1u;
            pending[lst] = false;
        }
        tc::fence_after();
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31, columns (w / 4) * HALF .. +HALF-1
        uint32_t r[16];
        const unsigned taddr = tmem + ((unsigned)(32 * (warp & 3)) << 16) + (unsigned)((warp >> 2) * HALF);
        if (HALF == 16) tc::ld16(taddr, r);
        else if (HALF == 8) tc::ld8(taddr, r);
        else tc::ld4(taddr, r);
        const int row = TILE * I0 + 32 * (warp & 3) + lane;
        const int c0 = (warp >> 2) * HALF;
        double dl[HALF];
#pragma unroll
        for (int c = 0; c < HALF; ++c) {
            dl[c] = 0.0;
            if (row < n && ok) {
                const size_t o = (size_t)(voff + row) * NR + c0 + c;
                const double y = (double)__uint_as_float(r[c]);
                out[o] = y;
                dl[c] = (double)x32[o] * y;
            }
        }
#pragma unroll
        for (int c = 0; c < HALF; ++c) {
            double v = dl[c];
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
            if (lane == 0) s_dot[warp][c] = v;
        }
        tc::fence_before();
        __syncthreads();
        if (tid < NR) {
            const int h = tid / HALF, c = tid % HALF;
            double t = 0.0;
            for (int w = 0; w < 4; ++w) t += s_dot[4 * h + w][c];
            B.unit_dot[(size_t)u * NR + tid] = t;
        }
    }
    // drain: both stages idle before the tensor memory is released
    for (int stg = 0; stg < 2; ++stg)
        if (pending[stg]) {
            if (!mbar_wait(&bar[stg], phase[stg])) ok = false;
            pending[stg] = false;
        }
    if (!ok && lane == 0) s_err = 1;
    tc::fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    if (tid == 0 && s_err) atomicExch(&P.st->error, 1);
    if (tid == 0) {
        __threadfence();
        s_last = (atomicAdd(&B.queue[1], 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        if (mode == 1) {
            __threadfence();
            if (tid < NR) {
                double t = 0.0;
                for (int q = 0; q < nunits; ++q) t += __ldcg(&B.unit_dot[(size_t)q * NR + tid]);
                B.scal[SC_PAP * NR + tid] = t;
            }
        }
        if (tid == 0) {
            B.queue[0] = 0;
            B.queue[1] = 0;
            __threadfence();
        }
    }
}

// ---- Tile SYMM on the tensor cores, asynchronous staging (32 right-hand sides)
// Same units (four tile rows of one subdomain, M = 128) and results as tile_symm_tc_kernel<32>,
// without register staging or transposes.  Every block column J of a unit arrives as raw FP32 by
// cp.async (16-byte chunks placed at their swizzled positions) into a ring of S stages:
//   * J >= I0 + 3: the stored tiles (I, J), K-major (128-byte swizzle);
//   * J <  I0:     the stored tiles (J, I) as they are, MN-major (the MMA reads A transposed;
//     128-byte swizzle with 32-byte atoms, the MN-major layout of 32-bit operands);
//   * the three mixed blocks I0 <= J < I0 + 3: a K-major panel assembled once per unit
//     (panel_kernel, before the first solve);
//   * X_J: 32 rows of x, N-contiguous, MN-major (BMN) or transposed to K-major by the CTA.
// The CTA splits the raw data in place, x = hi + lo with hi = x rounded to TF32 (the stage keeps
// hi, the low parts go to a double buffer at the same positions; with BMN = false X_J is also
// transposed there into K-major order), and one thread issues hi*hi + hi*lo + lo*hi
// (tcgen05.mma kind::tf32) and commits to the stage's mbarrier, which frees both the stage and
// the low-part buffer.  The copies of block t + S - 2 are
// in flight while block t is converted and multiplied.  Units are claimed from the work queue S - 2
// blocks ahead.  Every wait is bounded: on time-out the CTA records an error, drains its copies
// and MMAs, frees its tensor memory and returns.
namespace tc2 {
constexpr int S = 8;                         // raw stages
constexpr unsigned A_BYTES = 128 * 128;      // 128 rows x 32 FP32
constexpr unsigned B_BYTES = 32 * 128;       // 32 k-rows x 32 FP32
constexpr unsigned STAGE = A_BYTES + B_BYTES;
constexpr unsigned LOW = A_BYTES + 2 * B_BYTES;   // low parts of A; X_J high and low parts when K-major
constexpr unsigned SMEM = S * STAGE + 2 * LOW + 1024;
constexpr int RING = 8;                      // claimed units in flight (>= S - 1)
// MN-major TF32 operand: the 128-byte swizzle with 32-byte atoms (the only MN-major layout of
// 32-bit operands), rows of 128 bytes (32 MN elements) along K; in row r the 32-byte granule g sits
// at g ^ (r & 3).  32-element MN chunks LBO = 4096 bytes apart, 4-row K groups SBO = 512 bytes apart.
__device__ __forceinline__ unsigned swz_mn(int row, int chunk) {
    return (unsigned)(row * 128 + (((((chunk >> 1) ^ (row & 3)) << 1) | (chunk & 1)) << 4));
}
__device__ __forceinline__ uint64_t sdesc_mn(unsigned addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(4096 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)1 << 61);
}
// kind::tf32, M = 128, N = 32, A and B K-major (0) or MN-major (1)
__host__ __device__ constexpr uint32_t idesc(int a_mn, int b_mn) {
    return tc::idesc<32>() | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16);
}
__device__ __forceinline__ void cp16(unsigned dst, const void *src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct UnitInfo {
    int u, m, I0, tn, n, voff, fb;   // fb: first block of the unit in the CTA's block stream
    long long t0;
};
}  // namespace tc2

// K-major panels of the mixed blocks: unit u (tile rows I0 .. I0+3 of matrix m), p = 0..2, block
// column J = I0 + p: rows 32 q + r of S, columns 32 J .. 32 J + 31 (zero past the matrix)
__global__ void panel_kernel(TileSetDev ts, const int2 *units, int nunits, float *pan) {
    const int u = blockIdx.x / 3, p = blockIdx.x % 3;
    if (u >= nunits) return;
    const int m = units[u].x, I0 = 4 * units[u].y, J = I0 + p;
    const int tn = ts.mat_tn[m];
    const long long t0 = ts.mat_tile0[m];
    const float *tiles = reinterpret_cast<const float *>(ts.tiles);
    float *dst = pan + ((size_t)u * 3 + p) * 4096;
    for (int e = threadIdx.x; e < 4096; e += blockDim.x) {
        const int r = e >> 5, k = e & 31, q = r >> 5, rr = r & 31, I = I0 + q;
        float v = 0.f;
        if (J < tn && I < tn) {
            if (I <= J) v = tiles[(size_t)(t0 + (long long)I * tn - (long long)I * (I - 1) / 2 + (J - I)) * 1024 + rr * 32 + k];
            else v = tiles[(size_t)(t0 + (long long)J * tn - (long long)J * (J - 1) / 2 + (I - J)) * 1024 + k * 32 + rr];
        }
        dst[e] = v;
    }
}

template <bool BMN>
__global__ void __launch_bounds__(256, 1)
tile_symm_tc2_kernel(TileSetDev ts, DevProblem P, BlockDev B, const float *x32, const float *pan, double *out,
                     const int2 *units, int nunits, int slot, int mode) {
    pdl_enter();
    constexpr int S = tc2::S, RING = tc2::RING;
    extern __shared__ unsigned char tc2_smem[];
    __shared__ unsigned long long bar[S];
    __shared__ tc2::UnitInfo s_ring[RING];
    __shared__ unsigned s_tmem;
    __shared__ int s_nring, s_end, s_err, s_last;
    __shared__ double s_dot[8][16];
    if (mode != 0) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned base = smem_u32(tc2_smem);
    const unsigned pad = (1024u - (base & 1023u)) & 1023u;
    unsigned char *buf = tc2_smem + pad;     // 1024-byte aligned: S raw stages, then 2 low-part buffers
    const unsigned sbuf = base + pad;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(32u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_nring = 0;
        s_end = -1;
        s_err = 0;
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const unsigned tmem = s_tmem;
    const float *tiles = reinterpret_cast<const float *>(ts.tiles);
    auto tidx = [](long long t0, int tn, int a, int b) -> long long {
        return t0 + (long long)a * tn - (long long)a * (a - 1) / 2 + (b - a);
    };
    int pk = 0, pJ = 0;   // producer: ring counter of its unit, block column in the unit
    int ck = 0, cJ = 0;   // consumer
    int last_commit = -1;
    bool ok = true;
    for (int t = -(S - 2);; ++t) {
        const int pb = t + S - 2;
        if (tid == 0) {
            // claim units until block pb of the stream is covered or the queue is empty
            while (s_end < 0) {
                const int nr_ = s_nring;
                int endb = 0;
                if (nr_ > 0) endb = s_ring[(nr_ - 1) % RING].fb + s_ring[(nr_ - 1) % RING].tn;
                if (pb < endb) break;
                const int u = atomicAdd(&B.queue[0], 1);
                if (u >= nunits) {
                    s_end = endb;
                    break;
                }
                tc2::UnitInfo &N = s_ring[nr_ % RING];
                N.u = u;
                N.m = units[u].x;
                N.I0 = 4 * units[u].y;
                N.tn = ts.mat_tn[N.m];
                N.n = ts.mat_n[N.m];
                N.voff = ts.mat_voff[N.m];
                N.t0 = ts.mat_tile0[N.m];
                N.fb = endb;
                s_nring = nr_ + 1;
            }
        }
        if (!__syncthreads_and(ok)) break;
        const int end = s_end;
        if (end >= 0 && t >= end) break;
        // stage pb % S last held block t - 2 (and low-part buffer t & 1 too): its MMAs must be done
        if (t >= 2 && !mbar_wait(&bar[(t - 2) % S], (unsigned)(((t - 2) / S) & 1))) ok = false;
        if (end < 0 || pb < end) {
            const tc2::UnitInfo &U = s_ring[pk % RING];
            const int J = pJ, I0 = U.I0, tn = U.tn;
            const unsigned sa = sbuf + (unsigned)(pb % S) * tc2::STAGE, sb = sa + tc2::A_BYTES;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int q = tid + 256 * i, r = q >> 3, c = q & 7, qq = r >> 5, rr = r & 31, I = I0 + qq;
                const float *src = tiles;
                bool valid = true;
                if (J >= I0 + 3) {
                    valid = I < tn;
                    if (valid) src = tiles + (size_t)tidx(U.t0, tn, I, J) * 1024 + rr * 32 + 4 * c;
                } else if (J < I0) {
                    valid = I < tn;
                    if (valid) src = tiles + (size_t)tidx(U.t0, tn, J, I) * 1024 + rr * 32 + 4 * c;
                    tc2::cp16(sa + tc2::swz_mn(r, c), src, valid);
                    continue;
                } else {
                    src = pan + ((size_t)U.u * 3 + (J - I0)) * 4096 + r * 32 + 4 * c;
                }
                tc2::cp16(sa + tc::swz(r, c), src, valid);
            }
            {
                const int kk = tid >> 3, c = tid & 7, row = TILE * J + kk;
                const bool valid = row < U.n;
                tc2::cp16(sb + (BMN ? tc2::swz_mn(kk, c) : tc::swz(kk, c)),
                          valid ? (const void *)(x32 + (size_t)(U.voff + row) * 32 + 4 * c) : x32, valid);
            }
            if (++pJ == tn) {
                ++pk;
                pJ = 0;
            }
        }
        tc2::cp_commit();
        if (t < 0) continue;
        // block t: this thread's copies, then everyone's
        tc2::cp_wait<S - 2>();
        __syncthreads();
        const unsigned st = (unsigned)(t % S) * tc2::STAGE;
        const unsigned lo = (unsigned)S * tc2::STAGE + (unsigned)(t & 1) * tc2::LOW;
#pragma unroll
        for (int i = 0; i < 4; ++i) {   // 1024 A chunks of 16 bytes, split in place
            const unsigned off = (unsigned)(tid + 256 * i) * 16;
            tc::split_store(buf + st, buf + lo, off, *reinterpret_cast<const float4 *>(buf + st + off));
        }
        if (BMN) {
            const unsigned off = tc2::A_BYTES + (unsigned)tid * 16;
            tc::split_store(buf + st, buf + lo, off, *reinterpret_cast<const float4 *>(buf + st + off));
        } else {
            // X_J chunk (k-row kk, n = 4c .. 4c + 3) -> K-major [n][k] high and low parts
            const int kk = tid >> 3, c = tid & 7;
            const float4 v = *reinterpret_cast<const float4 *>(buf + st + tc2::A_BYTES + tc::swz(kk, c));
            const float xv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float h = tc::tf32_hi(xv[e]);
                const unsigned o = tc::swz(4 * c + e, kk >> 2) + 4u * (kk & 3);
                *reinterpret_cast<float *>(buf + lo + tc2::A_BYTES + o) = h;
                *reinterpret_cast<float *>(buf + lo + tc2::A_BYTES + tc2::B_BYTES + o) = xv[e] - h;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        const tc2::UnitInfo U = s_ring[ck % RING];
        if (tid == 0) {
            tc::fence_after();
            const bool amn = cJ < U.I0;       // stored tiles (J, I): A read transposed
            const uint32_t id = tc2::idesc(amn ? 1 : 0, BMN ? 1 : 0);
            const unsigned ahi = sbuf + st, alo = sbuf + lo;
            const unsigned bhi = BMN ? ahi + tc2::A_BYTES : alo + tc2::A_BYTES;
            const unsigned blo = BMN ? alo + tc2::A_BYTES : alo + tc2::A_BYTES + tc2::B_BYTES;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t dah = amn ? tc2::sdesc_mn(ahi + 1024u * kk) : tc::sdesc(ahi + 32u * kk);
                const uint64_t dal = amn ? tc2::sdesc_mn(alo + 1024u * kk) : tc::sdesc(alo + 32u * kk);
                const uint64_t dbh = BMN ? tc2::sdesc_mn(bhi + 1024u * kk) : tc::sdesc(bhi + 32u * kk);
                const uint64_t dbl = BMN ? tc2::sdesc_mn(blo + 1024u * kk) : tc::sdesc(blo + 32u * kk);
                tc::mma(tmem, dah, dbh, id, (cJ > 0 || kk > 0) ? 1u : 0u);
                tc::mma(tmem, dah, dbl, id, 1u);
                tc::mma(tmem, dal, dbh, id, 1u);
            }
            tc::commit(&bar[t % S]);
        }
        last_commit = t;
        if (cJ + 1 == U.tn) {
            // unit complete: accumulator -> rows of the output, dots with x per column
            if (!mbar_wait(&bar[t % S], (unsigned)((t / S) & 1))) ok = false;
            tc::fence_after();
            uint32_t r[16];
            tc::ld16(tmem + ((unsigned)(32 * (warp & 3)) << 16) + (unsigned)((warp >> 2) * 16), r);
            const int row = TILE * U.I0 + 32 * (warp & 3) + lane, c0 = (warp >> 2) * 16;
            double dl[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                dl[c] = 0.0;
                if (row < U.n && ok) {
                    const size_t o = (size_t)(U.voff + row) * 32 + c0 + c;
                    const double y = (double)__uint_as_float(r[c]);
                    out[o] = y;
                    dl[c] = (double)x32[o] * y;
                }
            }
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                double v = dl[c];
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
                if (lane == 0) s_dot[warp][c] = v;
            }
            tc::fence_before();
            __syncthreads();
            if (tid < 32) {
                const int h = tid / 16, c = tid % 16;
                double tsum = 0.0;
                for (int w = 0; w < 4; ++w) tsum += s_dot[4 * h + w][c];
                B.unit_dot[(size_t)U.u * 32 + tid] = tsum;
            }
        }
        if (++cJ == U.tn) {
            ++ck;
            cJ = 0;
        }
    }
    // drain: copies, then the MMAs of the last committed block
    tc2::cp_wait_all();
    if (last_commit >= 0 && !mbar_wait(&bar[last_commit % S], (unsigned)((last_commit / S) & 1))) ok = false;
    if (!ok && lane == 0) s_err = 1;
    tc::fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u) : "memory");
    if (tid == 0 && s_err) atomicExch(&P.st->error, 1);
    if (tid == 0) {
        __threadfence();
        s_last = (atomicAdd(&B.queue[1], 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        if (mode == 1) {
            __threadfence();
            if (tid < 32) {
                double tsum = 0.0;
                for (int q = 0; q < nunits; ++q) tsum += __ldcg(&B.unit_dot[(size_t)q * 32 + tid]);
                B.scal[SC_PAP * 32 + tid] = tsum;
            }
        }
        if (tid == 0) {
            B.queue[0] = 0;
            B.queue[1] = 0;
            __threadfence();
        }
    }
}

// ---- Tile SYMM on the tensor cores, warp-specialised (32 right-hand sides)
// Same units (four tile rows of one subdomain, M = 128) and results as tile_symm_tc_kernel<32>.
// The roles of a CTA (one per SM) hand 32-column blocks J over through a ring of NS stages (the
// bulk copies, at about 24 bytes per cycle and SM, and the ring's round-trip latency bound it):
//   * two producer lanes (warps 8 and 10, even and odd blocks: a lane's copy issue limits one): one
//     4 KB bulk copy (cp.async.bulk) of every stored tile the block needs, (I, J) for J >= I and
//     (J, I) for J < I, row-major as stored, into the tile's 4 KB slice of the stage (one 16 KB copy
//     when all four are transposed: they are adjacent in tile row J), and one 4 KB copy of the 32
//     rows of x (32 right-hand sides each);
//   * four converter warps, warp q for tile row I0 + q: read the raw tile into registers (vector
//     loads for a stored tile, transposing scalar loads for the transposed one), write its TF32
//     high part in place at the swizzled K-major position and its low part to the stage's low
//     buffer; warp q also splits columns 8q .. 8q + 7 of X_J^T (rows past the subdomain zero) into
//     the stage's X_hi | X_lo, the N = 64 operand;
//   * one MMA lane: per K step (K = 8, four per block) A_hi [X_hi | X_lo] as one N = 64 product and
//     A_lo X_hi (N = 32), tcgen05.mma kind::tf32, M = 128, into one of two FP32 accumulators of 64
//     columns in tensor memory (columns 0..31 hold hi*hi + lo*hi, 32..63 hi*lo; an MMA of N <= 128
//     takes the same time, so the stacking saves a third of the MMAs); commits free the stage and,
//     after the unit's last block, hand the accumulator to
//   * four epilogue warps (tensor-memory lane quadrants 0..3): y = the two halves summed in FP64,
//     rows to `out`; each lane keeps its column's share of x.y over the CTA's units and writes it
//     to unit_dot[4 CTA + warp] at the end.
// Units go to CTAs round-robin in the order of the unit list (longest rows first), so every role
// derives the same unit and block sequence.  Every wait is bounded and gives up at once when
// another role has given up: the CTA then records an error, drains its copies and MMAs in flight,
// frees its tensor memory and returns.  x32 carries 32 rows past the last subdomain: the copy of a
// subdomain's last block may read them (they are zeroed before use).
namespace tc3 {
constexpr int NS = 4;                            // stages
constexpr int CONV = 4, EPI = 4;                 // converter warps, epilogue warps
constexpr int PROD_WARP = CONV + EPI, MMA_WARP = CONV + EPI + 1, PROD_WARP2 = CONV + EPI + 2;
constexpr int THREADS = (CONV + EPI + 3) * 32;
constexpr unsigned A_BYTES = 128 * 128;          // 128 rows x 32 FP32
constexpr unsigned B_BYTES = 32 * 128;           // 32 rows (right-hand sides) x 32 FP32
// stage: A (raw, then high part) | A low part | X_hi | X_lo | raw x rows
constexpr unsigned ALO = A_BYTES, XS = 2 * A_BYTES, XRAW = 2 * A_BYTES + 2 * B_BYTES;
constexpr unsigned STAGE = 2 * A_BYTES + 3 * B_BYTES;
constexpr unsigned SMEM = NS * STAGE + 1024;
static_assert(NS % 2 == 0, "the two producer lanes own the even and the odd stages");
static_assert(STAGE % 1024 == 0, "stages start on 1024-byte boundaries (128-byte swizzle atoms)");
constexpr unsigned TMEM_COLS = 128;              // two accumulators of 64 columns (hi*hi + lo*hi | hi*lo)
__device__ __forceinline__ void bulk(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// bounded wait that also gives up when another role has set *abort
__device__ __forceinline__ bool wait(unsigned long long *bar, unsigned parity, volatile int *abort) {
    for (long long i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try(bar, parity)) return true;
        if (*abort) return false;
        if (i > 64) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void ld32(unsigned taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ long long tile_index(long long t0, int tn, int I, int J) {   // stored tile (I, J), I <= J
    return t0 + (long long)I * tn - (long long)I * (I - 1) / 2 + (J - I);
}
}  // namespace tc3

__global__ void __launch_bounds__(tc3::THREADS, 1)
tile_symm_tc3_kernel(TileSetDev ts, DevProblem P, BlockDev B, const float *x32, double *out, const int2 *units,
                     int nunits, int slot, int mode) {
    pdl_enter();
    constexpr int NS = tc3::NS, NR = 32;
    extern __shared__ unsigned char tc3_smem[];
    __shared__ __align__(8) unsigned long long full[NS], conv[NS], empty[NS], accf[2], acce[2];
    __shared__ unsigned s_tmem;
    __shared__ volatile int s_abort;
    __shared__ int s_last;
    __shared__ double s_red[tc3::THREADS / 32][32];
    if (mode != 0) {
        const int iter = P.st->iter_base + slot;
        if (skip_iter(P.st, iter)) return;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned base = smem_u32(tc3_smem);
    unsigned char *buf = tc3_smem + ((1024u - (base & 1023u)) & 1023u);   // 1024-byte aligned stages
    if (warp == tc3::MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(tc3::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&conv[s], tc3::CONV);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&accf[a], 1);
            mbar_init(&acce[a], tc3::EPI);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const unsigned tmem = s_tmem;
    const float *tiles = reinterpret_cast<const float *>(ts.tiles);
    bool ok = true;

    if (warp == tc3::PROD_WARP || warp == tc3::PROD_WARP2) {
        if (lane == 0) {
            const int par = (warp == tc3::PROD_WARP) ? 0 : 1;   // this lane's blocks: t % 2 == par
            long long t = 0, last[NS];
            for (int s = 0; s < NS; ++s) last[s] = -1;
            for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
                const int m = units[u].x, I0 = 4 * units[u].y, tn = ts.mat_tn[m];
                const long long t0 = ts.mat_tile0[m];
                const int nq = min(4, tn - I0);
                const float *xm = x32 + (size_t)ts.mat_voff[m] * NR;
                for (int J = 0; J < tn; ++J, ++t) {
                    if ((int)(t & 1) != par) continue;
                    const int s = (int)(t % NS);
                    if (t >= NS && !tc3::wait(&empty[s], (unsigned)(((t / NS) - 1) & 1), &s_abort)) {
                        ok = false;
                        break;
                    }
                    unsigned char *stg = buf + (size_t)s * tc3::STAGE;
                    mbar_arrive_tx(&full[s], 4096u * (unsigned)nq + tc3::B_BYTES);
                    if (J < I0) {
                        // the stored tiles (J, I0 .. I0 + nq - 1) are adjacent in tile row J
                        tc3::bulk(stg, tiles + (size_t)tc3::tile_index(t0, tn, J, I0) * (TILE * TILE), 4096u * (unsigned)nq,
                                  &full[s]);
                    } else {
                        for (int q = 0; q < nq; ++q) {
                            const int I = I0 + q;
                            const long long idx = (I <= J) ? tc3::tile_index(t0, tn, I, J) : tc3::tile_index(t0, tn, J, I);
                            tc3::bulk(stg + q * 4096, tiles + (size_t)idx * (TILE * TILE), 4096u, &full[s]);
                        }
                    }
                    tc3::bulk(stg + tc3::XRAW, xm + (size_t)TILE * J * NR, tc3::B_BYTES, &full[s]);
                    last[s] = t;
                }
            }
            if (!ok) s_abort = 1;
            // every copy this lane issued has landed before the CTA can leave (bounded waits)
            for (int s = 0; s < NS; ++s)
                if (last[s] >= 0) mbar_wait(&full[s], (unsigned)((last[s] / NS) & 1));
        }
    } else if (warp == tc3::MMA_WARP) {
        if (lane == 0) {
            constexpr uint32_t ID64 = tc::idesc<2 * NR>(), ID32 = tc::idesc<NR>();
            long long t = 0, lastc = -1;
            int k = 0;
            for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++k) {
                const int m = units[u].x, tn = ts.mat_tn[m];
                const int a = k & 1;
                if (k >= 2 && !tc3::wait(&acce[a], (unsigned)(((k >> 1) - 1) & 1), &s_abort)) {
                    ok = false;
                    break;
                }
                tc::fence_after();
                const unsigned d = tmem + (unsigned)(a * 2 * NR);
                for (int J = 0; J < tn; ++J, ++t) {
                    const int s = (int)(t % NS);
                    if (!tc3::wait(&conv[s], (unsigned)((t / NS) & 1), &s_abort)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after();
                    const unsigned a_hi = smem_u32(buf + (size_t)s * tc3::STAGE), a_lo = a_hi + tc3::ALO,
                                   b_hi = a_hi + tc3::XS;   // X_lo follows X_hi: rows 32..63 of B
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const unsigned off = 32u * kk;
                        tc::mma(d, tc::sdesc(a_hi + off), tc::sdesc(b_hi + off), ID64, (J > 0 || kk > 0) ? 1u : 0u);
                        tc::mma(d, tc::sdesc(a_lo + off), tc::sdesc(b_hi + off), ID32, 1u);
                    }
                    tc::commit(&empty[s]);
                    if (J == tn - 1) tc::commit(&accf[a]);
                    lastc = t;
                }
            }
            if (!ok) s_abort = 1;
            // every MMA issued has completed before the stages and the tensor memory are released
            if (lastc >= 0) mbar_wait(&empty[lastc % NS], (unsigned)((lastc / NS) & 1));
        }
    } else if (warp < tc3::CONV) {
        const int q = warp;
        long long t = 0;
        for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
            const int m = units[u].x, I = 4 * units[u].y + q, tn = ts.mat_tn[m], n = ts.mat_n[m];
            for (int J = 0; J < tn; ++J, ++t) {
                const int s = (int)(t % NS);
                ok = __all_sync(FULL, tc3::wait(&full[s], (unsigned)((t / NS) & 1), &s_abort));
                if (!ok) break;
                unsigned char *stg = buf + (size_t)s * tc3::STAGE;
                // X_J^T: columns 8q .. 8q + 7 (chunks 2q, 2q + 1) of every right-hand side `lane`
                {
                    const float *xr = reinterpret_cast<const float *>(stg + tc3::XRAW);
                    const int rows = n - TILE * J;   // rows of the block inside the subdomain
                    float4 xv[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int c = 2 * q + h;
                        xv[h].x = (4 * c + 0 < rows) ? xr[(4 * c + 0) * NR + lane] : 0.f;
                        xv[h].y = (4 * c + 1 < rows) ? xr[(4 * c + 1) * NR + lane] : 0.f;
                        xv[h].z = (4 * c + 2 < rows) ? xr[(4 * c + 2) * NR + lane] : 0.f;
                        xv[h].w = (4 * c + 3 < rows) ? xr[(4 * c + 3) * NR + lane] : 0.f;
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        tc::split_store(stg + tc3::XS, stg + tc3::XS + tc3::B_BYTES, tc::swz(lane, 2 * q + h), xv[h]);
                }
                if (I < tn) {   // rows of a missing tile row only reach accumulator rows that are not read
                    unsigned char *hi = stg + q * 4096, *lo = stg + tc3::ALO + q * 4096;
                    float4 v[8], h4[8];
                    unsigned off[8];
                    if (I <= J) {
                        const float4 *src = reinterpret_cast<const float4 *>(hi);
#pragma unroll
                        for (int it = 0; it < 8; ++it) v[it] = src[it * 32 + lane];
#pragma unroll
                        for (int it = 0; it < 8; ++it) {
                            const int p = it * 32 + lane;
                            off[it] = tc::swz(p >> 3, p & 7);
                        }
                    } else {
                        // stored tile (J, I): row `lane` of S_IJ is column `lane` of the stored tile
                        const float *src = reinterpret_cast<const float *>(hi);
#pragma unroll
                        for (int it = 0; it < 8; ++it) {
                            v[it] = make_float4(src[(4 * it + 0) * 32 + lane], src[(4 * it + 1) * 32 + lane],
                                                src[(4 * it + 2) * 32 + lane], src[(4 * it + 3) * 32 + lane]);
                            off[it] = tc::swz(lane, it);
                        }
                    }
                    __syncwarp();
                    // high parts in place, low parts to the stage's low buffer
#pragma unroll
                    for (int it = 0; it < 8; ++it) {
                        h4[it].x = tc::tf32_hi(v[it].x);
                        h4[it].y = tc::tf32_hi(v[it].y);
                        h4[it].z = tc::tf32_hi(v[it].z);
                        h4[it].w = tc::tf32_hi(v[it].w);
                        *reinterpret_cast<float4 *>(hi + off[it]) = h4[it];
                        *reinterpret_cast<float4 *>(lo + off[it]) =
                            make_float4(v[it].x - h4[it].x, v[it].y - h4[it].y, v[it].z - h4[it].z, v[it].w - h4[it].w);
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&conv[s]);
            }
        }
        if (!ok && lane == 0) s_abort = 1;
    } else {
        // epilogue: warp 4 + e reads tensor-memory lanes 32 e .. 32 e + 31 (rows of tile row I0 + e)
        const int e = warp - tc3::CONV;
        int k = 0;
        double dot = 0.0;   // lane l: this warp's share of x_l . y_l over the CTA's units
        for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++k) {
            const int m = units[u].x, I0 = 4 * units[u].y;
            const int n = ts.mat_n[m], voff = ts.mat_voff[m];
            const int a = k & 1;
            ok = __all_sync(FULL, tc3::wait(&accf[a], (unsigned)((k >> 1) & 1), &s_abort));
            if (!ok) break;
            tc::fence_after();
            uint32_t r[32], r2[32];
            tc3::ld32(tmem + ((unsigned)(32 * e) << 16) + (unsigned)(a * 2 * NR), r);
            tc3::ld32(tmem + ((unsigned)(32 * e) << 16) + (unsigned)(a * 2 * NR + NR), r2);
            tc::fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[a]);
            const int row = TILE * I0 + 32 * e + lane;
            double v[32];
            if (row < n) {
                const float4 *xr = reinterpret_cast<const float4 *>(x32 + (size_t)(voff + row) * NR);
                double2 *orow = reinterpret_cast<double2 *>(out + (size_t)(voff + row) * NR);
#pragma unroll
                for (int c4 = 0; c4 < 8; ++c4) {
                    const float4 xv = xr[c4];
                    const double y0 = (double)__uint_as_float(r[4 * c4 + 0]) + (double)__uint_as_float(r2[4 * c4 + 0]),
                                 y1 = (double)__uint_as_float(r[4 * c4 + 1]) + (double)__uint_as_float(r2[4 * c4 + 1]),
                                 y2 = (double)__uint_as_float(r[4 * c4 + 2]) + (double)__uint_as_float(r2[4 * c4 + 2]),
                                 y3 = (double)__uint_as_float(r[4 * c4 + 3]) + (double)__uint_as_float(r2[4 * c4 + 3]);
                    orow[2 * c4] = make_double2(y0, y1);
                    orow[2 * c4 + 1] = make_double2(y2, y3);
                    v[4 * c4 + 0] = (double)xv.x * y0;
                    v[4 * c4 + 1] = (double)xv.y * y1;
                    v[4 * c4 + 2] = (double)xv.z * y2;
                    v[4 * c4 + 3] = (double)xv.w * y3;
                }
            } else {
#pragma unroll
                for (int c = 0; c < 32; ++c) v[c] = 0.0;
            }
            // reduce-scatter over the lanes: afterwards lane l holds the warp's sum of column l
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                const bool upper = (lane & o) != 0;
#pragma unroll
                for (int i = 0; i < o; ++i) {
                    const double send = upper ? v[i] : v[i + o];
                    const double keep = upper ? v[i + o] : v[i];
                    v[i] = keep + __shfl_xor_sync(FULL, send, o);
                }
            }
            dot += v[0];
        }
        if (!ok && lane == 0) s_abort = 1;
        B.unit_dot[((size_t)blockIdx.x * tc3::EPI + e) * NR + lane] = dot;
        __threadfence();
    }
    if (!ok) atomicExch(&P.st->error, 1);
    tc::fence_before();
    __syncthreads();
    if (warp == tc3::MMA_WARP) {
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc3::TMEM_COLS)
                     : "memory");
    }
    if (tid == 0) {
        __threadfence();
        s_last = (atomicAdd(&B.queue[1], 1) == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        if (mode == 1) {
            // p.Ap of every column: the CTAs' partials, summed in a fixed order by all warps
            __threadfence();
            double tsum = 0.0;
            for (int q = warp; q < tc3::EPI * (int)gridDim.x; q += tc3::THREADS / 32)
                tsum += __ldcg(&B.unit_dot[(size_t)q * NR + lane]);
            s_red[warp][lane] = tsum;
            __syncthreads();
            if (tid < NR) {
                double t2 = 0.0;
                for (int w = 0; w < tc3::THREADS / 32; ++w) t2 += s_red[w][tid];
                B.scal[SC_PAP * NR + tid] = t2;
            }
        }
        if (tid == 0) {
            B.queue[0] = 0;
            B.queue[1] = 0;
            __threadfence();
        }
    }
}

// ---- Hybrid Total FETI cluster correction for nr columns ([row][rhs] layout)
// z_i = V_i^T x_i: one warp per column of V_i, lane = (row group, rhs)
__global__ void bhyb_vt_kernel(DevProblem P, HybDev H, BlockDev B, const double *x, double *z, int slot, int cond) {
    pdl_enter();
    if (hyb_skip(P, slot, cond)) return;
    const int nr = B.nr, lg = B.lg;
    const int d = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int j = lane & (nr - 1), g = lane >> lg, ng = 32 >> lg;
    const int e0 = P.loff[d], ni = P.loff[d + 1] - e0;
    const int z0 = H.zof[d], m = H.zof[d + 1] - z0;
    const double *V = H.V + H.voff[d];
    for (int c = wid; c < m; c += nw) {
        const double *col = V + (size_t)c * ni;
        double s = 0.0;
        for (int r = g; r < ni; r += ng) s += col[r] * x[(size_t)(e0 + r) * nr + j];
        for (int o = 16; o >= nr; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if (lane < nr) z[(size_t)(z0 + c) * nr + j] = s;
    }
}

// w_c = M_c z_c for nr columns; grid (ncl, row blocks); dot: per column p.Ap totals to correct
__global__ void __launch_bounds__(256) bhyb_m_kernel(DevProblem P, HybDev H, BlockDev B, const double *z, double *w,
                                                     int slot, int cond, double *dot, double *part, int *done) {
    pdl_enter();
    if (hyb_skip(P, slot, cond)) return;
    extern __shared__ double hz[];            // nc x nr
    __shared__ double s_cols[256];
    __shared__ int s_last;
    const int nr = B.nr, lg = B.lg;
    const int c = blockIdx.x;
    const int nc = H.cof[c + 1] - H.cof[c];
    for (int i = threadIdx.x; i < nc * nr; i += blockDim.x) hz[i] = 0.0;
    __syncthreads();
    for (int q = H.mem_ptr[c]; q < H.mem_ptr[c + 1]; ++q) {
        const int d = H.mem[q];
        const int z0 = H.zof[d], cnt = (H.zof[d + 1] - z0) * nr;
        for (int t = threadIdx.x; t < cnt; t += blockDim.x)
            hz[H.vmap[z0 + (t >> lg)] * nr + (t & (nr - 1))] += z[(size_t)z0 * nr + t];
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int j = lane & (nr - 1), g = lane >> lg, ng = 32 >> lg;
    const int r0 = blockIdx.y * HM_ROWS, r1 = min(nc, r0 + HM_ROWS);
    const double *M = H.M + H.mof[c];
    double zw = 0.0;
    for (int r = r0 + wid; r < r1; r += nw) {
        const double *col = M + (size_t)r * nc;
        double s = 0.0;
        for (int k = g; k < nc; k += ng) s += col[k] * hz[k * nr + j];
        for (int o = 16; o >= nr; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if (lane < nr) {
            w[(size_t)(H.cof[c] + r) * nr + j] = s;
            zw += s * hz[r * nr + j];
        }
    }
    if (dot == nullptr) return;
    // per-column partial of this CTA: lane j < nr of every warp holds column j
    s_cols[threadIdx.x] = (lane < nr) ? zw : 0.0;
    __syncthreads();
    const int cta = blockIdx.y * gridDim.x + blockIdx.x, ncta = gridDim.x * gridDim.y;
    if (threadIdx.x < nr) {
        double t = 0.0;
        for (int q = 0; q < nw; ++q) t += s_cols[q * 32 + threadIdx.x];
        part[(size_t)cta * nr + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(done, 1) == ncta - 1);
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (threadIdx.x < nr) {
            double t = 0.0;
            for (int q = 0; q < ncta; ++q) t += __ldcg(&part[(size_t)q * nr + threadIdx.x]);
            dot[threadIdx.x] -= t;
        }
        if (threadIdx.x == 0) *done = 0;
    }
}

// y_i -= V_i w_{c(i)} for nr columns: one thread per (row, rhs)
__global__ void bhyb_v_kernel(DevProblem P, HybDev H, BlockDev B, const double *w, double *y, int slot, int cond) {
    pdl_enter();
    if (hyb_skip(P, slot, cond)) return;
    extern __shared__ double wl[];            // m_i x nr
    const int nr = B.nr, lg = B.lg;
    const int d = blockIdx.x;
    const int e0 = P.loff[d], ni = P.loff[d + 1] - e0;
    const int z0 = H.zof[d], m = H.zof[d + 1] - z0;
    const int cb = H.cof[H.sub_cl[d]];
    for (int t = threadIdx.x; t < m * nr; t += blockDim.x)
        wl[t] = w[(size_t)(cb + H.vmap[z0 + (t >> lg)]) * nr + (t & (nr - 1))];
    __syncthreads();
    const double *V = H.V + H.voff[d];
    for (int t = threadIdx.x; t < ni * nr; t += blockDim.x) {
        const int r = t >> lg, jj = t & (nr - 1);
        double s = 0.0;
        for (int c = 0; c < m; ++c) s += V[(size_t)c * ni + r] * wl[c * nr + jj];
        y[(size_t)e0 * nr + t] -= s;
    }
}

__global__ void bchunk_end_kernel(DevProblem P, int chunk) {
    pdl_enter();
    if (threadIdx.x == 0 && blockIdx.x == 0) P.st->iter_base += chunk;
}

// ---- right-hand sides and primal recovery for nr columns (column-major local-DOF blocks)
__global__ void bsplit_rhs_kernel(const double *rhs, int nc, const int *gdof, const double *invm, double *f, int ntot,
                                  int nr) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)ntot * nr) return;
    const int j = (int)(i / ntot), k = (int)(i % ntot);
    const int gd = gdof[k];
    f[i] = gd >= 0 ? rhs[(size_t)j * nc + gd] * invm[k] : 0.0;
}

__global__ void bbvec_kernel(DevProblem P, BlockDev B, const int *rdof, const double *rsign, const double *rc,
                             const double *kf, int ntot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nr = B.nr;
    if (i >= P.NL * nr) return;
    const int e = (i >> B.lg), j = (i & (nr - 1));
    const double *k = kf + (size_t)j * ntot;
    double b = rsign[e] * k[rdof[e]] - rc[e];
    const int q = P.partner[e];
    if (q >= 0) b += rsign[q] * k[rdof[q]] - rc[q];
    B.bL[i] = b;
}

__global__ void bevec_kernel(DevProblem P, BlockDev B, const int *doff, const int *rofs, const double *R,
                             const double *f, int ntot) {
    __shared__ double sh[32 * KMAX];
    const int d = blockIdx.x % P.nd, j = blockIdx.x / P.nd;
    const int n = doff[d + 1] - doff[d], nk = P.kof[d + 1] - P.kof[d];
    const double *Rd = R + rofs[d];
    const double *fj = f + (size_t)j * ntot;
    double acc[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) acc[k] = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double fi = fj[doff[d] + i];
        for (int k = 0; k < nk; ++k) acc[k] += Rd[(size_t)k * n + i] * fi;
    }
    block_sum_k(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < nk; ++k) B.e[(size_t)(P.kof[d] + k) * B.nr + j] = -acc[k];
}

__global__ void bprimal_rhs_kernel(DevProblem P, BlockDev B, const int *tdof_g, const double *rsign, const double *f,
                                   double *g, int ntot) {
    const int nr = B.nr;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)ntot * nr;
         i += (long long)gridDim.x * blockDim.x)
        g[i] = f ? f[i] : 0.0;
}

__global__ void bprimal_bt_kernel(DevProblem P, BlockDev B, const int *tdof_g, const double *rsign, double *g,
                                  int ntot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nr = B.nr;
    if (i >= P.NT * nr) return;
    const int t = (i >> B.lg), j = (i & (nr - 1));
    double s = 0.0;
    for (int q = P.trow_ptr[t]; q < P.trow_ptr[t + 1]; ++q) {
        const int e = P.trow_idx[q];
        s += rsign[e] * B.x[(size_t)e * nr + j];
    }
    g[(size_t)j * ntot + tdof_g[t]] -= s;
}

__global__ void bprimal_merge_kernel(DevProblem P, BlockDev B, const int *doff, const int *rofs, const double *R,
                                     const double *u, const int *gdof, const double *invm, double *sol, int nc,
                                     int ntot) {
    const int d = blockIdx.x % P.nd, j = blockIdx.x / P.nd;
    const int n = doff[d + 1] - doff[d], nk = P.kof[d + 1] - P.kof[d];
    const double *Rd = R + rofs[d];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double val = u[(size_t)j * ntot + doff[d] + i];
        for (int k = 0; k < nk; ++k) val += Rd[(size_t)k * n + i] * B.alpha[(size_t)(P.akof[d] + k) * B.nr + j];
        const int gd = gdof[doff[d] + i];
        if (gd >= 0) atomicAdd(&sol[(size_t)j * nc + gd], val * invm[doff[d] + i]);
    }
}

}  // namespace
}  // namespace feti

// =============================================================================================
// Block solver host side
namespace feti {

void GpuSolver::Impl::ensure_block(int nr) {
    if (blk.nr == nr) return;
    if (blk.graph) { cudaGraphExecDestroy(blk.graph); blk.graph = nullptr; }
    const int NL = P.NL, NT = P.NT, nK = P.nK, nd = P.nd;
    BlockDev &B = blk.B;
    B.nr = nr;
    B.lg = __builtin_ctz(nr);
    B.x = alloc<double>((size_t)NL * nr); B.r = alloc<double>((size_t)NL * nr); B.w = alloc<double>((size_t)NL * nr);
    B.z = alloc<double>((size_t)NL * nr); B.y = alloc<double>((size_t)NL * nr); B.p = alloc<double>((size_t)NL * nr);
    B.Ap = alloc<double>((size_t)NL * nr); B.Ax = alloc<double>((size_t)NL * nr); B.bL = alloc<double>((size_t)NL * nr);
    // 32 rows past the last subdomain: the warp-specialised tensor-core SYMM copies whole 32-row blocks
    B.p32 = alloc<float>((size_t)(NL + TILE) * nr);
    B.uT = alloc<double>((size_t)NT * nr); B.vT = alloc<double>((size_t)NT * nr);
    // alpha carries KS zero rows past nK for the fixed-width G^T alpha loads
    B.d = alloc<double>((size_t)P.nP * nr); B.alpha = alloc<double>((size_t)(nK + P.KS) * nr);
    B.e = alloc<double>((size_t)P.nP * nr);
    CUDA_CHECK(cudaMemset(B.alpha, 0, sizeof(double) * (size_t)(nK + P.KS) * nr));
    // persistent grid of the flat block kernels: rows of all subdomains, UNR per thread in flight
    blk.flat_grid =
        std::max(1, std::min(nsm * FLAT_MIN_BLOCKS, (int)(((long long)NL * nr + 256LL * UNR - 1) / (256LL * UNR))));
    B.part = alloc<double>((size_t)2 * std::max(nd, blk.flat_grid) * nr);
    B.scal = alloc<double>((size_t)SC_COUNT * nr);
    B.rho_hist = alloc<double>((size_t)(opt.max_iterations + 64) * nr);
    B.tol = alloc<double>(nr); B.rmax = alloc<double>(nr); B.last_norm = alloc<double>(nr);
    B.conv = alloc<int>(nr);
    B.done = alloc<int>(DONE_COUNT);
    B.queue = alloc<int>(2);
    CUDA_CHECK(cudaMemset(B.done, 0, sizeof(int) * DONE_COUNT));
    CUDA_CHECK(cudaMemset(B.queue, 0, sizeof(int) * 2));
    CUDA_CHECK(cudaMemset(B.p, 0, sizeof(double) * NL * nr));
    // SYMM work units (subdomain, tile row), longest rows first
    std::vector<int2> units;
    const std::vector<int> &tn = F64.h_tn;
    std::vector<int> order(tn.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return tn[a] > tn[b]; });
    for (int m : order)
        for (int I = 0; I < tn[m]; ++I) units.push_back(make_int2(m, I));
    blk.units = upload(units);
    blk.nunits = (int)units.size();
    // tensor-core SYMM units: four tile rows each (M = 128)
    std::vector<int2> units4;
    for (int m : order)
        for (int I4 = 0; 4 * I4 < tn[m]; ++I4) units4.push_back(make_int2(m, I4));
    blk.units4 = upload(units4);
    blk.nunits4 = (int)units4.size();
    blk.pan = nullptr;   // rebuilt for these units at the first asynchronous tensor-core SYMM
    // per-unit dot products: one per unit, or four (one per epilogue warp) for the tensor-core units
    size_t max_units = std::max(units.size(), 4 * units4.size());
    if (opt.precond == PREC_DIRICHLET) {
        // SYMM units of the Dirichlet blocks S_dir (T space)
        std::vector<int2> du;
        const std::vector<int> &dtn = Dir.h_tn;
        std::vector<int> dorder(dtn.size());
        std::iota(dorder.begin(), dorder.end(), 0);
        std::stable_sort(dorder.begin(), dorder.end(), [&](int a, int b) { return dtn[a] > dtn[b]; });
        for (int m : dorder)
            for (int I = 0; I < dtn[m]; ++I) du.push_back(make_int2(m, I));
        blk.dunits = upload(du);
        blk.ndunits = (int)du.size();
        max_units = std::max(max_units, du.size());
    }
    B.unit_dot = alloc<double>(max_units * nr);
    blk.rhs = alloc<double>((size_t)std::max(1, n_caller) * nr);
    blk.sol = alloc<double>((size_t)std::max(1, n_caller) * nr);
    blk.f = alloc<double>((size_t)ntot * nr);
    blk.kf = alloc<double>((size_t)ntot * nr);
    blk.g = alloc<double>((size_t)ntot * nr);
    blk.zk = alloc<double>((size_t)ntot * nr);
    if (hybrid) {
        FETI_CHECK(sizeof(double) * (size_t)H.max_nc * nr <= 200 * 1024 &&
                       sizeof(double) * (size_t)hyb_max_m * nr <= 200 * 1024,
                   "FETI4ISolveMulti: a cluster's corner problem is too large for this many right-hand sides");
        int nz = 0, ncv = 0;
        CUDA_CHECK(cudaMemcpy(&nz, H.zof + P.nd, sizeof(int), cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(&ncv, H.cof + H.ncl, sizeof(int), cudaMemcpyDeviceToHost));
        bh_z = alloc<double>((size_t)nz * nr);
        bh_w = alloc<double>((size_t)ncv * nr);
        bh_part = alloc<double>((size_t)H.ncl * hyb_rows * nr);
        bh_done = alloc<int>(1);
        CUDA_CHECK(cudaMemset(bh_done, 0, sizeof(int)));
        cudaFuncSetAttribute(bhyb_m_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(bhyb_v_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    }
    blk.nr = nr;
}

void GpuSolver::Impl::launch_block_hybrid(const double *x, double *y, int slot, int cond, double *dot) {
    if (!hybrid) return;
    const int nr = blk.nr;
    launch_pdl(bhyb_vt_kernel, dim3(P.nd), dim3(256), 0, stream, P, H, blk.B, x, bh_z, slot, cond);
    launch_pdl(bhyb_m_kernel, dim3(H.ncl, hyb_rows), dim3(256), sizeof(double) * (size_t)H.max_nc * nr, stream, P, H,
               blk.B, bh_z, bh_w, slot, cond, dot, bh_part, bh_done);
    launch_pdl(bhyb_v_kernel, dim3(P.nd), dim3(256), sizeof(double) * (size_t)hyb_max_m * nr, stream, P, H, blk.B, bh_w,
               y, slot, cond);
}

// persistent launch: as many CTAs as are resident at once (they drain the unit queue)
template <int PR, int NR, int SRC>
static void symm_launch(int nsm, int ncta, size_t sm, cudaStream_t st, TileSetDev td, DevProblem P, BlockDev B,
                        const double *x64, const float *x32, double *out, const int2 *units, int nunits, int slot,
                        int mode) {
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaFuncSetAttribute(tile_symm_kernel<PR, NR, SRC>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        cudaFuncSetAttribute(tile_symm_kernel<PR, NR, SRC>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        int b = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, tile_symm_kernel<PR, NR, SRC>, 256, sm) != cudaSuccess ||
            b < 1)
            b = 1;
        per_sm = b;
    }
    const int grid = std::max(1, std::min(ncta, nsm * per_sm));
    launch_pdl(tile_symm_kernel<PR, NR, SRC>, dim3(grid), dim3(256), sm, st, td, P, B, x64, x32, out, units, nunits, slot,
               mode);
}

// w and u_T of the block PCG in one kernel (bwu_flat2_kernel); FETI4I_BLOCK_BWU=0 runs the two
// kernels it replaces
static bool bwu_enabled() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_BLOCK_BWU");
        return !(e && e[0] == '0');
    }();
    return on;
}

static bool symm_mma_enabled() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_SYMM_MMA");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <int NR>
static void symm_mma_launch(int nsm, int ncta, cudaStream_t st, TileSetDev td, DevProblem P, BlockDev B,
                            const double *x64, double *out, const int2 *units, int nunits, int slot, int mode) {
    static int per_sm = 0;
    if (per_sm == 0) {
        int b = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, tile_symm_mma_kernel<NR>, 256, 0) != cudaSuccess || b < 1)
            b = 1;
        per_sm = b;
    }
    const int grid = std::max(1, std::min(ncta, nsm * per_sm));
    launch_pdl(tile_symm_mma_kernel<NR>, dim3(grid), dim3(256), 0, st, td, P, B, x64, out, units, nunits, slot, mode);
}

// The asynchronous variant is opt-in (FETI4I_SYMM_TC2=1): on the heat workload of 512 subdomains it
// measured 71.1 ms per batch of 32 load cases against 57.1 ms with tile_symm_tc_kernel<32>.
static bool symm_tc2_enabled() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_SYMM_TC2");
        return e && e[0] == '1';
    }();
    return on;
}

// The warp-specialised tensor-core SYMM (tile_symm_tc3_kernel) serves 32 right-hand sides unless
// FETI4I_SYMM_TC3=0 selects tile_symm_tc_kernel<32>.
static bool symm_tc3_enabled() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_SYMM_TC3");
        return !(e && e[0] == '0');
    }();
    return on;
}

static void symm_tc3_launch(int nsm, cudaStream_t st, TileSetDev td, DevProblem P, BlockDev B, const float *x32,
                            double *out, const int2 *units, int nunits, int slot, int mode) {
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(tile_symm_tc3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tc3::SMEM));
        attr = true;
    }
    // one CTA per SM (its shared memory); CTAs never wait for one another
    const int grid = std::max(1, std::min(nunits, nsm));
    launch_pdl(tile_symm_tc3_kernel, dim3(grid), dim3(tc3::THREADS), (size_t)tc3::SMEM, st, td, P, B, x32, out, units,
               nunits, slot, mode);
}

static bool symm_tc2_bmn() {
    static const bool on = [] {
        const char *e = getenv("FETI4I_TC2_BMN");
        return !(e && e[0] == '0');
    }();
    return on;
}

static void symm_tc2_launch(int nsm, int nunits, cudaStream_t st, TileSetDev td, DevProblem P, BlockDev B,
                            const float *x32, const float *pan, double *out, const int2 *units, int slot, int mode) {
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(tile_symm_tc2_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tc2::SMEM));
        CUDA_CHECK(cudaFuncSetAttribute(tile_symm_tc2_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tc2::SMEM));
        attr = true;
    }
    const int grid = std::max(1, std::min(nunits, nsm));
    if (symm_tc2_bmn())
        launch_pdl(tile_symm_tc2_kernel<true>, dim3(grid), dim3(256), (size_t)tc2::SMEM, st, td, P, B, x32, pan, out,
                   units, nunits, slot, mode);
    else
        launch_pdl(tile_symm_tc2_kernel<false>, dim3(grid), dim3(256), (size_t)tc2::SMEM, st, td, P, B, x32, pan, out,
                   units, nunits, slot, mode);
}

template <int NR>
static void symm_tc_launch(int nsm, int nunits, cudaStream_t st, TileSetDev td, DevProblem P, BlockDev B,
                           const float *x32, double *out, const int2 *units, int slot, int mode) {
    constexpr size_t sm = 2 * (2 * 128 * 128 + 2 * NR * 128) + 1024;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(tile_symm_tc_kernel<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaFuncSetAttribute(tile_symm_tc_kernel<NR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        attr = true;
    }
    // two CTAs per SM fit (registers and shared memory); CTAs never wait for one another, so a
    // CTA that is not co-resident only starts later
    const int grid = std::max(1, std::min(nunits, nsm * 2));
    launch_pdl(tile_symm_tc_kernel<NR>, dim3(grid), dim3(tc::THREADS), sm, st, td, P, B, x32, out, units, nunits, slot, mode);
}

void GpuSolver::Impl::launch_symm(const TileSetHost &T, bool src32, const double *x64, const float *x32, double *out,
                                  int slot, int mode) {
    const int nr = blk.nr;
    const bool dir = &T == &Dir;
    const int2 *units = dir ? blk.dunits : blk.units;
    const int nunits = dir ? blk.ndunits : blk.nunits;
    if (!dir && opt.symm_tensor && T.prec == SCHUR_FP32 && src32 && nr == 32 && symm_tc3_enabled() &&
        !symm_tc2_enabled()) {
        symm_tc3_launch(nsm, stream, T.dev(), P, blk.B, x32, out, blk.units4, blk.nunits4, slot, mode);
        CUDA_CHECK(cudaGetLastError());
        return;
    }
    if (!dir && opt.symm_tensor && T.prec == SCHUR_FP32 && src32 && nr == 32 && symm_tc2_enabled()) {
        TileSetDev td = T.dev();
        FETI_CHECK(blk.pan != nullptr, "internal: tensor-core SYMM panels not built");
        symm_tc2_launch(nsm, blk.nunits4, stream, td, P, blk.B, x32, blk.pan, out, blk.units4, slot, mode);
        CUDA_CHECK(cudaGetLastError());
        return;
    }
    if (!dir && opt.symm_tensor && T.prec == SCHUR_FP32 && src32 && nr >= 8) {
        TileSetDev td = T.dev();
        switch (nr) {
        case 8: symm_tc_launch<8>(nsm, blk.nunits4, stream, td, P, blk.B, x32, out, blk.units4, slot, mode); break;
        case 16: symm_tc_launch<16>(nsm, blk.nunits4, stream, td, P, blk.B, x32, out, blk.units4, slot, mode); break;
        default: symm_tc_launch<32>(nsm, blk.nunits4, stream, td, P, blk.B, x32, out, blk.units4, slot, mode); break;
        }
        CUDA_CHECK(cudaGetLastError());
        return;
    }
    const size_t TB = (size_t)TILE * TILE * (T.prec == SCHUR_FP64 ? 8 : 4);
    const size_t sm = 8 * TB;
    const int ncta = (nunits + 7) / 8;
    TileSetDev td = T.dev();
    if (T.prec == SCHUR_FP64 && nr >= 8 && symm_mma_enabled()) {
        switch (nr) {
        case 8: symm_mma_launch<8>(nsm, ncta, stream, td, P, blk.B, x64, out, units, nunits, slot, mode); break;
        case 16: symm_mma_launch<16>(nsm, ncta, stream, td, P, blk.B, x64, out, units, nunits, slot, mode); break;
        default: symm_mma_launch<32>(nsm, ncta, stream, td, P, blk.B, x64, out, units, nunits, slot, mode); break;
        }
        CUDA_CHECK(cudaGetLastError());
        return;
    }
    FETI_CHECK(T.prec != SCHUR_BF16, "FETI4I: the multi right-hand-side solve supports FP64 and FP32 Schur storage");
#define SYMM(PR, NR_, S) symm_launch<PR, NR_, S>(nsm, ncta, sm, stream, td, P, blk.B, x64, x32, out, units, nunits, slot, mode)
#define SYMM_NR(PR, S)                       \
    switch (nr) {                            \
    case 4: SYMM(PR, 4, S); break;           \
    case 8: SYMM(PR, 8, S); break;           \
    case 16: SYMM(PR, 16, S); break;         \
    default: SYMM(PR, 32, S); break;         \
    }
    if (T.prec == SCHUR_FP64) { SYMM_NR(SCHUR_FP64, 0) }
    else if (src32) { SYMM_NR(SCHUR_FP32, 1) }
    else { SYMM_NR(SCHUR_FP32, 0) }
#undef SYMM_NR
#undef SYMM
    CUDA_CHECK(cudaGetLastError());
}

void GpuSolver::Impl::launch_block_iteration(int slot) {
    const int nd = P.nd;
    const int cgrid = (P.nK + CR - 1) / CR;
    BlockDev &B = blk.B;
    const bool mixed = opt.schur_precision != SCHUR_FP64;
    if (mixed) {
        launch_symm(F64, false, B.x, nullptr, B.Ax, slot, 3);
        launch_block_hybrid(B.x, B.Ax, slot, 3, nullptr);
        launch_pdl(br0_kernel, dim3(nd), dim3(TPB), 0, stream, P, B, 1, slot);
    }
    launch_pdl(bcoarse_kernel, dim3(cgrid), dim3(256), 0, stream, P, B, B.d, B.alpha, slot, 1);
    const int fgrid = blk.flat_grid;
    // the T-space gather has no register pressure (50 registers): twice the CTAs of the capped kernels
    const int ugrid = 2 * blk.flat_grid;
#define BW(PC)                                                                              \
    switch (P.KS) {                                                                         \
    case 1: launch_pdl(bw_flat2_kernel<PC, 1>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break;  \
    case 6: launch_pdl(bw_flat2_kernel<PC, 6>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break;  \
    default: launch_pdl(bw_flat2_kernel<PC, 0>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break; \
    }
#define BWU(PC)                                                                              \
    switch (P.KS) {                                                                          \
    case 1: launch_pdl(bwu_flat2_kernel<PC, 1>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break;  \
    case 6: launch_pdl(bwu_flat2_kernel<PC, 6>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break;  \
    default: launch_pdl(bwu_flat2_kernel<PC, 0>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break; \
    }
    const bool fused = bwu_enabled();
    switch (opt.precond) {
    case PREC_NONE: BW(PREC_NONE) break;
    case PREC_LUMPED:
        if (fused) { BWU(PREC_LUMPED) }
        else {
            BW(PREC_LUMPED)
            launch_pdl(bu_flat_kernel<PREC_LUMPED>, dim3(ugrid), dim3(256), 0, stream, P, B, slot);
        }
        launch_pdl(bell_flat2_kernel, dim3(fgrid), dim3(256), 0, stream, P, B, slot);
        break;
    case PREC_DIRICHLET:
        // u_T = B^T W w, then v_T = S_dir u_T (FP64 SYMM over the Dirichlet blocks)
        if (fused) { BWU(PREC_LUMPED) }
        else {
            BW(PREC_WEIGHT)
            launch_pdl(bu_flat_kernel<PREC_LUMPED>, dim3(ugrid), dim3(256), 0, stream, P, B, slot);
        }
        launch_symm(Dir, false, B.uT, nullptr, B.vT, slot, 2);
        break;
    default:
        if (fused) { BWU(PREC_WEIGHT) }
        else {
            BW(PREC_WEIGHT)
            launch_pdl(bu_flat_kernel<PREC_WEIGHT>, dim3(ugrid), dim3(256), 0, stream, P, B, slot);
        }
        break;
    }
#undef BWU
#undef BW
    if (opt.precond != PREC_NONE) {
        switch (P.KS) {
        case 1: launch_pdl(bz_kernel<1>, dim3(nd), dim3(TPBB), 0, stream, P, B, slot); break;
        case 6: launch_pdl(bz_kernel<6>, dim3(nd), dim3(TPBB), 0, stream, P, B, slot); break;
        default: launch_pdl(bz_kernel<0>, dim3(nd), dim3(TPBB), 0, stream, P, B, slot); break;
        }
        launch_pdl(bcoarse_kernel, dim3(cgrid), dim3(256), 0, stream, P, B, B.d, B.alpha, slot, 1);
        switch (P.KS) {
        case 1: launch_pdl(by_flat2_kernel<1>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break;
        case 6: launch_pdl(by_flat2_kernel<6>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break;
        default: launch_pdl(by_flat2_kernel<0>, dim3(fgrid), dim3(256), 0, stream, P, B, slot); break;
        }
    }
    launch_pdl(bp_kernel, dim3(blk.flat_grid), dim3(256), 0, stream, P, B, slot);
    if (mixed) launch_symm(Flow, true, nullptr, B.p32, B.Ap, slot, 1);
    else launch_symm(F64, false, B.p, nullptr, B.Ap, slot, 1);
    launch_block_hybrid(B.p, B.Ap, slot, 1, B.scal + SC_PAP * blk.nr);
    switch (P.KS) {
    case 1: launch_pdl(bupdate_kernel<1>, dim3(nd), dim3(TPBB), 0, stream, P, B, slot); break;
    case 6: launch_pdl(bupdate_kernel<6>, dim3(nd), dim3(TPBB), 0, stream, P, B, slot); break;
    default: launch_pdl(bupdate_kernel<0>, dim3(nd), dim3(TPBB), 0, stream, P, B, slot); break;
    }
}

// panels of the mixed blocks for the asynchronous tensor-core SYMM (built before any graph capture)
void GpuSolver::Impl::prepare_symm_panels() {
    if (blk.nr != 32 || !opt.symm_tensor || Flow.prec != SCHUR_FP32 || !symm_tc2_enabled() || blk.pan) return;
    blk.pan = alloc<float>((size_t)blk.nunits4 * 3 * 4096);
    panel_kernel<<<std::max(1, blk.nunits4 * 3), 256, 0, stream>>>(Flow.dev(), blk.units4, blk.nunits4, blk.pan);
    CUDA_CHECK(cudaGetLastError());
}

// y_j = F x_j for nrhs dual vectors (column j at j * n_lambda) through the multi right-hand-side
// F apply of the block PCG (tile SYMM in the given Schur precision, plus the HTFETI correction)
void GpuSolver::apply_F_multi(const double *x, double *y, int nrhs, int precision) {
    FETI_CHECK(!impl->implicit, "FETI4I: the multi right-hand-side F apply needs the explicit Schur complements");
    Impl &I = *impl;
    DevProblem &P = I.P;
    FETI_CHECK(nrhs >= 1 && nrhs <= 32, "FETI4IApplyDualOperatorMulti: 1..32 vectors per call");
    const TileSetHost &T = precision == SCHUR_FP64 ? I.F64 : I.Flow;
    FETI_CHECK(T.prec == precision, "FETI4I: the requested Schur precision was not prepared on the device");
    int nr = 4;
    while (nr < nrhs) nr *= 2;
    I.ensure_block(nr);
    I.prepare_symm_panels();
    BlockDev &B = I.blk.B;
    const int NL = P.NL;
    std::vector<double> xb((size_t)NL * nr, 0.0), yb((size_t)NL * nr);
    std::vector<float> xf((size_t)NL * nr);
    for (int e = 0; e < NL; ++e)
        for (int j = 0; j < nrhs; ++j) xb[(size_t)e * nr + j] = x[(size_t)j * I.n_lambda + I.h_lam[e]];
    for (size_t i = 0; i < xb.size(); ++i) xf[i] = (float)xb[i];
    CUDA_CHECK(cudaMemcpyAsync(B.p, xb.data(), xb.size() * sizeof(double), cudaMemcpyHostToDevice, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(B.p32, xf.data(), xf.size() * sizeof(float), cudaMemcpyHostToDevice, I.stream));
    CUDA_CHECK(cudaMemsetAsync(B.Ap, 0, sizeof(double) * (size_t)NL * nr, I.stream));
    I.launch_symm(T, precision != SCHUR_FP64, B.p, B.p32, B.Ap, 0, 0);
    I.launch_block_hybrid(B.p, B.Ap, 0, 0, nullptr);
    CUDA_CHECK(cudaMemcpyAsync(yb.data(), B.Ap, yb.size() * sizeof(double), cudaMemcpyDeviceToHost, I.stream));
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
    for (size_t i = 0; i < (size_t)nrhs * I.n_lambda; ++i) y[i] = 0.0;
    for (int e = 0; e < NL; ++e)
        for (int j = 0; j < nrhs; ++j) y[(size_t)j * I.n_lambda + I.h_lam[e]] += yb[(size_t)e * nr + j];
}

void GpuSolver::solve_multi(const double *rhs, int nrhs, int rhs_size, double *solutions, int solution_size,
                            SolveStats &stats, bool upload_rhs) {
    FETI_CHECK(!impl->implicit, "FETI4ISolveMulti needs the explicit Schur complements (FETI4I_EXT_SCHUR_EXPLICIT 1)");
    Impl &I = *impl;
    DevProblem &P = I.P;
    FETI_CHECK(nrhs >= 1 && nrhs <= 32, "FETI4ISolveMulti: 1..32 right-hand sides per call");
    int nr = 4;
    while (nr < nrhs) nr *= 2;
    I.ensure_block(nr);
    I.prepare_symm_panels();
    BlockDev &B = I.blk.B;
    const int nd = P.nd, nc = std::max(1, I.n_caller), ntot = I.ntot;
    const int cgrid = (P.nK + CR - 1) / CR;
    if (upload_rhs) {
        CUDA_CHECK(cudaMemsetAsync(I.blk.rhs, 0, sizeof(double) * (size_t)nc * nr, I.stream));
        const int ncp = std::min(rhs_size, I.n_caller);
        I.h2d_columns(I.blk.rhs, nc, rhs, rhs_size, (size_t)std::max(0, ncp), nrhs);
        const long long tot = (long long)ntot * nr;
        bsplit_rhs_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, I.stream>>>(I.blk.rhs, nc, I.d_gdof, I.d_invm, I.blk.f,
                                                                              ntot, nr);
        CUDA_CHECK(cudaMemsetAsync(I.blk.kf, 0, sizeof(double) * (size_t)ntot * nr, I.stream));
        if (I.hybrid)
            I.launch_kplus_dual_multi(I.blk.f, I.blk.kf, nrhs);
        else
            I.launch_kplus_multi(I.blk.f, I.blk.kf, nrhs, KPLUS_TOUCHED, I.blk.zk);
        bevec_kernel<<<nd * nr, TPB, 0, I.stream>>>(P, B, I.d_doff, I.d_rdofs, I.d_Rd, I.blk.f, ntot);
        bbvec_kernel<<<(P.NL * nr + 255) / 256, 256, 0, I.stream>>>(P, B, I.d_rdof, I.d_rsign, I.d_rc, I.blk.kf, ntot);
        CUDA_CHECK(cudaGetLastError());
    }
    // ---- block PCG
    const bool mixed = I.opt.schur_precision != SCHUR_FP64;
    DevState h{};
    h.conv_iter = -1;
    h.replace_iter = -1;
    h.true_iter = 0;
    h.max_it = I.opt.max_iterations;
    h.mixed = mixed ? 1 : 0;
    h.precision = I.opt.precision;
    h.delta = I.opt.reliable_delta;
    CUDA_CHECK(cudaEventRecord(I.ev0, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(I.st, &h, sizeof(h), cudaMemcpyHostToDevice, I.stream));
    bcoarse_kernel<<<cgrid, 256, 0, I.stream>>>(P, B, B.e, B.alpha, 0, 0);
    bgt_kernel<<<(P.NL * nr + 255) / 256, 256, 0, I.stream>>>(P, B, B.alpha, B.x);
    CUDA_CHECK(cudaMemsetAsync(B.p, 0, sizeof(double) * (size_t)P.NL * nr, I.stream));
    I.launch_symm(I.F64, false, B.x, nullptr, B.Ax, 0, 0);
    I.launch_block_hybrid(B.x, B.Ax, 0, 0, nullptr);
    br0_kernel<<<nd, TPB, 0, I.stream>>>(P, B, 0, 0);
    bcoarse_kernel<<<cgrid, 256, 0, I.stream>>>(P, B, B.d, B.alpha, 0, 0);
    bpnorm_kernel<<<nd, TPB, 0, I.stream>>>(P, B);
    btol_kernel<<<1, 32, 0, I.stream>>>(P, B);
    CUDA_CHECK(cudaGetLastError());
    const int chunk = std::max(1, I.opt.chunk);
    auto &G = I.blk;
    if (!(G.graph && G.graph_chunk == chunk && G.graph_prec == I.opt.schur_precision &&
          G.graph_precond == I.opt.precond)) {
        if (G.graph) { cudaGraphExecDestroy(G.graph); G.graph = nullptr; }
        cudaGraph_t g;
        CUDA_CHECK(cudaStreamBeginCapture(I.stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < chunk; ++j) I.launch_block_iteration(j);
        launch_pdl(bchunk_end_kernel, dim3(1), dim3(32), 0, I.stream, P, chunk);
        CUDA_CHECK(cudaStreamEndCapture(I.stream, &g));
        CUDA_CHECK(cudaGraphInstantiate(&G.graph, g, 0));
        cudaGraphDestroy(g);
        G.graph_chunk = chunk;
        G.graph_prec = I.opt.schur_precision;
        G.graph_precond = I.opt.precond;
    }
    DevState hs{};
    for (int done = 0; done < I.opt.max_iterations; done += chunk) {
        CUDA_CHECK(cudaGraphLaunch(G.graph, I.stream));
        CUDA_CHECK(cudaMemcpyAsync(&hs, I.st, sizeof(hs), cudaMemcpyDeviceToHost, I.stream));
        CUDA_CHECK(cudaStreamSynchronize(I.stream));
        if (hs.conv_iter >= 0) break;
    }
    bcoarse_kernel<<<cgrid, 256, 0, I.stream>>>(P, B, B.d, B.alpha, 0, 0);
    CUDA_CHECK(cudaEventRecord(I.ev1, I.stream));
    CUDA_CHECK(cudaMemcpyAsync(&hs, I.st, sizeof(hs), cudaMemcpyDeviceToHost, I.stream));
    std::vector<int> conv(nr);
    CUDA_CHECK(cudaMemcpyAsync(conv.data(), B.conv, sizeof(int) * nr, cudaMemcpyDeviceToHost, I.stream));
    CUDA_CHECK(cudaStreamSynchronize(I.stream));
    float ms = 0.f;
    CUDA_CHECK(cudaEventElapsedTime(&ms, I.ev0, I.ev1));
    stats.t_solve_ms = ms;
    stats.converged = hs.conv_iter >= 0;
    stats.iterations = stats.converged ? hs.conv_iter + 1 : std::min(hs.iter_base, I.opt.max_iterations);
    stats.replacements = hs.replacements;
    stats.final_norm = hs.last_norm;
    stats.kernel_launches = 9 + (stats.iterations + chunk - 1) / chunk * chunk * 11;
    stats.fapply_bytes = (mixed ? I.Flow : I.F64).alg_bytes;
    // ---- primal recovery for every column
    if (solutions) {
        bprimal_rhs_kernel<<<4096, 256, 0, I.stream>>>(P, B, I.d_tdof_g, I.d_rsign, I.hybrid ? I.blk.f : nullptr,
                                                      I.blk.g, ntot);
        bprimal_bt_kernel<<<(P.NT * nr + 255) / 256, 256, 0, I.stream>>>(P, B, I.d_tdof_g, I.d_rsign, I.blk.g, ntot);
        if (I.hybrid)
            I.launch_kplus_dual_multi(I.blk.g, I.blk.kf, nrhs);
        else
            I.launch_kplus_multi(I.blk.g, I.blk.kf, nrhs, KPLUS_PRIMAL, I.blk.zk);
        CUDA_CHECK(cudaMemsetAsync(I.blk.sol, 0, sizeof(double) * (size_t)nc * nr, I.stream));
        bprimal_merge_kernel<<<nd * nr, TPB, 0, I.stream>>>(P, B, I.d_doff, I.d_rdofs, I.d_Rd, I.blk.kf, I.d_gdof, I.d_invm,
                                                           I.blk.sol, nc, ntot);
        CUDA_CHECK(cudaGetLastError());
        const int ncp = std::min(solution_size, I.n_caller);
        I.d2h_columns(solutions, solution_size, I.blk.sol, nc, (size_t)std::max(0, ncp), nrhs);
        for (int j = 0; j < nrhs; ++j)
            for (int i = std::max(0, ncp); i < solution_size; ++i) solutions[(size_t)j * solution_size + i] = 0.0;
    }
}

}  // namespace feti
