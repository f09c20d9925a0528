// Device-resident Total-FETI dual iteration on one B200 (sm_100a).
//
// Dual vectors live in the replicated local layout: subdomain d owns rows
// loff[d]..loff[d+1] (its local multipliers, i.e. rows of B_i); a multiplier
// shared by two subdomains appears twice and both copies hold the same value.
// Assembly of a sum over subdomains is "own value + partner value".
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "decompose.h"
#include "prep.h"

namespace feti {

enum SchurPrecision { SCHUR_FP64 = 0, SCHUR_FP32 = 1, SCHUR_BF16 = 2 };

struct SolveOptions {
    double precision = 1e-5;
    int max_iterations = 200;
    int precond = PREC_DIRICHLET;
    int schur_precision = SCHUR_FP64;  // storage of the iteration operator
    int chunk = 16;                    // iterations per captured CUDA graph
    int tiles_per_item = 48;           // work-queue granularity of the tile SYMV
    int tile_kernel = 0;               // 0: register-prefetch SYMV, 1: TMA bulk-copy pipeline
    bool autotune = true;              // time the variants and item granularities per size class at upload
    bool symm_tensor = true;           // multi-RHS FP32 SYMM on the tensor cores (3xTF32) instead of CUDA cores
    bool schur_explicit = true;        // false: F applied through the K^+ factor (no stored S_i; FP64, Total FETI)
    double reliable_delta = 0.003;     // residual replacement threshold (mixed precision)
    bool use_graph = true;
};

struct SolveStats {
    int iterations = 0;
    int replacements = 0;
    double tol = 0.0;
    double final_norm = 0.0;
    double t_solve_ms = 0.0;       // device time of the dual PCG (events)
    double t_fapply_ms = 0.0;      // average device time of one F apply (operator precision)
    double fapply_bytes = 0.0;     // algorithmic bytes of one F apply
    int fapply_launches = 0;
    int kernel_launches = 0;       // kernels launched by the last solve
    bool converged = false;
};

class GpuSolver {
public:
    GpuSolver();
    ~GpuSolver();
    void upload(const Decomposition &dec, const Prep &prep, const SolveOptions &opt);
    // Dual PCG on device-resident b (lambda space), e (kernel space); outputs lambda and alpha.
    void set_rhs(const std::vector<double> &b, const std::vector<double> &e);
    void solve(SolveStats &st);
    void get_solution(std::vector<double> &lambda, std::vector<double> &alpha);
    // Whole solve on the device: caller right-hand side -> f_i, K^+ f_i, b, e, dual PCG,
    // primal recovery u_i = K^+ (f_i - B_i^T lambda) + R_i alpha_i, averaged into `solution`.
    // With upload_rhs == false the right-hand side of the previous call is reused.
    void solve_full(const double *rhs, int rhs_size, double *solution, int solution_size, SolveStats &st,
                    bool upload_rhs = true);
    // Several right-hand sides (1..32, rhs[j * rhs_size + i]) solved together: block PCG with
    // per-column scalars and stop tests, tile SYMM F apply; solutions[j * solution_size + i].
    void solve_multi(const double *rhs, int nrhs, int rhs_size, double *solutions, int solution_size, SolveStats &st,
                     bool upload_rhs = true);
    // Introspection through the device data (device preprocessing keeps S_i and K^+ only there):
    // S_i as a full ni x ni column-major matrix; x := K_i^+ x (local DOF order); b and e of the
    // caller right-hand side (multiplier order, dual kernel order).
    void subdomain_schur(int d, double *S);
    void subdomain_kplus(int d, double *x);
    void dual_rhs(const double *rhs, int rhs_size, double *b, double *e, int n_lambda, int n_kern);
    // y = F x in lambda space with the given operator precision (tests, benchmarks)
    void apply_F(const double *x_lambda, double *y_lambda, int precision);
    void apply_F_multi(const double *x, double *y, int nrhs, int precision);
    // partitioned dual problem, caller device vectors in the whole problem's multiplier numbering:
    // y += sum over the instance's subdomains of B S B^T x (precision of S), or of W B M B^T W x
    void apply_F_device(const double *x, double *y, int precision, void *stream);
    void apply_prec_device(const double *x, double *y, void *stream);
    // primal recovery from host lambda (whole numbering) and amplitudes (the instance's kernel numbering)
    void primal_from_dual(const double *rhs, int rhs_size, const double *lambda, const double *alpha, double *solution,
                          int solution_size);
    // average device time of `reps` F applies (inputs resident), returns ms
    double time_F(int precision, int reps);
    double fapply_bytes(int precision) const;
    // out[e] = v_e^T K_e u_e over the stored elements (u, v: caller DOF vectors of size n)
    void element_energies(const ElementData &el, const double *u, const double *v, int n, double *out);
    size_t device_bytes() const;
    double kplus_tile_fraction() const;   // applied / stored K+ factor tiles
    int device_id() const;
    void set_options(const SolveOptions &opt);
    std::string tuning() const;        // chosen SYMV variant and granularities

    struct Impl;
    Impl *impl;
};

bool cuda_available(std::string &why);

// Allocation-free batched tile SYMV on caller-owned device buffers (scratch in a static device array).
int tiled_symv_noalloc(const double *tiles, const long long *tile_offset, const int *order, const int *vector_offset,
                       int nmatrices, int max_order, const double *x, double *y, double *dot, void *stream);

}  // namespace feti
