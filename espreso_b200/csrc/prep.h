// Host preprocessing of one Total-FETI problem: subdomain factorisations,
// algebraic kernels, explicit Schur complements, preconditioner data and the
// coarse problem.  Timed separately from the GPU dual iteration.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "decompose.h"

namespace feti {

struct DevPrepStore;

// FETI4I_PRECONDITIONER values (src/config/ecf/solver/feti.h:40-47 of the reference)
enum Precond { PREC_NONE = 0, PREC_LUMPED = 1, PREC_WEIGHT = 2, PREC_DIRICHLET = 3, PREC_SUPER_DIRICHLET = 4,
               PREC_MAGIC = 5 };

struct SubPrep {
    int n = 0;              // local DOFs
    int ni = 0;             // local multipliers (rows of B_i)
    int nk = 0;             // kernel dimension (defect)
    int t = 0;              // touched DOFs (columns of B_i, fix DOFs included)
    std::vector<int> pos;   // local DOF -> factor position
    std::vector<int> tdof;  // T index -> local DOF (factor order of the tail)
    std::vector<int> trow;  // local multiplier row -> T index
    std::vector<double> Lp; // packed lower Cholesky factor of K_reg (factor order)
    std::vector<double> R;  // n x nk, local DOF order, orthonormal columns
    std::vector<double> S;  // ni x ni, column-major, B K_reg^-1 B^T
    std::vector<double> Sdir;  // t x t Schur complement of K onto T (Dirichlet preconditioner)
    // sparse preconditioner matrix on T, CSR in T order: K restricted to T (LUMPED, MAGIC), or
    // S_sd = K_TT - K_Tr diag(K_rr)^-1 K_rT over the untouched DOFs r (SUPER_DIRICHLET)
    std::vector<int> KT_ptr, KT_col;
    std::vector<double> KT_val;
    std::vector<double> f;  // subdomain right-hand side
    std::vector<double> G;  // nk x ni, row-major: G_i = -(B_i R_i)^T
    std::vector<int> fix_nodes;
    double kernel_residual = 0.0;  // ||K R||_F / (||K||_F) check of the detected kernel
    std::vector<double> ss_eigs;   // eigenvalues of the fix-DOF Schur block

    // kernel space of the dual problem restricted to this subdomain: the subdomain's own kernel
    // (Total FETI) or the cluster kernel R H_i (Hybrid Total FETI)
    int dnk = 0;                   // columns
    std::vector<double> Rd;        // n x dnk, local DOF order
    std::vector<double> Gd;        // dnk x ni, row-major: -(B_i Rd)^T

    // Hybrid Total FETI: corner rows of B0 touching this subdomain (one DOF per row)
    std::vector<int> b0_row;       // cluster-local B0 row
    std::vector<int> b0_dof;       // local DOF
    std::vector<double> b0_sign;
    std::vector<double> V;         // ni x (n0_i + nk), column-major: [B_i K^+ B0_i^T | G_i^T]
    // device preprocessing: B_i K^+ B0_i^T (ni x n0_i) and B0_i K^+ B0_i^T (n0_i x n0_i), column-major
    std::vector<double> BKB0, B0KB0;

    // x := K_reg^{-1} x (local DOF order)
    void kplus(double *x) const;
};

// One cluster of Hybrid Total FETI: subdomains glued at corners by B0.
struct ClusterPrep {
    std::vector<int> members;       // subdomains, ascending
    int n0 = 0;                     // B0 rows
    int ka = 0;                     // sum of the members' kernel dimensions
    std::vector<int> akofs;         // member -> offset in the ka block
    int nkc = 0;                    // cluster kernel dimension
    std::vector<double> H;          // ka x nkc, column-major: kernel of S_alpha
    std::vector<double> M;          // (n0+ka)^2, column-major: [g0; e0] -> [lambda0; alpha]
    double rho = 0.0;               // S_alpha regularisation weight
};

struct Prep {
    std::vector<SubPrep> sub;
    int n_lambda = 0;
    int n_kern = 0;                 // dual kernel space (GG^T order)
    std::vector<int> kofs;          // dual kernel offset per subdomain (its cluster's offset in HTFETI)
    int method = 0;                 // 0 Total FETI, 1 Hybrid Total FETI
    std::vector<int> sub_cluster;   // HTFETI: subdomain -> cluster
    std::vector<ClusterPrep> clusters;
    std::vector<double> GGt_inv;    // n_kern x n_kern, dense symmetric inverse
    std::vector<int> lam_owner;     // 2 per multiplier: (domain, row) packed as domain*2^20+row? (see owners)
    std::vector<int> own_dom, own_row;  // 2 entries per multiplier, -1 if absent
    double t_factor = 0.0, t_coarse = 0.0;
    bool device_prep = false;          // eliminations and Schur complements ran on the GPU
    // Total FETI with device preprocessing: S_i, Dirichlet blocks and K^+ as device tiles (the host
    // SubPrep::S, Sdir and Lp stay empty)
    std::shared_ptr<DevPrepStore> dstore;
    double t_device_factor_ms = 0.0;   // device time of those eliminations (events)
    double device_factor_flops = 0.0;
    int device_factor_launches = 0;
};

struct PrepOptions {
    int method = 0;                 // FETI_METHOD: 0 Total FETI, 1 Hybrid Total FETI
    std::vector<int> sub_cluster;   // HTFETI clusters (empty: one cluster)
    int precond = PREC_DIRICHLET;
    bool scaling = true;
    bool keep_dirichlet = false;
    int threads = 0;
    bool device = false;            // subdomain eliminations and S_i on the current CUDA device
    size_t device_mem = 0;          // bytes for one batch of dense subdomain matrices (0: half the free memory)
    int owned_first = 0, owned_count = 0;   // partitioned dual problem: prepare these subdomains only (count 0: all)
};

// rhs: caller DOF vector (size >= max DOF + 1); split per subdomain by multiplicity.
void preprocess(const ElementData &el, Decomposition &dec, const std::vector<double> &rhs, const PrepOptions &opt,
                Prep &out);

// x_i := K_c^+ x_i for the subdomains of every cluster (Hybrid Total FETI), x[d] in local DOF order;
// with Total FETI x_i := K_i^+ x_i.
void kplus_dual(const Prep &prep, std::vector<std::vector<double>> &x);

// Right-hand-side dependent vectors: b = sum_i B_i K_i^+ f_i - c (lambda space), e = -R^T f.
void make_rhs_vectors(const Decomposition &dec, const Prep &prep, std::vector<double> &b, std::vector<double> &e);

// Primal recovery u_i = K_i^+ (f_i - B_i^T lambda) + R_i alpha_i, merged to caller DOFs (averaged).
void primal_solution(const Decomposition &dec, const Prep &prep, const double *lambda, const double *alpha,
                     double *solution, int solution_size);

}  // namespace feti
