// CPU restatement of ESPRESO's projected dual PCG with explicit Schur complements,
// parallelised over the host cores with OpenMP.
//
// TEST INFRASTRUCTURE ONLY: used by the tests as a checker and by bench.py as the timed CPU
// baseline / reference arm.  The shipped library never links it.
//
// Restated from the reference (feeleewee/espreso), paths relative to its project:
//   PCG recurrences, stop rule, lambda_0 and the amplitudes  src/solver/specific/itersolver.cpp:1406-1724
//   projector (explicit GGtinvM stripe, GEMV)                   src/solver/specific/itersolver.cpp:5541-5623
//   F apply: per subdomain packed-upper SPMV of S_i on the
//     gathered multipliers, scatter-add                          src/solver/specific/cpu/itersolvercpu.cpp:49-70
//                                                                src/solver/generic/SparseMatrix.cpp:1057-1172
//   Apply_Prec: B1 scaling, B^T, K | S_dir, B, B1 scaling       src/solver/specific/cpu/itersolvercpu.cpp:520-602
//   dot products                                                 src/solver/specific/itersolver.cpp:6427-6467
// The numpy oracle (oracle/feti.py) builds every operator; this file only iterates.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

struct Problem {
    int ndom, n_lambda, n_kern, prec, nthreads;
    const int *loff, *lam;                 // local rows per subdomain, global multiplier per row
    const long long *soff;                 // packed S_i offsets
    const double *Sp;                      // packed upper, column-major (cblas_dspmv 'U')
    const int *l2r_ptr, *l2r_row;          // multiplier -> local rows
    const int *g_ptr, *g_col;              // G (n_kern x n_lambda), CSR
    const double *g_val;
    const int *gt_ptr, *gt_col;            // G^T (n_lambda x n_kern), CSR
    const double *gt_val;
    const double *GGtinv;                  // n_kern x n_kern, row-major
    const double *w, *sign;                // B1 scale and sign per local row
    const int *tofs, *trow;                // per subdomain offset into T space; row -> T index
    const int *m_ptr, *m_col;              // CSR preconditioner matrix over T space (LUMPED, MAGIC, SUPER_DIRICHLET)
    const double *m_val;
    const long long *doff;                 // packed dense preconditioner per subdomain (DIRICHLET)
    const double *Dp;
};

enum { NONE = 0, LUMPED = 1, WEIGHT = 2, DIRICHLET = 3, SUPER_DIRICHLET = 4, MAGIC = 5 };

// y = A x, A symmetric packed upper column-major of order n (cblas_dspmv, uplo 'U')
void spmv_packed(int n, const double *ap, const double *x, double *y) {
    for (int i = 0; i < n; ++i) y[i] = 0.0;
    for (int j = 0; j < n; ++j) {
        const double *col = ap + (size_t)j * (j + 1) / 2;
        const double xj = x[j];
        double s = 0.0;
#pragma omp simd reduction(+ : s)
        for (int i = 0; i < j; ++i) {
            y[i] += col[i] * xj;
            s += col[i] * x[i];
        }
        y[j] += s + col[j] * xj;
    }
}

struct Work {
    std::vector<double> yl, uT, vT, gx, ga;
};

double dot(const Problem &P, const double *a, const double *b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int i = 0; i < P.n_lambda; ++i) s += a[i] * b[i];
    return s;
}

// assemble y[l] = sum of the local rows of multiplier l
void assemble(const Problem &P, const double *yl, double *y) {
#pragma omp parallel for schedule(static)
    for (int l = 0; l < P.n_lambda; ++l) {
        double s = 0.0;
        for (int k = P.l2r_ptr[l]; k < P.l2r_ptr[l + 1]; ++k) s += yl[P.l2r_row[k]];
        y[l] = s;
    }
}

// y = F x = sum_i B_i S_i B_i^T x
void apply_F(const Problem &P, Work &W, const double *x, double *y) {
#pragma omp parallel
    {
        std::vector<double> xd;
#pragma omp for schedule(dynamic, 1)
        for (int d = 0; d < P.ndom; ++d) {
            const int r0 = P.loff[d], n = P.loff[d + 1] - r0;
            xd.resize(n);
            for (int r = 0; r < n; ++r) xd[r] = x[P.lam[r0 + r]];
            spmv_packed(n, P.Sp + P.soff[d], xd.data(), W.yl.data() + r0);
        }
    }
    assemble(P, W.yl.data(), y);
}

// mode 0: out = x - G^T (GG^T)^-1 G x;  mode 1: out = G^T (GG^T)^-1 x (x in kernel space);
// mode 2: out = (GG^T)^-1 G x (kernel space)
void projector(const Problem &P, Work &W, const double *x, double *out, int mode) {
    const int nk = P.n_kern;
    if (mode == 1) {
        std::memcpy(W.gx.data(), x, sizeof(double) * nk);
    } else {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nk; ++k) {
            double s = 0.0;
            for (int j = P.g_ptr[k]; j < P.g_ptr[k + 1]; ++j) s += P.g_val[j] * x[P.g_col[j]];
            W.gx[k] = s;
        }
    }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; ++k) {
        const double *row = P.GGtinv + (size_t)k * nk;
        double s = 0.0;
        for (int j = 0; j < nk; ++j) s += row[j] * W.gx[j];
        W.ga[k] = s;
    }
    if (mode == 2) {
        std::memcpy(out, W.ga.data(), sizeof(double) * nk);
        return;
    }
#pragma omp parallel for schedule(static)
    for (int l = 0; l < P.n_lambda; ++l) {
        double s = 0.0;
        for (int j = P.gt_ptr[l]; j < P.gt_ptr[l + 1]; ++j) s += P.gt_val[j] * W.ga[P.gt_col[j]];
        out[l] = mode == 0 ? x[l] - s : s;
    }
}

// y = sum_i W_i B_i M_i B_i^T W_i x (Apply_Prec)
void precondition(const Problem &P, Work &W, const double *x, double *y) {
    if (P.prec == NONE) {
        std::memcpy(y, x, sizeof(double) * P.n_lambda);
        return;
    }
#pragma omp parallel
    {
        std::vector<double> ut, vt;
#pragma omp for schedule(dynamic, 1)
        for (int d = 0; d < P.ndom; ++d) {
            const int r0 = P.loff[d], r1 = P.loff[d + 1];
            if (P.prec == WEIGHT) {
                for (int r = r0; r < r1; ++r) W.yl[r] = x[P.lam[r]] * P.w[r] * P.w[r];
                continue;
            }
            const int t0 = P.tofs[d], nt = P.tofs[d + 1] - t0;
            ut.assign(nt, 0.0);
            vt.resize(nt);
            for (int r = r0; r < r1; ++r) ut[P.trow[r]] += P.sign[r] * P.w[r] * x[P.lam[r]];
            if (P.prec == DIRICHLET) {
                spmv_packed(nt, P.Dp + P.doff[d], ut.data(), vt.data());
            } else {   // LUMPED, MAGIC (K - RegMat), SUPER_DIRICHLET (sparse S_dir): CSR over T space
                for (int i = 0; i < nt; ++i) {
                    double s = 0.0;
                    for (int j = P.m_ptr[t0 + i]; j < P.m_ptr[t0 + i + 1]; ++j) s += P.m_val[j] * ut[P.m_col[j] - t0];
                    vt[i] = s;
                }
            }
            for (int r = r0; r < r1; ++r) W.yl[r] = P.sign[r] * vt[P.trow[r]] * P.w[r];
        }
    }
    assemble(P, W.yl.data(), y);
}

}  // namespace

extern "C" {

// Projected PCG (Solve_RegCG) from b, e to lambda, alpha; returns the iteration count.
// stats[0] = final |w|, stats[1] = tolerance.
int oracle_pcg_solve(int ndom, int n_lambda, int n_kern, int prec, int nthreads, const int *loff, const int *lam,
                     const long long *soff, const double *Sp, const int *l2r_ptr, const int *l2r_row,
                     const int *g_ptr, const int *g_col, const double *g_val, const int *gt_ptr, const int *gt_col,
                     const double *gt_val, const double *GGtinv, const double *w, const double *sign,
                     const int *tofs, const int *trow, const int *m_ptr, const int *m_col, const double *m_val,
                     const long long *doff, const double *Dp, const double *b, const double *e, double precision,
                     int max_it, double *lambda, double *alpha, double *stats) {
    Problem P{ndom,  n_lambda, n_kern, prec,   nthreads, loff,  lam,   soff,   Sp,    l2r_ptr, l2r_row,
              g_ptr, g_col,    g_val,  gt_ptr, gt_col,   gt_val, GGtinv, w,   sign,  tofs,    trow,
              m_ptr, m_col,    m_val,  doff,   Dp};
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const int n = n_lambda;
    Work W;
    W.yl.resize(loff[ndom]);
    W.gx.resize(n_kern);
    W.ga.resize(n_kern);
    std::vector<double> x(n), Ax(n), r(n), u(n), wv(n, 0.0), y(n, 0.0), z(n), p(n, 0.0), Ap(n), wp(n), yp(n);
    projector(P, W, e, x.data(), 1);   // lambda_0 = G^T (GG^T)^-1 e
    apply_F(P, W, x.data(), Ax.data());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    projector(P, W, r.data(), u.data(), 0);
    const double tol = precision * std::fmin(std::sqrt(dot(P, u.data(), u.data())), std::sqrt(dot(P, b, b)));
    double norm = 0.0;
    int it = 0;
    for (it = 0; it < max_it; ++it) {
        wp.swap(wv);
        yp.swap(y);
        projector(P, W, r.data(), wv.data(), 0);
        if (prec == NONE) {
            std::memcpy(y.data(), wv.data(), sizeof(double) * n);
        } else {
            precondition(P, W, wv.data(), z.data());
            projector(P, W, z.data(), y.data(), 0);
        }
        const double yw = dot(P, y.data(), wv.data());
        if (it == 0) {
            std::memcpy(p.data(), y.data(), sizeof(double) * n);
        } else {
            const double beta = yw / dot(P, yp.data(), wp.data());
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) p[i] = y[i] + beta * p[i];
        }
        apply_F(P, W, p.data(), Ap.data());
        const double a = yw / dot(P, p.data(), Ap.data());
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            x[i] += a * p[i];
            r[i] -= a * Ap[i];
        }
        norm = std::sqrt(dot(P, wv.data(), wv.data()));
        if (norm < tol) break;
    }
    std::memcpy(lambda, x.data(), sizeof(double) * n);
    projector(P, W, r.data(), alpha, 2);   // amplitudes (GG^T)^-1 G r
    if (stats) {
        stats[0] = norm;
        stats[1] = tol;
    }
    return it < max_it ? it + 1 : max_it;
}

}  // extern "C"
