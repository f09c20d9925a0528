// Host dense kernels: a packed GEMM micro-kernel (AVX2/FMA through GCC vector
// extensions) and the blocked Cholesky / triangular routines built on it.
#include "dense.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace feti {
namespace dense {

typedef double v4d __attribute__((vector_size(32)));

namespace {

constexpr int MR = 8;    // rows of the micro-tile (2 x v4d)
constexpr int NR = 4;    // columns of the micro-tile
constexpr int KC = 256;  // depth of a packed panel
constexpr int MC = 128;  // rows of a packed A block

// pack A(m x k) rows [i0, i0+mb) into MR-row slivers: sliver s, depth p -> MR contiguous values
void pack_a(int mb, int kb, const double *A, int lda, double *Ap) {
    for (int s = 0; s < mb; s += MR) {
        int r = std::min(MR, mb - s);
        for (int p = 0; p < kb; ++p) {
            const double *col = A + (size_t)p * lda + s;
            double *dst = Ap + (size_t)s * kb + (size_t)p * MR;
            int i = 0;
            for (; i < r; ++i) dst[i] = col[i];
            for (; i < MR; ++i) dst[i] = 0.0;
        }
    }
}

// pack B(n x k) (C -= A B^T) into NR-column slivers
void pack_b(int nb, int kb, const double *B, int ldb, double *Bp) {
    for (int s = 0; s < nb; s += NR) {
        int c = std::min(NR, nb - s);
        for (int p = 0; p < kb; ++p) {
            const double *col = B + (size_t)p * ldb + s;
            double *dst = Bp + (size_t)s * kb + (size_t)p * NR;
            int j = 0;
            for (; j < c; ++j) dst[j] = col[j];
            for (; j < NR; ++j) dst[j] = 0.0;
        }
    }
}

inline v4d load4(const double *p) {
    v4d v;
    std::memcpy(&v, p, sizeof(v));
    return v;
}
inline void store4(double *p, v4d v) { std::memcpy(p, &v, sizeof(v)); }

// C(MR x NR) -= Ap(MR x kb) * Bp(NR x kb)^T
void micro_kernel(int kb, const double *Ap, const double *Bp, double *C, int ldc, int mr, int nr) {
    v4d c00 = {0, 0, 0, 0}, c01 = c00, c02 = c00, c03 = c00;
    v4d c10 = c00, c11 = c00, c12 = c00, c13 = c00;
    for (int p = 0; p < kb; ++p) {
        v4d a0 = load4(Ap + (size_t)p * MR);
        v4d a1 = load4(Ap + (size_t)p * MR + 4);
        const double *b = Bp + (size_t)p * NR;
        v4d b0 = {b[0], b[0], b[0], b[0]};
        v4d b1 = {b[1], b[1], b[1], b[1]};
        v4d b2 = {b[2], b[2], b[2], b[2]};
        v4d b3 = {b[3], b[3], b[3], b[3]};
        c00 += a0 * b0; c10 += a1 * b0;
        c01 += a0 * b1; c11 += a1 * b1;
        c02 += a0 * b2; c12 += a1 * b2;
        c03 += a0 * b3; c13 += a1 * b3;
    }
    if (mr == MR && nr == NR) {
        double *c;
        c = C + 0 * (size_t)ldc; store4(c, load4(c) - c00); store4(c + 4, load4(c + 4) - c10);
        c = C + 1 * (size_t)ldc; store4(c, load4(c) - c01); store4(c + 4, load4(c + 4) - c11);
        c = C + 2 * (size_t)ldc; store4(c, load4(c) - c02); store4(c + 4, load4(c + 4) - c12);
        c = C + 3 * (size_t)ldc; store4(c, load4(c) - c03); store4(c + 4, load4(c + 4) - c13);
        return;
    }
    double tmp[NR][MR];
    store4(tmp[0], c00); store4(tmp[0] + 4, c10);
    store4(tmp[1], c01); store4(tmp[1] + 4, c11);
    store4(tmp[2], c02); store4(tmp[2] + 4, c12);
    store4(tmp[3], c03); store4(tmp[3] + 4, c13);
    for (int j = 0; j < nr; ++j)
        for (int i = 0; i < mr; ++i) C[(size_t)j * ldc + i] -= tmp[j][i];
}

}  // namespace

void gemm_nt_sub(int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C, int ldc) {
    if (m <= 0 || n <= 0 || k <= 0) return;
    thread_local std::vector<double> Ap, Bp;
    for (int p0 = 0; p0 < k; p0 += KC) {
        int kb = std::min(KC, k - p0);
        int npad = (n + NR - 1) / NR * NR;
        if ((int)Bp.size() < npad * kb) Bp.resize((size_t)npad * kb);
        pack_b(n, kb, B + (size_t)p0 * ldb, ldb, Bp.data());
        for (int i0 = 0; i0 < m; i0 += MC) {
            int mb = std::min(MC, m - i0);
            int mpad = (mb + MR - 1) / MR * MR;
            if ((int)Ap.size() < mpad * kb) Ap.resize((size_t)mpad * kb);
            pack_a(mb, kb, A + (size_t)p0 * lda + i0, lda, Ap.data());
            for (int j = 0; j < n; j += NR) {
                int nr = std::min(NR, n - j);
                for (int i = 0; i < mb; i += MR) {
                    int mr = std::min(MR, mb - i);
                    micro_kernel(kb, Ap.data() + (size_t)i * kb, Bp.data() + (size_t)j * kb,
                                 C + (size_t)j * ldc + i0 + i, ldc, mr, nr);
                }
            }
        }
    }
}

namespace {
// unblocked Cholesky of an nb x nb diagonal block
int potf2(double *A, int n, int lda) {
    for (int j = 0; j < n; ++j) {
        double *cj = A + (size_t)j * lda;
        double d = cj[j];
        for (int p = 0; p < j; ++p) d -= A[(size_t)p * lda + j] * A[(size_t)p * lda + j];
        if (!(d > 0.0)) return j + 1;
        d = std::sqrt(d);
        cj[j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = cj[i];
            for (int p = 0; p < j; ++p) s -= A[(size_t)p * lda + i] * A[(size_t)p * lda + j];
            cj[i] = s / d;
        }
    }
    return 0;
}
}  // namespace

// Large problems outside a parallel region (the coarse problem) split their independent work over
// the host threads; every element sees the same operations in the same order either way.
static bool parallel_worth(double work) { return work > 4e6 && !omp_in_parallel() && omp_get_max_threads() > 1; }

void trsm_rlt(int m, int k, const double *L, int ldl, double *B, int ldb) {
    // column j of X: X_j = (B_j - sum_{p<j} X_p L(j,p)) / L(j,j); rows are independent
    const int RB = 256;
    const int nb = (m + RB - 1) / RB;
#pragma omp parallel for schedule(dynamic, 1) if (parallel_worth((double)m * k * k))
    for (int b = 0; b < nb; ++b) {
        const int i0 = b * RB, i1 = std::min(m, i0 + RB);
        for (int j = 0; j < k; ++j) {
            double *bj = B + (size_t)j * ldb;
            for (int p = 0; p < j; ++p) {
                double l = L[(size_t)p * ldl + j];
                if (l == 0.0) continue;
                const double *bp = B + (size_t)p * ldb;
                for (int i = i0; i < i1; ++i) bj[i] -= bp[i] * l;
            }
            double inv = 1.0 / L[(size_t)j * ldl + j];
            for (int i = i0; i < i1; ++i) bj[i] *= inv;
        }
    }
}

int potrf_lower(double *A, int n, int lda, int ncols) {
    const int NB = 96;
    for (int k = 0; k < ncols; k += NB) {
        int kb = std::min(NB, ncols - k);
        double *Akk = A + (size_t)k * lda + k;
        int info = potf2(Akk, kb, lda);
        if (info) return k + info;
        int m = n - k - kb;
        if (m <= 0) continue;
        double *P = Akk + kb;  // rows k+kb..n-1 of the panel
        trsm_rlt(m, kb, Akk, lda, P, lda);
        // trailing lower update A22 -= P P^T, by column blocks
        const int nblk = (m + NB - 1) / NB;
#pragma omp parallel for schedule(dynamic, 1) if (parallel_worth((double)m * m * kb))
        for (int b = 0; b < nblk; ++b) {
            const int j0 = b * NB, jb = std::min(NB, m - j0);
            gemm_nt_sub(m - j0, jb, kb, P + j0, lda, P + j0, lda,
                        A + (size_t)(k + kb + j0) * lda + k + kb + j0, lda);
        }
    }
    return 0;
}

void trtri_lower(double *L, int n, int ld) {
    // column-by-column: X = L^{-1}; X(j,j)=1/L(j,j); X(i,j) = -sum_{p=j}^{i-1} L(i,p) X(p,j) / L(i,i)
    // done blockwise-free but in the j-outer order with axpy over i for vectorisation
    // Columns from the right: with X22 = inverse of the trailing block (already
    // in place), x_jj = 1/l_jj and x_21 = -X22 (l_21 x_jj); X22 * v is formed
    // as a sum of contiguous column axpys.
    std::vector<double> y(n);
    const bool par = parallel_worth((double)n * n * n / 3.0);
    for (int j = n - 1; j >= 0; --j) {
        double xjj = 1.0 / L[(size_t)j * ld + j];
        int m = n - j - 1;
        double *l21 = L + (size_t)j * ld + j + 1;
        // y = X22 (l21 xjj): rows i in independent chunks, the sum over p in ascending order
        const int RB = 128;
        const int nb = (m + RB - 1) / RB;
#pragma omp parallel for schedule(static) if (par && m > 512)
        for (int b = 0; b < nb; ++b) {
            const int i0 = b * RB, i1 = std::min(m, i0 + RB);
            std::fill(y.begin() + i0, y.begin() + i1, 0.0);
            for (int p = 0; p < i1; ++p) {
                double v = l21[p] * xjj;
                if (v == 0.0) continue;
                const double *xc = L + (size_t)(j + 1 + p) * ld + j + 1;  // column p of X22, rows p..m-1
                for (int i = std::max(p, i0); i < i1; ++i) y[i] += xc[i] * v;
            }
        }
        L[(size_t)j * ld + j] = xjj;
        for (int i = 0; i < m; ++i) l21[i] = -y[i];
    }
}

void lauum_lower(const double *W, int n, int ldw, double *C, int ldc) {
    // C(i,j) = sum_{p >= max(i,j)} W(p,i) W(p,j); columns are independent
#pragma omp parallel for schedule(dynamic, 8) if (parallel_worth((double)n * n * n / 3.0))
    for (int j = 0; j < n; ++j) {
        const double *wj = W + (size_t)j * ldw;
        for (int i = j; i < n; ++i) {
            const double *wi = W + (size_t)i * ldw;
            double s = 0.0;
            for (int p = i; p < n; ++p) s += wi[p] * wj[p];
            C[(size_t)j * ldc + i] = s;
            C[(size_t)i * ldc + j] = s;
        }
    }
}

void pack_lower(const double *A, int n, int lda, double *P) {
    size_t o = 0;
    for (int j = 0; j < n; ++j) {
        const double *c = A + (size_t)j * lda;
        for (int i = j; i < n; ++i) P[o++] = c[i];
    }
}

void trsv_packed_lower(const double *P, int n, double *x) {
    size_t o = 0;
    for (int j = 0; j < n; ++j) {
        double xj = x[j] / P[o];
        x[j] = xj;
        const double *c = P + o + 1;
        int m = n - j - 1;
        for (int i = 0; i < m; ++i) x[j + 1 + i] -= c[i] * xj;
        o += n - j;
    }
}

void trsv_packed_lower_t(const double *P, int n, double *x) {
    // column j of L = row j of L^T; x(j) = (x(j) - sum_{i>j} L(i,j) x(i)) / L(j,j)
    std::vector<size_t> start(n);
    size_t o = 0;
    for (int j = 0; j < n; ++j) { start[j] = o; o += n - j; }
    for (int j = n - 1; j >= 0; --j) {
        const double *c = P + start[j];
        double s = x[j];
        int m = n - j - 1;
        for (int i = 0; i < m; ++i) s -= c[1 + i] * x[j + 1 + i];
        x[j] = s / c[0];
    }
}

void jacobi_eigen(const double *A0, int n, double *w, double *V) {
    std::vector<double> A(A0, A0 + (size_t)n * n);
    for (int i = 0; i < n * n; ++i) V[i] = 0.0;
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double a = A[(size_t)j * n + i];
                tot += a * a;
                if (i != j) off += a * a;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A[(size_t)q * n + p];
                if (apq == 0.0) continue;
                double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {  // columns p,q
                    double akp = A[(size_t)p * n + k], akq = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * akp - s * akq;
                    A[(size_t)q * n + k] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p,q
                    double apk = A[(size_t)k * n + p], aqk = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * apk - s * aqk;
                    A[(size_t)k * n + q] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
                    V[(size_t)p * n + k] = c * vkp - s * vkq;
                    V[(size_t)q * n + k] = s * vkp + c * vkq;
                }
            }
    }
    // sort ascending
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return A[(size_t)a * n + a] < A[(size_t)b * n + b]; });
    std::vector<double> Vs((size_t)n * n);
    for (int k = 0; k < n; ++k) {
        w[k] = A[(size_t)idx[k] * n + idx[k]];
        for (int i = 0; i < n; ++i) Vs[(size_t)k * n + i] = V[(size_t)idx[k] * n + i];
    }
    std::copy(Vs.begin(), Vs.end(), V);
}

}  // namespace dense
}  // namespace feti
