// Batched FP64 partial Cholesky of the augmented subdomain matrices [K_reg B~^T; B~ 0] on sm_100a.
//
// One batch holds the dense matrices of many subdomains (column-major, lower triangle used,
// leading dimension padded to 32 rows).  Per elimination step every subdomain of the batch that
// still has columns in the current phase contributes one "item" (panel columns [k0, k0+w), rows
// [k0, rend)), and three launches process all items of the step together:
//   diag_kernel    one CTA per item: Cholesky of the w x w diagonal block in shared memory;
//   trsm_kernel    one CTA per 64-row block below it: L_ik = A_ik L_kk^-T;
//   update_pipe_kernel  one CTA per 64 x 64 lower tile of the trailing block: A_IJ -= L_Ik L_Jk^T
//                  (FP64 MMA, 128-deep panels streamed by cp.async).
// Phases: untouched columns (rows of K only: the B~ rows are zero there and stay zero), touched
// columns (B~ rows included), fix columns after the host's regularisation of the fix-DOF block.
#include "gpu_prep.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "common.h"

#define PCHECK(x)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            throw ::feti::Error(std::string("CUDA error ") + cudaGetErrorString(e_) + " in " #x); \
    } while (0)

namespace feti {

namespace {

constexpr int PW = 128;   // panel width (k-depth of every trailing update)
constexpr int TE = 64;    // row block of the panel solve and tile edge of the trailing update
constexpr int BS = 64;    // column block of the kernel backward solve
constexpr int PT = 256;   // threads per CTA

struct SubD {
    long long a;          // offset of the dense matrix in the arena (doubles)
    int ld;               // leading dimension
    int n, N;             // columns eliminated (DOFs of K), rows (n + ni)
};

struct Item {
    int sub, k0, w, rend; // panel [k0, k0+w), rows [k0, rend)
    int trs0, upd0;       // first CTA of this item in the trsm / update grid
};

struct ElemD {
    long long val;        // offset of K_e in the batch value buffer
    int nd;               // element DOFs
    int pos;              // offset of its factor positions in the batch position buffer
    int sub;              // batch-local subdomain
};

struct JobD {
    int sub, n, n1, nc, ni, ns;
    int nrow;             // appended rows (B and B0)
    int m0;               // B0 rows
    long long vo;         // offset of the [B; B0] K^+ B0^T block in the staging buffer, -1 without B0
    long long boff;       // offset of its B~ rows in bpos / bsign
    long long s;          // offset of its S output in the staging buffer (doubles), -1 without
    long long fx;         // offset of its fix-DOF block in the fix buffer
};

// item whose first CTA is the largest one <= b (items with no CTAs share the next item's start)
template <int WHICH>
__device__ __forceinline__ int find_item(const Item *it, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int v = WHICH == 0 ? it[mid].trs0 : it[mid].upd0;
        if (v <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------------------------
// assembly and set-up

// Scatter-add of the element matrices of one colour into the lower triangles (elements of one
// colour share no DOF, so no two CTAs add into the same entry and the sums are deterministic).
__global__ void assemble_kernel(const ElemD *els, const int *list, int count, const double *vals, const int *epos,
                                const SubD *subs, double *arena) {
    for (int e = blockIdx.x; e < count; e += gridDim.x) {
        const ElemD E = els[list[e]];
        const SubD sd = subs[E.sub];
        double *A = arena + sd.a;
        const int nd = E.nd;
        for (int q = threadIdx.x; q < nd * nd; q += blockDim.x) {
            const int a = q / nd, c = q - a * nd;
            const int pa = epos[E.pos + a], pc = epos[E.pos + c];
            if (pa >= pc) A[(size_t)pc * sd.ld + pa] += vals[E.val + q];
        }
    }
}

// B~ rows below K: row n + r holds sign_r at the factor column of the row's DOF.
__global__ void brows_kernel(const JobD *jobs, const SubD *subs, const int *bpos, const double *bsign, double *arena) {
    const JobD J = jobs[blockIdx.y];
    const SubD sd = subs[J.sub];
    double *A = arena + sd.a;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < J.nrow; r += gridDim.x * blockDim.x)
        A[(size_t)bpos[J.boff + r] * sd.ld + J.n + r] = bsign[J.boff + r];
}

// Partial sums of ||K||_F^2 from the lower triangle (off-diagonal entries counted twice).
__global__ void knorm_kernel(const JobD *jobs, const SubD *subs, const double *arena, double *part) {
    const JobD J = jobs[blockIdx.y];
    const SubD sd = subs[J.sub];
    const double *A = arena + sd.a;
    const long long tot = (long long)J.n * J.n;
    double s = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(q / J.n), i = (int)(q - (long long)j * J.n);
        if (i >= j) {
            const double v = A[(size_t)j * sd.ld + i];
            s += (i > j ? 2.0 : 1.0) * v * v;
        }
    }
    __shared__ double red[PT / 32];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < PT / 32; ++w) t += red[w];
        part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
}

// ---------------------------------------------------------------------------------------------
// elimination step

// Cholesky of the w x w diagonal block of every item, blocked by 32 columns: warp 0 factors a 32 x 32
// block (one lane per row) and inverts it (one lane per column); all warps multiply the rows below
// by the inverse and update the rest of the panel block.  A non-positive pivot is recorded (first
// column per subdomain) and replaced by 1 so that the elimination stays finite.  The inverses of the
// 32 x 32 diagonal blocks go to `dinv` (four per item) for the panel solve.
constexpr int DB = 32;
constexpr int DSM = (PW * (PW + 1) + DB * (DB + 1) + (PW - DB) * (DB + 1)) * (int)sizeof(double);

__global__ void __launch_bounds__(PT) diag_kernel(const Item *items, const SubD *subs, double *arena, int *fail,
                                                  double *dinv) {
    extern __shared__ double dsm[];
    double(*D)[PW + 1] = reinterpret_cast<double(*)[PW + 1]>(dsm);
    double(*V)[DB + 1] = reinterpret_cast<double(*)[DB + 1]>(dsm + PW * (PW + 1));
    double(*T)[DB + 1] = reinterpret_cast<double(*)[DB + 1]>(dsm + PW * (PW + 1) + DB * (DB + 1));
    __shared__ int s_bad;
    const Item it = items[blockIdx.x];
    const SubD sd = subs[it.sub];
    double *A = arena + sd.a;
    const size_t ld = sd.ld;
    const int k0 = it.k0, w = it.w, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int q = tid; q < w * w; q += PT) {
        const int i = q % w, j = q / w;
        if (i >= j) D[i][j] = A[(size_t)(k0 + j) * ld + k0 + i];
    }
    if (tid == 0) s_bad = -1;
    __syncthreads();
    double *dout = dinv + (size_t)blockIdx.x * (PW / DB) * DB * DB;
    for (int c0 = 0; c0 < w; c0 += DB) {
        const int bw = min(DB, w - c0);
        if (warp == 0) {
            // factor the bw x bw block, lane = row
            for (int j = 0; j < bw; ++j) {
                if (lane == j) {
                    double d = D[c0 + j][c0 + j];
                    if (!(d > 0.0)) {
                        if (s_bad < 0) s_bad = c0 + j;
                        d = 1.0;
                    }
                    D[c0 + j][c0 + j] = sqrt(d);
                }
                __syncwarp();
                if (lane > j && lane < bw) D[c0 + lane][c0 + j] /= D[c0 + j][c0 + j];
                __syncwarp();
                if (lane > j && lane < bw)
                    for (int c = j + 1; c <= lane; ++c) D[c0 + lane][c0 + c] -= D[c0 + lane][c0 + j] * D[c0 + c][c0 + j];
                __syncwarp();
            }
            // inverse of the block, lane = column (zero above the diagonal and outside bw)
            for (int r = 0; r < DB; ++r) V[r][lane] = 0.0;
            if (lane < bw)
                for (int r = lane; r < bw; ++r) {
                    double sum = r == lane ? 1.0 : 0.0;
                    for (int k = lane; k < r; ++k) sum -= D[c0 + r][c0 + k] * V[k][lane];
                    V[r][lane] = sum / D[c0 + r][c0 + r];
                }
            __syncwarp();
            for (int r = 0; r < DB; ++r) dout[(size_t)(c0 / DB) * DB * DB + r * DB + lane] = V[r][lane];
        }
        __syncthreads();
        // rows below the block within the panel: X = P V^T, X[r][j] = sum_{m <= j} P[r][m] V[j][m]
        const int rb = c0 + bw, nr = w - rb;
        for (int q = tid; q < nr * bw; q += PT) {
            const int r = q % nr, j = q / nr;
            double sum = 0.0;
            for (int m = 0; m <= j; ++m) sum += D[rb + r][c0 + m] * V[j][m];
            T[r][j] = sum;
        }
        __syncthreads();
        for (int q = tid; q < nr * bw; q += PT) {
            const int r = q % nr, j = q / nr;
            D[rb + r][c0 + j] = T[r][j];
        }
        __syncthreads();
        // rest of the panel block: D[i][j] -= sum_m X[i][m] X[j][m], i >= j >= rb
        for (int q = tid; q < nr * nr; q += PT) {
            const int i = rb + q % nr, j = rb + q / nr;
            if (i < j) continue;
            double sum = 0.0;
            for (int m = 0; m < bw; ++m) sum += D[i][c0 + m] * D[j][c0 + m];
            D[i][j] -= sum;
        }
        __syncthreads();
    }
    if (tid == 0 && s_bad >= 0) atomicMin(&fail[it.sub], k0 + s_bad);
    for (int q = tid; q < w * w; q += PT) {
        const int i = q % w, j = q / w;
        if (i >= j) A[(size_t)(k0 + j) * ld + k0 + i] = D[i][j];
    }
}

// Row blocks below the diagonal block: X = P L_kk^-T by 32-column blocks,
// X_b = (P_b - sum_{c < b} X_c L_bc^T) V_b^T with the inverted diagonal blocks V_b of diag_kernel.
constexpr int TSM = (TE * (PW + 1) + DB * (PW + 1) + DB * (DB + 1) + TE * (DB + 1)) * (int)sizeof(double);

__global__ void __launch_bounds__(PT) trsm_kernel(const Item *items, int nitems, const SubD *subs, double *arena,
                                                  const double *dinv) {
    extern __shared__ double tsm[];
    double(*P)[PW + 1] = reinterpret_cast<double(*)[PW + 1]>(tsm);
    double(*Lb)[PW + 1] = reinterpret_cast<double(*)[PW + 1]>(tsm + TE * (PW + 1));
    double(*V)[DB + 1] = reinterpret_cast<double(*)[DB + 1]>(tsm + (TE + DB) * (PW + 1));
    double(*T)[DB + 1] = reinterpret_cast<double(*)[DB + 1]>(tsm + (TE + DB) * (PW + 1) + DB * (DB + 1));
    const int b = blockIdx.x, tid = threadIdx.x;
    const int ii = find_item<0>(items, nitems, b);
    const Item it = items[ii];
    const SubD sd = subs[it.sub];
    double *A = arena + sd.a;
    const size_t ld = sd.ld;
    const int k0 = it.k0, w = it.w;
    const int row0 = k0 + w + TE * (b - it.trs0);
    const int rows = min(TE, it.rend - row0);
    const double *vin = dinv + (size_t)ii * (PW / DB) * DB * DB;
    for (int q = tid; q < TE * w; q += PT) {
        const int r = q % TE, j = q / TE;
        P[r][j] = r < rows ? A[(size_t)(k0 + j) * ld + row0 + r] : 0.0;
    }
    for (int c0 = 0; c0 < w; c0 += DB) {
        const int bw = min(DB, w - c0);
        // rows c0.. of the factor block (columns < c0 + bw) and the inverse of its diagonal block
        for (int q = tid; q < bw * (c0 + bw); q += PT) {
            const int r = q % bw, c = q / bw;
            Lb[r][c] = A[(size_t)(k0 + c) * ld + k0 + c0 + r];
        }
        for (int q = tid; q < DB * DB; q += PT) V[q / DB][q % DB] = vin[(size_t)(c0 / DB) * DB * DB + q];
        __syncthreads();
        for (int q = tid; q < TE * bw; q += PT) {
            const int r = q % TE, m = q / TE;
            double sum = P[r][c0 + m];
            for (int c = 0; c < c0; ++c) sum -= P[r][c] * Lb[m][c];
            T[r][m] = sum;
        }
        __syncthreads();
        for (int q = tid; q < TE * bw; q += PT) {
            const int r = q % TE, j = q / TE;
            double sum = 0.0;
            for (int m = 0; m <= j; ++m) sum += T[r][m] * V[j][m];
            P[r][c0 + j] = sum;
        }
        __syncthreads();
    }
    for (int q = tid; q < TE * w; q += PT) {
        const int r = q % TE, j = q / TE;
        if (r < rows) A[(size_t)(k0 + j) * ld + row0 + r] = P[r][j];
    }
}

// Trailing update A_IJ -= L_Ik L_Jk^T of one 64 x 64 lower tile on the FP64 tensor-core path
// (mma.m8n8k4.f64): eight warps, each a 32 x 16 block of the tile as 4 x 2 fragments of 8 x 8.
// Panels are staged k-major with a stride of 72 doubles (8 mod 16), so the 8 x 4 fragment loads take
// the minimum of two shared-memory wavefronts.
constexpr int LDS = 72;

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// The panels stream through shared memory in k-chunks of KC with cp.async
// (two buffers, the next chunk in flight while the current one feeds the MMAs; rows beyond the
// block and k beyond w are zero-filled by the copy), and the C tile is loaded into registers before
// the first chunk so that its latency overlaps the staging.

__device__ __forceinline__ void cp_async8(double *dst, const double *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}

template <int KC>
__global__ void __launch_bounds__(PT, 2) update_pipe_kernel(const Item *items, int nitems, const SubD *subs,
                                                         double *arena) {
    extern __shared__ double upsm[];
    double(*buf)[2][KC][LDS] = reinterpret_cast<double(*)[2][KC][LDS]>(upsm);   // [stage][panel I / J][k][row]
    const int b = blockIdx.x, tid = threadIdx.x;
    const Item it = items[find_item<1>(items, nitems, b)];
    const SubD sd = subs[it.sub];
    double *A = arena + sd.a;
    const size_t ld = sd.ld;
    const int t = b - it.upd0;
    int I = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    while (I * (I + 1) / 2 > t) --I;
    const int J = t - I * (I + 1) / 2;
    const int k0 = it.k0, w = it.w;
    const int r0 = k0 + w;
    const int rI = r0 + TE * I, rJ = r0 + TE * J;
    const int nI = min(TE, it.rend - rI), nJ = min(TE, it.rend - rJ);
    const int nch = (w + KC - 1) / KC;
    // chunk c: 2 panels x 16 k x 64 rows = 2048 doubles, 8 per thread
    // thread tid copies row i = tid % 64 of both panels at k = tid / 64 + 4 u, u < KC / 4
    const int ci = tid & (TE - 1), ck = tid >> 6;
    const bool okI = ci < nI, okJ = ci < nJ;
    const double *srcI = A + (size_t)k0 * ld + rI + ci, *srcJ = A + (size_t)k0 * ld + rJ + ci;
    auto issue = [&](int c) {
        const int st = c & 1;
#pragma unroll
        for (int u = 0; u < KC / 4; ++u) {
            const int kk = ck + 4 * u, k = c * KC + kk;
            const bool kin = k < w;
            const size_t o = kin ? (size_t)k * ld : 0;
            // a copy that is switched off reads nothing; its address is the matrix start regardless
            cp_async8(&buf[st][0][kk][ci], (kin && okI) ? srcI + o : A, kin && okI);
            cp_async8(&buf[st][1][kk][ci], (kin && okJ) ? srcJ + o : A, kin && okJ);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    issue(0);
    if (nch > 1) issue(1);
    const int lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int g = lane >> 2, q4 = lane & 3;
    // the C tile in the accumulator layout, loaded while the first chunks are in flight
    double cv[4][2][2];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int r = wm * 32 + m * 8 + g;
#pragma unroll
        for (int n = 0; n < 2; ++n)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = wn * 16 + n * 8 + 2 * q4 + h;
                cv[m][n][h] = (r < nI && c < nJ) ? A[(size_t)(rJ + c) * ld + rI + r] : 0.0;
            }
    }
    double acc[4][2][2];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 2; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
    for (int c = 0; c < nch; ++c) {
        if (c + 1 < nch) asm volatile("cp.async.wait_group 1;" ::: "memory");
        else asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        const int st = c & 1;
#pragma unroll
        for (int kk = 0; kk < KC; kk += 4) {
            const double *la = &buf[st][0][kk + q4][wm * 32 + g];
            const double *lb = &buf[st][1][kk + q4][wn * 16 + g];
            double a[4], bb[2];
#pragma unroll
            for (int m = 0; m < 4; ++m) a[m] = la[m * 8];
#pragma unroll
            for (int n = 0; n < 2; ++n) bb[n] = lb[n * 8];
#pragma unroll
            for (int m = 0; m < 4; ++m)
#pragma unroll
                for (int n = 0; n < 2; ++n) dmma(acc[m][n], a[m], bb[n]);
        }
        __syncthreads();
        if (c + 2 < nch) issue(c + 2);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int r = wm * 32 + m * 8 + g;
#pragma unroll
        for (int n = 0; n < 2; ++n)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = wn * 16 + n * 8 + 2 * q4 + h;
                if (r < nI && c < nJ && (I != J || r >= c))
                    A[(size_t)(rJ + c) * ld + rI + r] = cv[m][n][h] - acc[m][n][h];
            }
    }
}

// ---------------------------------------------------------------------------------------------
// extraction

// dst (m x m, column-major, full) = scale * symmetric block at (r0, r0) read from the lower triangle
__global__ void copy_sym_kernel(const JobD *jobs, const SubD *subs, const double *arena, double *dst, int which,
                                double scale) {
    const JobD J = jobs[blockIdx.y];
    const SubD sd = subs[J.sub];
    const double *A = arena + sd.a;
    int r0, m;
    long long off;
    if (which == 0) { r0 = J.n; m = J.ni; off = J.s; }                  // -S
    else { r0 = J.nc; m = J.ns; off = J.fx; }                           // fix-DOF block
    if (off < 0) return;
    const long long tot = (long long)m * m;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(q / m), i = (int)(q - (long long)j * m);
        const double v = i >= j ? A[(size_t)(r0 + j) * sd.ld + r0 + i] : A[(size_t)(r0 + i) * sd.ld + r0 + j];
        dst[off + q] = scale * v;
    }
}

// -[B; B0] K^+ B0^T: rows n .. n + ni + m0 - 1, columns n + ni .. n + ni + m0 - 1 of the symmetric
// trailing block, (ni + m0) x m0 column-major
__global__ void copy_b0_kernel(const JobD *jobs, const SubD *subs, const double *arena, double *stage) {
    const JobD J = jobs[blockIdx.y];
    if (J.vo < 0) return;
    const SubD sd = subs[J.sub];
    const double *A = arena + sd.a;
    const int rows = J.ni + J.m0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rows * J.m0; q += gridDim.x * blockDim.x) {
        const int j = q / rows, r = q - j * rows;
        const int gi = J.n + r, gj = J.n + J.ni + j;
        const double v = gi >= gj ? A[(size_t)gj * sd.ld + gi] : A[(size_t)gi * sd.ld + gj];
        stage[J.vo + q] = -v;
    }
}


// A(nc + i, nc + j) += reg(i, j), i >= j
__global__ void add_reg_kernel(const JobD *jobs, const SubD *subs, double *arena, const double *reg) {   // reg at J.fx
    const JobD J = jobs[blockIdx.x];
    const SubD sd = subs[J.sub];
    double *A = arena + sd.a;
    for (int q = threadIdx.x; q < J.ns * J.ns; q += blockDim.x) {
        const int j = q / J.ns, i = q - j * J.ns;
        if (i >= j) A[(size_t)(J.nc + j) * sd.ld + J.nc + i] += reg[J.fx + q];
    }
}

// ---------------------------------------------------------------------------------------------
// device-resident outputs

constexpr int TL = 32;    // tile edge of the dual iteration's Schur and K^+ stores

struct TJob {
    int sub;              // batch-local subdomain
    int r0, m;            // symmetric block at (r0, r0) of size m (sym), or the leading m x m factor (kp)
    int tn;               // tiles per side
    long long tile0;      // first tile in the store
    int cta0;             // first CTA of this job
    double scale;
};

__device__ __forceinline__ int find_tjob(const TJob *tj, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tj[mid].cta0 <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Upper tiles of a symmetric block kept in the lower triangle: one CTA per tile (I <= J, row of
// tiles after row of tiles), tile[r][c] = scale * M(32 I + r, 32 J + c), zero beyond m.
__global__ void __launch_bounds__(PT) sym_tiles_kernel(const TJob *tj, int ntj, const SubD *subs,
                                                       const double *arena, double *out) {
    const TJob J_ = tj[find_tjob(tj, ntj, blockIdx.x)];
    const SubD sd = subs[J_.sub];
    const double *A = arena + sd.a;
    const int t = blockIdx.x - J_.cta0, tn = J_.tn;
    // row of tiles I: first tile I * tn - I (I - 1) / 2
    int lo = 0, hi = tn - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)mid * tn - (long long)mid * (mid - 1) / 2 <= t) lo = mid;
        else hi = mid - 1;
    }
    const int I = lo, J = I + (t - (int)((long long)I * tn - (long long)I * (I - 1) / 2));
    double *tile = out + (size_t)(J_.tile0 + t) * TL * TL;
    for (int q = threadIdx.x; q < TL * TL; q += PT) {
        const int r = q / TL, c = q % TL;
        const int i = TL * I + r, j = TL * J + c;
        double v = 0.0;
        if (i < J_.m && j < J_.m)
            v = i >= j ? A[(size_t)(J_.r0 + j) * sd.ld + J_.r0 + i] : A[(size_t)(J_.r0 + i) * sd.ld + J_.r0 + j];
        tile[q] = J_.scale * v;
    }
}

// Lower tiles of the leading factor (I >= J, column of tiles after column of tiles): tile[r][c] =
// L(32 I + r, 32 J + c); beyond m the diagonal is 1 and the rest 0.  A diagonal tile is replaced by
// the inverse of its lower triangle (forward substitution, one lane per column).
__global__ void __launch_bounds__(PT) kp_tiles_kernel(const TJob *tj, int ntj, const SubD *subs,
                                                      const double *arena, double *out) {
    __shared__ double T[TL][TL + 1];
    __shared__ double V[TL][TL + 1];
    const TJob J_ = tj[find_tjob(tj, ntj, blockIdx.x)];
    const SubD sd = subs[J_.sub];
    const double *A = arena + sd.a;
    const int t = blockIdx.x - J_.cta0, tn = J_.tn;
    // column of tiles J: first tile J * tn - J (J - 1) / 2
    int lo = 0, hi = tn - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)mid * tn - (long long)mid * (mid - 1) / 2 <= t) lo = mid;
        else hi = mid - 1;
    }
    const int J = lo, I = J + (t - (int)((long long)J * tn - (long long)J * (J - 1) / 2));
    const int m = J_.m;
    for (int q = threadIdx.x; q < TL * TL; q += PT) {
        const int c = q / TL, r = q % TL;     // rows contiguous in the arena's column
        const int i = TL * I + r, j = TL * J + c;
        double v;
        if (i < m && j < m) v = i >= j ? A[(size_t)j * sd.ld + i] : 0.0;
        else v = i == j ? 1.0 : 0.0;
        T[r][c] = v;
    }
    __syncthreads();
    double *tile = out + (size_t)(J_.tile0 + t) * TL * TL;
    if (I != J) {
        for (int q = threadIdx.x; q < TL * TL; q += PT) tile[q] = T[q / TL][q % TL];
        return;
    }
    if (threadIdx.x < TL) {
        const int c = threadIdx.x;
        for (int r = 0; r < c; ++r) V[r][c] = 0.0;
        for (int r = c; r < TL; ++r) {
            double sum = r == c ? 1.0 : 0.0;
            for (int k = c; k < r; ++k) sum -= T[r][k] * V[k][c];
            V[r][c] = sum / T[r][r];
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < TL * TL; q += PT) tile[q] = V[q / TL][q % TL];
}

// Kernel vectors: backward solve L_rr^T x_r = -L_sr^T N over 64-column blocks, descending.  One step
// per block J (the first step is the fix block itself, whose x = N is given): CTA `below` solves
// x_J = L_JJ^-T y_J and stores it; CTAs 0..below-1 subtract L_{J,i}^T x_J from y_i.  X and Y hold
// n x nk per subdomain, column after column.
struct BItem {
    int sub, c0, w;       // block rows [c0, c0 + w)
    int given;            // 1: x_J is known (the fix block), no solve and no store
    int nk;
    long long xo;         // offset of the subdomain's X / Y
    int n;                // rows of X / Y
    int cta0;
};

__global__ void __launch_bounds__(PT) bsolve_kernel(const BItem *items, int nitems, const SubD *subs,
                                                    const double *arena, double *X, double *Y) {
    __shared__ double D[BS][BS + 1];    // L_JJ (lower), or the tile L(J rows, i columns)
    __shared__ double x[BS][8];
    __shared__ double y[BS][8];
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].cta0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const BItem it = items[lo];
    const SubD sd = subs[it.sub];
    const double *A = arena + sd.a;
    const int tid = threadIdx.x, w = it.w, nk = it.nk, c0 = it.c0;
    const int l = blockIdx.x - it.cta0;
    const int below = (c0 + BS - 1) / BS;
    double *Xs = X + it.xo, *Ys = Y + it.xo;
    if (it.given) {
        for (int q = tid; q < BS * nk; q += PT) {
            const int r = q % BS, k = q / BS;
            x[r][k] = r < w ? Xs[(size_t)k * it.n + c0 + r] : 0.0;
        }
    } else {
        for (int q = tid; q < w * w; q += PT) {
            const int i = q % w, j = q / w;
            if (i >= j) D[i][j] = A[(size_t)(c0 + j) * sd.ld + c0 + i];
        }
        for (int q = tid; q < BS * nk; q += PT) {
            const int r = q % BS, k = q / BS;
            y[r][k] = r < w ? Ys[(size_t)k * it.n + c0 + r] : 0.0;
        }
        __syncthreads();
        for (int r = w - 1; r >= 0; --r) {
            if (tid < nk) x[r][tid] = y[r][tid] / D[r][r];
            __syncthreads();
            for (int q = tid; q < r * nk; q += PT) {
                const int i = q % r, k = q / r;
                y[i][k] -= D[r][i] * x[r][k];
            }
            __syncthreads();
        }
        if (l == below) {
            for (int q = tid; q < w * nk; q += PT) {
                const int r = q % w, k = q / w;
                Xs[(size_t)k * it.n + c0 + r] = x[r][k];
            }
            return;
        }
    }
    __syncthreads();
    // y_i -= L(J rows, i columns)^T x_J, i = block l: columns 64 l .. min(64 l + 64, c0) - 1
    const int cm = min(BS, c0 - BS * l);
    for (int q = tid; q < cm * w; q += PT) {
        const int r = q % w, c = q / w;
        D[r][c] = A[(size_t)(BS * l + c) * sd.ld + c0 + r];
    }
    __syncthreads();
    for (int q = tid; q < cm * nk; q += PT) {
        const int c = q % cm, k = q / cm;
        double sum = 0.0;
        for (int r = 0; r < w; ++r) sum += D[r][c] * x[r][k];
        Ys[(size_t)k * it.n + BS * l + c] -= sum;
    }
}

// ---------------------------------------------------------------------------------------------
// host side

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    void reserve(size_t m) {
        if (m <= n) return;
        if (p) PCHECK(cudaFree(p));
        p = nullptr;
        n = 0;
        PCHECK(cudaMalloc(&p, std::max<size_t>(m, 1) * sizeof(T)));
        n = m;
    }
    void put(const std::vector<T> &v) {
        reserve(v.size());
        if (!v.empty()) PCHECK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

struct Step {
    std::vector<Item> items;
    int ntrs = 0, nupd = 0;
};

// Steps of one phase: columns [lo(job), hi(job)) in PW panels, rows below up to rend(job).
template <typename Lo, typename Hi, typename Rend>
std::vector<Step> make_steps(int njobs, Lo lo, Hi hi, Rend rend, double &flops) {
    std::vector<Step> steps;
    for (int s = 0;; ++s) {
        Step st;
        for (int j = 0; j < njobs; ++j) {
            const int k0 = lo(j) + s * PW;
            if (k0 >= hi(j)) continue;
            Item it;
            it.sub = j;
            it.k0 = k0;
            it.w = std::min(PW, hi(j) - k0);
            it.rend = rend(j);
            it.trs0 = st.ntrs;
            it.upd0 = st.nupd;
            const int below = it.rend - k0 - it.w;
            const int nb = below > 0 ? (below + TE - 1) / TE : 0;
            st.ntrs += nb;
            st.nupd += nb * (nb + 1) / 2;
            st.items.push_back(it);
            const double w = it.w, r = below;
            flops += w * w * w / 3.0 + r * w * w + r * r * w;
        }
        if (st.items.empty()) break;
        steps.push_back(std::move(st));
    }
    return steps;
}

}  // namespace

DevPrepStore::~DevPrepStore() {
    if (s_tiles) cudaFree(s_tiles);
    if (dir_tiles) cudaFree(dir_tiles);
    if (kp_tiles) cudaFree(kp_tiles);
}

void device_factor(const ElementData &el, std::vector<DevFactorJob> &jobs, const RegulariseFn &regularise,
                   size_t mem_budget, DevFactorTimes *times, DevPrepStore *store, int ndom) {
    const double t_start = now_s();
    DevFactorTimes tm;
    const int nj = (int)jobs.size();
    if (nj == 0) {
        if (times) *times = tm;
        return;
    }
    const bool resident = store != nullptr;
    if (resident) {
        // tile stores for every subdomain (slots without a job get no tiles)
        std::vector<int> sn(ndom, 0), st(ndom, 0), kn(ndom, 0);
        bool dir = false;
        for (const DevFactorJob &J : jobs) {
            FETI_CHECK(J.slot >= 0 && J.slot < ndom, "FETI4I: device factorisation job outside the store");
            sn[J.slot] = J.ni;
            kn[J.slot] = J.n;
            if (J.want_sdir) {
                st[J.slot] = J.n - J.n1;
                dir = true;
            }
        }
        auto offsets = [&](const std::vector<int> &m, bool lower) {
            std::vector<long long> o(ndom + 1, 0);
            for (int d = 0; d < ndom; ++d) {
                const long long t = (m[d] + TL - 1) / TL;
                o[d + 1] = o[d] + t * (t + 1) / 2;
            }
            (void)lower;
            return o;
        };
        store->nd = ndom;
        store->s_tile0 = offsets(sn, false);
        store->kp_tile0 = offsets(kn, true);
        const size_t tb = (size_t)TL * TL * sizeof(double);
        PCHECK(cudaMalloc(&store->s_tiles, std::max<long long>(store->s_tile0[ndom], 1) * tb));
        PCHECK(cudaMalloc(&store->kp_tiles, std::max<long long>(store->kp_tile0[ndom], 1) * tb));
        if (dir) {
            store->dir_tile0 = offsets(st, false);
            PCHECK(cudaMalloc(&store->dir_tiles, std::max<long long>(store->dir_tile0[ndom], 1) * tb));
        }
    }
    if (mem_budget == 0) {
        size_t fr = 0, tot = 0;
        PCHECK(cudaMemGetInfo(&fr, &tot));
        mem_budget = fr / 2;
    }
    PCHECK(cudaFuncSetAttribute(diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DSM));
    // k-chunks of 16 (32 measured 9 % slower on 4 subdomains of 12^3, 2 % faster on 512)
    constexpr int UPSM16 = 2 * 2 * 16 * LDS * (int)sizeof(double);
    PCHECK(cudaFuncSetAttribute(update_pipe_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, UPSM16));
    PCHECK(cudaFuncSetAttribute(trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TSM));

    // per-job sizes and batches
    struct Sz {
        int ld, N;
        size_t a, s, fx, vals, pos, v;
    };
    std::vector<Sz> sz(nj);
    for (int j = 0; j < nj; ++j) {
        const DevFactorJob &J = jobs[j];
        FETI_CHECK(J.n > 0 && J.ns >= 0 && J.n1 >= 0 && J.n1 + J.ns <= J.n, "FETI4I: invalid device factorisation job");
        Sz &z = sz[j];
        FETI_CHECK(J.b0pos.size() == J.b0sign.size(), "FETI4I: corner rows incomplete");
        z.N = J.n + J.ni + (int)J.b0pos.size();
        z.ld = (z.N + 31) / 32 * 32;
        z.a = (size_t)z.ld * z.N;
        z.s = (resident || !J.S) ? 0 : (size_t)J.ni * J.ni;
        z.fx = (size_t)J.ns * J.ns;
        z.v = J.b0pos.empty() ? 0 : (size_t)(J.ni + J.b0pos.size()) * J.b0pos.size();
        z.vals = 0;
        for (int k = 0; k < J.nelem; ++k) {
            const int e = J.elems[k];
            const size_t nd = (size_t)(el.dof_ptr[e + 1] - el.dof_ptr[e]);
            z.vals += nd * nd;
        }
        z.pos = J.elpos.size();
    }
    std::vector<int> bstart{0};
    {
        size_t cur = 0;
        for (int j = 0; j < nj; ++j) {
            const size_t bytes = 8 * (sz[j].a + sz[j].s + sz[j].fx + sz[j].vals + sz[j].v +
                                      (resident ? 16 * (size_t)jobs[j].n : 0)) +
                                 4 * sz[j].pos;
            if (j > bstart.back() && cur + bytes > mem_budget) {
                bstart.push_back(j);
                cur = 0;
            }
            cur += bytes;
        }
        bstart.push_back(nj);
    }

    DevBuf<double> arena, stage, fxb, vals, bsign, reg, part, dX, dY, dinvb;
    DevBuf<TJob> dtj;
    DevBuf<BItem> dbi;
    DevBuf<int> epos, bpos, fail, list;
    DevBuf<SubD> dsubs;
    DevBuf<JobD> djobs;
    DevBuf<ElemD> dels;
    DevBuf<Item> ditems;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    PCHECK(cudaEventCreate(&ev0));
    PCHECK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evg{ev0, ev1};
    constexpr int KN_BLOCKS = 64;
    double *pinned = nullptr;   // staging of the element values
    size_t pinned_n = 0;
    struct PinGuard {
        double *&p;
        ~PinGuard() {
            if (p) cudaFreeHost(p);
        }
    } ping{pinned};

    // Element values: when the jobs use most of the element array and it takes a small share of the
    // device memory, it goes to the device once and the assembly reads it in place.
    bool all_vals = false;
    {
        size_t used = 0;
        for (const Sz &z : sz) used += z.vals;
        size_t fr = 0, tot = 0;
        PCHECK(cudaMemGetInfo(&fr, &tot));
        const size_t bytes = el.vals.size() * sizeof(double);
        if (used > 0 && used * 2 >= el.vals.size() && bytes < fr / 8) {
            vals.reserve(el.vals.size());
            PCHECK(cudaMemcpy(vals.p, el.vals.data(), bytes, cudaMemcpyHostToDevice));
            all_vals = true;
        }
    }
    double th_setup = now_s() - t_start, th_stage = 0.0, th_wait = 0.0, th_reg = 0.0, th_out = 0.0;
    double th_gather = 0.0, th_h2d = 0.0;
    for (size_t bi = 0; bi + 1 < bstart.size(); ++bi) {
        double tq = now_s();
        const int j0 = bstart[bi], j1 = bstart[bi + 1], nb = j1 - j0;
        // layout of the batch
        std::vector<SubD> subs(nb);
        std::vector<JobD> jd(nb);
        size_t a_tot = 0, st_tot = 0, fx_tot = 0, v_tot = 0, p_tot = 0, b_tot = 0;
        for (int q = 0; q < nb; ++q) {
            const DevFactorJob &J = jobs[j0 + q];
            const Sz &z = sz[j0 + q];
            subs[q] = SubD{(long long)a_tot, z.ld, J.n, z.N};
            a_tot += z.a;
            JobD &d = jd[q];
            d.sub = q;
            d.n = J.n;
            d.n1 = J.n1;
            d.nc = J.n - J.ns;
            d.ni = J.ni;
            d.ns = J.ns;
            d.m0 = (int)J.b0pos.size();
            d.nrow = J.ni + d.m0;
            d.boff = (long long)b_tot;
            b_tot += d.nrow;
            d.s = z.s ? (long long)st_tot : -1;
            st_tot += z.s;
            d.vo = z.v ? (long long)st_tot : -1;
            st_tot += z.v;
            d.fx = (long long)fx_tot;
            fx_tot += z.fx;
            v_tot += z.vals;
            p_tot += z.pos;
        }
        // element data, colour lists, B~ rows
        size_t hv_n = 0;
        std::vector<const double *> src;   // K_e of every batch element (gathered in parallel below)
        std::vector<int> hp;
        hp.reserve(p_tot);
        std::vector<ElemD> he;
        std::vector<std::vector<int>> colors;
        std::vector<int> hbp;
        std::vector<double> hbs;
        hbp.reserve(b_tot);
        hbs.reserve(b_tot);
        for (int q = 0; q < nb; ++q) {
            const DevFactorJob &J = jobs[j0 + q];
            FETI_CHECK((int)J.elcolor.size() == J.nelem, "FETI4I: element colours missing");
            if ((int)colors.size() < J.ncolors) colors.resize(J.ncolors);
            size_t po = 0;
            for (int k = 0; k < J.nelem; ++k) {
                const int e = J.elems[k];
                const int nd = (int)(el.dof_ptr[e + 1] - el.dof_ptr[e]);
                ElemD E;
                E.val = all_vals ? (long long)el.val_ptr[e] : (long long)hv_n;
                E.nd = nd;
                E.pos = (int)(hp.size());
                E.sub = q;
                src.push_back(el.vals.data() + el.val_ptr[e]);
                hv_n += (size_t)nd * nd;
                hp.insert(hp.end(), J.elpos.begin() + po, J.elpos.begin() + po + nd);
                po += nd;
                colors[J.elcolor[k]].push_back((int)he.size());
                he.push_back(E);
            }
            FETI_CHECK(po == J.elpos.size(), "FETI4I: element DOF positions do not match the elements");
            FETI_CHECK((int)J.bpos.size() == J.ni && (int)J.bsign.size() == J.ni, "FETI4I: B rows missing");
            hbp.insert(hbp.end(), J.bpos.begin(), J.bpos.end());
            hbs.insert(hbs.end(), J.bsign.begin(), J.bsign.end());
            for (int p : J.b0pos) FETI_CHECK(p >= J.n1 && p < J.n, "FETI4I: a corner DOF is not on the subdomain interface");
            hbp.insert(hbp.end(), J.b0pos.begin(), J.b0pos.end());
            hbs.insert(hbs.end(), J.b0sign.begin(), J.b0sign.end());
        }
        std::vector<int> hl;
        std::vector<std::pair<int, int>> cl;   // (offset, count) per colour
        for (auto &c : colors) {
            cl.emplace_back((int)hl.size(), (int)c.size());
            hl.insert(hl.end(), c.begin(), c.end());
        }
        arena.reserve(a_tot);
        stage.reserve(st_tot);
        fxb.reserve(fx_tot);
        // element values: parallel gather into pinned memory, one copy to the device (unless the
        // whole element array is already there)
        const double tg0 = now_s();
        if (all_vals) hv_n = 0;
        if (hv_n > pinned_n) {
            if (pinned) PCHECK(cudaFreeHost(pinned));
            pinned = nullptr;
            pinned_n = 0;
            PCHECK(cudaMallocHost(&pinned, hv_n * sizeof(double)));
            pinned_n = hv_n;
        }
        if (!all_vals) {
            const long long ne_ = (long long)he.size();
#pragma omp parallel for schedule(static)
            for (long long k = 0; k < ne_; ++k)
                std::memcpy(pinned + he[k].val, src[k], sizeof(double) * (size_t)he[k].nd * he[k].nd);
        }
        const double tg1 = now_s();
        if (!all_vals) {
            vals.reserve(hv_n);
            if (hv_n) PCHECK(cudaMemcpy(vals.p, pinned, hv_n * sizeof(double), cudaMemcpyHostToDevice));
        }
        th_gather += tg1 - tg0;
        th_h2d += now_s() - tg1;
        epos.put(hp);
        dels.put(he);
        list.put(hl);
        bpos.put(hbp);
        bsign.put(hbs);
        dsubs.put(subs);
        djobs.put(jd);
        std::vector<int> hf(nb, INT_MAX);
        fail.put(hf);
        part.reserve((size_t)nb * KN_BLOCKS);

        // elimination schedule
        double flops = 0.0;
        auto jn = [&](int q) { return jobs[j0 + q].n; };
        auto jn1 = [&](int q) { return jobs[j0 + q].n1; };
        auto jnc = [&](int q) { return jobs[j0 + q].n - jobs[j0 + q].ns; };
        auto jN = [&](int q) { return sz[j0 + q].N; };
        auto zero = [](int) { return 0; };
        std::vector<Step> ph1 = make_steps(nb, zero, jn1, jn, flops);
        std::vector<Step> ph2 = make_steps(nb, jn1, jnc, jN, flops);
        std::vector<Step> ph3 = make_steps(nb, jnc, jn, jN, flops);
        std::vector<Item> all;
        auto offsets = [&](std::vector<Step> &ph) {
            std::vector<size_t> o;
            for (auto &s : ph) {
                o.push_back(all.size());
                all.insert(all.end(), s.items.begin(), s.items.end());
            }
            return o;
        };
        std::vector<size_t> o1 = offsets(ph1), o2 = offsets(ph2), o3 = offsets(ph3);
        ditems.put(all);
        size_t maxitems = 0;   // inverted 32 x 32 diagonal blocks of the largest step
        for (auto *ph : {&ph1, &ph2, &ph3})
            for (auto &st : *ph) maxitems = std::max(maxitems, st.items.size());
        dinvb.reserve(std::max<size_t>(maxitems, 1) * (PW / DB) * DB * DB);
        tm.flops += flops;

        th_stage += now_s() - tq;
        tq = now_s();
        PCHECK(cudaEventRecord(ev0));
        PCHECK(cudaMemset(arena.p, 0, a_tot * sizeof(double)));
        for (int q = 0; q < nb; ++q) {
            const DevFactorJob &J = jobs[j0 + q];
            if (!J.dense) continue;
            PCHECK(cudaMemcpy2D(arena.p + subs[q].a, (size_t)subs[q].ld * sizeof(double), J.dense,
                                (size_t)J.n * sizeof(double), (size_t)J.n * sizeof(double), J.n,
                                cudaMemcpyHostToDevice));
        }
        for (auto &c : cl) {
            if (c.second == 0) continue;
            assemble_kernel<<<std::min(c.second, 65535), 128>>>(dels.p, list.p + c.first, c.second, vals.p, epos.p,
                                                               dsubs.p, arena.p);
            ++tm.launches;
        }
        brows_kernel<<<dim3(8, nb), PT>>>(djobs.p, dsubs.p, bpos.p, bsign.p, arena.p);
        knorm_kernel<<<dim3(KN_BLOCKS, nb), PT>>>(djobs.p, dsubs.p, arena.p, part.p);
        tm.launches += 2;
        PCHECK(cudaGetLastError());
        auto run = [&](std::vector<Step> &ph, std::vector<size_t> &off) {
            for (size_t s = 0; s < ph.size(); ++s) {
                const Item *it = ditems.p + off[s];
                const int ni = (int)ph[s].items.size();
                diag_kernel<<<ni, PT, DSM>>>(it, dsubs.p, arena.p, fail.p, dinvb.p);
                ++tm.launches;
                if (ph[s].ntrs > 0) {
                    trsm_kernel<<<ph[s].ntrs, PT, TSM>>>(it, ni, dsubs.p, arena.p, dinvb.p);
                    ++tm.launches;
                }
                if (ph[s].nupd > 0) {
                    update_pipe_kernel<16><<<ph[s].nupd, PT, UPSM16>>>(it, ni, dsubs.p, arena.p);
                    ++tm.launches;
                }
            }
            PCHECK(cudaGetLastError());
        };
        // symmetric-block or factor tiles of this batch into a store
        auto tiles = [&](int which, double *out, const std::vector<long long> &t0, double scale) {
            std::vector<TJob> tj;
            int ctas = 0;
            for (int q = 0; q < nb; ++q) {
                const DevFactorJob &J = jobs[j0 + q];
                TJob t;
                t.sub = q;
                if (which == 0) { t.r0 = J.n; t.m = J.ni; }
                else if (which == 1) { if (!J.want_sdir) continue; t.r0 = J.n1; t.m = J.n - J.n1; }
                else { t.r0 = 0; t.m = J.n; }
                t.tn = (t.m + TL - 1) / TL;
                t.tile0 = t0[J.slot];
                t.cta0 = ctas;
                t.scale = scale;
                const int cnt = t.tn * (t.tn + 1) / 2;
                if (cnt == 0) continue;
                ctas += cnt;
                tj.push_back(t);
            }
            if (ctas == 0) return;
            dtj.put(tj);
            if (which == 2) kp_tiles_kernel<<<ctas, PT>>>(dtj.p, (int)tj.size(), dsubs.p, arena.p, out);
            else sym_tiles_kernel<<<ctas, PT>>>(dtj.p, (int)tj.size(), dsubs.p, arena.p, out);
            ++tm.launches;
            PCHECK(cudaGetLastError());
        };
        run(ph1, o1);
        if (resident && store->dir_tiles) tiles(1, store->dir_tiles, store->dir_tile0, 1.0);   // Dirichlet
        run(ph2, o2);
        copy_sym_kernel<<<dim3(1, nb), PT>>>(djobs.p, dsubs.p, arena.p, fxb.p, 2, 1.0);       // fix block
        ++tm.launches;
        PCHECK(cudaGetLastError());
        PCHECK(cudaEventRecord(ev1));
        PCHECK(cudaEventSynchronize(ev1));
        th_wait += now_s() - tq;
        tq = now_s();
        float ms = 0.f;
        PCHECK(cudaEventElapsedTime(&ms, ev0, ev1));
        tm.device_ms += ms;

        // host: fix-block regularisation (skipped for subdomains whose elimination already failed)
        PCHECK(cudaMemcpy(hf.data(), fail.p, nb * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<double> hfx(fx_tot), hreg(fx_tot, 0.0);
        if (fx_tot) PCHECK(cudaMemcpy(hfx.data(), fxb.p, fx_tot * sizeof(double), cudaMemcpyDeviceToHost));
        for (int q = 0; q < nb; ++q)
            if (jobs[j0 + q].ns > 0 && hf[q] == INT_MAX) regularise(j0 + q, hfx.data() + jd[q].fx, hreg.data() + jd[q].fx);
        reg.put(hreg);
        th_reg += now_s() - tq;
        tq = now_s();
        PCHECK(cudaEventRecord(ev0));
        add_reg_kernel<<<nb, 64>>>(djobs.p, dsubs.p, arena.p, reg.p);
        ++tm.launches;
        run(ph3, o3);
        copy_b0_kernel<<<dim3(16, nb), PT>>>(djobs.p, dsubs.p, arena.p, stage.p);
        ++tm.launches;
        std::vector<BItem> bitems;
        std::vector<std::vector<size_t>> bsteps;   // item ranges per backward-solve step
        size_t x_tot = 0;
        if (resident) {
            tiles(0, store->s_tiles, store->s_tile0, -1.0);
            tiles(2, store->kp_tiles, store->kp_tile0, 1.0);
            // kernel vectors: X = [x_r; N], Y = 0
            std::vector<long long> xo(nb);
            int maxb = 0;
            for (int q = 0; q < nb; ++q) {
                const DevFactorJob &J = jobs[j0 + q];
                FETI_CHECK(J.nk >= 0 && J.nk <= 8, "FETI4I: kernel dimension above 8");
                xo[q] = (long long)x_tot;
                x_tot += (size_t)J.n * J.nk;
                maxb = std::max(maxb, (J.n - J.ns + BS - 1) / BS);
            }
            std::vector<double> hx(std::max<size_t>(x_tot, 1), 0.0);
            for (int q = 0; q < nb; ++q) {
                const DevFactorJob &J = jobs[j0 + q];
                FETI_CHECK((int)J.N.size() >= J.ns * J.nk, "FETI4I: kernel eigenvectors missing");
                for (int k = 0; k < J.nk; ++k)
                    for (int r = 0; r < J.ns; ++r) hx[xo[q] + (size_t)k * J.n + (J.n - J.ns) + r] = J.N[(size_t)k * J.ns + r];
            }
            dX.put(hx);
            dY.reserve(hx.size());
            PCHECK(cudaMemset(dY.p, 0, hx.size() * sizeof(double)));
            for (int step = 0; step <= maxb; ++step) {
                std::vector<size_t> rng{bitems.size()};
                int ctas = 0;
                for (int q = 0; q < nb; ++q) {
                    const DevFactorJob &J = jobs[j0 + q];
                    if (J.nk == 0) continue;
                    const int nr = J.n - J.ns, nbr = (nr + BS - 1) / BS;
                    BItem b;
                    b.sub = q;
                    b.nk = J.nk;
                    b.xo = xo[q];
                    b.n = J.n;
                    b.cta0 = ctas;
                    int cnt;
                    if (step == 0) {
                        b.c0 = nr;
                        b.w = J.ns;
                        b.given = 1;
                        cnt = nbr;
                    } else {
                        const int blk = nbr - step;
                        if (blk < 0) continue;
                        b.c0 = BS * blk;
                        b.w = std::min(BS, nr - b.c0);
                        b.given = 0;
                        cnt = blk + 1;
                    }
                    if (cnt == 0) continue;
                    ctas += cnt;
                    bitems.push_back(b);
                }
                rng.push_back(bitems.size());
                rng.push_back((size_t)ctas);
                bsteps.push_back(rng);
            }
            dbi.put(bitems);
            for (auto &r : bsteps) {
                const int cnt = (int)(r[1] - r[0]), ctas = (int)r[2];
                if (ctas == 0) continue;
                bsolve_kernel<<<ctas, PT>>>(dbi.p + r[0], cnt, dsubs.p, arena.p, dX.p, dY.p);
                ++tm.launches;
            }
            PCHECK(cudaGetLastError());
        } else {
            copy_sym_kernel<<<dim3(256, nb), PT>>>(djobs.p, dsubs.p, arena.p, stage.p, 0, -1.0);
            tm.launches += 1;
            PCHECK(cudaGetLastError());
        }
        PCHECK(cudaEventRecord(ev1));
        PCHECK(cudaEventSynchronize(ev1));
        th_wait += now_s() - tq;
        tq = now_s();
        PCHECK(cudaEventElapsedTime(&ms, ev0, ev1));
        tm.device_ms += ms;

        // results
        PCHECK(cudaMemcpy(hf.data(), fail.p, nb * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<double> hpart((size_t)nb * KN_BLOCKS);
        PCHECK(cudaMemcpy(hpart.data(), part.p, hpart.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int q = 0; q < nb; ++q) {
            DevFactorJob &J = jobs[j0 + q];
            J.fail_col = hf[q] == INT_MAX ? -1 : hf[q];
            double s = 0.0;
            for (int k = 0; k < KN_BLOCKS; ++k) s += hpart[(size_t)q * KN_BLOCKS + k];
            J.knorm = std::sqrt(s);
            if (jd[q].vo >= 0 && (J.V || J.F0)) {
                const int m0 = jd[q].m0, rows = J.ni + m0;
                std::vector<double> blk((size_t)rows * m0);
                PCHECK(cudaMemcpy(blk.data(), stage.p + jd[q].vo, blk.size() * sizeof(double), cudaMemcpyDeviceToHost));
                for (int c = 0; c < m0; ++c) {
                    if (J.V)
                        for (int r = 0; r < J.ni; ++r) J.V[(size_t)c * J.ni + r] = blk[(size_t)c * rows + r];
                    if (J.F0)
                        for (int r = 0; r < m0; ++r) J.F0[(size_t)c * m0 + r] = blk[(size_t)c * rows + J.ni + r];
                }
            }
            if (resident) {
                if (J.Rp && J.nk > 0) {
                    size_t o = 0;
                    for (int p = 0; p < q; ++p) o += (size_t)jobs[j0 + p].n * jobs[j0 + p].nk;
                    PCHECK(cudaMemcpy(J.Rp, dX.p + o, (size_t)J.n * J.nk * sizeof(double), cudaMemcpyDeviceToHost));
                }
                continue;
            }
            if (J.S) PCHECK(cudaMemcpy(J.S, stage.p + jd[q].s, sz[j0 + q].s * sizeof(double), cudaMemcpyDeviceToHost));
        }
        th_out += now_s() - tq;
        ++tm.batches;
    }
    tm.total_s = now_s() - t_start;
    FETI_LOG(2, "FETI4I: device factorisation: setup %.3f s, staging %.3f s (element gather %.3f s, copy %.3f s), "
                "device waits %.3f s, fix blocks %.3f s, results %.3f s\n", th_setup, th_stage, th_gather, th_h2d,
             th_wait, th_reg, th_out);
    if (times) *times = tm;
}

}  // namespace feti
