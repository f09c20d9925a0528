// Device factorisation and Schur-complement assembly of the subdomain matrices (sm_100a, FP64).
//
// The host's symbolic phase fixes the factor order of every subdomain matrix K_i:
// [untouched DOFs | DOFs touched by B_i, fix DOFs excluded | fix DOFs].  The device appends the
// signed rows of B_i below K_i and runs one partial Cholesky over the n columns of K_i:
//
//     [ K_reg   B~^T ]      eliminate the first n columns      trailing ni x ni block
//     [ B~      0    ]   ------------------------------------>  = -B~ K_reg^-1 B~^T = -S_i
//
// (B~ row r holds sign_r at the factor position of the row's DOF).  The same elimination leaves
// the Cholesky factor of K_reg in the leading n x n block (the K^+ of the dual iteration) and,
// snapshotted after the untouched columns, the Dirichlet-preconditioner Schur complement of K onto
// the touched DOFs.  Between the last touched column and the fix columns the host regularises the
// fix-DOF Schur block (the algebraic kernel detection).  This replaces the host dense path in
// prep.cpp, which computes the same quantities (SparseSolverMKL.cpp:1207-1428 of the reference
// assembles S_i with PARDISO's Schur-complement mode on the host).
#pragma once

#include <functional>
#include <vector>

#include "decompose.h"

namespace feti {

// Device-resident results of device_factor for Total FETI: the tile stores the dual iteration
// reads, handed to the GPU solver without a host copy.  Subdomain d's tiles start at tile0[d]
// (tile0 has ndom + 1 entries); a tile is 32 x 32 doubles, row-major.
struct DevPrepStore {
    int nd = 0;
    double *s_tiles = nullptr;       // S_i: upper tiles (I <= J), row of tiles after row of tiles
    std::vector<long long> s_tile0;
    double *dir_tiles = nullptr;     // Dirichlet Schur complements, same layout (null without them)
    std::vector<long long> dir_tile0;
    double *kp_tiles = nullptr;      // K_reg factor: lower tiles (I >= J), column of tiles after column,
    std::vector<long long> kp_tile0; // diagonal tiles replaced by the inverse of their triangle
    ~DevPrepStore();
};

struct DevFactorJob {
    // inputs
    int slot = 0;                // subdomain index (tile offsets in a DevPrepStore)
    int n = 0;                   // DOFs
    int n1 = 0;                  // untouched DOFs (eliminated first)
    int ns = 0;                  // fix DOFs (eliminated last)
    int ni = 0;                  // rows of B_i
    const double *dense = nullptr;  // instead of elements: the n x n matrix itself (column-major)
    const int *elems = nullptr;  // element ids of the subdomain (into ElementData)
    int nelem = 0;
    std::vector<int> elpos;      // factor position of every element DOF, element after element
    std::vector<int> elcolor;    // per element: colour (elements of one colour share no DOF)
    int ncolors = 0;
    std::vector<int> bpos;       // per B row: factor position of its DOF (>= n1)
    std::vector<double> bsign;   // per B row: sign
    // Hybrid Total FETI: the corner rows B0 of the subdomain (one DOF each, factor position >= n1),
    // appended after the B rows; the trailing block then also holds B K^+ B0^T and B0 K^+ B0^T
    std::vector<int> b0pos;
    std::vector<double> b0sign;
    double *V = nullptr;         // ni x m0: B K_reg^-1 B0^T (column-major), copied back
    double *F0 = nullptr;        // m0 x m0: B0 K_reg^-1 B0^T, copied back
    bool want_sdir = false;      // snapshot the Schur complement onto the touched DOFs
    // set by the regularisation callback: kernel dimension and the kernel eigenvectors N (ns x nk)
    int nk = 0;
    std::vector<double> N;
    // outputs (host buffers sized by the caller)
    double *Rp = nullptr;        // n x nk: kernel [-L_rr^-T L_sr^T N; N] in factor order (store mode)
    double *S = nullptr;         // ni x ni, column-major, full symmetric (without a store: the
                                 // coarse problem's dense inverse)
    double knorm = 0.0;          // Frobenius norm of the assembled K
    int fail_col = -1;           // first column with a non-positive pivot, -1 if none
};

struct DevFactorTimes {
    double total_s = 0.0;        // wall time of device_factor
    double device_ms = 0.0;      // device time of the factorisation kernels (events)
    double flops = 0.0;          // algorithmic FP64 flops of the eliminations
    int batches = 0;
    int launches = 0;
};

// regularise(job, Sss, reg): Sss is the ns x ns fix-DOF Schur block (column-major, full); the
// callback writes reg (ns x ns, column-major), which is added to the block before its columns are
// eliminated, and sets the job's nk and N.  It runs on the host between the elimination phases of
// each batch.
using RegulariseFn = std::function<void(int job, const double *Sss, double *reg)>;

// Factorises every job on the current CUDA device, in batches whose dense matrices fit
// `mem_budget` bytes (0: half of the free device memory).  With `store` (sized by this call for
// `ndom` subdomains; jobs' slots index it) S_i, the Dirichlet blocks and the K^+ factor stay on the
// device as tiles and only the kernels Rp come back; without it S is copied to the host (the dense
// inverse of the coarse problem).  Throws feti::Error on CUDA errors.
void device_factor(const ElementData &el, std::vector<DevFactorJob> &jobs, const RegulariseFn &regularise,
                   size_t mem_budget, DevFactorTimes *times, DevPrepStore *store = nullptr, int ndom = 0);

}  // namespace feti
