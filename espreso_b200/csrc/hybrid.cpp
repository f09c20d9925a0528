// Hybrid Total FETI host preprocessing: corner gluing, the cluster coarse problem
// and the cluster kernels (see hybrid.h for the reference files restated).
//
// The cluster solve of multKplusGlobal_Kinv,
//     g0 = B0 K^+ x,  e0 = -R^T x,
//     alpha = S_alpha^-1 (G0 F0^-1 g0 - e0),  lambda0 = F0^-1 (g0 - G0^T alpha),
//     K_c^+ x = K^+ x - K^+ B0^T lambda0 + R alpha,
// is linear in (g0, e0).  It is kept as one dense symmetric matrix per cluster,
//     [lambda0; alpha] = M [g0; e0],
//     M = [ A - A G0^T S^-1 G0 A    A G0^T S^-1 ]
//         [ S^-1 G0 A              -S^-1        ],   A = F0^-1, S = S_alpha regularised,
// so the device applies the whole cluster correction of one F apply as
//     F_c = sum_i B_i S_i B_i^T - V M V^T,  V_i = [B_i K_i^+ B0_i^T | G_i^T].
#include "hybrid.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "common.h"
#include "dense.h"

namespace feti {

namespace {

// inv := A^-1 for a symmetric positive definite n x n matrix (A is overwritten)
bool spd_inverse(std::vector<double> &A, int n, std::vector<double> &inv) {
    inv.assign((size_t)n * n, 0.0);
    if (n == 0) return true;
    if (dense::potrf_lower(A.data(), n, n, n) != 0) return false;
    std::vector<double> W((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) W[(size_t)j * n + i] = A[(size_t)j * n + i];
    dense::trtri_lower(W.data(), n, n);
    dense::lauum_lower(W.data(), n, n, inv.data(), n);
    return true;
}

}  // namespace

void hybrid_corners(const Decomposition &dec, const std::vector<int> &sub_cluster, Prep &prep,
                    std::vector<int> &n0) {
    const int dpn = dec.dpn;
    const int nint = (int)dec.interval_domains.size();
    // corner nodes (fetidata.cpp:146-188): the middle node of every interval shared by two
    // or more domains; every len/3-th node on surface intervals.  The surface cursor advances
    // only on intervals shared by two or more domains, as in the reference.
    std::vector<int> ext_list;
    for (int p = 0; p < nint; ++p)
        if (dec.interval_ext[p]) ext_list.push_back(p);
    std::vector<std::pair<int, int>> corners;  // (node, interval)
    size_t ei = 0;
    for (int p = 0; p < nint; ++p) {
        if (dec.interval_domains[p].size() == 1) continue;
        const int b = dec.interval_ptr[p], e = dec.interval_ptr[p + 1];
        if (ei < ext_list.size() && ext_list[ei] == p) {
            ++ei;
            const int inc = std::max((e - b) / 3, 1);
            for (int i = b; i < e; i += inc) corners.emplace_back(dec.node_order[i], p);
        } else {
            corners.emplace_back(dec.node_order[b + (e - b) / 2], p);
        }
    }
    // B0 rows (equalityconstraints.cpp:504-555): per corner, per pair of consecutive domains of
    // one cluster, per DOF; +1 in the first domain, -1 in the second.  Every cluster numbers
    // its own rows (one cluster per process in the reference).
    int ncl = 0;
    for (int c : sub_cluster) ncl = std::max(ncl, c + 1);
    n0.assign(ncl, 0);
    for (auto &S : prep.sub) { S.b0_row.clear(); S.b0_dof.clear(); S.b0_sign.clear(); }
    std::vector<int> cd, cls;
    for (const auto &cn : corners) {
        const int node = cn.first;
        const std::vector<int> &doms = dec.interval_domains[cn.second];
        cls.clear();
        for (int d : doms) cls.push_back(sub_cluster[d]);
        std::sort(cls.begin(), cls.end());
        cls.erase(std::unique(cls.begin(), cls.end()), cls.end());
        for (int c : cls) {
            cd.clear();
            for (int d : doms)
                if (sub_cluster[d] == c) cd.push_back(d);
            for (size_t k = 0; k + 1 < cd.size(); ++k) {
                const int d1 = cd[k], d2 = cd[k + 1];
                const int l1 = dec.g2l[d1].at(node), l2 = dec.g2l[d2].at(node);
                for (int comp = 0; comp < dpn; ++comp) {
                    const int r = n0[c]++;
                    SubPrep &A = prep.sub[d1], &B = prep.sub[d2];
                    A.b0_row.push_back(r); A.b0_dof.push_back(dpn * l1 + comp); A.b0_sign.push_back(1.0);
                    B.b0_row.push_back(r); B.b0_dof.push_back(dpn * l2 + comp); B.b0_sign.push_back(-1.0);
                }
            }
        }
    }
}

void hybrid_prepare(const Decomposition &dec, Prep &prep, const std::vector<int> &n0, int threads) {
    const int nd = dec.ndom;
    const int ncl = (int)n0.size();
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
    prep.clusters.assign(ncl, ClusterPrep());
    for (int c = 0; c < ncl; ++c) prep.clusters[c].n0 = n0[c];
    for (int d = 0; d < nd; ++d) prep.clusters[prep.sub_cluster[d]].members.push_back(d);
    for (int c = 0; c < ncl; ++c) {
        ClusterPrep &C = prep.clusters[c];
        FETI_CHECK(!C.members.empty(), "FETI4I: cluster " + std::to_string(c) + " has no subdomains");
        C.akofs.assign(C.members.size() + 1, 0);
        for (size_t i = 0; i < C.members.size(); ++i) C.akofs[i + 1] = C.akofs[i] + prep.sub[C.members[i]].nk;
        C.ka = C.akofs.back();
        FETI_CHECK(C.ka <= 4096, "FETI4I: a cluster holds too many subdomain kernels; split it into more clusters");
    }

    // per subdomain: X = K^+ B0^T, V = [B X | G^T], local F0 block and B0 R
    std::vector<std::vector<double>> F0loc(nd), B0R(nd);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int d = 0; d < nd; ++d) {
        SubPrep &S = prep.sub[d];
        const DomainRows &D = dec.dom[d];
        const int m0 = (int)S.b0_row.size(), nk = S.nk, n = S.n, ni = S.ni;
        S.V.assign((size_t)ni * (m0 + nk), 0.0);
        F0loc[d].assign((size_t)m0 * m0, 0.0);
        B0R[d].assign((size_t)m0 * nk, 0.0);
        if (!S.BKB0.empty() || (m0 > 0 && S.Lp.empty())) {
            // device preprocessing: both blocks come from the eliminated [K B^T B0^T; B; B0]
            FETI_CHECK(S.BKB0.size() == (size_t)ni * m0 && S.B0KB0.size() == (size_t)m0 * m0,
                       "FETI4I: corner blocks of the device preprocessing missing");
            std::copy(S.BKB0.begin(), S.BKB0.end(), S.V.begin());
            F0loc[d] = S.B0KB0;
        } else {
            std::vector<double> x(n);
            for (int j = 0; j < m0; ++j) {
                std::fill(x.begin(), x.end(), 0.0);
                x[S.b0_dof[j]] = S.b0_sign[j];
                S.kplus(x.data());
                for (int r = 0; r < ni; ++r) S.V[(size_t)j * ni + r] = D.sign[r] * x[D.dof[r]];
                for (int l = 0; l < m0; ++l) F0loc[d][(size_t)j * m0 + l] = S.b0_sign[l] * x[S.b0_dof[l]];
            }
        }
        for (int k = 0; k < nk; ++k) {
            for (int r = 0; r < ni; ++r) S.V[(size_t)(m0 + k) * ni + r] = S.G[(size_t)k * ni + r];
            for (int j = 0; j < m0; ++j) B0R[d][(size_t)k * m0 + j] = S.b0_sign[j] * S.R[(size_t)k * n + S.b0_dof[j]];
        }
    }

    std::vector<std::string> errors(ncl);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int c = 0; c < ncl; ++c) {
        try {
            ClusterPrep &C = prep.clusters[c];
            const int N0 = C.n0, ka = C.ka;
            // F0 = sum B0_i K_i^+ B0_i^T (cluster.cpp:1293-1478) and G0 = -(B0 R)^T (:1226-1291)
            std::vector<double> F0((size_t)N0 * N0, 0.0), G0((size_t)ka * N0, 0.0);  // G0 column-major ka x N0
            for (size_t mi = 0; mi < C.members.size(); ++mi) {
                const int d = C.members[mi];
                const SubPrep &S = prep.sub[d];
                const int m0 = (int)S.b0_row.size();
                for (int j = 0; j < m0; ++j)
                    for (int l = 0; l < m0; ++l)
                        F0[(size_t)S.b0_row[j] * N0 + S.b0_row[l]] += F0loc[d][(size_t)j * m0 + l];
                for (int k = 0; k < S.nk; ++k)
                    for (int j = 0; j < m0; ++j)
                        G0[(size_t)S.b0_row[j] * ka + C.akofs[mi] + k] = -B0R[d][(size_t)k * m0 + j];
            }
            std::vector<double> A;
            FETI_CHECK(spd_inverse(F0, N0, A), "FETI4I: the corner problem F0 of a cluster is singular");
            // T = A G0^T (N0 x ka), S_alpha = G0 T (cluster.cpp:1480-1560)
            std::vector<double> T((size_t)N0 * ka, 0.0), Sa((size_t)ka * ka, 0.0);
            for (int k = 0; k < ka; ++k)
                for (int q = 0; q < N0; ++q) {
                    const double g = G0[(size_t)q * ka + k];
                    if (g == 0.0) continue;
                    const double *a = &A[(size_t)q * N0];
                    double *t = &T[(size_t)k * N0];
                    for (int i = 0; i < N0; ++i) t[i] += a[i] * g;
                }
            for (int k = 0; k < ka; ++k)
                for (int q = 0; q < N0; ++q) {
                    const double t = T[(size_t)k * N0 + q];
                    if (t == 0.0) continue;
                    for (int i = 0; i < ka; ++i) Sa[(size_t)k * ka + i] += G0[(size_t)q * ka + i] * t;
                }
            for (int j = 0; j < ka; ++j)
                for (int i = j + 1; i < ka; ++i) {
                    const double v = 0.5 * (Sa[(size_t)j * ka + i] + Sa[(size_t)i * ka + j]);
                    Sa[(size_t)j * ka + i] = Sa[(size_t)i * ka + j] = v;
                }
            // kernel of S_alpha: the cluster's rigid modes in subdomain amplitudes
            std::vector<double> ev(ka), EV((size_t)ka * ka);
            dense::jacobi_eigen(Sa.data(), ka, ev.data(), EV.data());
            double emax = 0.0;
            for (double v : ev) emax = std::max(emax, std::fabs(v));
            auto in_kernel = [&](int i) { return emax == 0.0 || std::fabs(ev[i]) <= 1e-8 * emax; };
            int nkc = 0;
            for (int i = 0; i < ka; ++i)
                if (in_kernel(i)) ++nkc;
            FETI_CHECK(nkc > 0, "FETI4I: S_alpha of a cluster is not singular (a cluster must float)");
            C.nkc = nkc;
            C.H.assign((size_t)ka * nkc, 0.0);
            for (int i = 0, col = 0; i < ka; ++i)
                if (in_kernel(i)) {
                    std::copy(&EV[(size_t)i * ka], &EV[(size_t)(i + 1) * ka], &C.H[(size_t)col * ka]);
                    ++col;
                }
            // regularisation by the kernel, weighted by the mean of the diagonal (cluster.cpp:1626-1628)
            double rho = 0.0;
            for (int i = 0; i < ka; ++i) rho += Sa[(size_t)i * ka + i];
            rho = (ka > 0 && rho > 0.0) ? rho / ka : 1.0;
            C.rho = rho;
            for (int j = 0; j < ka; ++j)
                for (int i = 0; i < ka; ++i) {
                    double h = 0.0;
                    for (int k = 0; k < nkc; ++k) h += C.H[(size_t)k * ka + i] * C.H[(size_t)k * ka + j];
                    Sa[(size_t)j * ka + i] += rho * h;
                }
            std::vector<double> Sinv;
            FETI_CHECK(spd_inverse(Sa, ka, Sinv), "FETI4I: the regularised S_alpha of a cluster is not positive definite");
            // U = T Sinv (N0 x ka); M = [[A - U T^T, U], [U^T, -Sinv]]
            std::vector<double> U((size_t)N0 * ka, 0.0);
            for (int k = 0; k < ka; ++k)
                for (int q = 0; q < ka; ++q) {
                    const double sv = Sinv[(size_t)k * ka + q];
                    const double *t = &T[(size_t)q * N0];
                    double *u = &U[(size_t)k * N0];
                    for (int i = 0; i < N0; ++i) u[i] += t[i] * sv;
                }
            const int nc = N0 + ka;
            C.M.assign((size_t)nc * nc, 0.0);
            for (int j = 0; j < N0; ++j)
                for (int i = 0; i < N0; ++i) {
                    double sum = A[(size_t)j * N0 + i];
                    for (int k = 0; k < ka; ++k) sum -= U[(size_t)k * N0 + i] * T[(size_t)k * N0 + j];
                    C.M[(size_t)j * nc + i] = sum;
                }
            for (int k = 0; k < ka; ++k)
                for (int i = 0; i < N0; ++i) {
                    C.M[(size_t)(N0 + k) * nc + i] = U[(size_t)k * N0 + i];
                    C.M[(size_t)i * nc + N0 + k] = U[(size_t)k * N0 + i];
                }
            for (int j = 0; j < ka; ++j)
                for (int i = 0; i < ka; ++i) C.M[(size_t)(N0 + j) * nc + N0 + i] = -Sinv[(size_t)j * ka + i];
        } catch (const std::exception &ex) {
            errors[c] = ex.what();
        }
    }
    for (int c = 0; c < ncl; ++c)
        if (!errors[c].empty()) throw Error(errors[c] + " (cluster " + std::to_string(c) + ")");

    // dual kernel space: R_c restricted to subdomain i = R_i H_i, G = -(B1 R_c)^T
    prep.kofs.assign(nd + 1, 0);
    std::vector<int> ckof(ncl + 1, 0);
    for (int c = 0; c < ncl; ++c) ckof[c + 1] = ckof[c] + prep.clusters[c].nkc;
    prep.n_kern = ckof[ncl];
    for (int c = 0; c < ncl; ++c) {
        const ClusterPrep &C = prep.clusters[c];
        for (size_t mi = 0; mi < C.members.size(); ++mi) {
            const int d = C.members[mi];
            SubPrep &S = prep.sub[d];
            const int n = S.n, ni = S.ni, nkc = C.nkc;
            S.dnk = nkc;
            S.Rd.assign((size_t)n * nkc, 0.0);
            S.Gd.assign((size_t)nkc * ni, 0.0);
            for (int kc = 0; kc < nkc; ++kc)
                for (int k = 0; k < S.nk; ++k) {
                    const double h = C.H[(size_t)kc * C.ka + C.akofs[mi] + k];
                    if (h == 0.0) continue;
                    for (int i = 0; i < n; ++i) S.Rd[(size_t)kc * n + i] += S.R[(size_t)k * n + i] * h;
                    for (int r = 0; r < ni; ++r) S.Gd[(size_t)kc * ni + r] += S.G[(size_t)k * ni + r] * h;
                }
            prep.kofs[d] = ckof[c];
        }
    }
    prep.kofs[nd] = prep.n_kern;
}

}  // namespace feti
