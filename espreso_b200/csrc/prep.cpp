// Host preprocessing: subdomain K assembly, partial Cholesky with the fix
// DOFs last, algebraic kernel detection on the fix-DOF Schur block, explicit
// Schur complements S_i = B_i K_reg^-1 B_i^T, Dirichlet/lumped preconditioner
// data and the coarse problem (GG^T)^-1.
#include "prep.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <numeric>

#include "common.h"
#include "dense.h"
#include "gpu_prep.h"
#include "hybrid.h"

namespace feti {

namespace {

// Breadth-first distances on the subdomain node graph (nodes sharing an element).
std::vector<int> bfs(const std::vector<std::vector<int>> &adj, int src) {
    std::vector<int> dist(adj.size(), -1);
    std::deque<int> q;
    dist[src] = 0;
    q.push_back(src);
    while (!q.empty()) {
        int v = q.front();
        q.pop_front();
        for (int w : adj[v])
            if (dist[w] < 0) { dist[w] = dist[v] + 1; q.push_back(w); }
    }
    return dist;
}

// Three mutually distant nodes whose DOFs are all touched by B: the fix set
// on which the kernel of K is detected (the algebraic regularisation of
// src/solver/generic/SparseMatrix.cpp:3540-4495 works on a Schur complement
// of K onto a small DOF set in the same way).  Distances are breadth-first over
// the element edges, so on a structured mesh they are Manhattan distances: the
// third node maximises da + db, which keeps it off the line through a and b
// (three collinear nodes would leave a rotation free).
std::vector<int> choose_fix_nodes(const std::vector<std::vector<int>> &adj, const std::vector<char> &cand) {
    int n = (int)adj.size();
    int a = -1;
    for (int i = 0; i < n; ++i)
        if (cand[i]) { a = i; break; }
    FETI_CHECK(a >= 0, "FETI4I: a subdomain has no DOF glued to other subdomains or fixed by Dirichlet conditions");
    std::vector<int> fix{a};
    std::vector<int> da = bfs(adj, a);
    int b = -1;
    for (int i = 0; i < n; ++i)
        if (cand[i] && i != a && (b < 0 || da[i] > da[b])) b = i;
    if (b < 0) return fix;
    fix.push_back(b);
    std::vector<int> db = bfs(adj, b);
    int c = -1;
    for (int i = 0; i < n; ++i) {
        if (!cand[i] || i == a || i == b) continue;
        if (c < 0) { c = i; continue; }
        const int si = da[i] + db[i], sc = da[c] + db[c];
        if (si > sc || (si == sc && std::min(da[i], db[i]) > std::min(da[c], db[c]))) c = i;
    }
    if (c >= 0) fix.push_back(c);
    return fix;
}

void orthonormalize(std::vector<double> &R, int n, int k) {
    for (int pass = 0; pass < 2; ++pass)
        for (int j = 0; j < k; ++j) {
            double *rj = R.data() + (size_t)j * n;
            for (int i = 0; i < j; ++i) {
                const double *ri = R.data() + (size_t)i * n;
                double s = 0.0;
                for (int p = 0; p < n; ++p) s += ri[p] * rj[p];
                for (int p = 0; p < n; ++p) rj[p] -= s * ri[p];
            }
            double nr = 0.0;
            for (int p = 0; p < n; ++p) nr += rj[p] * rj[p];
            nr = std::sqrt(nr);
            FETI_CHECK(nr > 0.0, "FETI4I: degenerate kernel basis");
            for (int p = 0; p < n; ++p) rj[p] /= nr;
        }
}

}  // namespace

void SubPrep::kplus(double *x) const {
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) y[pos[i]] = x[i];
    dense::trsv_packed_lower(Lp.data(), n, y.data());
    dense::trsv_packed_lower_t(Lp.data(), n, y.data());
    for (int i = 0; i < n; ++i) x[i] = y[pos[i]];
}

// Per-subdomain state between the symbolic phase, the numeric factorisation (host or device) and
// the kernel / G phase.
struct SubWork {
    int n1 = 0;                     // untouched DOFs (factor positions 0..n1-1)
    int ns = 0;                     // fix DOFs (the last ns factor positions)
    double rho = 0.0;               // largest diagonal entry of K: weight of the regularisation
    std::vector<int> fixdofs;
    std::vector<int> eldof;         // device path: factor position of every element DOF
    std::vector<int> elcolor;       // device path: element colours (one colour shares no node)
    int ncolors = 0;
    std::vector<double> Kfix;       // n x ns: columns of K at the fix DOFs, factor-order rows
    double knorm = 0.0;             // ||K||_F
    std::vector<double> V;          // ns x ns: eigenvectors of the fix-DOF Schur block
    int defect = 0;
};

// Element DOFs of element e as local DOF indices of subdomain d.
static void element_local_dofs(const ElementData &el, const Decomposition &dec, int d, int e, std::vector<int> &eldof) {
    const int dpn = dec.dpn;
    const auto &g2l = dec.g2l[d];
    const int nd = (int)(el.dof_ptr[e + 1] - el.dof_ptr[e]);
    eldof.resize(nd);
    for (int k = 0; k < nd; ++k) {
        const int dof = el.dofs[el.dof_ptr[e] + k];
        eldof[k] = dpn * g2l.at(dec.dof_node[dof]) + dec.dof_comp[dof];
    }
}

// Symbolic phase: fix nodes, factor order [untouched | touched, not fix | fix], T numbering,
// K restricted to T (lumped preconditioner), the largest diagonal entry of K.  With `device`
// also the element DOF positions, element colours and the fix columns of K for the device
// factorisation.
static void prep_symbolic(const ElementData &el, const Decomposition &dec, int d, const PrepOptions &opt, SubPrep &S,
                          SubWork &W, bool device) {
    const DomainRows &D = dec.dom[d];
    const int dpn = dec.dpn;
    const int n = D.ndofs;
    const int nn = (int)D.nodes.size();
    const auto &g2l = dec.g2l[d];
    S.n = n;
    S.ni = (int)D.lam.size();

    std::vector<std::vector<int>> adj(nn);
    std::vector<int> eldof;
    // touched DOFs and candidate fix nodes
    std::vector<char> touched(n, 0);
    for (int r = 0; r < S.ni; ++r) touched[D.dof[r]] = 1;
    std::vector<char> cand(nn, 0);
    for (int a = 0; a < nn; ++a) {
        bool all = true;
        for (int c = 0; c < dpn; ++c) all = all && touched[dpn * a + c];
        cand[a] = all;
    }
    // node graph: the 12 edges of a HEXA8 element, all node pairs of other elements
    static const int kHexEdges[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                         {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    for (int e : D.elems) {
        int64_t nb = el.node_ptr[e], ne_ = el.node_ptr[e + 1];
        if (ne_ - nb == 8) {
            for (const auto &ed : kHexEdges) {
                const int u = g2l.at(el.nodes[nb + ed[0]]), v = g2l.at(el.nodes[nb + ed[1]]);
                adj[u].push_back(v);
                adj[v].push_back(u);
            }
            continue;
        }
        for (int64_t i = nb; i < ne_; ++i)
            for (int64_t j = nb; j < ne_; ++j)
                if (i != j) adj[g2l.at(el.nodes[i])].push_back(g2l.at(el.nodes[j]));
    }
    for (auto &v : adj) { std::sort(v.begin(), v.end()); v.erase(std::unique(v.begin(), v.end()), v.end()); }
    S.fix_nodes = choose_fix_nodes(adj, cand);
    std::vector<char> isfix(n, 0);
    W.fixdofs.clear();
    for (int a : S.fix_nodes)
        for (int c = 0; c < dpn; ++c) { isfix[dpn * a + c] = 1; W.fixdofs.push_back(dpn * a + c); }
    const int ns = (int)W.fixdofs.size();
    W.ns = ns;

    // factor order: [untouched | touched, not fix | fix]
    S.pos.assign(n, -1);
    int p = 0;
    for (int i = 0; i < n; ++i) if (!touched[i]) S.pos[i] = p++;
    const int n1 = p;
    W.n1 = n1;
    for (int i = 0; i < n; ++i) if (touched[i] && !isfix[i]) S.pos[i] = p++;
    for (int i : W.fixdofs) S.pos[i] = p++;
    S.t = n - n1;
    S.tdof.resize(S.t);
    for (int i = 0; i < n; ++i) if (S.pos[i] >= n1) S.tdof[S.pos[i] - n1] = i;
    S.trow.resize(S.ni);
    for (int r = 0; r < S.ni; ++r) S.trow[r] = S.pos[D.dof[r]] - n1;

    // K diagonal, K restricted to T (lumped), device-path element data
    std::vector<double> diag(n, 0.0);
    S.f.assign(n, 0.0);
    std::vector<std::vector<std::pair<int, double>>> KT(S.t);
    // SUPER_DIRICHLET: the columns K_rT of the untouched DOFs r (r -> (T index, value))
    const bool super_dir = opt.precond == PREC_SUPER_DIRICHLET;
    std::vector<std::vector<std::pair<int, double>>> KrT(super_dir ? n1 : 0);
    if (device) {
        W.eldof.clear();
        W.Kfix.assign((size_t)n * ns, 0.0);
    }
    for (int e : D.elems) {
        element_local_dofs(el, dec, d, e, eldof);
        const int nd = (int)eldof.size();
        const double *Ke = el.vals.data() + el.val_ptr[e];
        for (int a = 0; a < nd; ++a) {
            const int pa = S.pos[eldof[a]];
            diag[eldof[a]] += Ke[(size_t)a * nd + a];
            if (pa >= n1)
                for (int b = 0; b < nd; ++b) {
                    int pb = S.pos[eldof[b]];
                    if (pb >= n1) KT[pa - n1].emplace_back(pb - n1, Ke[(size_t)a * nd + b]);
                    else if (super_dir) KrT[pb].emplace_back(pa - n1, Ke[(size_t)a * nd + b]);
                }
        }
        if (device) {
            for (int a = 0; a < nd; ++a) W.eldof.push_back(S.pos[eldof[a]]);
            // column pb of K at a fix DOF, row pa (the host path's dense assembly order)
            for (int a = 0; a < nd; ++a)
                for (int b = 0; b < nd; ++b) {
                    const int pb = S.pos[eldof[b]];
                    if (pb >= n - ns) W.Kfix[(size_t)(pb - (n - ns)) * n + S.pos[eldof[a]]] += Ke[(size_t)a * nd + b];
                }
        }
    }
    W.rho = *std::max_element(diag.begin(), diag.end());
    if (super_dir) {
        // S_sd = K_TT - K_Tr diag(K_rr)^-1 K_rT (clustercpu.cpp:254-311, diagonalized_K_rr): every
        // untouched DOF r adds -K_ir K_jr / K_rr to the T pairs (i, j) it couples
        std::vector<int> rdof(n1);
        for (int i = 0; i < n; ++i) if (S.pos[i] < n1) rdof[S.pos[i]] = i;
        for (int r = 0; r < n1; ++r) {
            auto &col = KrT[r];
            if (col.empty()) continue;
            std::sort(col.begin(), col.end(), [](auto &x, auto &y) { return x.first < y.first; });
            size_t m = 0;   // sum duplicates (element contributions)
            for (size_t k = 0; k < col.size(); ++k) {
                if (m > 0 && col[m - 1].first == col[k].first) col[m - 1].second += col[k].second;
                else col[m++] = col[k];
            }
            col.resize(m);
            const double inv = 1.0 / diag[rdof[r]];
            for (auto &ci : col)
                for (auto &cj : col) KT[ci.first].emplace_back(cj.first, -ci.second * cj.second * inv);
        }
    }
    if (opt.precond == PREC_LUMPED || opt.precond == PREC_MAGIC || super_dir) {
        // MAGIC stores K - RegMat (cluster.cpp:413-433): on T the same entries as LUMPED's K
        S.KT_ptr.assign(S.t + 1, 0);
        for (int i = 0; i < S.t; ++i) {
            auto &row = KT[i];
            std::sort(row.begin(), row.end(), [](auto &x, auto &y) { return x.first < y.first; });
            int last = -1;
            for (auto &kv : row) {
                if (kv.first == last) { S.KT_val.back() += kv.second; continue; }
                S.KT_col.push_back(kv.first);
                S.KT_val.push_back(kv.second);
                last = kv.first;
            }
            S.KT_ptr[i + 1] = (int)S.KT_col.size();
        }
    }
    if (device) {
        // greedy element colouring: elements of one colour share no node
        const int ne = (int)D.elems.size();
        W.elcolor.assign(ne, 0);
        std::vector<uint64_t> used(nn, 0);
        W.ncolors = 0;
        for (int k = 0; k < ne; ++k) {
            const int e = D.elems[k];
            uint64_t mask = 0;
            for (int64_t i = el.node_ptr[e]; i < el.node_ptr[e + 1]; ++i) mask |= used[g2l.at(el.nodes[i])];
            int c = 0;
            while (c < 64 && ((mask >> c) & 1u)) ++c;
            FETI_CHECK(c < 64, "FETI4I: more than 64 element colours in a subdomain");
            W.elcolor[k] = c;
            W.ncolors = std::max(W.ncolors, c + 1);
            for (int64_t i = el.node_ptr[e]; i < el.node_ptr[e + 1]; ++i) used[g2l.at(el.nodes[i])] |= (uint64_t)1 << c;
        }
    }
}

// Kernel detection on the fix-DOF Schur block Sss (ns x ns, full, column-major): defect, the
// regularisation reg = rho V_k V_k^T over the kernel eigenvectors (ns x ns, column-major).
static void fix_block(SubPrep &S, SubWork &W, const double *Sss, double *reg) {
    const int ns = W.ns;
    std::vector<double> A(Sss, Sss + (size_t)ns * ns), ev(ns);
    W.V.assign((size_t)ns * ns, 0.0);
    dense::jacobi_eigen(A.data(), ns, ev.data(), W.V.data());
    S.ss_eigs = ev;
    // defect: the last eigenvalue before a jump of more than 1e5 (SparseMatrix.cpp:3657-3661)
    int defect = 0;
    double scale = std::fabs(ev[ns - 1]);
    for (int k = ns - 2; k >= 0; --k)
        if (std::fabs(ev[k]) < 1e-5 * std::fabs(ev[k + 1])) { defect = k + 1; break; }
    if (defect == 0 && scale > 0 && std::fabs(ev[0]) < 1e-10 * scale) defect = 1;
    FETI_CHECK(defect > 0, "FETI4I: subdomain stiffness matrix is not singular (Total FETI expects floating subdomains)");
    S.nk = defect;
    W.defect = defect;
    const std::vector<double> &V = W.V;
    for (int j = 0; j < ns; ++j)
        for (int i = 0; i < ns; ++i) {
            double r = 0.0;
            for (int k = 0; k < defect; ++k) r += V[(size_t)k * ns + i] * V[(size_t)k * ns + j];
            reg[(size_t)j * ns + i] = W.rho * r;
        }
}

// Host numeric phase: dense K in factor order, partial Cholesky with the fix-block
// regularisation in between, S_i = B (K_reg^-1)_TT B^T, the packed factor.
static void prep_numeric_host(const ElementData &el, const Decomposition &dec, int d, const PrepOptions &opt,
                              SubPrep &S, SubWork &W) {
    const DomainRows &D = dec.dom[d];
    const int n = S.n, n1 = W.n1, ns = W.ns;
    std::vector<int> eldof;
    std::vector<double> A((size_t)n * n, 0.0);
    for (int e : D.elems) {
        element_local_dofs(el, dec, d, e, eldof);
        const int nd = (int)eldof.size();
        const double *Ke = el.vals.data() + el.val_ptr[e];
        for (int a = 0; a < nd; ++a) {
            const int pa = S.pos[eldof[a]];
            for (int b = 0; b < nd; ++b) A[(size_t)S.pos[eldof[b]] * n + pa] += Ke[(size_t)a * nd + b];
        }
    }
    // Frobenius norm of K and its columns at the fix DOFs for the kernel check
    double knorm = 0.0;
    for (size_t i = 0; i < A.size(); ++i) knorm += A[i] * A[i];
    W.knorm = std::sqrt(knorm);
    W.Kfix.assign((size_t)n * ns, 0.0);
    for (int j = 0; j < ns; ++j)
        std::memcpy(&W.Kfix[(size_t)j * n], &A[(size_t)(n - ns + j) * n], sizeof(double) * n);

    // 1) eliminate the untouched DOFs: trailing block = Schur complement onto T
    int info = dense::potrf_lower(A.data(), n, n, n1);
    FETI_CHECK(info == 0, "FETI4I: interior block of a subdomain stiffness matrix is not positive definite");
    if (opt.precond == PREC_DIRICHLET) {
        S.Sdir.assign((size_t)S.t * S.t, 0.0);
        for (int j = 0; j < S.t; ++j)
            for (int i = j; i < S.t; ++i) {
                double v = A[(size_t)(n1 + j) * n + n1 + i];
                S.Sdir[(size_t)j * S.t + i] = v;
                S.Sdir[(size_t)i * S.t + j] = v;
            }
    }
    // 2) eliminate the touched, non-fix DOFs
    double *At = A.data() + (size_t)n1 * n + n1;
    info = dense::potrf_lower(At, S.t, n, S.t - ns);
    FETI_CHECK(info == 0, "FETI4I: fix-node choice does not remove the rigid-body modes of a subdomain");
    // 3) kernel of the fix-DOF Schur block, regularisation, last columns
    double *Ass = A.data() + (size_t)(n - ns) * n + (n - ns);
    std::vector<double> Sss((size_t)ns * ns), reg((size_t)ns * ns);
    for (int j = 0; j < ns; ++j)
        for (int i = 0; i < ns; ++i) Sss[(size_t)j * ns + i] = (i >= j) ? Ass[(size_t)j * n + i] : Ass[(size_t)i * n + j];
    fix_block(S, W, Sss.data(), reg.data());
    for (int j = 0; j < ns; ++j)
        for (int i = j; i < ns; ++i) Ass[(size_t)j * n + i] += reg[(size_t)j * ns + i];
    info = dense::potrf_lower(Ass, ns, n, ns);
    FETI_CHECK(info == 0, "FETI4I: regularised fix block is not positive definite");

    // 4) S_i = B (K_reg^-1)_TT B^T with (K_reg^-1)_TT = W^T W, W = L_TT^-1
    std::vector<double> Wt((size_t)S.t * S.t, 0.0), KiTT((size_t)S.t * S.t);
    for (int j = 0; j < S.t; ++j)
        for (int i = j; i < S.t; ++i) Wt[(size_t)j * S.t + i] = A[(size_t)(n1 + j) * n + n1 + i];
    dense::trtri_lower(Wt.data(), S.t, S.t);
    dense::lauum_lower(Wt.data(), S.t, S.t, KiTT.data(), S.t);
    S.S.assign((size_t)S.ni * S.ni, 0.0);
    for (int k = 0; k < S.ni; ++k)
        for (int j = 0; j < S.ni; ++j)
            S.S[(size_t)k * S.ni + j] = D.sign[j] * D.sign[k] * KiTT[(size_t)S.trow[k] * S.t + S.trow[j]];

    // packed factor (host K^+ solves, device K^+ tiles, kernel below)
    S.Lp.resize((size_t)n * (n + 1) / 2);
    dense::pack_lower(A.data(), n, n, S.Lp.data());
}

// Kernel R = [-K_rr^-1 K_rs N; N] from the packed factor: R_r = -L_rr^-T (L_sr^T N); its check
// against the fix columns of K; orthonormal columns; G_i = -(B_i R_i)^T.
static void finish_kernel(const Decomposition &dec, int d, SubPrep &S, SubWork &W, const std::vector<double> &Rp);

static void prep_finish(const Decomposition &dec, int d, SubPrep &S, SubWork &W) {
    const int n = S.n, ns = W.ns, defect = W.defect;
    const int nr = n - ns;
    const double *Lp = S.Lp.data();
    std::vector<double> Rp((size_t)n * defect, 0.0);
    for (int k = 0; k < defect; ++k) {
        double *x = &Rp[(size_t)k * n];
        for (int s = 0; s < ns; ++s) {
            double v = W.V[(size_t)k * ns + s];
            x[nr + s] = v;
            for (int j = 0; j < nr; ++j) x[j] += Lp[dense::packed_index(n, nr + s, j)] * v;
        }
        for (int j = nr - 1; j >= 0; --j) {
            const double *cj = Lp + dense::packed_index(n, j, j) - j;   // cj[i] = L(i, j), i >= j
            double s = x[j];
            for (int i = j + 1; i < nr; ++i) s -= cj[i] * x[i];
            x[j] = s / cj[j];
        }
        for (int j = 0; j < nr; ++j) x[j] = -x[j];
    }
    finish_kernel(dec, d, S, W, Rp);
}

// Rp (n x defect, factor order) -> R in local DOF order, the kernel check, orthonormal columns, G.
static void finish_kernel(const Decomposition &dec, int d, SubPrep &S, SubWork &W, const std::vector<double> &Rp) {
    const DomainRows &D = dec.dom[d];
    const int n = S.n, ns = W.ns, defect = W.defect;
    S.R.assign((size_t)n * defect, 0.0);
    for (int k = 0; k < defect; ++k)
        for (int i = 0; i < n; ++i) S.R[(size_t)k * n + i] = Rp[(size_t)k * n + S.pos[i]];
    // kernel check on the fix columns: (K R) rows at the fix DOFs use the saved columns
    {
        double res = 0.0;
        for (int k = 0; k < defect; ++k)
            for (int j = 0; j < ns; ++j) {
                double s = 0.0;
                for (int i = 0; i < n; ++i) s += W.Kfix[(size_t)j * n + i] * Rp[(size_t)k * n + i];
                res += s * s;
            }
        double rn = 0.0;
        for (double v : Rp) rn += v * v;
        S.kernel_residual = std::sqrt(res) / (W.knorm * std::sqrt(rn));
    }
    orthonormalize(S.R, n, defect);

    // G_i = -(B_i R_i)^T (row-major nk x ni)
    S.G.assign((size_t)defect * S.ni, 0.0);
    for (int k = 0; k < defect; ++k)
        for (int j = 0; j < S.ni; ++j) S.G[(size_t)k * S.ni + j] = -D.sign[j] * S.R[(size_t)k * n + D.dof[j]];
    W.Kfix.clear();
    W.Kfix.shrink_to_fit();
}

static void prep_subdomain(const ElementData &el, const Decomposition &dec, int d, const PrepOptions &opt, SubPrep &S) {
    SubWork W;
    prep_symbolic(el, dec, d, opt, S, W, false);
    prep_numeric_host(el, dec, d, opt, S, W);
    prep_finish(dec, d, S, W);
}

// Device path: symbolic phase on the host threads, every subdomain's elimination and Schur
// complement on the GPU (gpu_prep.cu), kernels and G on the host threads.
static void prep_all_device(const ElementData &el, const Decomposition &dec, const PrepOptions &opt,
                            std::vector<SubPrep> &sub, const std::vector<int> &order, int nthreads,
                            std::vector<std::string> &errors, DevFactorTimes &dt,
                            std::shared_ptr<DevPrepStore> &dstore) {
    const int nd = dec.ndom;
    const double t0 = now_s();
    std::vector<SubWork> work(nd);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int k = 0; k < nd; ++k) {
        const int d = order[k];
        try {
            prep_symbolic(el, dec, d, opt, sub[d], work[d], true);
        } catch (const std::exception &ex) {
            errors[d] = ex.what();
        }
    }
    std::vector<int> ids;   // subdomains of the device jobs, largest first
    for (int k = 0; k < nd; ++k)
        if (errors[order[k]].empty()) ids.push_back(order[k]);
    // S_i, the Dirichlet blocks and K^+ stay on the device (the tile stores of the dual iteration);
    // Hybrid Total FETI appends its corner rows B0, and B K^+ B0^T, B0 K^+ B0^T come back for the
    // cluster problems.
    std::shared_ptr<DevPrepStore> store = std::make_shared<DevPrepStore>();
    std::vector<std::vector<double>> Rps(nd);
    std::vector<DevFactorJob> jobs(ids.size());
    for (size_t q = 0; q < ids.size(); ++q) {
        const int d = ids[q];
        SubPrep &S = sub[d];
        SubWork &W = work[d];
        const DomainRows &D = dec.dom[d];
        DevFactorJob &J = jobs[q];
        J.n = S.n;
        J.n1 = W.n1;
        J.ns = W.ns;
        J.ni = S.ni;
        J.elems = D.elems.data();
        J.nelem = (int)D.elems.size();
        J.elpos = std::move(W.eldof);
        J.elcolor = std::move(W.elcolor);
        J.ncolors = W.ncolors;
        J.bpos.resize(S.ni);
        for (int r = 0; r < S.ni; ++r) J.bpos[r] = S.pos[D.dof[r]];
        J.bsign = D.sign;
        J.want_sdir = opt.precond == PREC_DIRICHLET;
        J.slot = d;
        if (!S.b0_dof.empty()) {
            const int m0 = (int)S.b0_dof.size();
            J.b0pos.resize(m0);
            for (int j = 0; j < m0; ++j) J.b0pos[j] = S.pos[S.b0_dof[j]];
            J.b0sign = S.b0_sign;
            S.BKB0.assign((size_t)S.ni * m0, 0.0);
            S.B0KB0.assign((size_t)m0 * m0, 0.0);
            J.V = S.BKB0.data();
            J.F0 = S.B0KB0.data();
        }
    }
    auto reg = [&](int q, const double *Sss, double *r) {
        const int d = ids[q];
        try {
            fix_block(sub[d], work[d], Sss, r);
            DevFactorJob &J = jobs[q];
            J.nk = work[d].defect;
            J.N.assign(work[d].V.begin(), work[d].V.begin() + (size_t)J.nk * J.ns);
            Rps[d].assign((size_t)J.n * J.nk, 0.0);
            J.Rp = Rps[d].data();
        } catch (const std::exception &ex) {
            errors[d] = ex.what();
            std::fill(r, r + (size_t)work[d].ns * work[d].ns, 0.0);
        }
    };
    const double t1 = now_s();
    device_factor(el, jobs, reg, opt.device_mem, &dt, store.get(), nd);
    const double t2 = now_s();
    dstore = store;
    for (size_t q = 0; q < ids.size(); ++q) {
        const int d = ids[q];
        const DevFactorJob &J = jobs[q];
        if (J.fail_col >= 0 && errors[d].empty()) {
            if (J.fail_col < J.n1)
                errors[d] = "FETI4I: interior block of a subdomain stiffness matrix is not positive definite";
            else if (J.fail_col < J.n - J.ns)
                errors[d] = "FETI4I: fix-node choice does not remove the rigid-body modes of a subdomain";
            else
                errors[d] = "FETI4I: regularised fix block is not positive definite";
        }
        work[d].knorm = J.knorm;
    }
    jobs.clear();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int k = 0; k < (int)ids.size(); ++k) {
        const int d = ids[k];
        if (!errors[d].empty()) continue;
        try {
            finish_kernel(dec, d, sub[d], work[d], Rps[d]);
        } catch (const std::exception &ex) {
            errors[d] = ex.what();
        }
    }
    FETI_LOG(2, "FETI4I: device preprocessing: symbolic %.3f s, device %.3f s (kernels %.1f ms, %.1f GFLOP, %d batches), kernels/G %.3f s\n",
             t1 - t0, t2 - t1, dt.device_ms, dt.flops * 1e-9, dt.batches, now_s() - t2);
}

void preprocess(const ElementData &el, Decomposition &dec, const std::vector<double> &rhs, const PrepOptions &opt,
                Prep &out) {
    const int dpn = dec.dpn;
    double t0 = now_s();
    // K diagonals for the B1 scaling (diagonal of each subdomain matrix)
    std::vector<std::vector<double>> diags(dec.ndom);
    for (int d = 0; d < dec.ndom; ++d) {
        diags[d].assign(dec.dom[d].ndofs, 0.0);
        for (int e : dec.dom[d].elems) {
            int nd = (int)(el.dof_ptr[e + 1] - el.dof_ptr[e]);
            const double *Ke = el.vals.data() + el.val_ptr[e];
            for (int a = 0; a < nd; ++a) {
                int dof = el.dofs[el.dof_ptr[e] + a];
                diags[d][dpn * dec.g2l[d].at(dec.dof_node[dof]) + dec.dof_comp[dof]] += Ke[(size_t)a * nd + a];
            }
        }
    }
    compute_weights(dec, opt.scaling ? &diags : nullptr);
    // partitioned dual problem: the weights need every subdomain's diagonal; the rest only the owned block
    if (opt.owned_count > 0) {
        FETI_CHECK(opt.method == 0, "FETI4I: a partitioned dual problem (owned subdomain range) is Total FETI only");
        restrict_subdomains(dec, opt.owned_first, opt.owned_count);
    }

    out.sub.assign(dec.ndom, SubPrep());
    out.n_lambda = dec.n_lambda;
    // largest subdomains first
    std::vector<int> order(dec.ndom);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return dec.dom[a].ndofs > dec.dom[b].ndofs; });
    int nthreads = opt.threads > 0 ? opt.threads : omp_get_max_threads();
    std::vector<std::string> errors(dec.ndom);
    out.device_prep = opt.device;
    std::vector<int> n0;
    if (opt.method == 1) {
        // Hybrid Total FETI: clusters glued at corners (the corner rows depend on the numbering only)
        out.sub_cluster = opt.sub_cluster.empty() ? std::vector<int>(dec.ndom, 0) : opt.sub_cluster;
        FETI_CHECK((int)out.sub_cluster.size() == dec.ndom,
                   "FETI4I: the cluster partition must list one cluster per subdomain");
        for (int c : out.sub_cluster) FETI_CHECK(c >= 0, "FETI4I: negative cluster index");
        hybrid_corners(dec, out.sub_cluster, out, n0);
    }
    if (opt.device) {
        DevFactorTimes dt;
        prep_all_device(el, dec, opt, out.sub, order, nthreads, errors, dt, out.dstore);
        out.t_device_factor_ms = dt.device_ms;
        out.device_factor_flops = dt.flops;
        out.device_factor_launches = dt.launches;
    } else {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
        for (int k = 0; k < dec.ndom; ++k) {
            int d = order[k];
            try {
                prep_subdomain(el, dec, d, opt, out.sub[d]);
            } catch (const std::exception &ex) {
                errors[d] = ex.what();
            }
        }
    }
    for (int d = 0; d < dec.ndom; ++d)
        if (!errors[d].empty()) throw Error(errors[d] + " (subdomain " + std::to_string(d) + ")");

    // subdomain right-hand sides: caller DOF value divided by its multiplicity
    for (int d = 0; d < dec.ndom; ++d) {
        SubPrep &S = out.sub[d];
        const DomainRows &D = dec.dom[d];
        for (int a = 0; a < (int)D.nodes.size(); ++a)
            for (int c = 0; c < dpn; ++c) {
                int dof = dec.node_dof[(size_t)D.nodes[a] * dpn + c];
                double v = (dof >= 0 && dof < (int)rhs.size()) ? rhs[dof] : 0.0;
                S.f[dpn * a + c] = v / dec.node_ndom[D.nodes[a]];
            }
    }
    out.t_factor = now_s() - t0;
    FETI_LOG(2, "FETI4I: subdomain preprocessing %.3f s\n", out.t_factor);

    // coarse problem: dual kernel space, owners of every multiplier, GG^T and its inverse
    double t1 = now_s();
    out.method = opt.method;
    if (opt.method == 1) {
        // Hybrid Total FETI: cluster problems and cluster kernels in the dual problem
        hybrid_prepare(dec, out, n0, nthreads);
    } else {
        out.kofs.assign(dec.ndom + 1, 0);
        for (int d = 0; d < dec.ndom; ++d) {
            SubPrep &S = out.sub[d];
            S.dnk = S.nk;
            S.Rd = S.R;
            S.Gd = S.G;
            out.kofs[d + 1] = out.kofs[d] + S.nk;
        }
        out.n_kern = out.kofs[dec.ndom];
    }
    out.own_dom.assign((size_t)2 * dec.n_lambda, -1);
    out.own_row.assign((size_t)2 * dec.n_lambda, -1);
    for (int d = 0; d < dec.ndom; ++d)
        for (int r = 0; r < (int)dec.dom[d].lam.size(); ++r) {
            int l = dec.dom[d].lam[r];
            int slot = out.own_dom[2 * (size_t)l] < 0 ? 0 : 1;
            FETI_CHECK(out.own_dom[2 * (size_t)l + slot] < 0, "FETI4I: a multiplier is shared by more than two subdomains");
            out.own_dom[2 * (size_t)l + slot] = d;
            out.own_row[2 * (size_t)l + slot] = r;
        }
    const int nK = out.n_kern;
    std::vector<double> GG((size_t)nK * nK, 0.0);
    for (int l = 0; l < dec.n_lambda; ++l) {
        for (int s1 = 0; s1 < 2; ++s1) {
            int d1 = out.own_dom[2 * (size_t)l + s1];
            if (d1 < 0) continue;
            int r1 = out.own_row[2 * (size_t)l + s1];
            const SubPrep &A1 = out.sub[d1];
            for (int s2 = 0; s2 < 2; ++s2) {
                int d2 = out.own_dom[2 * (size_t)l + s2];
                if (d2 < 0) continue;
                int r2 = out.own_row[2 * (size_t)l + s2];
                const SubPrep &A2 = out.sub[d2];
                for (int a = 0; a < A1.dnk; ++a)
                    for (int b = 0; b < A2.dnk; ++b)
                        GG[(size_t)(out.kofs[d2] + b) * nK + out.kofs[d1] + a] +=
                            A1.Gd[(size_t)a * A1.ni + r1] * A2.Gd[(size_t)b * A2.ni + r2];
            }
        }
    }
    out.GGt_inv.assign((size_t)nK * nK, 0.0);
    if (opt.device && nK > 0) {
        // (G G^T)^-1 as the trailing block of the eliminated [G G^T I; I 0] on the device
        std::vector<DevFactorJob> cj(1);
        DevFactorJob &J = cj[0];
        J.n = nK;
        J.ni = nK;
        J.dense = GG.data();
        J.bpos.resize(nK);
        std::iota(J.bpos.begin(), J.bpos.end(), 0);
        J.bsign.assign(nK, 1.0);
        J.S = out.GGt_inv.data();
        DevFactorTimes ct;
        device_factor(el, cj, [](int, const double *, double *) {}, 0, &ct);
        FETI_CHECK(J.fail_col < 0, "FETI4I: the coarse problem G G^T is singular");
        out.t_device_factor_ms += ct.device_ms;
        out.device_factor_flops += ct.flops;
        out.device_factor_launches += ct.launches;
    } else {
        int info = dense::potrf_lower(GG.data(), nK, nK, nK);
        FETI_CHECK(info == 0, "FETI4I: the coarse problem G G^T is singular");
        std::vector<double> Wc((size_t)nK * nK, 0.0);
        for (int j = 0; j < nK; ++j)
            for (int i = j; i < nK; ++i) Wc[(size_t)j * nK + i] = GG[(size_t)j * nK + i];
        dense::trtri_lower(Wc.data(), nK, nK);
        dense::lauum_lower(Wc.data(), nK, nK, out.GGt_inv.data(), nK);
    }
    out.t_coarse = now_s() - t1;
    FETI_LOG(2, "FETI4I: coarse problem %.3f s\n", out.t_coarse);
}

void kplus_dual(const Prep &prep, std::vector<std::vector<double>> &x) {
    const int nd = (int)prep.sub.size();
    if (prep.method != 1) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int d = 0; d < nd; ++d) prep.sub[d].kplus(x[d].data());
        return;
    }
    // cluster solve (cluster.cpp:796-916) with the cluster matrix M
    const int ncl = (int)prep.clusters.size();
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < ncl; ++c) {
        const ClusterPrep &C = prep.clusters[c];
        const int nc = C.n0 + C.ka;
        std::vector<double> z(nc, 0.0), w(nc, 0.0), kx;
        for (size_t mi = 0; mi < C.members.size(); ++mi) {
            const int d = C.members[mi];
            const SubPrep &S = prep.sub[d];
            kx = x[d];
            S.kplus(kx.data());
            for (size_t j = 0; j < S.b0_row.size(); ++j) z[S.b0_row[j]] += S.b0_sign[j] * kx[S.b0_dof[j]];
            for (int k = 0; k < S.nk; ++k) {
                double s = 0.0;
                for (int i = 0; i < S.n; ++i) s += S.R[(size_t)k * S.n + i] * x[d][i];
                z[C.n0 + C.akofs[mi] + k] = -s;
            }
        }
        for (int j = 0; j < nc; ++j)
            for (int i = 0; i < nc; ++i) w[i] += C.M[(size_t)j * nc + i] * z[j];
        for (size_t mi = 0; mi < C.members.size(); ++mi) {
            const int d = C.members[mi];
            const SubPrep &S = prep.sub[d];
            std::vector<double> &v = x[d];
            for (size_t j = 0; j < S.b0_row.size(); ++j) v[S.b0_dof[j]] -= S.b0_sign[j] * w[S.b0_row[j]];
            S.kplus(v.data());
            for (int k = 0; k < S.nk; ++k) {
                const double a = w[C.n0 + C.akofs[mi] + k];
                for (int i = 0; i < S.n; ++i) v[i] += S.R[(size_t)k * S.n + i] * a;
            }
        }
    }
}

void make_rhs_vectors(const Decomposition &dec, const Prep &prep, std::vector<double> &b, std::vector<double> &e) {
    b.assign(dec.n_lambda, 0.0);
    e.assign(prep.n_kern, 0.0);
    const int nd = dec.ndom;
    std::vector<std::vector<double>> kf(nd);
    for (int d = 0; d < nd; ++d) kf[d] = prep.sub[d].f;
    kplus_dual(prep, kf);
    for (int d = 0; d < nd; ++d) {
        const SubPrep &S = prep.sub[d];
        for (int k = 0; k < S.dnk; ++k) {
            double s = 0.0;
            for (int i = 0; i < S.n; ++i) s += S.Rd[(size_t)k * S.n + i] * S.f[i];
            e[prep.kofs[d] + k] -= s;
        }
    }
    for (int d = 0; d < nd; ++d) {
        const DomainRows &D = dec.dom[d];
        for (size_t r = 0; r < D.lam.size(); ++r) b[D.lam[r]] += D.sign[r] * kf[d][D.dof[r]] - D.c[r];
    }
}

void primal_solution(const Decomposition &dec, const Prep &prep, const double *lambda, const double *alpha,
                     double *solution, int solution_size) {
    const int dpn = dec.dpn;
    const int nd = dec.ndom;
    std::vector<std::vector<double>> u(nd);
    for (int d = 0; d < nd; ++d) {
        const DomainRows &D = dec.dom[d];
        u[d] = prep.sub[d].f;
        for (size_t r = 0; r < D.lam.size(); ++r) u[d][D.dof[r]] -= D.sign[r] * lambda[D.lam[r]];
    }
    kplus_dual(prep, u);
#pragma omp parallel for schedule(dynamic, 1)
    for (int d = 0; d < nd; ++d) {
        const SubPrep &S = prep.sub[d];
        for (int k = 0; k < S.dnk; ++k) {
            double a = alpha[prep.kofs[d] + k];
            for (int i = 0; i < S.n; ++i) u[d][i] += S.Rd[(size_t)k * S.n + i] * a;
        }
    }
    std::vector<double> cnt(solution_size, 0.0);
    for (int i = 0; i < solution_size; ++i) solution[i] = 0.0;
    for (int d = 0; d < nd; ++d) {
        const DomainRows &D = dec.dom[d];
        for (int a = 0; a < (int)D.nodes.size(); ++a)
            for (int c = 0; c < dpn; ++c) {
                int dof = dec.node_dof[(size_t)D.nodes[a] * dpn + c];
                if (dof < 0 || dof >= solution_size) continue;
                solution[dof] += u[d][dpn * a + c];
                cnt[dof] += 1.0;
            }
    }
    for (int i = 0; i < solution_size; ++i)
        if (cnt[i] > 0) solution[i] /= cnt[i];
}

}  // namespace feti
