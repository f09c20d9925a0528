// Subdomain decomposition and ESPRESO-compatible multiplier numbering (host).
#include "decompose.h"

#include <algorithm>
#include <array>
#include <numeric>
#include <unordered_map>

#include "common.h"

namespace feti {

namespace {

// HEXA8 faces (node positions inside the element), reference hexahedron8.cpp:12-19
const int kHexFaces[6][4] = {{0, 1, 5, 4}, {3, 2, 1, 0}, {4, 5, 6, 7}, {7, 6, 2, 3}, {1, 2, 6, 5}, {3, 0, 4, 7}};

}  // namespace

Decomposition decompose(const ElementData &el, int ndomains_hint, const std::vector<int> &dir_dofs,
                        const std::vector<double> &dir_vals) {
    Decomposition dec;
    const double tdec = now_s();
    const size_t ne = el.nelem();
    FETI_CHECK(ne > 0, "FETI4I: the stiffness matrix has no elements");

    // DOFs per node (uniform), node <-> DOF maps
    int dpn = -1, maxnode = -1, maxdof = -1;
    for (size_t e = 0; e < ne; ++e) {
        int nn = (int)(el.node_ptr[e + 1] - el.node_ptr[e]);
        int nd = (int)(el.dof_ptr[e + 1] - el.dof_ptr[e]);
        FETI_CHECK(nn > 0 && nd % nn == 0, "FETI4I: element DOF count is not a multiple of its node count");
        if (dpn < 0) dpn = nd / nn;
        FETI_CHECK(dpn == nd / nn, "FETI4I: all elements must have the same number of DOFs per node");
        for (int64_t i = el.node_ptr[e]; i < el.node_ptr[e + 1]; ++i) maxnode = std::max(maxnode, el.nodes[i]);
        for (int64_t i = el.dof_ptr[e]; i < el.dof_ptr[e + 1]; ++i) maxdof = std::max(maxdof, el.dofs[i]);
    }
    dec.dpn = dpn;
    dec.n_nodes = maxnode + 1;
    dec.node_dof.assign((size_t)dec.n_nodes * dpn, -1);
    dec.dof_node.assign(maxdof + 1, -1);
    dec.dof_comp.assign(maxdof + 1, -1);
    for (size_t e = 0; e < ne; ++e) {
        int nn = (int)(el.node_ptr[e + 1] - el.node_ptr[e]);
        for (int a = 0; a < nn; ++a) {
            int node = el.nodes[el.node_ptr[e] + a];
            FETI_CHECK(node >= 0, "FETI4I: negative node index (check indexBase)");
            for (int c = 0; c < dpn; ++c) {
                int dof = el.dofs[el.dof_ptr[e] + (int64_t)a * dpn + c];
                FETI_CHECK(dof >= 0, "FETI4I: negative DOF index (check indexBase)");
                int &slot = dec.node_dof[(size_t)node * dpn + c];
                FETI_CHECK(slot < 0 || slot == dof, "FETI4I: inconsistent node/DOF association between elements");
                slot = dof;
                dec.dof_node[dof] = node;
                dec.dof_comp[dof] = c;
            }
        }
    }

    FETI_LOG(3, "FETI4I: decompose t_maps %.3f s\n", now_s() - tdec);
    // element -> domain
    dec.elem_domain.resize(ne);
    if (!el.partition.empty()) {
        FETI_CHECK(el.partition.size() == ne, "FETI4I: subdomain partition size differs from the element count");
        int mx = 0;
        for (size_t e = 0; e < ne; ++e) {
            FETI_CHECK(el.partition[e] >= 0, "FETI4I: negative subdomain index in partition");
            dec.elem_domain[e] = el.partition[e];
            mx = std::max(mx, el.partition[e]);
        }
        dec.ndom = mx + 1;
    } else {
        int nd = std::max(1, std::min<int>(ndomains_hint, (int)ne));
        for (size_t e = 0; e < ne; ++e) dec.elem_domain[e] = (int)((e * (size_t)nd) / ne);
        dec.ndom = nd;
    }
    dec.dom.resize(dec.ndom);
    for (size_t e = 0; e < ne; ++e) dec.dom[dec.elem_domain[e]].elems.push_back((int)e);
    for (int d = 0; d < dec.ndom; ++d) FETI_CHECK(!dec.dom[d].elems.empty(), "FETI4I: empty subdomain in partition");

    FETI_LOG(3, "FETI4I: decompose t_elemdom %.3f s\n", now_s() - tdec);
    // node -> sorted domain list (CSR): the domains of each node's elements, bucketed by node
    std::vector<int> dptr(dec.n_nodes + 1, 0), dlist;
    {
        std::vector<int> cnt(dec.n_nodes + 1, 0);
        for (size_t e = 0; e < ne; ++e)
            for (int64_t i = el.node_ptr[e]; i < el.node_ptr[e + 1]; ++i) cnt[el.nodes[i] + 1]++;
        for (int n = 0; n < dec.n_nodes; ++n) cnt[n + 1] += cnt[n];
        std::vector<int> bucket(cnt[dec.n_nodes]);
        {
            std::vector<int> fill(cnt.begin(), cnt.end() - 1);
            for (size_t e = 0; e < ne; ++e)
                for (int64_t i = el.node_ptr[e]; i < el.node_ptr[e + 1]; ++i) bucket[fill[el.nodes[i]]++] = dec.elem_domain[e];
        }
        std::vector<int> len(dec.n_nodes, 0);
#pragma omp parallel for schedule(static)
        for (int n = 0; n < dec.n_nodes; ++n) {
            int *b = bucket.data() + cnt[n], *e = bucket.data() + cnt[n + 1];
            std::sort(b, e);
            len[n] = (int)(std::unique(b, e) - b);
        }
        for (int n = 0; n < dec.n_nodes; ++n) dptr[n + 1] = dptr[n] + len[n];
        dlist.resize(dptr[dec.n_nodes]);
#pragma omp parallel for schedule(static)
        for (int n = 0; n < dec.n_nodes; ++n)
            std::copy(bucket.begin() + cnt[n], bucket.begin() + cnt[n] + len[n], dlist.begin() + dptr[n]);
    }
    dec.node_ndom.resize(dec.n_nodes);
    for (int n = 0; n < dec.n_nodes; ++n) dec.node_ndom[n] = dptr[n + 1] - dptr[n];

    FETI_LOG(3, "FETI4I: decompose t_nodedom %.3f s\n", now_s() - tdec);
    // nodes on the external surface: faces owned by one element (HEXA8 only).  Faces are bucketed
    // by their smallest node; a face appearing once in its bucket is external.
    std::vector<char> ext(dec.n_nodes, 0);
    {
        std::vector<int> cnt(dec.n_nodes + 1, 0);
        auto face_key = [&](size_t e, int f, int (&k)[4]) {
            const int *en = &el.nodes[el.node_ptr[e]];
            for (int i = 0; i < 4; ++i) k[i] = en[kHexFaces[f][i]];
            std::sort(k, k + 4);
        };
        int k[4];
        for (size_t e = 0; e < ne; ++e) {
            if (el.node_ptr[e + 1] - el.node_ptr[e] != 8) continue;
            for (int f = 0; f < 6; ++f) {
                face_key(e, f, k);
                cnt[k[0] + 1]++;
            }
        }
        for (int n = 0; n < dec.n_nodes; ++n) cnt[n + 1] += cnt[n];
        std::vector<std::array<int, 3>> rest(cnt[dec.n_nodes]);   // the other three nodes of each face
        {
            std::vector<int> fill(cnt.begin(), cnt.end() - 1);
            for (size_t e = 0; e < ne; ++e) {
                if (el.node_ptr[e + 1] - el.node_ptr[e] != 8) continue;
                for (int f = 0; f < 6; ++f) {
                    face_key(e, f, k);
                    rest[fill[k[0]]++] = {k[1], k[2], k[3]};
                }
            }
        }
        std::vector<char> extf(rest.size(), 0);
#pragma omp parallel for schedule(dynamic, 1024)
        for (int n = 0; n < dec.n_nodes; ++n) {
            auto *b = rest.data() + cnt[n], *e = rest.data() + cnt[n + 1];
            std::sort(b, e);
            for (auto *q = b; q < e;) {
                auto *r = q + 1;
                while (r < e && *r == *q) ++r;
                if (r - q == 1) extf[q - rest.data()] = 1;
                q = r;
            }
        }
        for (int n = 0; n < dec.n_nodes; ++n)
            for (int i = cnt[n]; i < cnt[n + 1]; ++i)
                if (extf[i]) {
                    ext[n] = 1;
                    for (int v : rest[i]) ext[v] = 1;
                }
    }

    FETI_LOG(3, "FETI4I: decompose t_faces %.3f s\n", now_s() - tdec);
    // final node order: by (domain list with "longer first on a common prefix", surface group, node ID)
    std::vector<int> used;
    for (int n = 0; n < dec.n_nodes; ++n)
        if (dptr[n + 1] > dptr[n]) used.push_back(n);
    auto cmp_key = [&](int a, int b) -> int {  // -1, 0, 1 on (domain list, group)
        int la = dptr[a + 1] - dptr[a], lb = dptr[b + 1] - dptr[b];
        int m = std::min(la, lb);
        for (int i = 0; i < m; ++i) {
            int x = dlist[dptr[a] + i], y = dlist[dptr[b] + i];
            if (x != y) return x < y ? -1 : 1;
        }
        if (la != lb) return la > lb ? -1 : 1;
        int ga = ext[a] ? 0 : 1, gb = ext[b] ? 0 : 1;
        if (ga != gb) return ga < gb ? -1 : 1;
        return 0;
    };
    std::sort(used.begin(), used.end(), [&](int a, int b) {
        int c = cmp_key(a, b);
        return c != 0 ? c < 0 : a < b;
    });
    dec.node_order = used;
    dec.interval_ptr.push_back(0);
    for (size_t i = 1; i <= used.size(); ++i)
        if (i == used.size() || cmp_key(used[i - 1], used[i]) != 0) dec.interval_ptr.push_back((int)i);
    const int nint = (int)dec.interval_ptr.size() - 1;
    dec.interval_domains.resize(nint);
    dec.node_interval.assign(dec.n_nodes, -1);
    for (int p = 0; p < nint; ++p)
        for (int i = dec.interval_ptr[p]; i < dec.interval_ptr[p + 1]; ++i) dec.node_interval[used[i]] = p;
    dec.interval_ext.assign(nint, 0);
    for (int p = 0; p < nint; ++p) {
        int n = used[dec.interval_ptr[p]];
        dec.interval_domains[p].assign(dlist.begin() + dptr[n], dlist.begin() + dptr[n + 1]);
        dec.interval_ext[p] = ext[n];
    }

    FETI_LOG(3, "FETI4I: decompose t_order %.3f s\n", now_s() - tdec);
    // domain local node numbering (interval by interval)
    dec.g2l.assign(dec.ndom, std::unordered_map<int, int>());
    for (int p = 0; p < nint; ++p)
        for (int d : dec.interval_domains[p])
            for (int i = dec.interval_ptr[p]; i < dec.interval_ptr[p + 1]; ++i) {
                int node = used[i];
                dec.g2l[d][node] = (int)dec.dom[d].nodes.size();
                dec.dom[d].nodes.push_back(node);
            }
    for (int d = 0; d < dec.ndom; ++d) dec.dom[d].ndofs = dpn * (int)dec.dom[d].nodes.size();

    FETI_LOG(3, "FETI4I: decompose t_g2l %.3f s\n", now_s() - tdec);
    // Dirichlet nodes per (component, interval); values by (node, comp)
    std::vector<char> dmask((size_t)dec.n_nodes * dpn, 0);
    std::vector<double> dval((size_t)dec.n_nodes * dpn, 0.0);
    FETI_CHECK(dir_dofs.size() == dir_vals.size(), "FETI4I: Dirichlet indices/values size mismatch");
    for (size_t i = 0; i < dir_dofs.size(); ++i) {
        int dof = dir_dofs[i];
        FETI_CHECK(dof >= 0 && dof < (int)dec.dof_node.size() && dec.dof_node[dof] >= 0,
                   "FETI4I: Dirichlet index does not belong to any element");
        size_t k = (size_t)dec.dof_node[dof] * dpn + dec.dof_comp[dof];
        FETI_CHECK(!dmask[k], "FETI4I: Dirichlet DOFs have to be unique");
        dmask[k] = 1;
        dval[k] = dir_vals[i];
    }
    // per interval and component: Dirichlet node count
    std::vector<int> dcount((size_t)nint * dpn, 0), dsize(nint, 0);
    for (int p = 0; p < nint; ++p)
        for (int i = dec.interval_ptr[p]; i < dec.interval_ptr[p + 1]; ++i)
            for (int c = 0; c < dpn; ++c)
                if (dmask[(size_t)used[i] * dpn + c]) { dcount[(size_t)p * dpn + c]++; dsize[p]++; }

    // interval offsets (one rank): Dirichlet block, then gluing block
    std::vector<int64_t> doff(nint), goff(nint);
    int64_t off = 0;
    for (int p = 0; p < nint; ++p) { doff[p] = off; off += (int64_t)dec.interval_domains[p].size() * dsize[p]; }
    dec.n_dirichlet = (int)off;
    for (int p = 0; p < nint; ++p) {
        goff[p] = off;
        int64_t m = dec.interval_domains[p].size();
        if (m > 1) off += ((int64_t)dpn * (dec.interval_ptr[p + 1] - dec.interval_ptr[p]) - dsize[p]) * (m * (m - 1) / 2);
    }
    FETI_CHECK(off < (int64_t)INT32_MAX, "FETI4I: too many Lagrange multipliers for 32-bit indices");
    dec.n_lambda = (int)off;

    auto pair_index = [](int a, int b, int m) { return a * m - a * (a + 1) / 2 + (b - a - 1); };
    for (int p = 0; p < nint; ++p) {
        const std::vector<int> &doms = dec.interval_domains[p];
        int m = (int)doms.size();
        for (int k = 0; k < m; ++k) {
            DomainRows &D = dec.dom[doms[k]];
            const auto &g2l = dec.g2l[doms[k]];
            // Dirichlet rows (redundant: every domain of the interval)
            int64_t lm = 0;
            for (int c = 0; c < dpn; ++c) {
                int cnt = dcount[(size_t)p * dpn + c];
                int64_t base = doff[p] + (int64_t)k * cnt + lm;
                int t = 0;
                for (int i = dec.interval_ptr[p]; i < dec.interval_ptr[p + 1]; ++i) {
                    int node = used[i];
                    size_t key = (size_t)node * dpn + c;
                    if (!dmask[key]) continue;
                    D.lam.push_back((int)(base + t++));
                    D.dof.push_back(dpn * g2l.at(node) + c);
                    D.sign.push_back(1.0);
                    D.c.push_back(dval[key]);
                    D.other.push_back(-1);
                    D.node.push_back(node);
                    D.comp.push_back(c);
                }
                lm += (int64_t)m * cnt;
            }
        }
        if (m > 1) {
            int npairs = m * (m - 1) / 2;
            for (int k = 0; k < m; ++k) {
                DomainRows &D = dec.dom[doms[k]];
                const auto &g2l = dec.g2l[doms[k]];
                int64_t counter = 0;
                for (int c = 0; c < dpn; ++c)
                    for (int i = dec.interval_ptr[p]; i < dec.interval_ptr[p + 1]; ++i) {
                        int node = used[i];
                        if (dmask[(size_t)node * dpn + c]) continue;
                        int64_t base = goff[p] + counter * npairs;
                        for (int a = 0; a < k; ++a) {
                            D.lam.push_back((int)(base + pair_index(a, k, m)));
                            D.sign.push_back(-1.0);
                            D.other.push_back(doms[a]);
                            D.dof.push_back(dpn * g2l.at(node) + c); D.c.push_back(0.0); D.node.push_back(node); D.comp.push_back(c);
                        }
                        for (int b = k + 1; b < m; ++b) {
                            D.lam.push_back((int)(base + pair_index(k, b, m)));
                            D.sign.push_back(1.0);
                            D.other.push_back(doms[b]);
                            D.dof.push_back(dpn * g2l.at(node) + c); D.c.push_back(0.0); D.node.push_back(node); D.comp.push_back(c);
                        }
                        ++counter;
                    }
            }
        }
    }
    FETI_LOG(3, "FETI4I: decompose t_rows %.3f s\n", now_s() - tdec);
    // rows in ascending multiplier order
    for (auto &D : dec.dom) {
        size_t n = D.lam.size();
        std::vector<size_t> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return D.lam[a] < D.lam[b]; });
        auto permute_i = [&](std::vector<int> &v) { std::vector<int> t(n); for (size_t i = 0; i < n; ++i) t[i] = v[ord[i]]; v.swap(t); };
        auto permute_d = [&](std::vector<double> &v) { std::vector<double> t(n); for (size_t i = 0; i < n; ++i) t[i] = v[ord[i]]; v.swap(t); };
        permute_i(D.lam); permute_i(D.dof); permute_i(D.other); permute_i(D.node); permute_i(D.comp);
        permute_d(D.sign); permute_d(D.c);
        D.w.assign(n, 1.0);
    }
    FETI_LOG(3, "FETI4I: decompose done %.3f s\n", now_s() - tdec);
    return dec;
}

void compute_weights(Decomposition &dec, const std::vector<std::vector<double>> *diags) {
    const int dpn = dec.dpn;
    for (int d = 0; d < dec.ndom; ++d) {
        DomainRows &D = dec.dom[d];
        for (size_t i = 0; i < D.lam.size(); ++i) {
            if (D.other[i] < 0) { D.w[i] = 1.0; continue; }
            int node = D.node[i], c = D.comp[i];
            if (!diags) { D.w[i] = 1.0 / dec.node_ndom[node]; continue; }
            // K-diagonal ratio: diagonal of the partner over the sum over all sharing domains
            double tot = 0.0;
            for (int q : dec.interval_domains[dec.node_interval[node]]) tot += (*diags)[q][dpn * dec.g2l[q].at(node) + c];
            int o = D.other[i];
            double mine = (*diags)[o][dpn * dec.g2l[o].at(node) + c];
            D.w[i] = mine / tot;
        }
    }
}

void restrict_subdomains(Decomposition &dec, int first, int count) {
    FETI_CHECK(first >= 0 && count > 0 && first + count <= dec.ndom,
               "FETI4I: the owned subdomain range [" + std::to_string(first) + ", " + std::to_string(first + count) +
                   ") is outside the " + std::to_string(dec.ndom) + " subdomains");
    dec.dom = std::vector<DomainRows>(dec.dom.begin() + first, dec.dom.begin() + first + count);
    dec.g2l = std::vector<std::unordered_map<int, int>>(dec.g2l.begin() + first, dec.g2l.begin() + first + count);
    dec.ndom = count;
}

}  // namespace feti
