// Subdomain decomposition and multiplier numbering of a FETI4I problem.
//
// The rules restate ESPRESO's single-process numbering:
//   node intervals and their order ...... src/mesh/preprocessing/arrangement.cpp:32-241
//   Dirichlet and gluing multipliers .... src/assembler/constraints/equalityconstraints.cpp:25-285
//   interval offsets .................... src/assembler/constraints/constraints.cpp:198-260
//   duplicity / K-diagonal scaling ...... src/assembler/constraints/equalityconstraints.cpp:287-423
#pragma once

#include <cstdint>
#include <unordered_map>
#include <vector>

namespace feti {

struct ElementData {
    int type = 0;        // FETI4IMatrixType
    int index_base = 0;
    std::vector<int> etype;
    std::vector<int64_t> node_ptr, dof_ptr, val_ptr;
    std::vector<int> nodes, dofs;     // already shifted by index_base
    std::vector<double> vals;         // row-major dofsSize^2 per element
    std::vector<int> partition;       // element -> subdomain (optional)
    std::vector<int> sub_cluster;     // subdomain -> cluster for Hybrid Total FETI (optional)
    size_t nelem() const { return etype.size(); }
};

struct DomainRows {
    std::vector<int> nodes;           // local node -> global node
    std::vector<int> elems;           // elements of the domain
    // one entry per local multiplier (B1 row), ascending multiplier index
    std::vector<int> lam, dof, other, node, comp;
    std::vector<double> sign, c, w;
    int ndofs = 0;
};

struct Decomposition {
    int dpn = 0;
    int ndom = 0;
    int n_nodes = 0;
    int n_lambda = 0;
    int n_dirichlet = 0;
    std::vector<int> elem_domain;
    std::vector<int> node_dof;        // node*dpn + c -> caller DOF, -1 if absent
    std::vector<int> dof_node, dof_comp;  // caller DOF -> node, component
    std::vector<int> node_order;      // final node order (interval by interval)
    std::vector<int> interval_ptr;    // into node_order
    std::vector<std::vector<int>> interval_domains;
    std::vector<char> interval_ext;   // 1 for intervals of the external-surface group
    std::vector<int> node_ndom;       // number of domains sharing each node
    std::vector<int> node_interval;   // node -> interval index
    std::vector<DomainRows> dom;
    std::vector<std::unordered_map<int, int>> g2l;  // per domain: global node -> local node
};

// Build the numbering.  `dirichlet` holds caller DOFs (already shifted) and values.
Decomposition decompose(const ElementData &el, int ndomains_hint, const std::vector<int> &dir_dofs,
                        const std::vector<double> &dir_vals);

// Duplicity weights: 1/ndomains, or with scaling K-diagonal ratios; diags[d] in local DOF order.
void compute_weights(Decomposition &dec, const std::vector<std::vector<double>> *diags);

// Keep subdomains [first, first + count) only (a partitioned dual problem: the subdomain block of one
// process).  Multiplier indices, weights, multiplicities and the caller-DOF maps stay global.
void restrict_subdomains(Decomposition &dec, int first, int count);

}  // namespace feti
