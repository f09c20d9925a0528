// Hybrid Total FETI (HTFETI): subdomains of a cluster are glued at corner nodes by
// B0, and the dual iteration uses the cluster's generalised inverse K_c^+ and the
// cluster kernels.  Restated from ESPRESO:
//   corner nodes ............ src/mesh/preprocessing/fetidata.cpp:146-188
//   B0 corner rows .......... src/assembler/constraints/equalityconstraints.cpp:504-555
//   B0 compression .......... src/solver/specific/cluster.cpp:1186-1224
//   G0, F0, S_alpha ......... src/solver/specific/cluster.cpp:1226-1700
//   cluster kernels R H ..... src/solver/specific/cluster.cpp:1776-1800
//   cluster solve ........... src/solver/specific/cluster.cpp:796-916 (multKplusGlobal_Kinv)
#pragma once

#include <vector>

#include "decompose.h"
#include "prep.h"

namespace feti {

// Corner B0 rows of every subdomain (SubPrep::b0_*), and the number of rows of every cluster.
void hybrid_corners(const Decomposition &dec, const std::vector<int> &sub_cluster, Prep &prep,
                    std::vector<int> &n0);

// After the subdomain factorisations: V_i = [B_i K^+ B0_i^T | G_i^T], F0, G0, S_alpha and its
// kernel H, the cluster matrix M, the cluster kernels R_i H_i and the dual G.
void hybrid_prepare(const Decomposition &dec, Prep &prep, const std::vector<int> &n0, int threads);

}  // namespace feti
