// FETI4I C API of the B200 dual solver (src/app/apiwrapper/wrapper.cpp of the
// reference is the interface being replaced).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/feti4i.h"
#include "../../include/feti4i_ext.h"
#include "common.h"
#include "decompose.h"
#include "gpu_solver.h"
#include "prep.h"

namespace feti {

int g_verbose = 0;
static thread_local std::string t_last_error;
void set_last_error(const std::string &m) { t_last_error = m; }
const char *last_error() { return t_last_error.c_str(); }
void clear_last_error() { t_last_error.clear(); }

}  // namespace feti

using namespace feti;

struct FETI4IStructMatrix {
    ElementData el;
};

struct FETI4IStructInstance {
    ElementData el;              // copy of the element data (the reference copies too, wrapper.cpp:156-162)
    std::vector<double> rhs;
    std::vector<int> l2g;
    std::vector<int> dir_idx;
    std::vector<double> dir_val;
    int iopt[FETI4I_INTEGER_OPTIONS_SIZE];
    double ropt[FETI4I_REAL_OPTIONS_SIZE];
    double ext[FETI4I_EXT_OPTIONS_SIZE];
    Decomposition dec_full;      // numbering of the whole problem
    Decomposition dec;           // the subdomains this instance prepares (all, or the owned block)
    Prep prep;
    std::unique_ptr<GpuSolver> gpu;
    SolveOptions sopt;
    SolveStats stats;
    std::vector<double> b, e, lambda, alpha;
    double t_prep = 0.0, t_upload = 0.0, t_solve_wall = 0.0;
    bool rhs_on_device = false;
    int multi_on_device = 0;
};

namespace {

std::mutex g_mutex;
std::list<FETI4IStructMatrix *> g_matrices;
std::list<FETI4IStructInstance *> g_instances;
double g_ext[FETI4I_EXT_OPTIONS_SIZE] = {0, 1, 0, 48, 16, 0.003, 0, 0, 1, 1, 1, 1, 0, 0, 0};

template <typename F>
void guarded(F &&f) {
    std::lock_guard<std::mutex> lock(g_mutex);
    clear_last_error();
    try {
        f();
    } catch (const std::exception &ex) {
        set_last_error(ex.what());
        FETI_LOG(1, "FETI4I error: %s\n", ex.what());
    }
}

FETI4IStructInstance *check_instance(FETI4IInstance inst) {
    FETI_CHECK(inst && std::find(g_instances.begin(), g_instances.end(), inst) != g_instances.end(),
               "FETI4I: invalid instance handle");
    return inst;
}
FETI4IStructMatrix *check_matrix(FETI4IMatrix m) {
    FETI_CHECK(m && std::find(g_matrices.begin(), g_matrices.end(), m) != g_matrices.end(),
               "FETI4I: invalid matrix handle");
    return m;
}

// Caller integers (FETI4IInt: 32 or 64 bit, by FETI4I_INT_WIDTH) -> the library's 32-bit indices.
int narrow(FETI4IInt v, const char *what) {
    FETI_CHECK(v >= (FETI4IInt)INT32_MIN && v <= (FETI4IInt)INT32_MAX,
               std::string("FETI4I: ") + what + " does not fit the library's 32-bit indices");
    return (int)v;
}
std::vector<int> narrow_all(const FETI4IInt *v, size_t n, const char *what) {
    std::vector<int> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = narrow(v[i], what);
    return out;
}

void add_element(ElementData &el, int type, int nn, const FETI4IInt *nodes, int nd, const FETI4IInt *dofs,
                 const double *values) {
    // elements whose first dofsSize values are all zero are skipped, as in the
    // reference (src/app/apiwrapper/wrapper.cpp:151)
    bool zero = true;
    for (int i = 0; i < nd && zero; ++i) zero = values[i] == 0.0;
    if (zero) return;
    if (el.node_ptr.empty()) { el.node_ptr.push_back(0); el.dof_ptr.push_back(0); el.val_ptr.push_back(0); }
    el.etype.push_back(type);
    for (int i = 0; i < nn; ++i) el.nodes.push_back(narrow(nodes[i] - el.index_base, "a node index"));
    for (int i = 0; i < nd; ++i) el.dofs.push_back(narrow(dofs[i] - el.index_base, "a DOF index"));
    el.vals.insert(el.vals.end(), values, values + (size_t)nd * nd);
    el.node_ptr.push_back((int64_t)el.nodes.size());
    el.dof_ptr.push_back((int64_t)el.dofs.size());
    el.val_ptr.push_back((int64_t)el.vals.size());
}

// The decomposition depends on the element structure, the partition and the Dirichlet DOFs only;
// a matrix update with the same structure keeps it.
bool same_structure(const ElementData &a, const ElementData &b) {
    return a.etype == b.etype && a.node_ptr == b.node_ptr && a.dof_ptr == b.dof_ptr && a.nodes == b.nodes &&
           a.dofs == b.dofs && a.partition == b.partition && a.index_base == b.index_base;
}

void build(FETI4IStructInstance *I, bool keep_decomposition = false) {
    const int *io = I->iopt;
    g_verbose = io[FETI4I_VERBOSE_LEVEL];
    FETI_CHECK(io[FETI4I_FETI_METHOD] == 0 || io[FETI4I_FETI_METHOD] == 1,
               "FETI4I: FETI_METHOD " + std::to_string(io[FETI4I_FETI_METHOD]) +
                   " is not supported (0 TOTAL_FETI, 1 HYBRID_FETI)");
    FETI_CHECK(io[FETI4I_CGSOLVER] == 0, "FETI4I: only CGSOLVER 0 (PCG) is supported by this build");
    int prec = io[FETI4I_PRECONDITIONER];
    FETI_CHECK(prec >= 0 && prec <= 5, "FETI4I: PRECONDITIONER " + std::to_string(prec) + " is not supported (0..5)");
    FETI_CHECK(I->ropt[FETI4I_PRECISION] > 0, "FETI4I: PRECISION must be positive");
    FETI_CHECK(io[FETI4I_MAX_ITERATIONS] > 0, "FETI4I: MAX_ITERATIONS must be positive");
    double t0 = now_s();
    if (!keep_decomposition) {
        I->dec_full = decompose(I->el, io[FETI4I_SUBDOMAINS], I->dir_idx, I->dir_val);
        FETI_LOG(2, "FETI4I: decomposition %.3f s\n", now_s() - t0);
    }
    I->dec = I->dec_full;   // preprocess keeps the owned subdomains of a partitioned problem
    PrepOptions po;
    po.method = io[FETI4I_FETI_METHOD];
    if (po.method == 1 && !I->el.sub_cluster.empty()) {
        FETI_CHECK((int)I->el.sub_cluster.size() == I->dec.ndom,
                   "FETI4I: the cluster partition lists " + std::to_string(I->el.sub_cluster.size()) +
                       " subdomains, the problem has " + std::to_string(I->dec.ndom));
        po.sub_cluster = I->el.sub_cluster;
    }
    po.precond = prec;
    po.owned_first = (int)I->ext[FETI4I_EXT_OWNED_FIRST];
    po.owned_count = (int)I->ext[FETI4I_EXT_OWNED_COUNT];
    FETI_CHECK(po.owned_count == 0 || io[FETI4I_FETI_METHOD] == 0,
               "FETI4I: a partitioned dual problem (FETI4I_EXT_OWNED_COUNT > 0) is Total FETI only");
    po.scaling = I->ext[FETI4I_EXT_SCALING] != 0.0;
    po.threads = (int)I->ext[FETI4I_EXT_HOST_THREADS];
    // the device preprocessing runs with the GPU path; HOST_ONLY instances preprocess on the host
    po.device = I->ext[FETI4I_EXT_DEVICE_PREP] != 0.0 && I->ext[FETI4I_EXT_HOST_ONLY] == 0.0;
    // batch size of the device eliminations in bytes (tests force one subdomain per batch)
    if (const char *b = std::getenv("FETI4I_DEVICE_PREP_BATCH_BYTES")) po.device_mem = std::strtoull(b, nullptr, 10);
    // the previous device solver (and its tile stores) goes first: a rebuild must not hold two
    // copies of the device data at once
    I->gpu.reset();
    I->prep = Prep();
    preprocess(I->el, I->dec, I->rhs, po, I->prep);
    I->t_prep = now_s() - t0;
    FETI_LOG(1, "FETI4I: %d subdomains, %d multipliers, %d kernel vectors, preprocessing %.2f s\n", I->dec.ndom,
             I->dec.n_lambda, I->prep.n_kern, I->t_prep);
    SolveOptions &so = I->sopt;
    so.precision = I->ropt[FETI4I_PRECISION];
    so.max_iterations = io[FETI4I_MAX_ITERATIONS];
    // SUPER_DIRICHLET and MAGIC apply a sparse matrix on the touched DOFs, as LUMPED does: the
    // device iteration runs them through the LUMPED kernels with the matrix the preparation built
    so.precond = (prec == PREC_SUPER_DIRICHLET || prec == PREC_MAGIC) ? (int)PREC_LUMPED : prec;
    so.schur_precision = (int)I->ext[FETI4I_EXT_SCHUR_PRECISION];
    FETI_CHECK(so.schur_precision >= 0 && so.schur_precision <= 2, "FETI4I: invalid Schur precision");
    so.tiles_per_item = std::max(1, (int)I->ext[FETI4I_EXT_TILES_PER_ITEM]);
    so.chunk = std::max(1, (int)I->ext[FETI4I_EXT_GRAPH_CHUNK]);
    so.reliable_delta = I->ext[FETI4I_EXT_RELIABLE_DELTA];
    so.tile_kernel = (int)I->ext[FETI4I_EXT_TILE_KERNEL];
    so.autotune = I->ext[FETI4I_EXT_AUTOTUNE] != 0.0;
    so.symm_tensor = I->ext[FETI4I_EXT_SYMM_TENSOR] != 0.0;
    so.schur_explicit = I->ext[FETI4I_EXT_SCHUR_EXPLICIT] != 0.0;
    I->gpu.reset();
    I->rhs_on_device = false;
    if (I->ext[FETI4I_EXT_HOST_ONLY] == 0.0) {
        double t1 = now_s();
        I->gpu.reset(new GpuSolver());
        I->gpu->upload(I->dec, I->prep, so);
        I->t_upload = now_s() - t1;
    }
}

}  // namespace

extern "C" {

const char *FETI4IGetLastError(void) { return last_error(); }

void FETI4ISetDefaultIntegerOptions(FETI4IInt *options) {
    guarded([&] {
        FETI_CHECK(options, "FETI4I: null options array");
        // defaults of src/config/ecf/input/feti4ilibrary.cpp:7 and src/config/ecf/solver/feti.cpp
        options[FETI4I_SUBDOMAINS] = 4;
        options[FETI4I_MAX_ITERATIONS] = 200;
        options[FETI4I_FETI_METHOD] = 0;
        options[FETI4I_PRECONDITIONER] = 3;
        options[FETI4I_CGSOLVER] = 0;
        options[FETI4I_N_MICS] = 2;
        options[FETI4I_VERBOSE_LEVEL] = 1;
        options[FETI4I_MEASURE_LEVEL] = 0;
        options[FETI4I_PRINT_MATRICES] = 0;
        options[FETI4I_SC_SIZE] = 200;
    });
}

void FETI4ISetDefaultRealOptions(FETI4IReal *options) {
    guarded([&] {
        FETI_CHECK(options, "FETI4I: null options array");
        options[FETI4I_PRECISION] = 1e-5;
    });
}

void FETI4ICreateStiffnessMatrix(FETI4IMatrix *matrix, FETI4IInt type, FETI4IInt indexBase) {
    guarded([&] {
        FETI_CHECK(matrix, "FETI4I: null matrix pointer");
        FETI_CHECK(type == FETI4I_REAL_SYMMETRIC_POSITIVE_DEFINITE,
                   "FETI4I: only REAL_SYMMETRIC_POSITIVE_DEFINITE matrices are supported by the explicit-Schur solver");
        auto *m = new FETI4IStructMatrix();
        m->el.type = (int)type;
        m->el.index_base = narrow(indexBase, "indexBase");
        g_matrices.push_back(m);
        *matrix = m;
    });
}

void FETI4IAddElement(FETI4IMatrix matrix, FETI4IInt type, FETI4IInt nodesSize, FETI4IInt *nodes, FETI4IInt dofsSize,
                      FETI4IInt *dofs, FETI4IReal *values) {
    guarded([&] {
        auto *m = check_matrix(matrix);
        FETI_CHECK(nodesSize > 0 && dofsSize > 0 && nodes && dofs && values, "FETI4I: invalid element data");
        add_element(m->el, (int)type, narrow(nodesSize, "nodesSize"), nodes, narrow(dofsSize, "dofsSize"), dofs,
                    values);
    });
}

void FETI4IAddElements(FETI4IMatrix matrix, FETI4IInt type, FETI4IInt nelems, FETI4IInt nodesSize, FETI4IInt *nodes,
                       FETI4IInt dofsSize, FETI4IInt *dofs, FETI4IReal *values) {
    guarded([&] {
        auto *m = check_matrix(matrix);
        FETI_CHECK(nelems >= 0 && nodesSize > 0 && dofsSize > 0 && nodes && dofs && values, "FETI4I: invalid element data");
        m->el.etype.reserve(m->el.etype.size() + nelems);
        m->el.vals.reserve(m->el.vals.size() + (size_t)nelems * dofsSize * dofsSize);
        const int nn = narrow(nodesSize, "nodesSize"), nd = narrow(dofsSize, "dofsSize");
        for (FETI4IInt e = 0; e < nelems; ++e)
            add_element(m->el, (int)type, nn, nodes + (size_t)e * nn, nd, dofs + (size_t)e * nd,
                        values + (size_t)e * nd * nd);
    });
}

void FETI4ISetSubdomainPartition(FETI4IMatrix matrix, FETI4IInt size, FETI4IInt *elem2sub) {
    guarded([&] {
        auto *m = check_matrix(matrix);
        FETI_CHECK(size == (FETI4IInt)m->el.nelem(), "FETI4I: partition size differs from the number of added elements");
        m->el.partition = narrow_all(elem2sub, (size_t)size, "a subdomain index");
    });
}

void FETI4ISetClusterPartition(FETI4IMatrix matrix, FETI4IInt nsubdomains, const FETI4IInt *sub2cluster) {
    guarded([&] {
        auto *m = check_matrix(matrix);
        FETI_CHECK(nsubdomains >= 0 && (nsubdomains == 0 || sub2cluster), "FETI4I: invalid cluster partition");
        m->el.sub_cluster = narrow_all(sub2cluster, (size_t)nsubdomains, "a cluster index");
    });
}

void FETI4ISetExtendedOption(FETI4IInt key, FETI4IReal value) {
    guarded([&] {
        FETI_CHECK(key >= 0 && key < FETI4I_EXT_OPTIONS_SIZE, "FETI4I: unknown extended option");
        g_ext[key] = value;
    });
}

void FETI4ISetExtendedOptions(FETI4IInstance instance, FETI4IInt key, FETI4IReal value) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(key >= 0 && key < FETI4I_EXT_OPTIONS_SIZE, "FETI4I: unknown extended option");
        if (I->ext[key] == value) return;
        I->ext[key] = value;
        if (key == FETI4I_EXT_TRUNCATE) return;   // read by the next solve
        if (I->gpu && (key == FETI4I_EXT_RELIABLE_DELTA || key == FETI4I_EXT_GRAPH_CHUNK ||
                       key == FETI4I_EXT_SYMM_TENSOR)) {
            SolveOptions so = I->sopt;
            so.reliable_delta = I->ext[FETI4I_EXT_RELIABLE_DELTA];
            so.chunk = std::max(1, (int)I->ext[FETI4I_EXT_GRAPH_CHUNK]);
            so.symm_tensor = I->ext[FETI4I_EXT_SYMM_TENSOR] != 0.0;
            I->gpu->set_options(so);
            I->sopt = so;
            return;
        }
        build(I, true);   // preprocessing-dependent option: same decomposition, new preparation
    });
}

void FETI4ICreateInstance(FETI4IInstance *instance, FETI4IMatrix matrix, FETI4IInt size, FETI4IReal *rhs, FETI4IInt *l2g,
                          FETI4IMPIInt neighbours_size, FETI4IMPIInt *neighbours, FETI4IInt dirichlet_size,
                          FETI4IInt *dirichlet_indices, FETI4IReal *dirichlet_values, FETI4IInt *integer_options,
                          FETI4IReal *real_options) {
    guarded([&] {
        FETI_CHECK(instance, "FETI4I: null instance pointer");
        auto *m = check_matrix(matrix);
        FETI_CHECK(neighbours_size == 0, "FETI4I: this build runs on one process (neighbours_size must be 0)");
        FETI_CHECK(integer_options && real_options, "FETI4I: null options");
        FETI_CHECK(size >= 0 && (size == 0 || rhs), "FETI4I: invalid right-hand side");
        std::unique_ptr<FETI4IStructInstance> I(new FETI4IStructInstance());
        I->el = m->el;
        I->rhs.assign(rhs, rhs + size);
        if (l2g) I->l2g = narrow_all(l2g, (size_t)size, "an l2g entry");
        for (FETI4IInt i = 0; i < dirichlet_size; ++i) {
            I->dir_idx.push_back(narrow(dirichlet_indices[i] - m->el.index_base, "a Dirichlet index"));
            I->dir_val.push_back(dirichlet_values[i]);
        }
        for (int k = 0; k < FETI4I_INTEGER_OPTIONS_SIZE; ++k) I->iopt[k] = narrow(integer_options[k], "an option");
        std::memcpy(I->ropt, real_options, sizeof(I->ropt));
        std::memcpy(I->ext, g_ext, sizeof(I->ext));
        (void)neighbours;
        build(I.get());
        g_instances.push_back(I.get());
        *instance = I.release();
    });
}

// The internal dual PCG needs the whole dual problem; a partitioned instance (one process's block of
// subdomains) is driven through the device-operator entry points instead.
static void check_whole(FETI4IStructInstance *I) {
    FETI_CHECK(I->ext[FETI4I_EXT_OWNED_COUNT] == 0.0,
               "FETI4I: this instance holds a block of the subdomains (FETI4I_EXT_OWNED_COUNT); it is solved by a "
               "partitioned driver through FETI4IApplyDualOperatorDevice, FETI4IApplyPreconditionerDevice and "
               "FETI4IPrimalFromDual");
}

// The reference's output formatting (FETISolver.cpp:130-147): every value truncated to
// dplaces = 1 / precision / max(1, 10^ceil(log10 max|u|)) places.  The reference applies it to the
// subdomain primal values before they are gathered; here it is applied to the caller's (averaged)
// solution vector, so values on subdomain interfaces may differ from the reference's by one unit of
// 1 / dplaces.
static void truncate_like_reference(double *u, size_t n, double precision) {
    double gmax = 0.0;
    for (size_t i = 0; i < n; ++i) gmax = std::max(gmax, std::fabs(u[i]));
    if (gmax == 0.0) return;
    const double dplaces = 1.0 / precision / std::max(1.0, std::pow(10.0, std::ceil(std::log10(gmax))));
    for (size_t i = 0; i < n; ++i) u[i] = std::trunc(dplaces * u[i]) / dplaces;
}

static void solve_instance(FETI4IStructInstance *I) {
    FETI_CHECK(I->gpu, "FETI4I: instance was created with FETI4I_EXT_HOST_ONLY; no device solver");
    make_rhs_vectors(I->dec, I->prep, I->b, I->e);
    I->gpu->set_rhs(I->b, I->e);
    I->rhs_on_device = true;
    I->gpu->solve(I->stats);
    I->gpu->get_solution(I->lambda, I->alpha);
    FETI_LOG(1, "FETI4I: PCG %s after %d iterations (|w| %.3e, tol %.3e), %.3f ms on the device\n",
             I->stats.converged ? "converged" : "stopped", I->stats.iterations, I->stats.final_norm, I->stats.tol,
             I->stats.t_solve_ms);
}

void FETI4ISolve(FETI4IInstance instance, FETI4IInt solution_size, FETI4IReal *solution) {
    guarded([&] {
        auto *I = check_instance(instance);
        check_whole(I);
        FETI_CHECK(solution_size >= 0 && (solution_size == 0 || solution), "FETI4I: invalid solution array");
        FETI_CHECK(I->gpu, "FETI4I: instance was created with FETI4I_EXT_HOST_ONLY; no device solver");
        double t0 = now_s();
        I->gpu->solve_full(I->rhs.data(), (int)I->rhs.size(), solution, solution_size, I->stats, true);
        if (I->ext[FETI4I_EXT_TRUNCATE] != 0.0)
            truncate_like_reference(solution, (size_t)solution_size, I->ropt[FETI4I_PRECISION]);
        I->rhs_on_device = true;
        I->t_solve_wall = (now_s() - t0) * 1e3;
        I->lambda.clear();
        FETI_LOG(1, "FETI4I: PCG %s after %d iterations (|w| %.3e, tol %.3e), %.3f ms on the device\n",
                 I->stats.converged ? "converged" : "stopped", I->stats.iterations, I->stats.final_norm, I->stats.tol,
                 I->stats.t_solve_ms);
    });
}

void FETI4ISolveMulti(FETI4IInstance instance, FETI4IInt nrhs, FETI4IInt size, const FETI4IReal *rhs,
                      FETI4IReal *solutions) {
    guarded([&] {
        auto *I = check_instance(instance);
        check_whole(I);
        FETI_CHECK(I->gpu, "FETI4I: instance was created with FETI4I_EXT_HOST_ONLY; no device solver");
        FETI_CHECK(rhs && solutions && size > 0, "FETI4ISolveMulti: invalid arrays");
        double t0 = now_s();
        I->gpu->solve_multi(rhs, nrhs, size, solutions, size, I->stats, true);
        if (I->ext[FETI4I_EXT_TRUNCATE] != 0.0)
            for (FETI4IInt j = 0; j < nrhs; ++j)
                truncate_like_reference(solutions + (size_t)j * size, (size_t)size, I->ropt[FETI4I_PRECISION]);
        I->t_solve_wall = (now_s() - t0) * 1e3;
        I->multi_on_device = nrhs;
    });
}

FETI4IReal FETI4ISolveMultiResident(FETI4IInstance instance, FETI4IInt nrhs) {
    double ms = -1.0;
    guarded([&] {
        auto *I = check_instance(instance);
        check_whole(I);
        FETI_CHECK(I->gpu && I->multi_on_device == nrhs, "FETI4ISolveMultiResident: call FETI4ISolveMulti first");
        I->gpu->solve_multi(nullptr, nrhs, 0, nullptr, 0, I->stats, false);
        ms = I->stats.t_solve_ms;
    });
    return ms;
}

FETI4IReal FETI4ISolveResident(FETI4IInstance instance) {
    double ms = -1.0;
    guarded([&] {
        auto *I = check_instance(instance);
        check_whole(I);
        FETI_CHECK(I->gpu && I->rhs_on_device, "FETI4I: no right-hand side on the device (call FETI4ISolve first)");
        I->gpu->solve(I->stats);
        I->lambda.clear();
        ms = I->stats.t_solve_ms;
    });
    return ms;
}

void FETI4ISetSolvePrecision(FETI4IInstance instance, FETI4IInt precision) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        SolveOptions so = I->sopt;
        so.schur_precision = precision;
        I->gpu->set_options(so);
        I->sopt = so;
    });
}

void FETI4IUpdateStiffnessMatrix(FETI4IInstance instance, FETI4IMatrix stiffnessMatrix) {
    guarded([&] {
        auto *I = check_instance(instance);
        auto *m = check_matrix(stiffnessMatrix);
        std::vector<int> part = I->el.partition;
        ElementData el = m->el;
        if (el.partition.empty() && part.size() == el.nelem()) el.partition = part;
        const bool keep = same_structure(el, I->el);
        I->el = std::move(el);
        build(I, keep);
    });
}

void FETI4IUpdateStiffnessMatrixScaled(FETI4IInstance instance, FETI4IMatrix stiffnessMatrix, FETI4IInt size,
                                       const FETI4IReal *scale) {
    guarded([&] {
        auto *I = check_instance(instance);
        auto *m = check_matrix(stiffnessMatrix);
        const ElementData &src = m->el;
        FETI_CHECK(size == (FETI4IInt)src.nelem() && (size == 0 || scale),
                   "FETI4I: one scale per stored element of the matrix is required");
        std::vector<int> part = I->el.partition;
        const bool keep = same_structure(src, I->el) ||
                          (src.partition.empty() && part.size() == src.nelem() && [&] {
                              ElementData probe;
                              probe.etype = src.etype; probe.node_ptr = src.node_ptr; probe.dof_ptr = src.dof_ptr;
                              probe.nodes = src.nodes; probe.dofs = src.dofs; probe.partition = part;
                              probe.index_base = src.index_base;
                              return same_structure(probe, I->el);
                          }());
        // K_e := scale_e * K_e of the matrix object (element after element, in parallel)
        I->el.vals.resize(src.vals.size());
        const long long ne = (long long)src.nelem();
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < ne; ++e) {
            const double s_ = scale[e];
            for (int64_t k = src.val_ptr[e]; k < src.val_ptr[e + 1]; ++k) I->el.vals[k] = s_ * src.vals[k];
        }
        if (!keep) {
            std::vector<double> v = std::move(I->el.vals);
            I->el = src;
            I->el.vals = std::move(v);
            if (I->el.partition.empty() && part.size() == I->el.nelem()) I->el.partition = part;
        }
        build(I, keep);
    });
}

void FETI4IUpdateRhs(FETI4IInstance instance, FETI4IInt size, FETI4IReal *values) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(size >= 0 && (size == 0 || values), "FETI4I: invalid right-hand side");
        I->rhs.assign(values, values + size);
        // subdomain loads: value / multiplicity (src/assembler/physics/precomputed.cpp:61-65)
        const int dpn = I->dec.dpn;
        for (int d = 0; d < I->dec.ndom; ++d) {
            SubPrep &S = I->prep.sub[d];
            const DomainRows &D = I->dec.dom[d];
            for (int a = 0; a < (int)D.nodes.size(); ++a)
                for (int c = 0; c < dpn; ++c) {
                    int dof = I->dec.node_dof[(size_t)D.nodes[a] * dpn + c];
                    double v = (dof >= 0 && dof < (int)I->rhs.size()) ? I->rhs[dof] : 0.0;
                    S.f[dpn * a + c] = v / I->dec.node_ndom[D.nodes[a]];
                }
        }
        I->rhs_on_device = false;
    });
}

void FETI4IUpdateDirichlet(FETI4IInstance instance, FETI4IInt size, FETI4IInt *indices, FETI4IReal *values) {
    guarded([&] {
        auto *I = check_instance(instance);
        std::vector<int> idx;
        std::vector<double> val;
        for (FETI4IInt i = 0; i < size; ++i) {
            idx.push_back(narrow(indices[i] - I->el.index_base, "a Dirichlet index"));
            val.push_back(values[i]);
        }
        std::vector<int> a = idx, b = I->dir_idx;
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        I->dir_idx = idx;
        I->dir_val = val;
        if (a == b) {
            // same constrained DOFs: only the values c of the Dirichlet rows change
            const int dpn = I->dec.dpn;
            std::vector<double> byk((size_t)I->dec.n_nodes * dpn, 0.0);
            for (size_t i = 0; i < idx.size(); ++i)
                byk[(size_t)I->dec.dof_node[idx[i]] * dpn + I->dec.dof_comp[idx[i]]] = val[i];
            for (Decomposition *dc : {&I->dec, &I->dec_full})
                for (auto &D : dc->dom)
                    for (size_t r = 0; r < D.lam.size(); ++r)
                        if (D.other[r] < 0) D.c[r] = byk[(size_t)D.node[r] * dpn + D.comp[r]];
            I->rhs_on_device = false;
        } else {
            build(I);
        }
    });
}

void FETI4IDestroy(void *ptr) {
    guarded([&] {
        for (auto it = g_matrices.begin(); it != g_matrices.end(); ++it)
            if (*it == ptr) { delete *it; g_matrices.erase(it); return; }
        for (auto it = g_instances.begin(); it != g_instances.end(); ++it)
            if (*it == ptr) { delete *it; g_instances.erase(it); return; }
    });
}

void FETI4IGetStats(FETI4IInstance instance, FETI4IInt size, FETI4IReal *stats) {
    guarded([&] {
        auto *I = check_instance(instance);
        double v[FETI4I_STAT_SIZE] = {0};
        v[FETI4I_STAT_ITERATIONS] = I->stats.iterations;
        v[FETI4I_STAT_CONVERGED] = I->stats.converged ? 1 : 0;
        v[FETI4I_STAT_DUAL_SIZE] = I->dec.n_lambda;
        v[FETI4I_STAT_KERNEL_SIZE] = I->prep.n_kern;
        v[FETI4I_STAT_SUBDOMAINS] = I->dec.ndom;
        v[FETI4I_STAT_PREP_SECONDS] = I->t_prep;
        v[FETI4I_STAT_UPLOAD_SECONDS] = I->t_upload;
        v[FETI4I_STAT_SOLVE_MS] = I->stats.t_solve_ms;
        v[FETI4I_STAT_SOLVE_WALL_MS] = I->t_solve_wall;
        v[FETI4I_STAT_FAPPLY_BYTES] = I->gpu ? I->gpu->fapply_bytes(I->sopt.schur_precision) : 0.0;
        v[FETI4I_STAT_REPLACEMENTS] = I->stats.replacements;
        v[FETI4I_STAT_KERNEL_LAUNCHES] = I->stats.kernel_launches;
        v[FETI4I_STAT_DEVICE_BYTES] = I->gpu ? (double)I->gpu->device_bytes() : 0.0;
        v[FETI4I_STAT_FINAL_NORM] = I->stats.final_norm;
        v[FETI4I_STAT_TOLERANCE] = I->stats.tol;
        v[FETI4I_STAT_ELEMENTS] = (double)I->el.nelem();
        v[FETI4I_STAT_PREP_DEVICE_MS] = I->prep.t_device_factor_ms;
        v[FETI4I_STAT_PREP_DEVICE_FLOPS] = I->prep.device_factor_flops;
        v[FETI4I_STAT_KPLUS_TILES] = I->gpu ? I->gpu->kplus_tile_fraction() : 0.0;
        for (int i = 0; i < size && i < FETI4I_STAT_SIZE; ++i) stats[i] = v[i];
    });
}

const char *FETI4IGetTuning(FETI4IInstance instance) {
    static thread_local std::string t;
    t.clear();
    guarded([&] {
        auto *I = check_instance(instance);
        if (I->gpu) t = I->gpu->tuning();
    });
    return t.c_str();
}

void FETI4IGetDualSolution(FETI4IInstance instance, FETI4IReal *lambda, FETI4IReal *amplitudes) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu && I->rhs_on_device, "FETI4I: no solution yet");
        if (I->lambda.empty()) I->gpu->get_solution(I->lambda, I->alpha);
        if (lambda) std::copy(I->lambda.begin(), I->lambda.end(), lambda);
        if (amplitudes) std::copy(I->alpha.begin(), I->alpha.end(), amplitudes);
    });
}

void FETI4IGetSubdomainInfo(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *info) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(subdomain >= 0 && subdomain < I->dec.ndom, "FETI4I: subdomain index out of range");
        const SubPrep &S = I->prep.sub[subdomain];
        info[0] = S.n; info[1] = S.ni; info[2] = S.nk; info[3] = S.t;
    });
}

void FETI4IGetSubdomainMultipliers(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *lambda, FETI4IInt *dof,
                                   FETI4IReal *sign, FETI4IReal *weight, FETI4IReal *c) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(subdomain >= 0 && subdomain < I->dec.ndom, "FETI4I: subdomain index out of range");
        const DomainRows &D = I->dec.dom[subdomain];
        for (size_t r = 0; r < D.lam.size(); ++r) {
            if (lambda) lambda[r] = D.lam[r];
            if (dof) dof[r] = D.dof[r];
            if (sign) sign[r] = D.sign[r];
            if (weight) weight[r] = D.w[r];
            if (c) c[r] = D.c[r];
        }
    });
}

void FETI4IGetSubdomainNodes(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *nodes) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(subdomain >= 0 && subdomain < I->dec.ndom, "FETI4I: subdomain index out of range");
        const DomainRows &D = I->dec.dom[subdomain];
        std::copy(D.nodes.begin(), D.nodes.end(), nodes);
    });
}

void FETI4IGetSubdomainSchur(FETI4IInstance instance, FETI4IInt subdomain, FETI4IReal *S) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(subdomain >= 0 && subdomain < I->dec.ndom, "FETI4I: subdomain index out of range");
        const SubPrep &P = I->prep.sub[subdomain];
        if (P.S.empty() && I->gpu) I->gpu->subdomain_schur(subdomain, S);   // device preprocessing
        else std::copy(P.S.begin(), P.S.end(), S);
    });
}

void FETI4IGetSubdomainKernel(FETI4IInstance instance, FETI4IInt subdomain, FETI4IReal *R) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(subdomain >= 0 && subdomain < I->dec.ndom, "FETI4I: subdomain index out of range");
        const SubPrep &P = I->prep.sub[subdomain];
        std::copy(P.R.begin(), P.R.end(), R);
    });
}

FETI4IInt FETI4IGetSubdomainCorners(FETI4IInstance instance, FETI4IInt subdomain, FETI4IInt *rows, FETI4IInt *dofs,
                                    FETI4IReal *signs) {
    FETI4IInt count = -1;
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(subdomain >= 0 && subdomain < I->dec.ndom, "FETI4I: subdomain index out of range");
        const SubPrep &S = I->prep.sub[subdomain];
        count = (FETI4IInt)S.b0_row.size();
        if (rows) std::copy(S.b0_row.begin(), S.b0_row.end(), rows);
        if (dofs) std::copy(S.b0_dof.begin(), S.b0_dof.end(), dofs);
        if (signs) std::copy(S.b0_sign.begin(), S.b0_sign.end(), signs);
    });
    return count;
}

void FETI4IGetClusterInfo(FETI4IInstance instance, FETI4IInt *info) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(info, "FETI4I: null info array");
        const Prep &P = I->prep;
        info[0] = P.method;
        info[1] = P.method == 1 ? (FETI4IInt)P.clusters.size() : I->dec.ndom;
        int n0 = 0;
        for (const auto &C : P.clusters) n0 += C.n0;
        info[2] = n0;
        info[3] = P.n_kern;
    });
}

void FETI4IApplySubdomainKplus(FETI4IInstance instance, FETI4IInt subdomain, FETI4IReal *x) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(subdomain >= 0 && subdomain < I->dec.ndom, "FETI4I: subdomain index out of range");
        if (I->prep.sub[subdomain].Lp.empty() && I->gpu) I->gpu->subdomain_kplus(subdomain, x);   // device factor
        else I->prep.sub[subdomain].kplus(x);
    });
}

void FETI4IGetDualRhs(FETI4IInstance instance, FETI4IReal *b, FETI4IReal *e) {
    guarded([&] {
        auto *I = check_instance(instance);
        std::vector<double> bb, ee;
        if (I->prep.dstore && I->gpu) {   // device preprocessing: K^+ only on the device
            bb.assign(I->dec.n_lambda, 0.0);
            ee.assign(I->prep.n_kern, 0.0);
            I->gpu->dual_rhs(I->rhs.data(), (int)I->rhs.size(), bb.data(), ee.data(), I->dec.n_lambda,
                             I->prep.n_kern);
        } else {
            make_rhs_vectors(I->dec, I->prep, bb, ee);
        }
        if (b) std::copy(bb.begin(), bb.end(), b);
        if (e) std::copy(ee.begin(), ee.end(), e);
    });
}

void FETI4IApplyDualOperator(FETI4IInstance instance, FETI4IInt precision, FETI4IReal *x, FETI4IReal *y) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        I->gpu->apply_F(x, y, precision);
    });
}

void FETI4IApplyDualOperatorMulti(FETI4IInstance instance, FETI4IInt precision, FETI4IInt nrhs, FETI4IReal *x,
                                  FETI4IReal *y) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        FETI_CHECK(x && y, "FETI4IApplyDualOperatorMulti: invalid arrays");
        I->gpu->apply_F_multi(x, y, (int)nrhs, precision);
    });
}

FETI4IReal FETI4ITimeDualOperator(FETI4IInstance instance, FETI4IInt precision, FETI4IInt reps) {
    double ms = -1.0;
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        ms = I->gpu->time_F((int)precision, std::max(1, (int)reps));
    });
    return ms;
}

void FETI4IElementEnergies(FETI4IInstance instance, FETI4IInt size, const FETI4IReal *u, const FETI4IReal *v,
                           FETI4IReal *out) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        FETI_CHECK(size > 0 && u && v && out, "FETI4I: invalid vectors");
        I->gpu->element_energies(I->el, u, v, size, out);
    });
}

void FETI4IApplyDualOperatorDevice(FETI4IInstance instance, FETI4IInt precision, const FETI4IReal *x, FETI4IReal *y,
                                   void *stream) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        FETI_CHECK(x && y, "FETI4IApplyDualOperatorDevice: null vector");
        I->gpu->apply_F_device(x, y, (int)precision, stream);
    });
}

void FETI4IApplyPreconditionerDevice(FETI4IInstance instance, const FETI4IReal *x, FETI4IReal *y, void *stream) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        FETI_CHECK(x && y, "FETI4IApplyPreconditionerDevice: null vector");
        I->gpu->apply_prec_device(x, y, stream);
    });
}

void FETI4IPrimalFromDual(FETI4IInstance instance, const FETI4IReal *lambda, const FETI4IReal *amplitudes,
                          FETI4IInt solution_size, FETI4IReal *solution) {
    guarded([&] {
        auto *I = check_instance(instance);
        FETI_CHECK(I->gpu, "FETI4I: no device solver");
        FETI_CHECK(lambda && amplitudes && solution_size >= 0 && (solution_size == 0 || solution),
                   "FETI4IPrimalFromDual: invalid arrays");
        I->gpu->primal_from_dual(I->rhs.data(), (int)I->rhs.size(), lambda, amplitudes, solution, (int)solution_size);
    });
}

int FETI4ITiledSymvNoAlloc(const FETI4IReal *tiles, const long long *tile_offset, const FETI4IInt *order,
                           const FETI4IInt *vector_offset, FETI4IInt nmatrices, FETI4IInt max_order,
                           const FETI4IReal *x, FETI4IReal *y, FETI4IReal *dot, void *stream) {
    int rc = -1;
    guarded([&] {
#if FETI4I_INT_WIDTH == 32
        rc = tiled_symv_noalloc(tiles, tile_offset, order, vector_offset, nmatrices, max_order, x, y, dot, stream);
#else
        (void)tiles; (void)tile_offset; (void)order; (void)vector_offset; (void)nmatrices; (void)max_order;
        (void)x; (void)y; (void)dot; (void)stream;
        FETI_CHECK(false, "FETI4ITiledSymvNoAlloc reads 32-bit device index arrays: call it through the "
                          "FETI4I_INT_WIDTH 32 library");
#endif
    });
    return rc;
}

}  // extern "C"
