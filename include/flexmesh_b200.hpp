// flexmesh_b200.hpp — C++ drop-in for the FlexMesh hot path over the C ABI
// (fm_api.h).  Same names and argument meaning as the reference's
//   FEM/adaptive_fem_engine.hpp   build_csr_sparsity_pattern_rigorous (:1069),
//                                 assemble_global_threadlocal (:1126),
//                                 assemble_global_residual_only (:990),
//                                 pcg_solve_ilu0 (:1283),
//                                 tet_element_stiffness_rigorous (:511),
//                                 generate_unit_cube_mesh (:2219)
//   FEM/nonlinear_solver.hpp      NewtonSolverConfig, NewtonSolverResult,
//                                 NonlinearNewtonSolver::solve (:23-238)
//   FEM/constitutive_models.hpp   NeoHookeanParameters, NeoHookeanMaterial (:30-52)
// Mesh/CSR arguments are templates: the reference's own MeshTopology and
// SparseCSR (or anything with the same fields: nodes[i].x/.y/.z,
// elements[e].nodes[4], elements[e].volume; n_rows/row_ptr/col_idx/val) pass
// straight through.  Free functions use a per-thread default context on
// device 0 unless a Context is given.  Errors throw flexmesh_b200::Error
// (the reference's functions are noexcept and degrade silently; here a
// device-side problem is reported).
#pragma once

#include <array>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "fm_api.h"

namespace flexmesh_b200 {

class Error : public std::runtime_error {
public:
    Error(fm_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
    fm_status status;
};

class Context {
public:
    explicit Context(int device = 0, void* cuda_stream = nullptr) {
        fm_status s = fm_create(&c_, device, cuda_stream);
        if (s != FM_OK) throw Error(s, "fm_create failed");
    }
    ~Context() { fm_destroy(c_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    fm_ctx* get() const { return c_; }
    void check(fm_status s, const char* what) const {
        if (s == FM_OK) return;
        char buf[512];
        fm_last_error(c_, buf, sizeof buf);
        throw Error(s, std::string(what) + ": " + buf);
    }
    // identity of the mesh last uploaded (to skip re-uploads)
    const void* mesh_key = nullptr;
    size_t mesh_nodes = 0, mesh_elems = 0;

private:
    fm_ctx* c_ = nullptr;
};

inline Context& default_context() {
    thread_local Context ctx(0);
    return ctx;
}

// ---------------------------------------------------------------------------
// mesh hand-over
// ---------------------------------------------------------------------------
template <class Mesh>
void set_mesh(Context& ctx, const Mesh& mesh, bool use_stored_volume = true) {
    const size_t nn = mesh.nodes.size(), ne = mesh.elements.size();
    if (ctx.mesh_key == &mesh && ctx.mesh_nodes == nn && ctx.mesh_elems == ne) return;
    std::vector<double> xyz(3 * nn), vol(ne);
    std::vector<uint32_t> conn(4 * ne);
    for (size_t n = 0; n < nn; ++n) {
        xyz[3 * n] = mesh.nodes[n].x;
        xyz[3 * n + 1] = mesh.nodes[n].y;
        xyz[3 * n + 2] = mesh.nodes[n].z;
    }
    for (size_t e = 0; e < ne; ++e) {
        for (int v = 0; v < 4; ++v) conn[4 * e + v] = (uint32_t)mesh.elements[e].nodes[v];
        vol[e] = mesh.elements[e].volume;
    }
    ctx.check(fm_set_mesh(ctx.get(), (uint32_t)nn, xyz.data(), (uint32_t)ne, conn.data(),
                          use_stored_volume ? vol.data() : nullptr),
              "fm_set_mesh");
    ctx.mesh_key = &mesh;
    ctx.mesh_nodes = nn;
    ctx.mesh_elems = ne;
}

// generate_unit_cube_mesh (:2219): node coordinates and connectivity
inline void generate_unit_cube(int N, std::vector<double>& xyz, std::vector<uint32_t>& conn) {
    uint32_t nn = 0, ne = 0;
    if (fm_unit_cube_sizes(N, &nn, &ne) != FM_OK) throw Error(FM_ERR_ARG, "bad N");
    xyz.resize(3 * (size_t)nn);
    conn.resize(4 * (size_t)ne);
    fm_unit_cube(N, xyz.data(), conn.data());
}

// ---------------------------------------------------------------------------
// free functions
// ---------------------------------------------------------------------------
// build_csr_sparsity_pattern_rigorous (:1069).  fill = FM_PATTERN_REFERENCE
// reproduces the reference's column fill exactly (with its defect);
// FM_PATTERN_SOLVE lists every neighbour column (what the solves need).
template <class Mesh, class CSR>
void build_csr_sparsity_pattern_rigorous(Context& ctx, const Mesh& mesh, CSR& K,
                                         fm_pattern fill = FM_PATTERN_SOLVE) {
    set_mesh(ctx, mesh);
    uint32_t nn, ne, n;
    uint64_t nnz;
    fm_sizes(ctx.get(), &nn, &ne, &n, &nnz);
    K.n_rows = n;
    K.row_ptr.assign(n + 1, 0);
    K.col_idx.assign(nnz, 0);
    K.val.assign(nnz, 0.0);
    ctx.check(fm_build_pattern(ctx.get(), fill, K.row_ptr.data(), K.col_idx.data(), nullptr),
              "fm_build_pattern");
}
template <class Mesh, class CSR>
void build_csr_sparsity_pattern_rigorous(const Mesh& mesh, CSR& K) {
    build_csr_sparsity_pattern_rigorous(default_context(), mesh, K);
}

// assemble_global_threadlocal (:1126): K.val (solve pattern) and f_int for
// the problem's (E, nu).  K must hold the solve pattern of the same mesh.
template <class Mesh, class Prob, class CSR>
void assemble_global_threadlocal(Context& ctx, const Mesh& mesh, const Prob& prob,
                                 const double* u, CSR& K, std::vector<double>& f_int) {
    set_mesh(ctx, mesh);
    ctx.check(fm_set_material(ctx.get(), prob.E, prob.nu, nullptr), "fm_set_material");
    uint32_t nn, ne, n;
    uint64_t nnz;
    fm_sizes(ctx.get(), &nn, &ne, &n, &nnz);
    if (K.val.size() != nnz) throw Error(FM_ERR_ARG, "K does not hold this mesh's pattern");
    f_int.assign(n, 0.0);
    ctx.check(fm_assemble_host(ctx.get(), u, K.val.data(), f_int.data()), "fm_assemble_host");
}
template <class Mesh, class Prob, class CSR>
void assemble_global_threadlocal(const Mesh& mesh, const Prob& prob, const double* u, CSR& K,
                                 std::vector<double>& f_int) {
    assemble_global_threadlocal(default_context(), mesh, prob, u, K, f_int);
}

// assemble_global_residual_only (:990)
template <class Mesh, class Prob>
void assemble_global_residual_only(Context& ctx, const Mesh& mesh, const Prob& prob,
                                   const double* u, std::vector<double>& f_int) {
    set_mesh(ctx, mesh);
    ctx.check(fm_set_material(ctx.get(), prob.E, prob.nu, nullptr), "fm_set_material");
    uint32_t nn, ne, n;
    uint64_t nnz;
    fm_sizes(ctx.get(), &nn, &ne, &n, &nnz);
    f_int.assign(n, 0.0);
    ctx.check(fm_assemble_host(ctx.get(), u, nullptr, f_int.data()), "fm_assemble_host");
}
template <class Mesh, class Prob>
void assemble_global_residual_only(const Mesh& mesh, const Prob& prob, const double* u,
                                   std::vector<double>& f_int) {
    assemble_global_residual_only(default_context(), mesh, prob, u, f_int);
}

// pcg_solve_ilu0 (:1283): factorizes A on entry, x in/out, returns the
// iteration count (max_iter when not converged), same stop tests.
template <class CSR>
int pcg_solve_ilu0(Context& ctx, const CSR& A, const double* b, double* x, uint32_t N,
                   double tol = 1e-10, int max_iter = 1000) {
    int iters = 0;
    double rel = 0.0;
    ctx.check(fm_csr_pcg_ilu0(ctx.get(), N, A.row_ptr.data(), A.col_idx.data(), A.val.data(), b,
                              x, tol, max_iter, &iters, &rel),
              "fm_csr_pcg_ilu0");
    return iters;
}
template <class CSR>
int pcg_solve_ilu0(const CSR& A, const double* b, double* x, uint32_t N, double tol = 1e-10,
                   int max_iter = 1000) {
    return pcg_solve_ilu0(default_context(), A, b, x, N, tol, max_iter);
}

// ---------------------------------------------------------------------------
// material and Newton solver API (FEM/constitutive_models.hpp:30-52,
// FEM/nonlinear_solver.hpp:23-238)
// ---------------------------------------------------------------------------
struct NeoHookeanParameters {
    double E = 210e9;
    double nu = 0.3;
    double rho = 7850;
    double mu() const noexcept { return E / (2.0 * (1.0 + nu)); }
    double lambda() const noexcept { return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)); }
    double bulk_modulus() const noexcept { return E / (3.0 * (1.0 - 2.0 * nu)); }
};

struct NeoHookeanMaterial {
    explicit NeoHookeanMaterial(const NeoHookeanParameters& p = NeoHookeanParameters())
        : params(p) {}
    NeoHookeanParameters params;
};

struct LoadStep {
    double load_factor{1.0};
    std::array<double, 3> force{0.0, 0.0, 0.0};
    double magnitude{1.0};
    std::string description;
};

struct BoundaryConditions {
    std::vector<std::tuple<int, int, double>> dirichlet_bcs;  // (node, dof, value at full load)
    std::vector<std::tuple<int, double, double, double>> neumann_bcs;
};

struct NewtonSolverConfig {
    int max_iterations = 50;
    double tol_absolute = 1e-8;
    double tol_relative = 1e-6;
    int max_line_search = 10;
    double line_search_alpha = 1.0;
    double line_search_beta = 0.5;
    bool reuse_tangent = false;       // not used: the tangent is rebuilt every iteration
    bool verbose = true;
    double energy_convergence_tol = 1e-2;  // not used: the stop tests are on the residual
    // B200 additions
    double inner_tol = 1e-12;         // PCG tolerance of each Newton correction
    int max_pcg = 5000;
    fm_precision precision = FM_FP64;
    int ilu_every = 1;                // ILU(0) refactored every ilu_every solves
    int initial_guess = 0;            // FM_MIXED: PCG from the projected previous correction
};

struct NewtonSolverResult {
    bool converged = false;
    int num_iterations = 0;
    double final_residual_norm = 0;
    double final_residual_relative = 0;
    double final_energy_change = 0;
    int pcg_iterations = 0;
    std::vector<double> residual_history;   // ||R|| before each solve
    std::vector<double> step_size_history;  // alpha of each accepted step
    std::vector<double> energy_history;     // not computed (empty)
};

namespace detail {
// optional fields of a caller's config type (the reference's
// NewtonSolverConfig has none of the B200 additions)
template <class T, class = void>
struct has_inner_tol : std::false_type {};
template <class T>
struct has_inner_tol<T, std::void_t<decltype(std::declval<const T&>().inner_tol)>>
    : std::true_type {};
template <class T, class = void>
struct has_max_pcg : std::false_type {};
template <class T>
struct has_max_pcg<T, std::void_t<decltype(std::declval<const T&>().max_pcg)>>
    : std::true_type {};
template <class T, class = void>
struct has_precision : std::false_type {};
template <class T>
struct has_precision<T, std::void_t<decltype(std::declval<const T&>().precision)>>
    : std::true_type {};
template <class T, class = void>
struct has_ilu_every : std::false_type {};
template <class T>
struct has_ilu_every<T, std::void_t<decltype(std::declval<const T&>().ilu_every)>>
    : std::true_type {};
template <class T, class = void>
struct has_initial_guess : std::false_type {};
template <class T>
struct has_initial_guess<T, std::void_t<decltype(std::declval<const T&>().initial_guess)>>
    : std::true_type {};
}  // namespace detail

// NonlinearNewtonSolver with the engine's mathematics: element tangent and
// force of tet_element_stiffness_rigorous, CSR assembly, elimination BCs,
// ILU(0)-PCG corrections, Armijo backtracking on ||R|| with
// (1 - 0.1 alpha) and up to max_line_search trials, as the reference's
// solve() (:156-187).  The constrained DOFs of u are set to
// load.load_factor * value before the iterations.
// Mesh, Material, BCs, load and config are templates: the reference's own
// atlas::fem::MeshTopology, NeoHookeanMaterial (.params.E, .params.nu),
// BoundaryConditions (.dirichlet_bcs), LoadStep (.load_factor) and
// NewtonSolverConfig (max_iterations, tol_absolute, tol_relative,
// max_line_search) pass unchanged; the B200 fields of this header's
// NewtonSolverConfig (inner_tol, max_pcg, precision, ilu_every,
// initial_guess) are read where present.
template <class Mesh, class Material = NeoHookeanMaterial, class BCs = BoundaryConditions>
class NonlinearNewtonSolver {
public:
    NonlinearNewtonSolver(const Mesh& mesh, const Material& mat, const BCs& bcs,
                          Context* ctx = nullptr)
        : mesh_(mesh), material_(mat), bcs_(bcs), ctx_(ctx ? ctx : &default_context()) {}

    template <class Load, class Config = NewtonSolverConfig>
    NewtonSolverResult solve(std::vector<double>& u, const Load& load,
                             const Config& config = Config()) const {
        Context& ctx = *ctx_;
        set_mesh(ctx, mesh_);
        const size_t n = 3 * mesh_.nodes.size();
        if (u.size() != n) u.assign(n, 0.0);
        ctx.check(fm_set_material(ctx.get(), material_.params.E, material_.params.nu, nullptr),
                  "fm_set_material");
        std::vector<uint8_t> mask(n, 0);
        std::vector<double> value(n, 0.0);
        for (const auto& bc : bcs_.dirichlet_bcs) {
            const size_t d = 3 * (size_t)std::get<0>(bc) + (size_t)std::get<1>(bc);
            if (d >= n) throw Error(FM_ERR_ARG, "dirichlet dof out of range");
            mask[d] = 1;
            value[d] = std::get<2>(bc);
        }
        ctx.check(fm_set_bc(ctx.get(), mask.data(), value.data()), "fm_set_bc");
        fm_newton_config g;
        fm_newton_config_default(&g);
        g.newton_rtol = config.tol_relative;
        g.newton_atol = config.tol_absolute;
        g.max_newton = config.max_iterations;
        g.line_search = config.max_line_search > 0 ? config.max_line_search : 0;
        g.ls_c = 0.1;
        if constexpr (detail::has_inner_tol<Config>::value) g.inner_tol = config.inner_tol;
        if constexpr (detail::has_max_pcg<Config>::value) g.max_pcg = config.max_pcg;
        if constexpr (detail::has_precision<Config>::value) g.precision = config.precision;
        if constexpr (detail::has_ilu_every<Config>::value) g.ilu_every = config.ilu_every;
        if constexpr (detail::has_initial_guess<Config>::value)
            g.initial_guess = config.initial_guess;
        fm_newton_result res;
        const fm_status s = fm_newton_step_cfg_host(ctx.get(), u.data(), load.load_factor, &g,
                                                    &res);
        if (s != FM_OK && s != FM_ERR_NOT_CONVERGED) ctx.check(s, "fm_newton_step_cfg_host");
        NewtonSolverResult r;
        r.converged = s == FM_OK;
        r.num_iterations = res.newton_iters;
        r.final_residual_norm = res.rnorm;
        r.final_residual_relative = res.final_relres;
        r.pcg_iterations = res.pcg_iters;
        int cnt = 0;
        fm_newton_history(ctx.get(), nullptr, 0, &cnt);
        std::vector<fm_newton_record> h((size_t)cnt);
        if (cnt) fm_newton_history(ctx.get(), h.data(), cnt, &cnt);
        for (const auto& rec : h) {
            r.residual_history.push_back(rec.rnorm);
            if (rec.alpha > 0.0) r.step_size_history.push_back(rec.alpha);
        }
        return r;
    }

private:
    const Mesh& mesh_;
    const Material& material_;
    const BCs& bcs_;
    Context* ctx_;
};

}  // namespace flexmesh_b200
