// A caller written against the reference's own types, switched to the B200
// path by swapping the namespace of the calls: atlas::fem::MeshTopology
// from the reference's generate_unit_cube_mesh, its BoundaryConditions,
// NeoHookeanMaterial, LoadStep, NewtonSolverConfig, SparseCSR and
// ProblemDescriptor go unchanged into flexmesh_b200::NonlinearNewtonSolver,
// build_csr_sparsity_pattern_rigorous, assemble_global_threadlocal and
// pcg_solve_ilu0.  The same assembly and PCG are also run through the
// reference's own functions on the CPU for comparison.
//
// Built by oracle/Makefile (target refdemo) against the reference headers
// into oracle/_ref/ref_types_demo.  Usage: ref_types_demo <out.bin> [N]
// Writes u (3 Nn doubles) followed by: total Newton iterations, max
// relative K and f difference against the reference's assembly, PCG
// iterations (B200, reference) and max relative x difference.
#include "fem/nonlinear_solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "flexmesh_b200.hpp"

namespace af = atlas::fem;
namespace fb = flexmesh_b200;

static double max_rel(const std::vector<double>& a, const std::vector<double>& b) {
    double d = 0.0, s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) {
        d = std::max(d, std::fabs(a[i] - b[i]));
        s = std::max(s, std::fabs(b[i]));
    }
    return s > 0 ? d / s : d;
}

int main(int argc, char** argv) {
    if (argc < 2) return 1;
    const int N = argc > 2 ? std::atoi(argv[2]) : 4;
    const af::MeshTopology mesh = af::generate_unit_cube_mesh(N);
    af::BoundaryConditions bcs;
    for (size_t n = 0; n < mesh.nodes.size(); ++n) {
        if (mesh.nodes[n].z < 1e-12)
            for (int d = 0; d < 3; ++d) bcs.dirichlet_bcs.emplace_back((int)n, d, 0.0);
        else if (mesh.nodes[n].z > 1.0 - 1e-12)
            bcs.dirichlet_bcs.emplace_back((int)n, 2, -0.1);
    }
    af::NeoHookeanParameters p;
    p.E = 1.0;
    p.nu = 0.3;
    const af::NeoHookeanMaterial mat(p);
    af::NewtonSolverConfig cfg;
    cfg.tol_relative = 1e-10;
    cfg.tol_absolute = 0.0;
    cfg.max_iterations = 200;
    cfg.max_line_search = 10;
    cfg.verbose = false;

    fb::Context ctx(0);
    fb::NonlinearNewtonSolver<af::MeshTopology, af::NeoHookeanMaterial, af::BoundaryConditions>
        solver(mesh, mat, bcs, &ctx);
    af::Solution u(3 * mesh.nodes.size(), 0.0);
    int newton = 0;
    for (int s = 1; s <= 5; ++s) {
        af::LoadStep load;
        load.load_factor = s / 5.0;
        const auto r = solver.solve(u, load, cfg);
        newton += r.num_iterations;
        if (!r.converged) {
            std::fprintf(stderr, "load step %d did not converge\n", s);
            return 2;
        }
    }

    // free functions on the reference's SparseCSR / ProblemDescriptor, at u
    af::SparseCSR K;
    fb::build_csr_sparsity_pattern_rigorous(ctx, mesh, K);
    af::ProblemDescriptor prob;
    prob.E = 1.0;
    prob.nu = 0.3;
    std::vector<double> f;
    fb::assemble_global_threadlocal(ctx, mesh, prob, u.data(), K, f);
    af::SparseCSR Kr = K;
    std::vector<double> fr;
    af::assemble_global_threadlocal(mesh, prob, u.data(), Kr, fr);
    const double dK = max_rel(K.val, Kr.val), df = max_rel(f, fr);

    // PCG-ILU(0) on the assembled K with the Dirichlet DOFs eliminated
    // (zero rows and columns, unit diagonal) and a unit right-hand side on
    // the free DOFs
    const uint32_t n = K.n_rows;
    std::vector<char> fixed(n, 0);
    for (const auto& bc : bcs.dirichlet_bcs) fixed[3 * std::get<0>(bc) + std::get<1>(bc)] = 1;
    for (af::SparseCSR* A : {&K, &Kr})
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k)
                if (fixed[i] || fixed[A->col_idx[k]]) A->val[k] = (A->col_idx[k] == i) ? 1.0 : 0.0;
    std::vector<double> b(n, 1.0), x(n, 0.0), xr(n, 0.0);
    for (uint32_t i = 0; i < n; ++i)
        if (fixed[i]) b[i] = 0.0;
    const int it = fb::pcg_solve_ilu0(ctx, K, b.data(), x.data(), n, 1e-10, 2000);
    const int itr = af::pcg_solve_ilu0(Kr, b.data(), xr.data(), n, 1e-10, 2000);
    const double dx = max_rel(x, xr);

    FILE* fo = std::fopen(argv[1], "wb");
    if (!fo) return 3;
    std::fwrite(u.data(), sizeof(double), u.size(), fo);
    const double meta[6] = {(double)newton, dK, df, (double)it, (double)itr, dx};
    std::fwrite(meta, sizeof(double), 6, fo);
    std::fclose(fo);
    std::printf("newton %d dK %.3e df %.3e pcg %d/%d dx %.3e\n", newton, dK, df, it, itr, dx);
    return 0;
}
