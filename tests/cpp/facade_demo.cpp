// A reference-style caller of the C++ drop-in (include/flexmesh_b200.hpp):
// the small unit-cube problem (bottom clamped, top u_z = -0.1 in 5 load
// steps) through NonlinearNewtonSolver::solve, plus pcg_solve_ilu0 on the
// reference's 2-D Poisson validation matrix.  Writes u and the PCG result
// to the file given as argv[1] (raw doubles) for the test to compare.
#include <cmath>
#include <cstdio>
#include <vector>

#include "flexmesh_b200.hpp"

namespace fb = flexmesh_b200;

struct Node {
    double x, y, z;
};
struct Tet {
    std::array<uint32_t, 4> nodes;
    double volume;
};
struct Mesh {
    std::vector<Node> nodes;
    std::vector<Tet> elements;
};
struct CSR {
    uint32_t n_rows = 0;
    std::vector<uint32_t> row_ptr, col_idx;
    std::vector<double> val;
};

int main(int argc, char** argv) {
    const int N = argc > 2 ? std::atoi(argv[2]) : 4;
    std::vector<double> xyz;
    std::vector<uint32_t> conn;
    fb::generate_unit_cube(N, xyz, conn);
    Mesh mesh;
    for (size_t n = 0; n < xyz.size() / 3; ++n) mesh.nodes.push_back({xyz[3 * n], xyz[3 * n + 1], xyz[3 * n + 2]});
    for (size_t e = 0; e < conn.size() / 4; ++e) {
        Tet t;
        for (int v = 0; v < 4; ++v) t.nodes[v] = conn[4 * e + v];
        const Node &a = mesh.nodes[t.nodes[0]], &b = mesh.nodes[t.nodes[1]],
                   &c = mesh.nodes[t.nodes[2]], &d = mesh.nodes[t.nodes[3]];
        const double u0 = b.x - a.x, u1 = b.y - a.y, u2 = b.z - a.z;
        const double v0 = c.x - a.x, v1 = c.y - a.y, v2 = c.z - a.z;
        const double w0 = d.x - a.x, w1 = d.y - a.y, w2 = d.z - a.z;
        t.volume = std::fabs(u0 * (v1 * w2 - v2 * w1) - u1 * (v0 * w2 - v2 * w0) +
                             u2 * (v0 * w1 - v1 * w0)) / 6.0;
        mesh.elements.push_back(t);
    }
    fb::BoundaryConditions bcs;
    for (size_t n = 0; n < mesh.nodes.size(); ++n) {
        if (mesh.nodes[n].z < 1e-12)
            for (int d = 0; d < 3; ++d) bcs.dirichlet_bcs.emplace_back((int)n, d, 0.0);
        else if (mesh.nodes[n].z > 1.0 - 1e-12)
            bcs.dirichlet_bcs.emplace_back((int)n, 2, -0.1);
    }
    fb::NeoHookeanParameters p;
    p.E = 1.0;
    p.nu = 0.3;
    fb::NeoHookeanMaterial mat(p);
    fb::NonlinearNewtonSolver<Mesh> solver(mesh, mat, bcs);
    fb::NewtonSolverConfig cfg;
    cfg.tol_absolute = 0.0;
    cfg.tol_relative = 1e-10;
    cfg.max_iterations = 200;
    cfg.max_line_search = 0;
    std::vector<double> u(3 * mesh.nodes.size(), 0.0);
    int newton = 0;
    for (int s = 1; s <= 5; ++s) {
        fb::LoadStep load;
        load.load_factor = s / 5.0;
        fb::NewtonSolverResult r = solver.solve(u, load, cfg);
        if (!r.converged) {
            std::fprintf(stderr, "load step %d did not converge\n", s);
            return 2;
        }
        newton += r.num_iterations;
    }
    // pcg_solve_ilu0 on the 2-D Poisson matrix (diagonal first, as the
    // reference's validation runner builds it)
    const uint32_t g = 16, n = g * g;
    const double h = 1.0 / (g + 1), ih2 = 1.0 / (h * h);
    CSR A;
    A.n_rows = n;
    A.row_ptr.push_back(0);
    std::vector<double> xe(n), b(n, 0.0), x(n, 0.0);
    for (uint32_t i = 0; i < g; ++i)
        for (uint32_t j = 0; j < g; ++j) {
            const uint32_t row = i * g + j;
            xe[row] = std::sin(3.14159265358979323846 * (i + 1) * h) *
                      std::sin(3.14159265358979323846 * (j + 1) * h);
            A.col_idx.push_back(row);
            A.val.push_back(4.0 * ih2);
            if (i > 0) { A.col_idx.push_back(row - g); A.val.push_back(-ih2); }
            if (i + 1 < g) { A.col_idx.push_back(row + g); A.val.push_back(-ih2); }
            if (j > 0) { A.col_idx.push_back(row - 1); A.val.push_back(-ih2); }
            if (j + 1 < g) { A.col_idx.push_back(row + 1); A.val.push_back(-ih2); }
            A.row_ptr.push_back((uint32_t)A.col_idx.size());
        }
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t k = A.row_ptr[i]; k < A.row_ptr[i + 1]; ++k) b[i] += A.val[k] * xe[A.col_idx[k]];
    const int its = fb::pcg_solve_ilu0(A, b.data(), x.data(), n, 1e-10, 4000);
    double err = 0.0, nrm = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        err += (x[i] - xe[i]) * (x[i] - xe[i]);
        nrm += xe[i] * xe[i];
    }
    FILE* f = std::fopen(argv[1], "wb");
    std::fwrite(u.data(), sizeof(double), u.size(), f);
    const double meta[3] = {(double)newton, (double)its, std::sqrt(err / nrm)};
    std::fwrite(meta, sizeof(double), 3, f);
    std::fclose(f);
    std::printf("facade ok: newton %d pcg %d poisson rel err %.3e\n", newton, its, std::sqrt(err / nrm));
    return 0;
}
