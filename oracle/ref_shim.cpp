// ref_shim.cpp — C entry points over the reference's own headers
// (TEST INFRASTRUCTURE).  Built by oracle/Makefile into oracle/_ref/ from
// the reference sources where they lie; nothing of the reference is copied.
// Used only to pin the C oracle and to generate golden fixtures, and as the
// reference-kind CPU baseline.  Every function calls the reference's code
// unchanged; the only code here is marshalling between flat arrays and the
// reference's MeshTopology / SparseCSR containers.
#include "fem/adaptive_fem_engine.hpp"

#include <omp.h>

#include <cstdint>
#include <cstring>
#include <vector>

using namespace atlas::fem;

namespace {
struct RefMesh {
    MeshTopology mesh;
};

MeshTopology mesh_from_arrays(uint32_t n_nodes, const double* xyz, uint32_t n_elems,
                              const uint32_t* conn, const double* vol) {
    MeshTopology m;
    m.nodes.resize(n_nodes);
    for (uint32_t n = 0; n < n_nodes; ++n) {
        m.nodes[n].x = xyz[3 * n];
        m.nodes[n].y = xyz[3 * n + 1];
        m.nodes[n].z = xyz[3 * n + 2];
        m.nodes[n].id = n;
    }
    m.elements.resize(n_elems);
    m.states.resize(n_elems);
    for (uint32_t e = 0; e < n_elems; ++e) {
        for (int v = 0; v < 4; ++v) m.elements[e].nodes[v] = conn[4 * (size_t)e + v];
        m.elements[e].volume = vol[e];
        m.elements[e].id = e;
    }
    m.n_dofs = 3 * n_nodes;
    return m;
}

SparseCSR csr_from_arrays(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                          const double* val) {
    SparseCSR A;
    A.n_rows = n;
    A.row_ptr.assign(row_ptr, row_ptr + n + 1);
    A.col_idx.assign(col_idx, col_idx + row_ptr[n]);
    if (val) A.val.assign(val, val + row_ptr[n]);
    else A.val.assign(row_ptr[n], 0.0);
    return A;
}
}  // namespace

extern "C" {

// generate_unit_cube_mesh (FEM/adaptive_fem_engine.hpp:2219)
void* ref_mesh_new(int N) {
    auto* h = new RefMesh;
    h->mesh = generate_unit_cube_mesh(N);
    return h;
}
void ref_mesh_free(void* h) { delete static_cast<RefMesh*>(h); }
void ref_mesh_sizes(void* h, uint32_t* n_nodes, uint32_t* n_elems, uint32_t* n2e_len) {
    auto& m = static_cast<RefMesh*>(h)->mesh;
    *n_nodes = (uint32_t)m.n_nodes();
    *n_elems = (uint32_t)m.n_elements();
    *n2e_len = (uint32_t)m.node_to_elem_data.size();
}
void ref_mesh_get(void* h, double* xyz, uint32_t* conn, double* vol, uint32_t* n2e_ptr,
                  uint32_t* n2e) {
    auto& m = static_cast<RefMesh*>(h)->mesh;
    for (size_t n = 0; n < m.n_nodes(); ++n) {
        xyz[3 * n] = m.nodes[n].x;
        xyz[3 * n + 1] = m.nodes[n].y;
        xyz[3 * n + 2] = m.nodes[n].z;
    }
    for (size_t e = 0; e < m.n_elements(); ++e) {
        for (int v = 0; v < 4; ++v) conn[4 * e + v] = m.elements[e].nodes[v];
        vol[e] = m.elements[e].volume;
    }
    std::memcpy(n2e_ptr, m.node_to_elem_ptr.data(), sizeof(uint32_t) * m.node_to_elem_ptr.size());
    std::memcpy(n2e, m.node_to_elem_data.data(), sizeof(uint32_t) * m.node_to_elem_data.size());
}

// tet_volume (FEM/mesh_adaptation.hpp:123)
double ref_tet_volume(const double* a, const double* b, const double* c, const double* d) {
    MeshNode n[4];
    const double* p[4] = {a, b, c, d};
    for (int q = 0; q < 4; ++q) {
        n[q].x = p[q][0];
        n[q].y = p[q][1];
        n[q].z = p[q][2];
    }
    return tet_volume(n[0], n[1], n[2], n[3]);
}

// build_csr_sparsity_pattern_rigorous (:1069) on an arbitrary mesh
uint64_t ref_pattern(uint32_t n_nodes, const double* xyz, uint32_t n_elems, const uint32_t* conn,
                     uint32_t* row_ptr, uint32_t* col_idx) {
    std::vector<double> vol(n_elems, 1.0);
    MeshTopology m = mesh_from_arrays(n_nodes, xyz, n_elems, conn, vol.data());
    SparseCSR K;
    build_csr_sparsity_pattern_rigorous(m, K);
    if (row_ptr) std::memcpy(row_ptr, K.row_ptr.data(), sizeof(uint32_t) * K.row_ptr.size());
    if (col_idx) std::memcpy(col_idx, K.col_idx.data(), sizeof(uint32_t) * K.col_idx.size());
    return K.row_ptr.back();
}

// tet_element_stiffness_rigorous (:511)
void ref_element(const double* x12, const double* u12, double E, double nu, double* K144,
                 double* f12) {
    MeshNode n[4];
    for (int q = 0; q < 4; ++q) {
        n[q].x = x12[3 * q];
        n[q].y = x12[3 * q + 1];
        n[q].z = x12[3 * q + 2];
    }
    ElementState st;
    tet_element_stiffness_rigorous(n, u12, st, E, nu, K144, f12);
}

// assemble_global_threadlocal (:1126) with the given thread count; the
// CSR pattern is the caller's (reference or solve pattern).
void ref_assemble(uint32_t n_nodes, const double* xyz, uint32_t n_elems, const uint32_t* conn,
                  const double* vol, double E, double nu, const double* u, const uint32_t* row_ptr,
                  const uint32_t* col_idx, double* K_val, double* f_int, int threads) {
    MeshTopology m = mesh_from_arrays(n_nodes, xyz, n_elems, conn, vol);
    ProblemDescriptor prob;
    prob.E = E;
    prob.nu = nu;
    SparseCSR K = csr_from_arrays(3 * n_nodes, row_ptr, col_idx, nullptr);
    std::vector<double> f;
    omp_set_num_threads(threads);
    assemble_global_threadlocal(m, prob, u, K, f);
    std::memcpy(K_val, K.val.data(), sizeof(double) * K.val.size());
    std::memcpy(f_int, f.data(), sizeof(double) * f.size());
}

// assemble_global_residual_only (:990)
void ref_residual(uint32_t n_nodes, const double* xyz, uint32_t n_elems, const uint32_t* conn,
                  const double* vol, double E, double nu, const double* u, double* f_int,
                  int threads) {
    MeshTopology m = mesh_from_arrays(n_nodes, xyz, n_elems, conn, vol);
    ProblemDescriptor prob;
    prob.E = E;
    prob.nu = nu;
    std::vector<double> f;
    omp_set_num_threads(threads);
    assemble_global_residual_only(m, prob, u, f);
    std::memcpy(f_int, f.data(), sizeof(double) * f.size());
}

// Timing-only helper for per-element E: the reference element kernel
// (:511) driven through a slot-map scatter in element order (the
// reference's threadlocal assembly takes one scalar E per problem).
void ref_assemble_slotmap(uint32_t n_nodes, const double* xyz, uint32_t n_elems,
                          const uint32_t* conn, const double* vol, const double* E_elem, double nu,
                          const double* u, const int32_t* slot, uint64_t nnz, double* K_val,
                          double* f_int) {
    std::memset(K_val, 0, sizeof(double) * nnz);
    std::memset(f_int, 0, sizeof(double) * 3 * (size_t)n_nodes);
    ElementState st;
    for (uint32_t e = 0; e < n_elems; ++e) {
        if (vol[e] < 1e-30) continue;
        MeshNode n[4];
        double ue[12];
        for (int a = 0; a < 4; ++a) {
            uint32_t id = conn[4 * (size_t)e + a];
            n[a].x = xyz[3 * id];
            n[a].y = xyz[3 * id + 1];
            n[a].z = xyz[3 * id + 2];
            for (int d = 0; d < 3; ++d) ue[3 * a + d] = u[3 * (size_t)id + d];
        }
        double Ke[144], fe[12];
        tet_element_stiffness_rigorous(n, ue, st, E_elem[e], nu, Ke, fe);
        const int32_t* s = slot + 144 * (size_t)e;
        for (int q = 0; q < 144; ++q)
            if (s[q] >= 0) K_val[s[q]] += Ke[q];
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) f_int[3 * (size_t)conn[4 * (size_t)e + a] + d] += fe[3 * a + d];
    }
}

// ILU0Preconditioner::factorize (:305); O(n^2), small n only.
// Writes L_val/U_val (full nnz copies as the reference keeps them), diag
// and the reference's level array; returns max_level.
int ref_ilu0(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* val,
             double* L_val, double* U_val, double* diag, int* level) {
    SparseCSR A = csr_from_arrays(n, row_ptr, col_idx, val);
    auto f = ILU0Preconditioner::factorize(A);
    std::memcpy(L_val, f.L_val.data(), sizeof(double) * f.L_val.size());
    std::memcpy(U_val, f.U_val.data(), sizeof(double) * f.U_val.size());
    std::memcpy(diag, f.diag.data(), sizeof(double) * n);
    if (level) std::memcpy(level, f.symbolic.level.data(), sizeof(int) * n);
    return f.max_level;
}

// factorize + ILU0Preconditioner::solve (:473)
void ref_ilu0_solve(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                    const double* val, const double* r, double* y) {
    SparseCSR A = csr_from_arrays(n, row_ptr, col_idx, val);
    auto f = ILU0Preconditioner::factorize(A);
    ILU0Preconditioner::solve(f, r, y, n);
}

// pcg_solve_ilu0 (:1283)
int ref_pcg_ilu0(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* val,
                 const double* b, double* x, double tol, int max_iter, int threads) {
    SparseCSR A = csr_from_arrays(n, row_ptr, col_idx, val);
    omp_set_num_threads(threads);
    return pcg_solve_ilu0(A, b, x, n, tol, max_iter);
}

// SparseCSR::matvec (FEM/fem_types.hpp:310)
void ref_spmv(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* val,
              const double* x, double* y) {
    SparseCSR A = csr_from_arrays(n, row_ptr, col_idx, val);
    A.matvec(x, y);
}

// MeshColoring::compute (:1554), O(E^2): small meshes only
uint32_t ref_mesh_coloring(uint32_t n_nodes, const double* xyz, uint32_t n_elems,
                           const uint32_t* conn, const double* vol, uint32_t* colors) {
    MeshTopology m = mesh_from_arrays(n_nodes, xyz, n_elems, conn, vol);
    const MeshColoring mc = MeshColoring::compute(m);
    std::memcpy(colors, mc.element_colors.data(), sizeof(uint32_t) * n_elems);
    return mc.n_colors;
}

// sl3_retraction(G, 0) (CORE/lie_operator.cpp:300) on a Matrix3x3 whose
// data array is G9
void ref_sl3_retraction(const double* G9, double* out9) {
    atlas::Matrix3x3 G;
    for (int i = 0; i < 9; ++i) G.data[i] = G9[i];
    const atlas::Matrix3x3 R = atlas::sl3_retraction(G, atlas::Matrix3x3::zero());
    for (int i = 0; i < 9; ++i) out9[i] = R.data[i];
}

// neo_hookean_response (:79) with the J given
void ref_nh_response(const double* F9, double E, double nu, double J, double* sig6) {
    neo_hookean_response(F9, E, nu, sig6, J);
}

// CheckpointFile::save (:1350) of the reference's own unit cube N with the
// given solution (also copied into MeshNode::u, v, w) and states F/stress
// (nullable: the ElementState defaults)
int ref_checkpoint_save(const char* path, int N, const double* u, const double* F,
                        const double* stress, uint32_t load_step, uint32_t adapt_iter) {
    MeshTopology mesh = generate_unit_cube_mesh(N);
    std::vector<double> uu(u, u + mesh.n_dofs);
    for (size_t n = 0; n < mesh.nodes.size(); ++n) {
        mesh.nodes[n].u = u[3 * n];
        mesh.nodes[n].v = u[3 * n + 1];
        mesh.nodes[n].w = u[3 * n + 2];
    }
    for (size_t e = 0; e < mesh.states.size(); ++e) {
        if (F) std::memcpy(mesh.states[e].F_data, F + 9 * e, sizeof(double) * 9);
        if (stress) std::memcpy(mesh.states[e].stress, stress + 6 * e, sizeof(double) * 6);
    }
    return CheckpointFile::save(path, mesh, uu, load_step, adapt_iter) ? 0 : 1;
}

// CheckpointFile::load (:1402): sizes, the solution, and the states
int ref_checkpoint_load(const char* path, uint32_t* n_nodes, uint32_t* n_elems, uint32_t* n_dofs,
                        uint32_t* load_step, uint32_t* adapt_iter, double* u_out, double* F_out,
                        double* stress_out, uint32_t cap_dofs, uint32_t cap_elems) {
    MeshTopology mesh;
    std::vector<double> u;
    if (!CheckpointFile::load(path, mesh, u, *load_step, *adapt_iter)) return 1;
    *n_nodes = (uint32_t)mesh.nodes.size();
    *n_elems = (uint32_t)mesh.elements.size();
    *n_dofs = mesh.n_dofs;
    if (u.size() <= cap_dofs && u_out) std::memcpy(u_out, u.data(), sizeof(double) * u.size());
    if (mesh.states.size() <= cap_elems)
        for (size_t e = 0; e < mesh.states.size(); ++e) {
            if (F_out) std::memcpy(F_out + 9 * e, mesh.states[e].F_data, sizeof(double) * 9);
            if (stress_out) std::memcpy(stress_out + 6 * e, mesh.states[e].stress, sizeof(double) * 6);
        }
    return 0;
}

}  // extern "C"
