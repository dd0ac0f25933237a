// fm_kernels.hpp — host launchers of the FlexMesh sm_100a kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fm_device.cuh"

namespace fm {

// Mesh/material data resident on the device (read by assembly kernels).
struct MeshDev {
    uint32_t n_nodes = 0, n_elems = 0;
    const double* xyz = nullptr;       // 3*n_nodes
    const uint4* conn = nullptr;       // n_elems, bit 31 of .x = element skipped
    const uint32_t* nbr_ptr = nullptr; // n_nodes+1
    const uint32_t* nbr = nullptr;     // node neighbours, sorted
    const uint32_t* inc_ptr = nullptr; // n_nodes+1
    const uint32_t* inc = nullptr;     // incident elements, ascending
    const uint8_t* mask = nullptr;     // n_dofs Dirichlet mask (may be null)
    // material: mode 0 scalar (mu_s, lam_s), 1 per-element E (m0) with
    // mu = E c_mu, lam = E c_lam, 2 per-element Lame (m0 = mu, m1 = lam)
    int mat_mode = 0;
    const double* m0 = nullptr;
    const double* m1 = nullptr;
    double mu_s = 0, lam_s = 0, c_mu = 0, c_lam = 0, inv_cnu = 0;
    // per-element records of the assembly's element pass (n_elems *
    // kElemRecBytes bytes, 16-byte aligned)
    void* elem_rec = nullptr;
    // structural scatter data of the node pass, built once per mesh:
    // inc_pos[i]: positions (4 x u8) of incidence i's tet vertices in the
    // owner's neighbour list; nbr_members[j]: bit l set when the owner's
    // l-th incident tet (not skipped) holds the edge to neighbour entry j
    const uint32_t* inc_pos = nullptr;
    const uint32_t* nbr_members = nullptr;
};
constexpr size_t kElemRecBytes = 224;


// A10/A11/A12: assembly in two passes, an element pass (each tet's
// kinematics, stress, vertex forces and tangent scalars, once) and a
// node-owner pass that writes every CSR row block once.  K (double or float,
// may be null for a residual-only call), f (FP64, may be null), R = -f with
// zeros on constrained DOFs (may be null).  m.elem_rec is required.
void launch_assemble(const MeshDev& m, const double* u, double* K, double* f, double* R,
                     int apply_bc, unsigned* status, cudaStream_t s);
void launch_assemble(const MeshDev& m, const double* u, float* K, double* f, double* R,
                     int apply_bc, unsigned* status, cudaStream_t s);
// Element-centric scatter through an int32 slot map (reference pattern).
// K and f must be zeroed by the caller; Ke_scratch holds 144*n_elems doubles.
void launch_assemble_slotmap(const MeshDev& m, const double* u, const int32_t* slot, double* K,
                             double* f, double* Ke_scratch, unsigned* status, cudaStream_t s);
// Batched element kernel (full 12x12 + 12 per element)
void launch_elements(uint32_t n, const double* x, const double* u, const double* E, double nu,
                     double* K, double* f, unsigned* status, cudaStream_t s);

// SpMV on the node-block solve pattern (y = A x); with dot != null also
// finishes dot(x, y) into *dot through the deterministic grid reduction.
template <typename T>
void launch_spmv_nodes(uint32_t n_nodes, const uint32_t* nbr_ptr, const uint32_t* nbr,
                       const T* val, const T* x, T* y, T* partials, unsigned* counter,
                       double* dot, cudaStream_t s);
// Generic scalar CSR SpMV (ascending or any column order)
template <typename T>
void launch_spmv_csr(uint32_t n, const uint32_t* rp, const uint32_t* ci, const T* val, const T* x,
                     T* y, T* partials, unsigned* counter, double* dot, cudaStream_t s);

// Sync-free ILU(0) and triangular solves on a CSR with ascending columns.
// order: a topological order of the rows (dependency levels); done: one
// flag per row, released with the given epoch.
struct CsrDev {
    uint32_t n = 0;
    const uint32_t* rp = nullptr;
    const uint32_t* ci = nullptr;
    const uint32_t* dpos = nullptr;   // index of the first column >= row (diag slot if present)
    const uint32_t* upos = nullptr;   // index of the first column > row
    const uint32_t* fwd_order = nullptr;
    const uint32_t* bwd_order = nullptr;
    uint32_t max_row = 0;
};
template <typename T>
void launch_ilu0_csr(const CsrDev& A, const T* a_val, T* lu, T* diag, unsigned* done,
                     unsigned epoch, unsigned* status, int grid, cudaStream_t s);
template <typename T>
void launch_trsv_lower_csr(const CsrDev& A, const T* lu, const T* r, T* z, unsigned* done,
                           unsigned epoch, unsigned* status, int grid, cudaStream_t s);
template <typename T>
void launch_trsv_upper_csr(const CsrDev& A, const T* lu, const T* diag, const T* z, T* y,
                           unsigned* done, unsigned epoch, unsigned* status, int grid,
                           cudaStream_t s);
// persistent grid sizes (all blocks co-resident) for the sync-free kernels
int persistent_grid_ilu0_csr(int device, bool fp32, const CsrDev& A);
int persistent_grid_trsv_csr(int device, bool fp32);

// PCG vector kernels; all reductions deterministic (fixed grid kRedBlocks).
template <typename T>
void launch_dot(uint32_t n, const T* x, const T* y, T* partials, unsigned* counter, double* out,
                cudaStream_t s);
// r = b - r (r holds A x on entry); *rr = r.r
template <typename T>
void launch_residual_init(uint32_t n, const T* b, T* r, T* partials, unsigned* counter,
                          double* rr, cudaStream_t s);
// p = z; rz = r.z; bb = b.b (both into sc)
template <typename T>
void launch_pcg_start(uint32_t n, const T* r, const T* z, const T* b, T* p, T* partials,
                      unsigned* counter, DevScalars* sc, cudaStream_t s);
// alpha = rz/pAp; x += alpha p; r -= alpha Ap
template <typename T>
void launch_pcg_update_xr(uint32_t n, const T* p, const T* Ap, T* x, T* r, DevScalars* sc,
                          cudaStream_t s);
// rz_new = r.z; relres = sqrt(rz_new / max(bb,1e-300))
template <typename T>
void launch_pcg_rz(uint32_t n, const T* r, const T* z, T* partials, unsigned* counter,
                   DevScalars* sc, cudaStream_t s);
// beta = rz_new/rz; p = z + beta p; rz = rz_new (rotation done by thread 0
// of the grid after all blocks read rz: see kernel)
template <typename T>
void launch_pcg_update_p(uint32_t n, const T* z, T* p, DevScalars* sc, cudaStream_t s);

// Newton helpers
void launch_set_bc_values(uint32_t n, const uint8_t* mask, const double* val, double frac,
                          double* u, cudaStream_t s);
// free-DOF squared norm of R into *out
void launch_norm2(uint32_t n, const double* R, double* partials, unsigned* counter, double* out,
                  cudaStream_t s);
// b32 = R * inv_scale (FP32), x32 = 0 (x32 nullable)
void launch_to_f32_scaled(uint32_t n, const double* R, double inv_scale, float* b32, float* x32,
                          cudaStream_t s);
// x *= g
void launch_scale_f32(uint32_t n, float* x, float g, cudaStream_t s);
// u += du (FP64)
void launch_axpy_u(uint32_t n, const double* du, double* u, cudaStream_t s);
// u += scale * du32
void launch_axpy_u_f32(uint32_t n, const float* du, double scale, double* u, cudaStream_t s);
// load-step predictor pieces
void launch_bc_increment(uint32_t n, const uint8_t* mask, const double* val, double frac,
                         const double* u, double* v, float* v32, double* partials,
                         unsigned* counter, double* out, cudaStream_t s);
template <typename T>
void launch_predictor_rhs(uint32_t n, const uint8_t* mask, const double* f, const T* Kv,
                          double* R, cudaStream_t s);
template <typename T>
void launch_apply_bc_nodes(uint32_t nn, const uint32_t* nbr_ptr, const uint32_t* nbr,
                           const uint8_t* mask, T* K, cudaStream_t s);
// y = scale * x (FP32 -> FP64)
void launch_f32_to_f64_scaled(uint32_t n, const float* x, double scale, double* y,
                              cudaStream_t s);
// Element state update (fm_states.cu): per element F_sl3 (9, the
// reference's column-major Matrix3x3 data) and Mandel stress (6); elements
// with a degenerate reference Jacobian keep their previous state.
// counts[0] += tets with |det F_sl3 - 1| > 1e-8, counts[1] += tets whose
// state is not finite.
void launch_element_states(const MeshDev& m, const double* u, double nu, double* F,
                           double* stress, unsigned* counts, cudaStream_t s);
// one warp waits (bounded by the limit that travels with status) for *flag
// to reach epoch 1; nothing sets it, so the wait times out
void launch_wait_probe(const unsigned* flag, unsigned* status, cudaStream_t s);
// y = u + alpha du (line-search trial point)
void launch_trial(uint32_t n, const double* u, double alpha, const double* du, double* y,
                  cudaStream_t s);

}  // namespace fm
