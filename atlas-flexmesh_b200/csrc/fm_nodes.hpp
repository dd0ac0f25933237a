// fm_nodes.hpp — node-block ILU(0) / triangular-solve schedule and launchers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fm {

// Topological orders of the mesh nodes for the factorization/forward solve
// (fwd: node level = 1 + max level of its lower neighbours) and the
// backward solve (bwd: from the top), plus the widest level of each, which
// sizes the persistent grids.
struct NodeSched {
    uint32_t n_nodes = 0;
    const uint32_t* nbr_ptr = nullptr;
    const uint32_t* nbr = nullptr;
    const uint32_t* self_pos = nullptr;  // index of n inside its own neighbour list
    const uint32_t* fwd_order = nullptr;
    const uint32_t* bwd_order = nullptr;
    // per position of the orders: {node, nbr_ptr[node], degree, self_pos[node]}
    const uint4* fwd_rec = nullptr;
    const uint4* bwd_rec = nullptr;
    uint32_t max_width_fwd = 0, max_width_bwd = 0;
    // ILU(0) update map (fm_setup.cpp ilu_edge_maps): per node offset, entries
    const uint32_t* emap_ptr = nullptr;
    const uint8_t* emap = nullptr;
};

// y = U^-1 L^-1 r using tmp for the intermediate (both overwritten);
// dinv holds the reciprocal pivots written by the factorization
template <typename T>
void launch_trsv_nodes(const NodeSched& S, const T* lu, const T* dinv, const T* r, T* tmp, T* y,
                       unsigned* status, int device, cudaStream_t s);
// LU (nnz entries, a_ii kept on diagonal slots), pivots d and their
// reciprocals dinv (three kernels: LU and dinv filled with the wait
// sentinel, then the factorization)
template <typename T>
void launch_ilu0_nodes(const NodeSched& S, const T* a, T* lu, uint64_t nnz, T* d, T* dinv,
                       unsigned* status, int device, cudaStream_t s);
template <typename T>
void launch_fill_sentinel(uint32_t n, T* x, cudaStream_t s);

// Slab-partitioned push solves (fm_trsv_push.cu) on the plan of
// fm_setup.cpp push_plan: CTA g of the grid (clusters of `cluster` CTAs)
// walks positions pos_*[g] .. pos_*[g+1] of rec_* ({node, first neighbour
// entry, degree, self position}; node ~0u: a hole), half-warp v every
// (2 warps)-th of them from the v-th.
struct PushSolve {
    uint32_t n_ctas = 0, cluster = 0, warps32 = 0, warps64 = 0;  // warps per CTA
    uint32_t max_slot_f = 0, max_slot_b = 0;
    const uint32_t* pos_f = nullptr;
    const uint32_t* pos_b = nullptr;
    const uint4* rec_f = nullptr;
    const uint4* rec_b = nullptr;
    const uint32_t* src = nullptr;     // per neighbour entry: reader-side slot or ~0u
    const uint32_t* push_f = nullptr;  // 8 per node: rank << 20 | slot, ~0u after the last
    const uint32_t* push_b = nullptr;
    const uint32_t* nslot_f = nullptr;  // slots per CTA
    const uint32_t* nslot_b = nullptr;
};
// most warps per CTA of the push kernels of this value width (register budget)
constexpr int push_max_warps(size_t value_bytes) { return value_bytes == 4 ? 32 : 16; }
// dynamic shared memory of one CTA of a direction with max_slot slots
size_t push_smem_bytes(uint32_t max_slot, size_t value_bytes);
// clusters of `cluster` CTAs (warps each, smem bytes) that can be resident
// at once for both directions' kernels of this value width (0: none)
int push_max_clusters(size_t value_bytes, int cluster, int warps, size_t smem);
// y = U^-1 L^-1 r through tmp (three kernels: tmp's sentinel fill, the
// forward solve, which also fills y unless y aliases r, and the backward);
// returns the first launch error, with nothing left half-done on success
template <typename T>
cudaError_t launch_trsv_push(const PushSolve& P, const NodeSched& S, const T* lu, const T* dinv,
                             const T* r, T* tmp, T* y, unsigned* status, cudaStream_t s);

}  // namespace fm
