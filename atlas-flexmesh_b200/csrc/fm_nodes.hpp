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
};

// y = U^-1 L^-1 r using tmp for the intermediate (both overwritten);
// dinv holds the reciprocal pivots written by the factorization
template <typename T>
void launch_trsv_nodes(const NodeSched& S, const T* lu, const T* dinv, const T* r, T* tmp, T* y,
                       unsigned* status, int device, cudaStream_t s);
// LU (a_ii kept on diagonal slots), pivots d and their reciprocals dinv
template <typename T>
void launch_ilu0_nodes(const NodeSched& S, const T* a, T* lu, T* d, T* dinv, unsigned* done,
                       unsigned epoch, unsigned* status, int device, cudaStream_t s);
template <typename T>
void launch_fill_sentinel(uint32_t n, T* x, cudaStream_t s);

}  // namespace fm
