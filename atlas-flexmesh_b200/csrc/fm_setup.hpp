// fm_setup.hpp — host-side (CPU) structures built once per mesh.
//
// Everything here is integer work done at fm_set_mesh time: node neighbour
// lists, node->element incidence, the two CSR patterns of the reference,
// element->CSR slot maps and the ILU(0) dependency levels/schedules that
// the sync-free device kernels walk.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define FM_HD __host__ __device__
#else
#define FM_HD
#endif

namespace fm {

// Node-level CSR of sorted unique neighbour sets (self included), the
// std::set<uint32_t> per node that build_csr_sparsity_pattern_rigorous
// builds (FEM/adaptive_fem_engine.hpp:1076-1085).
struct NodeGraph {
    uint32_t n_nodes = 0;
    std::vector<uint32_t> ptr;   // n_nodes+1
    std::vector<uint32_t> nbr;   // sorted per node
    std::vector<uint32_t> self;  // position of n inside its own list
    uint32_t max_deg = 0;
};

struct Incidence {
    std::vector<uint32_t> ptr;   // n_nodes+1
    std::vector<uint32_t> elem;  // ascending element id per node
    uint32_t max_inc = 0;
};

// A1: unit cube generator, numbering as generate_unit_cube_mesh (:2219-2294)
void unit_cube(int N, double* xyz, uint32_t* conn);

NodeGraph build_node_graph(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn);
Incidence build_incidence(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn);

// DOF-level CSR: row_ptr[3n+d] = 9*ptr[n] + 3*d*deg(n) for both patterns.
void csr_row_ptr(const NodeGraph& g, uint32_t* row_ptr);
// Solve pattern: every row of node n lists 3*nbr[k]+q ascending.
void csr_solve_cols(const NodeGraph& g, uint32_t* col_idx);
// Reference pattern: neighbour-major fill across the node's 3 rows (:1109-1119).
void csr_reference_cols(const NodeGraph& g, uint32_t* col_idx);
// slot[e][(i*3+di)*12 + j*3+dj]; last duplicate wins, missing -> -1 (:1141-1150)
void slot_map(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n_elems,
              const uint32_t* conn, int32_t* slot);

// True dependency levels of a CSR with ascending columns.
// lower=true: depth(i) = 1 + max depth(j<i in row i); else from the bottom.
// ptr gets levels+1 entries, rows the stable sort by depth.
uint32_t csr_levels(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, bool lower,
                    std::vector<uint32_t>& ptr, std::vector<uint32_t>& rows);

// Node-granular levels of the solve pattern: node n depends on the nodes
// before (lower) / after (upper) it in its neighbour list.
uint32_t node_levels(const NodeGraph& g, bool lower, std::vector<uint32_t>& ptr,
                     std::vector<uint32_t>& order);

// Structural map of the ILU(0) updates (node granularity): for node n and
// its k-th lower neighbour m (k < self[n]), entry t of
// map[ptr[n] + sum_{k'<k} (deg(m') - self(m')) + t], t = 0 .. deg(m) - self(m) - 1,
// is the position in n's neighbour list of m's neighbour number self(m) + t
// (m itself, then its upper neighbours), or 0xff when n does not neighbour
// it.  Neighbour lists hold at most 32 nodes, so a position fits a byte.
void ilu_edge_maps(const NodeGraph& g, std::vector<uint32_t>& ptr, std::vector<uint8_t>& map);

// Plan of the slab-partitioned push solves (fm_trsv_push.cu).  The node
// range is cut into n_clusters contiguous slabs, one per thread-block
// cluster of `cluster` CTAs.  Both solves only ever wait on nodes on one
// side in the numbering (lower for the forward, upper for the backward), so
// a chain of dependencies leaves a slab at most n_clusters - 1 times: every
// other dependency hop stays inside one cluster.  There the producer stores
// its three values into a shared-memory slot of each CTA that reads them
// (one slot per producer and reading CTA, no reuse), and the readers poll
// their own shared memory; across slabs values go through global memory as
// in the grid-wide solves.  Inside a slab, blocks of `block` consecutive
// nodes are dealt round-robin to the cluster's CTAs, so that every CTA holds
// a share of each level (block is chosen to keep the busiest CTA's share of
// any level small).
constexpr uint32_t kPushMax = 9;  // reading CTAs per producer, at most (>= cluster size)
struct PushPlan {
    uint32_t n_ctas = 0, cluster = 0, block = 0;
    uint32_t max_level_share = 0;  // most nodes of one level in one CTA
    // CTA g's nodes are positions pos_f[g] .. pos_f[g + 1] of order_f (and
    // likewise backward), sorted by that direction's level and padded with
    // holes (~0u) so that positions 2i and 2i + 1 of a CTA, which one warp
    // resolves together, are never two nodes of different levels
    std::vector<uint32_t> pos_f, pos_b;  // n_ctas + 1 each
    std::vector<uint32_t> order_f, order_b;
    // per neighbour entry e of node n (graph order): the neighbour's slot in
    // n's CTA when the neighbour is on the solve's side and in n's slab, else
    // ~0u (read from global memory).  Lower entries serve the forward solve,
    // upper ones the backward; the self entry is ~0u.
    std::vector<uint32_t> src;
    // kPushMax per node and direction: rank << 20 | slot of each reading CTA
    // of the node's slab, ~0u after the last
    std::vector<uint32_t> push_f, push_b;
    std::vector<uint32_t> nslot_f, nslot_b;  // slots per CTA
    uint32_t max_slot_f = 0, max_slot_b = 0;
};

// CTA of node n: its slab's first CTA plus the round-robin rank of its block
// (slab s holds nodes ceil(s n_nodes / n_clusters) .. ceil((s+1) n_nodes / n_clusters) - 1)
FM_HD inline uint32_t push_slab_begin(uint32_t s, uint32_t n_nodes, uint32_t n_clusters) {
    return (uint32_t)(((uint64_t)s * n_nodes + n_clusters - 1) / n_clusters);
}
FM_HD inline uint32_t push_cta(uint32_t n, uint32_t n_nodes, uint32_t n_clusters,
                               uint32_t cluster, uint32_t block) {
    const uint32_t s = (uint32_t)((uint64_t)n * n_clusters / n_nodes);
    return s * cluster + ((n - push_slab_begin(s, n_nodes, n_clusters)) / block) % cluster;
}

// Builds the plan for n_clusters clusters of `cluster` CTAs (cluster <=
// kPushMax) from the level orders and level pointers of node_levels.  block
// = 0 picks the block size in 16 .. 512 with the smallest busiest-CTA level
// share whose slot counts stay within max_slots (ties: the smaller size).
// Returns false when a side of some node has more than 16 neighbours (the
// solves give each node a half-warp) or no block size keeps the slots
// within max_slots.
bool push_plan(const NodeGraph& g, const std::vector<uint32_t>& fwd_ptr,
               const std::vector<uint32_t>& fwd_order, const std::vector<uint32_t>& bwd_ptr,
               const std::vector<uint32_t>& bwd_order, uint32_t n_clusters, uint32_t cluster,
               uint32_t block, uint32_t max_slots, PushPlan& plan);

}  // namespace fm
