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

// Plan of a triangular solve on one thread-block cluster: warp
// gw = cta * warps_per_cta + w takes positions lvl_ptr[l] + gw, + gw + W, ...
// of each dependency level (W = all warps).  The three values a node
// produces live, from its level to the last level that reads them, in a
// slot of its writer CTA's shared-memory pool.  Levels are grouped in
// windows of `window` levels closed by a cluster barrier; a slot whose last
// read falls in window t is reset (to the wait sentinel) by its CTA after
// the barrier closing window t and handed out again from window t + 2 on.
struct ClusterPlan {
    uint32_t n_levels = 0, n_ctas = 0, warps_per_cta = 0, window = 1;
    uint32_t max_per_warp = 0;   // nodes one warp takes in one level, at most
    uint32_t max_cnt = 0;        // neighbours on the solve's side of one node, at most
    uint32_t slots_per_cta = 0;  // pool entries the busiest CTA needs
    std::vector<uint32_t> lvl_ptr;  // n_levels + 1 positions
    // per position: {node, first neighbour entry, deg | sk << 8 | cnt << 16, own slot}
    std::vector<uint32_t> rec;      // 4 words per position
    // slots CTA c resets after window t: reset[reset_ptr[t * n_ctas + c] ...
    // reset_ptr[t * n_ctas + c + 1])
    std::vector<uint32_t> reset_ptr, reset;
    // lane groups (lanes = true): a level's positions in groups of 32, group
    // i of level l is global group lvl_gptr[l] + i, taken by warp
    // (global group) mod W, lane = position within the group
    bool lanes = false;
    uint32_t n_groups = 0;
    std::vector<uint32_t> lvl_gptr;  // n_levels + 1
};

// Builds the plan of one direction (lower: forward solve over the levels
// ptr/order of node_levels(g, true, ...)) and writes, for every neighbour
// entry on that side (lower entries for the forward solve, upper ones for
// the backward), the neighbour's slot as (cta << 16) | index into nslot
// (g.nbr.size() entries; the other side's entries are left as they are).
// Returns false when a CTA pool would need more than max_slots_per_cta
// entries or a side has more than 32 neighbours.
bool cluster_plan(const NodeGraph& g, bool lower, const std::vector<uint32_t>& ptr,
                  const std::vector<uint32_t>& order, uint32_t n_ctas, uint32_t warps_per_cta,
                  uint32_t window, uint32_t max_slots_per_cta, ClusterPlan& plan,
                  std::vector<uint32_t>& nslot, bool lanes = false);

// Structural map of the ILU(0) updates (node granularity): for node n and
// its k-th lower neighbour m (k < self[n]), entry t of
// map[ptr[n] + sum_{k'<k} (deg(m') - self(m')) + t], t = 0 .. deg(m) - self(m) - 1,
// is the position in n's neighbour list of m's neighbour number self(m) + t
// (m itself, then its upper neighbours), or 0xff when n does not neighbour
// it.  Neighbour lists hold at most 32 nodes, so a position fits a byte.
void ilu_edge_maps(const NodeGraph& g, std::vector<uint32_t>& ptr, std::vector<uint8_t>& map);

// Cards of the cluster solves are ordered by (level, warp, node): position
// level_start + gw + j W of a level of `width` positions is warp gw's j-th
// node there, and warp gw holds q + (gw < r) of the level's cards
// (width = q W + r), starting at
FM_HD inline uint32_t first_card(uint32_t level_start, uint32_t width, uint32_t W,
                                 uint32_t gw) {
    const uint32_t q = width / W, r = width % W;
    return level_start + gw * q + (gw < r ? gw : r);
}
// card index of every position of the levels lvl_ptr
void cluster_card_index(const std::vector<uint32_t>& lvl_ptr, uint32_t W,
                        std::vector<uint32_t>& card_of_pos);

}  // namespace fm
