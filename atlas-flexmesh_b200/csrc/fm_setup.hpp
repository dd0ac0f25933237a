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

}  // namespace fm
