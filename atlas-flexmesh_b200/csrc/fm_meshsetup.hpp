// fm_meshsetup.hpp — the per-mesh structures built on the device.
//
// build_csr_sparsity_pattern_rigorous (FEM/adaptive_fem_engine.hpp:1069)
// forms every node's neighbour set with a std::set and the node->element
// lists of generate_unit_cube_mesh (:2279-2291) are built serially; here the
// same structures (and those the B200 kernels need on top) come from a few
// device passes:
//   incidence   node -> incident tets, ascending (counting sort + a warp
//               sort of each node's list);
//   node graph  sorted unique neighbour set of every node (self included)
//               and the position of the node in its own set;
//   levels      the ILU(0) dependency depth of every node in both
//               directions, by one sync-free pass over the nodes in ticket
//               order (a node waits only on nodes with earlier tickets), and
//               the level lists as a stable sort of the nodes by depth;
//   ILU maps    fm_setup.hpp ilu_edge_maps; assembly scatter structures
//               (vertex positions per incidence, tet bitmask per edge).
// Every output equals the host construction in fm_setup.cpp entry for entry.
#pragma once

#include <cstdint>
#include <vector>

#include "fm_devbuf.hpp"
#include "fm_setup.hpp"

namespace fm {

// device outputs (owned by the caller; resized here)
struct MeshSetupDev {
    DevBuf<uint32_t>* inc_ptr;      // n_nodes + 1
    DevBuf<uint32_t>* inc_e;        // 4 n_elems
    DevBuf<uint32_t>* nbr_ptr;      // n_nodes + 1
    DevBuf<uint32_t>* nbr;          // neighbour entries
    DevBuf<uint32_t>* self_pos;     // n_nodes
    DevBuf<uint32_t>* node_fwd;     // forward level order (n_nodes)
    DevBuf<uint32_t>* node_bwd;     // backward level order
    DevBuf<uint4>* node_fwd_rec;    // {node, first entry, degree, self} per position
    DevBuf<uint4>* node_bwd_rec;
    DevBuf<uint32_t>* emap_ptr;     // n_nodes + 1
    DevBuf<uint8_t>* emap;
    DevBuf<uint32_t>* inc_pos;      // 4 x u8 per incidence
    DevBuf<uint32_t>* nbr_members;  // tet bitmask per neighbour entry
};

// host copies that host-side planning and the exports use
struct MeshSetupHost {
    NodeGraph graph;
    uint32_t max_inc = 0;
    std::vector<uint32_t> lp, lo, up, uo;  // node levels: (ptr, order) forward, backward
};

enum { kSetupOk = 0, kSetupLimits = 1, kSetupTimeout = 2 };

// conn: n_elems uint4 on the device, bit 31 of .x marking a skipped tet (the
// incidence and graph include it; the tet bitmasks do not).  status: the
// context's status word (its bounded-wait limit follows it).  *result:
// kSetupLimits when a node has more than 32 neighbours or incident tets,
// kSetupTimeout when a dependency wait of the level pass expired.
cudaError_t build_mesh_device(uint32_t n_nodes, uint32_t n_elems, const uint4* conn,
                              MeshSetupDev& d, MeshSetupHost& h, unsigned* status, int* result,
                              cudaStream_t s);

// Element -> CSR slot map of tets e0 .. e0+count-1 (144 int32 per tet,
// slot[(i*3+di)*12 + j*3+dj]) for the solve pattern or, reference != 0, the
// reference's own column fill (last duplicate wins, missing -1).
void launch_slot_map(uint32_t e0, uint32_t count, const uint4* conn, const uint32_t* nbr_ptr,
                     const uint32_t* nbr, int reference, int32_t* slot, cudaStream_t s);

// Element colouring of MeshColoring::compute (FEM/adaptive_fem_engine.hpp:
// 1549-1602): greedy first fit in element order, elements sharing a node
// differ; the same colours as the reference's O(E^2) construction, in
// O(E * incident tets) through the node incidence.  Returns the colour count.
uint32_t mesh_coloring(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn,
                       uint32_t* colors);

}  // namespace fm
