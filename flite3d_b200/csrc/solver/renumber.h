// Node renumbering for locality (host side of flite_create).
//
// The device numbers the nodes of every level in an order of its own: the
// boundary nodes stay the prefix 0..Nb-1 (the reference relies on boundary
// nodes being numbered first, def_par:5292, 5482, 11094, 12504), and within the
// boundary and the interior part, level 1 is ordered along a Morton
// (Z-order) curve of the node coordinates and every coarse level by the
// smallest new number of its children.  Consecutive nodes are then close in
// space, so a block of 256 nodes and its neighbours form a compact set that
// a gather stages in shared memory, and the node arrays of neighbouring
// nodes share cache lines.
//
// Edges keep their numbers, and every per-node list stays in the reference's
// order (incident edges in edge order, restriction children in the order of
// the original fine numbering), so every sum is formed in the same order as
// without renumbering: results are identical bit for bit.  Node arrays cross
// the C ABI in the caller's numbering.
#pragma once
#include <cstdint>
#include <vector>

#include "flite_gpu.h"

namespace flite {

// The levels of flite_create in the device numbering: the per-level
// permutation (perm[new] = old, iperm[old] = new, 0-based) and copies of
// the node-indexed and node-valued arrays of the descriptors.
struct Renumbered {
    std::vector<std::vector<int>> perm, iperm;
    std::vector<flite_level_desc> desc;
    bool identity = true;
    // storage behind desc
    std::vector<std::vector<int32_t>> side_idx, bnd_idx, node_ind, parent, engine_idx;
    std::vector<std::vector<double>> volume, wall_dist, coords, coord_move, rweight, volume_prev, volume_prev2;
};

// mode 0: identity; 1: locality order.  Throws std::runtime_error on
// inconsistent descriptors.
void renumber_levels(int nlevels, const flite_level_desc *lv, int mode, Renumbered &out);
// the same with a given numbering (perm, iperm per level; identity when the
// device numbering is the caller's): the levels of a moving mesh's next step
void renumber_as(int nlevels, const flite_level_desc *lv, const std::vector<std::vector<int>> &perm,
                 const std::vector<std::vector<int>> &iperm, bool identity, Renumbered &out);
// the descriptors of out in the numbering of out.perm / out.iperm
void permute_levels(int nlevels, const flite_level_desc *lv, Renumbered &out);

// process-wide default of flite_create (flite_set_node_order)
int default_node_order();

}  // namespace flite
