// Host-side partition plan for the persistent PCG kernel.
//
// The node set is cut into G parts by recursive coordinate bisection (each
// cut at the proportional median of the longer bounding-box side), one part
// per thread block of the persistent launch.  A part owns its nodes; it also
// holds every element touching an owned node and, as ghosts, the nodes of
// those elements it does not own.  Within a part, elements are ordered by
// colour so that one colour's rows can be added into shared memory without
// atomics; local node numbering is owned nodes first, then ghosts.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "plategpu.h"

namespace pg {

struct HostPlan {
    int Nn = 0, Ne = 0, npe = 4, colors = 0, G = 0;
    // per part: [node_off[g], node_off[g+1]) local nodes (owned first), nown[g] owned
    std::vector<int> node_off, nown, nodes;
    // per part: [elem_off[g], elem_off[g+1]) elements; color_off[g*(colors+1)+c] absolute
    std::vector<int> elem_off, color_off, elems;
    std::vector<int> lnode;  // npe local node indices per part element
    // node -> (element*4 + position) incidence, for block-diagonal assembly
    std::vector<int> inc_ptr, inc_idx;
    // the colouring actually used (the caller's, or a greedy one when the
    // caller's colouring had node-sharing elements of one colour)
    std::vector<uint32_t> color_offsets, elements_by_color;
    bool recolored = false;
    int max_nloc = 0, max_nown = 0, max_nel = 0;
};

// Checks the problem arrays; returns "" when valid, else the reason.
std::string validate_problem(const pg_problem& p, bool need_rhs);

// Builds the colouring (caller's or greedy) and node incidence.
std::string build_structure(const pg_problem& p, HostPlan& plan);

// Partitions into G parts (G <= node_count) and fills the part arrays.
std::string build_partition(const pg_problem& p, int G, HostPlan& plan);

// 64-bit FNV-1a over the problem's mesh, colouring, material and
// constraint arrays (not F): the key of the plan cache.
uint64_t problem_hash(const pg_problem& p);

}  // namespace pg
