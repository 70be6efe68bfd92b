// Host-side partition plan for the persistent PCG kernel.
//
// The node set is cut into G parts, one per thread block of the persistent
// launch: nodes sorted by y are cut into R strips (R ~ sqrt(G * height /
// width)), and each strip, sorted by x, into its share of the G blocks, so
// parts are near-square for any G and any node cloud.  A part owns its
// nodes.  Its work items ("tasks") are the (element, owned node) incidences:
// a task computes the node's 3 rows of Ke u_e.  Tasks are ordered node by
// node, so a node's K u is the sum of a contiguous run of task results (an
// owner-computes gather: no scatter, no atomics, fixed summation order).
// Nodes of a part's elements that it does not own are its ghosts (ring 1);
// with rings = 2 the nodes of the elements around ring-1 nodes that are in
// neither set form ring 2, and ring-1 nodes get tasks too (the polynomial
// smoother needs K t on owned and ring-1 rows).  Local numbering: owned
// nodes, then ring 1, then ring 2; tasks: owned nodes' tasks, then ring-1
// nodes' tasks.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "plategpu.h"

namespace pg {

struct HostPlan {
    int Nn = 0, Ne = 0, npe = 4, colors = 0, G = 0, rings = 1;
    // per part: [node_off[g], node_off[g+1]) local nodes (owned first), nown[g] owned
    std::vector<int> node_off, nown, nodes;
    // per part: [task_off[g], task_off[g+1]) tasks (global task numbering)
    std::vector<int> task_off;
    std::vector<int> task_elem;           // element of each task
    std::vector<uint8_t> task_pos;        // position of the owned node in the element
    std::vector<uint16_t> task_nodes;     // npe local node ids per task, owned node first,
                                          // then the element's next nodes cyclically
    // per part: n1[g] = owned + ring-1 nodes (the nodes with tasks when
    // rings = 2, else nown[g]); n1[g]+1 task offsets (relative to the part)
    // at tp_off[g]; the owned nodes' tasks are the first tptr[nown] of them
    std::vector<int> tptr, tp_off, n1;
    // node -> (element*4 + position) incidence, for block-diagonal assembly
    std::vector<int> inc_ptr, inc_idx;
    // the colouring actually used (the caller's, or a greedy one when the
    // caller's colouring had node-sharing elements of one colour)
    std::vector<uint32_t> color_offsets, elements_by_color;
    bool recolored = false;
    int max_nloc = 0, max_nown = 0, max_ntask = 0, max_ntask_own = 0, max_n1 = 0;

    // Two-level coarse space: one aggregate per part (its owned nodes), 3
    // modes each (the plate's rigid-body motions: w = 1; w = y, thx = 1;
    // w = x, thy = -1, in coordinates about the aggregate centre scaled by
    // its size h).  C = 3 G coarse DOFs.
    bool coarse = false;
    int C = 0, max_kagg = 0;
    std::vector<double> node_basis;  // per part-local node: dx, dy, 1/h of its aggregate
    std::vector<int> node_slot;      // per part-local node: index in the part's aggregate list
    std::vector<int> cagg_off, cagg; // per part: aggregates touching its local nodes (own first)
    std::vector<int> ainv_off;       // per part: first row of its A_c^-1 rows (3 per aggregate)
    std::vector<int> ainv_src;       // [rows]: the A_c^-1 row each part row copies (3 a + m)
    std::vector<double> ainv;        // rows of A_c^-1, [rows][C] (host set-up only)
    std::vector<int> coarse_owner;   // [Nn] aggregate (part) owning each node
    std::vector<double> coarse_geom; // [G][3] aggregate centre x, y and 1/size
    int dropped_modes = 0;           // coarse modes dropped as numerically dependent
};

// Checks the problem arrays; returns "" when valid, else the reason.
std::string validate_problem(const pg_problem& p, bool need_rhs);

// Builds the colouring (caller's or greedy) and node incidence.
std::string build_structure(const pg_problem& p, HostPlan& plan);

// The part (0 .. G - 1) of each of the Nn nodes (xy: [2 Nn]) under the
// strip partition above: sorted by (y, x, node id) into R strips, each
// strip sorted by (x, y, node id) and cut into its blocks; G >= 1.
void strip_partition(const float* xy, int Nn, int G, std::vector<int>& part_of);
// Partitions into G parts (G <= node_count) and fills the part arrays, with
// a ghost halo of `rings` (1 or 2) element layers.
std::string build_partition(const pg_problem& p, int G, int rings, HostPlan& plan);

// Coarse space of the two-level preconditioner from the element matrices
// ke64 ([Ne][(3 npe)^2], FP64): per-node basis data, per-part aggregate
// lists, and the rows of A_c^-1 = (P^T A P)^-1 each part needs.
std::string build_coarse(const pg_problem& p, const std::vector<double>& ke64, HostPlan& plan);
// The part of build_coarse that needs no element matrices: aggregate owners
// and geometry, per-node basis data, per-part aggregate lists and the
// source row of each part row of A_c^-1 (ainv_src); plan.ainv stays empty
// and plan.coarse false (the dense steps then run on the device).
std::string build_coarse_meta(const pg_problem& p, HostPlan& plan);

// Team schedule of a batch of independent plates.  A plate of n nodes gets
// a team of d blocks: a power of two, or every block of the device for the
// largest plates, with at most caps[i] nodes per block (so its parts fit in
// shared memory) and about part_nodes (default 400) nodes per block otherwise (fewer blocks
// per plate cost less block time, since an iteration's latency hardly
// depends on the part size).  Team sizes that fit side by side form a
// phase, one persistent launch; inside a phase the blocks are shared out
// among the team sizes in proportion to their estimated work (sqrt(n)
// iterations of n + 300 d node-equivalents), one team per size at least,
// and each size's plates go to its teams longest first to the least-loaded
// team.  Plates of different kinds (element types: the launch's kernel is
// specialised for one) never share a phase.
// Teams of one size form a class; a class's plates sit in one queue,
// largest estimated work first, and each team takes the next plate of its
// class's queue when it is free (a device-side counter per class), so the
// estimates only order the queue.  queue_off / queue / team_load keep the
// static assignment those estimates predict (each plate to the least
// loaded team of its size), for reporting.
struct BatchPhase {
    int kind = 4;                         // nodes per element of all its plates
    int grid = 0;                         // blocks of the launch
    std::vector<int> team_base, team_size;
    std::vector<int> team_class;          // [teams] class of each team
    std::vector<int> class_off, class_queue;  // [classes + 1]; plates, class by class
    std::vector<int> log_off;             // [teams + 1] each team's claim slots (its class's plates)
    std::vector<int> queue_off, queue;    // per team, the predicted plates in solve order
    std::vector<double> team_load;        // estimated work per team (predicted assignment)
};
struct BatchSchedule {
    std::vector<BatchPhase> phases;
    std::vector<int> plate_phase, plate_team, plate_size;  // [count]; team index within its phase
};
std::string schedule_batch(const std::vector<int>& nodes, const std::vector<int>& caps,
                           const std::vector<int>& kinds, int sms, BatchSchedule& out, int part_nodes = 400);

}  // namespace pg
