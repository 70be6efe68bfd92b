/*
 * plategpu.h -- C ABI of the B200 (sm_100a) matrix-free plate-bending PCG
 * solver.
 *
 * This is the drop-in boundary for the GPU plate solve of
 * cseifert512/gpu-gauntlet: the entry points below are what the
 * reference's GPU-solver module would bind through an N-API addon.  Every
 * argument is a plain pointer or a size; no C++ or torch type crosses this
 * boundary; no exception, exit or abort either: every call returns a
 * pg_status and pg_last_error() describes the last failure.  There is no CPU
 * fallback: without a usable CUDA device every solve fails with PG_ECUDA.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   pg_solve         solveGPU(mesh, material, coloring, F, constrainedDOFs,
 *                    options) -> GPUSolveResult   src/lib/plate/gpu/solver.ts:80-104
 *                    (with solveGPUInternal :109-185 and runGPUPCG :190-553)
 *   pg_problem       PlateMesh, PlateMaterial, ElementColoring
 *                    src/lib/plate/types.ts:14-102; F and constrainedDOFs as
 *                    solveGPU receives them
 *   pg_options       GPUSolverOptions  src/lib/plate/gpu/solver.ts:35-42
 *   pg_info          GPUSolveResult    src/lib/plate/gpu/solver.ts:47-60
 *   pg_apply_k       gpuApplyK + apply_k_q4 / apply_k_dkt
 *                    src/lib/plate/gpu/solver.ts:413-461 (single-colour K.x
 *                    test pattern of src/lib/plate/gpu/single_color_test.ts)
 *   pg_block_jacobi  computeBlockDiagonal + invertBlockDiagonal
 *                    src/lib/plate/solver.ts:188-304 as solveGPUInternal calls
 *                    them (gpu/solver.ts:130-131)
 *   pg_is_available  isWebGPUAvailable  src/lib/plate/gpu/context.ts:19
 *   pg_clear_cache   clearPipelineCache src/lib/plate/gpu/solver.ts:601-603
 *   pg_solve_load_cases  solveGPU called once per load of the same plate
 *                    (gpu/solver.ts:80-104); the lockstep solve of several
 *                    loads has no reference counterpart
 *
 * Semantics kept from the reference: F arrives with the boundary conditions
 * applied (applyBCsToRHS); constrained DOFs are identity rows, (K p)_c = p_c,
 * so the solution is 0 there; the block-Jacobi preconditioner is built
 * inside the solve from mesh and material; defaults tolerance 1e-6,
 * max_iterations 1000; the reference stop rule is ||r|| < tol or
 * ||r|| / ||b|| < tol on the recursive residual; |p.Ap| < 1e-30 is a
 * breakdown that returns converged = 0.
 */
#ifndef PLATEGPU_H
#define PLATEGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_ABI_VERSION 1

typedef enum pg_status {
    PG_OK = 0,
    PG_EINVAL = 1,        /* malformed problem or options */
    PG_ENOMEM = 2,        /* device or host allocation failed */
    PG_ECUDA = 3,         /* CUDA runtime error / no device */
    PG_ETIMEOUT = 4,      /* a wait for another block's data ran past its time limit */
    PG_ENONFINITE = 5,    /* NaN or Inf in the inputs or the iteration */
    PG_EUNSUPPORTED = 6   /* a request this build does not serve */
} pg_status;

typedef enum pg_precision {
    PG_PREC_FP64 = 0,  /* plain FP64 block-Jacobi PCG */
    PG_PREC_MIXED = 1  /* FP32 inner iterations, FP64 solution and
                          FP64 true-residual replacement */
} pg_precision;

typedef enum pg_preconditioner {
    PG_PRECOND_BLOCK_JACOBI = 0, /* 3x3 block Jacobi, as the reference (solver.ts:188-339) */
    PG_PRECOND_TWO_LEVEL = 1     /* block Jacobi + Galerkin coarse correction on one
                                    aggregate per thread block (3 rigid-body modes each) */
} pg_preconditioner;

typedef enum pg_smoother {
    PG_SMOOTHER_BLOCK_JACOBI = 0, /* u = D^-1 r, D the 3x3 nodal blocks (the reference's) */
    PG_SMOOTHER_CHEBYSHEV = 1     /* u = a D^-1 r - b D^-1 K D^-1 r: two Chebyshev steps
                                     for D^-1 K on [hi/20, hi], hi = 1.1 lambda_max
                                     (power-iteration estimate); one more K product per
                                     iteration on a 2-ring ghost halo, no extra exchange */
} pg_smoother;

typedef enum pg_stop_rule {
    PG_STOP_REFERENCE = 0, /* ||r|| < tol  or  ||r||/||b|| < tol  (gpu/solver.ts:516) */
    PG_STOP_RELATIVE = 1   /* ||r||/||b|| < tol only */
} pg_stop_rule;

typedef enum pg_stop_reason {
    PG_STOP_CONVERGED = 0,
    PG_STOP_MAX_ITER = 1,
    PG_STOP_BREAKDOWN = 2, /* |p.Ap| < 1e-30 (pcg.ts:154, gpu/solver.ts:496) */
    PG_STOP_ZERO_RHS = 3,  /* ||b|| < 1e-30: x = 0, 0 iterations */
    PG_STOP_STAGNATED = 4  /* mixed precision: the FP64 residual did not halve over three
                              residual replacements (FP32 cannot resolve the problem);
                              with pg_options.fallback the call re-solves in FP64 */
} pg_stop_reason;

/* One plate problem, in the reference's host layout. */
typedef struct pg_problem {
    uint32_t node_count;
    uint32_t element_count;
    uint32_t nodes_per_element;        /* 4 = Q4 Mindlin quad, 3 = DKT triangle */
    const float* nodes;                /* [2*node_count] x0,y0,x1,y1,...      */
    const uint32_t* elements;          /* [nodes_per_element*element_count]   */
    uint32_t color_count;
    const uint32_t* color_offsets;     /* [color_count+1], offsets into:      */
    const uint32_t* elements_by_color; /* [element_count] element ids by colour */
    double E, nu, t;                   /* PlateMaterial                        */
    const float* elem_t;               /* optional [element_count] thickness,
                                          overrides t (NULL = uniform t)       */
    const float* F;                    /* [3*node_count] load vector           */
    const uint8_t* constrained;        /* [3*node_count] 1 = constrained DOF   */
} pg_problem;

typedef struct pg_options {
    uint32_t struct_size;         /* sizeof(pg_options); set by pg_options_default */
    double tolerance;             /* default 1e-6 */
    int32_t max_iterations;       /* default 1000 */
    int32_t precision;            /* pg_precision, default PG_PREC_FP64 */
    int32_t stop_rule;            /* pg_stop_rule, default PG_STOP_REFERENCE */
    int32_t ctas;                 /* persistent grid size; 0 = automatic */
    int32_t threads;              /* threads per CTA; 0 = automatic */
    double wait_timeout_ms;       /* limit on each wait for another block's data; default 1000 */
    int32_t reliable_interval;    /* mixed: max inner iterations between FP64
                                     residual replacements; 0 = automatic (200) */
    double reliable_delta;        /* mixed: replace when the FP32 residual fell
                                     by this factor; 0 = automatic (0.1) */
    int32_t phase_timing;         /* 1: record per-phase device time (pg_info.phase_us) */
    int32_t test_stall;           /* test hook: 1 makes block 0 wait once for a value no
                                     block ever writes, so the call must end with
                                     PG_ETIMEOUT after wait_timeout_ms */
    int32_t preconditioner;       /* pg_preconditioner, default PG_PRECOND_BLOCK_JACOBI */
    int32_t trace_iteration;      /* > 0: time-stamp that iteration in every block
                                     (pg_info.trace_ns) */
    int32_t smoother;             /* pg_smoother, default PG_SMOOTHER_BLOCK_JACOBI (also the
                                     smoother of the two-level preconditioner) */
    int32_t fallback;             /* mixed precision: 1 (default) continues in FP64 when the
                                     mixed solve stagnates (PG_STOP_STAGNATED): an FP64 solve
                                     of the correction K d = F - K x_m from the stagnated x_m,
                                     stopped by the same rule on x_m + d; 0 returns the
                                     stagnated result */
    int32_t batch_part_nodes;     /* batches: preferred nodes per block of a plate's team
                                     (0 = automatic, 400); plategpu.autotune picks it per
                                     GPU and batch */
} pg_options;

/* Per-solve result (GPUSolveResult plus extended statistics). */
typedef struct pg_info {
    int32_t status;               /* pg_status of the call */
    int32_t iterations;
    int32_t converged;
    int32_t stop_reason;          /* pg_stop_reason */
    double final_residual;        /* ||r|| of the recursive residual (reference meaning) */
    double true_rel_residual;     /* ||F - K x|| / ||F||, recomputed in FP64 on the GPU */
    double b_norm;                /* ||F|| */
    double setup_ms;              /* device: element stiffness + block-Jacobi setup (about 0
                                     once the plan's set-up has been done) */
    double solve_ms;              /* device: persistent PCG launch */
    double total_ms;              /* host wall clock of the whole call (gpuTimeMs) */
    int32_t ctas;
    int32_t threads;
    int32_t reliable_updates;     /* mixed precision: FP64 residual replacements */
    int32_t plan_cached;          /* 1 when the partition plan was reused */
    int32_t reductions;           /* grid-wide reductions (one per iteration, plus
                                     one per residual replacement) */
    int32_t shared_bytes;         /* dynamic shared memory per block */
    int32_t coarse_dim;           /* two-level: coarse DOFs kept (0 otherwise) */
    int32_t fallback;             /* 1 when a stagnated mixed solve was finished by an FP64
                                     correction (iterations, stop_reason and converged are
                                     then the correction's; the residuals refer to the final
                                     x and F; solve_ms covers both) */
    double phase_us[8];           /* with phase_timing, block 0's time (SM cycles at
                                     the nominal clock) in: K.u; gather, dots and
                                     publishing w; block reduction and publishing the
                                     partials; the Chebyshev smoother's K t; the
                                     exchange wait; the barrier after the decision;
                                     thread 0's decision; the other vector updates */
    double trace_ns[6];           /* with trace_iteration, over all blocks: spread of
                                     iteration starts; spread of partial publication;
                                     first start to last publication; last publication
                                     to the first block holding every partial; spread
                                     of exchange completion; whole iteration */
    double smoother_lambda_max;   /* Chebyshev smoother: the lambda_max(D^-1 K) estimate used */
    int32_t global_path;          /* 1 when the plate's parts did not fit one block's shared
                                     memory and the solve ran as flexible PCG over global
                                     memory: FP32 vectors, FP64 x, dot products and true-
                                     residual stop; block Jacobi, or damped block-Jacobi
                                     smoothing steps when the two-level preconditioner or
                                     the Chebyshev smoother was asked for */
    int32_t reserved;
    double plan_ms;               /* host wall time in this call of: building the partition
                                     plan (pg_solve; 0 when the plan was cached), */
    double coarse_ms;             /* the two-level coarse space (A_c on the device, its
                                     factorisation and inverse; 0 once done for the plan), */
    double eigen_ms;              /* the Chebyshev smoother's lambda_max estimate (0 once
                                     done for the plan) */
} pg_info;

typedef struct pg_ctx pg_ctx;

/* pg_options filled with the reference defaults. */
void pg_options_default(pg_options* opt);

/* 1 when a CUDA device of compute capability 10.x can be used. */
int pg_is_available(void);

/* Context on CUDA device `device`: owns a stream, device buffers and the
 * cache of partition plans.  One context per host thread (calls on one
 * context are serialised by an internal mutex). */
int pg_create(int device, pg_ctx** out);
void pg_destroy(pg_ctx* ctx);

/* Message of the last failing call on ctx (or of pg_create when ctx is NULL). */
const char* pg_last_error(const pg_ctx* ctx);

/* Drops every cached partition plan and device buffer of ctx. */
int pg_clear_cache(pg_ctx* ctx);

/* Runs all work of ctx on `stream` (a cudaStream_t; NULL = the context's
 * own stream). */
int pg_set_stream(pg_ctx* ctx, void* stream);

/* Solves K x = F.  x_out: [3*node_count] FP64 (the TypeScript wrapper
 * narrows it to the reference's Float32Array).  info may be NULL. */
int pg_solve(pg_ctx* ctx, const pg_problem* prob, const pg_options* opt, double* x_out,
             pg_info* info);

/* Load cases: solves K x_k = F_k for `count` loads of one plate (prob->F is
 * not read).  F: [count][3*node_count] float, x_out: [count][3*node_count]
 * FP64, infos (optional): [count].  Up to cases_per_launch cases (0 =
 * automatic: the widest of 4 and 2 whose shared-memory layout still holds
 * the element blocks, else the widest that fits, else 1; or 1, 2, 4) run in
 * lockstep in one persistent launch: one
 * exchange round per iteration for all of them, each element block read
 * once for all of them, each case with its own PCG scalars and stop.  The
 * launch runs until its last case stops; each case's info carries that
 * launch's solve_ms.  In mixed precision a residual replacement asked for
 * by one case runs for all (only the cases that asked replace their
 * residual), and a case that stagnates is solved again alone in FP64
 * (pg_options.fallback).  A solve of one load (pg_solve) is the
 * reference's solveGPU (gpu/solver.ts:80-104); the reference solves load
 * cases by calling it once per load. */
int pg_solve_load_cases(pg_ctx* ctx, const pg_problem* prob, int count, const float* F,
                        const pg_options* opt, int cases_per_launch, double* x_out, pg_info* infos);

/* Device-resident solves.  A plan holds the partition of one mesh and its
 * device copies (nodes, elements, colouring, constraints, material).  The
 * first solve on a plan computes the element stiffness, block-Jacobi and
 * task set-up on the device (they depend only on the plan's own copies, so
 * later solves reuse them); every pg_plan_solve_device runs the persistent
 * PCG for a new load.  F_dev is
 * a device float [3*node_count], x_dev a device double [3*node_count]; work
 * runs on the context stream and the call returns after its one readback
 * of the result record (x_dev is unspecified when the call fails).  A plan
 * must not outlive its context. */
typedef struct pg_plan pg_plan;
int pg_plan_create(pg_ctx* ctx, const pg_problem* prob, const pg_options* opt, pg_plan** out);
int pg_plan_solve_device(pg_plan* plan, const pg_options* opt, const float* F_dev,
                         double* x_dev, pg_info* info);
void pg_plan_destroy(pg_plan* plan);

/* Batches of independent plates (no counterpart in the reference, whose
 * solveGPU takes one plate).  All plates of a batch are solved by one
 * persistent launch: the grid is cut into teams of blocks, each plate gets a
 * team sized to it (a power of two; large plates more blocks) and is
 * partitioned for that team, and every team works through its own queue of
 * plates, longest first, with no waiting between teams.  Team sizes that
 * cannot share the device (the largest plates may need every block) run in
 * separate phases: one launch each, back to back.  Plates may mix Q4
 * and DKT elements, sizes, materials and supports; the options (precision,
 * preconditioner, smoother, tolerance, ...) apply to every plate.
 * pg_batch_create plans the batch and copies each problem's F to the device;
 * pg_batch_solve solves it, with new loads when F is non-NULL (F[i] NULL
 * keeps plate i's load); x_out[i] (host, 3*node_count doubles, may be NULL)
 * and infos[i] (may be NULL) receive each plate's result.  infos[i].solve_ms
 * is the plate's own start-to-end time inside the launch.  A plate too large
 * for a batch (more nodes than every block together holds) is rejected with
 * PG_EUNSUPPORTED: solve it with pg_solve. */
typedef struct pg_batch_info {
    int32_t status;
    int32_t count;                /* plates */
    int32_t teams;                /* teams of blocks in the launch */
    int32_t grid;                 /* blocks of the largest launch */
    int32_t converged;            /* plates that converged */
    int32_t shared_bytes;         /* dynamic shared memory per block */
    int32_t phases;               /* launches (team sizes that do not fit side by side
                                     run in separate phases) */
    int32_t fallbacks;            /* plates re-solved in FP64 after a stagnated mixed solve
                                     (one launch each, after the batch; in solve_ms) */
    double setup_ms;              /* device: element set-up queued by this call (0 once done) */
    double solve_ms;              /* device: the batch launch (CUDA events) */
    double total_ms;              /* host wall clock of the call */
    double plate_ms_p50;          /* per-plate start-to-end time in the launch: median, */
    double plate_ms_p99;          /*   99th percentile */
    double plate_ms_max;          /*   and largest */
    double solves_per_s;          /* count / solve_ms */
    int32_t graph;                /* 1 when the phase launches ran as one captured CUDA graph */
} pg_batch_info;

typedef struct pg_batch pg_batch;
int pg_batch_create(pg_ctx* ctx, const pg_problem* probs, int count, const pg_options* opt,
                    pg_batch** out);
int pg_batch_solve(pg_batch* batch, const pg_options* opt, const float* const* F,
                   double* const* x_out, pg_info* infos, pg_batch_info* info);
void pg_batch_destroy(pg_batch* batch);
/* pg_batch_create + pg_batch_solve + pg_batch_destroy in one call. */
int pg_solve_batch(pg_ctx* ctx, const pg_problem* probs, int count, const pg_options* opt,
                   double* const* x_out, pg_info* infos, pg_batch_info* info);
/* Host-only: the schedule pg_batch_create uses for plates of these node
 * counts on `sms` blocks with at most `cap` nodes per block: per plate its
 * phase, team size and predicted team (index within the phase) [count
 * each]; per phase its grid [count, the first *phases_out entries used].
 * At run time the teams of one size share one queue of their plates
 * (largest estimated work first) and a free team takes the next one, so
 * the team that solves a plate can differ from the prediction. */
int pg_batch_schedule(const uint32_t* node_counts, int count, int sms, int cap, int32_t* plate_phase,
                      int32_t* plate_size, int32_t* plate_team, int32_t* phase_grid,
                      int32_t* phases_out);
/* Host-only: the thread block (part) owning each node in a solve over
 * `ctas` blocks (pg_info.ctas; at most node_count are used): nodes sorted
 * by (y, x, node id) are cut into R = round(sqrt(ctas * height / width))
 * strips, each strip sorted by (x, y, node id) is cut into its share of the
 * blocks.  nodes: [2*node_count] x0,y0,...; part_of: [node_count].  No
 * counterpart in the reference (its solver does not partition the mesh).
 * PG_EINVAL for NULL arrays, ctas < 1, or coordinates that are not finite. */
int pg_partition_nodes(const float* nodes, uint32_t node_count, int ctas, int32_t* part_of);

/* Nodal bending moments of a solution, as computeMoments
 * (postprocess.ts:40-264): curvatures at each element's centroid (Q4
 * shape derivatives at xi = eta = 0, DKT linear-triangle derivatives), Mx =
 * D (kx + nu ky), My = D (ky + nu kx), Mxy = D (1 - nu) kxy / 2 with the
 * plate's uniform D (E, nu, t of the problem; like the reference, elem_t is
 * not used), averaged over the elements around each node; degenerate
 * triangles are left out.  FP64 on the device.  x: [3*node_count]. */
int pg_moments(pg_ctx* ctx, const pg_problem* prob, const double* x, double* Mx, double* My,
               double* Mxy);
/* The same on a plan's device-resident solution: x_dev [3*node_count] ->
 * M_dev [3][node_count] (Mx, My, Mxy), on the context stream. */
int pg_plan_moments_device(pg_plan* plan, const double* x_dev, double* M_dev);

/* Test hook: y = K x in FP64 with the reference BC rule (y_c = x_c). */
int pg_apply_k(pg_ctx* ctx, const pg_problem* prob, const double* x, double* y);

/* Test hook: inverted 3x3 block diagonal (9 doubles per node, row-major),
 * constrained rows/columns replaced by identity before inversion and
 * |det| < 1e-30 blocks replaced by identity (solver.ts:231-304). */
int pg_block_jacobi(pg_ctx* ctx, const pg_problem* prob, double* binv_out);

/* y = K x (same operator and BC rule as pg_apply_k) without allocating
 * anything.  No counterpart in the reference: it is for callers that may
 * not call cudaMalloc -- code whose device memory belongs to another
 * allocator with no untracked blocks to spare (a framework's caching
 * allocator, a fixed memory budget), or code that must not allocate once it
 * is running (a real-time loop, a driver callback).
 *   - prob's nodes, elements, elements_by_color, elem_t (optional) and
 *     constrained, and x and y ([3*node_count] doubles), are DEVICE pointers
 *     on the calling thread's current device; color_offsets is a HOST
 *     pointer; F is not used.  The colouring must be valid (no two elements
 *     of one colour share a node); it is not checked.
 *   - The element matrices go to a static device array of 8 MiB that the
 *     library holds on every GPU it is loaded on until the process exits:
 *     at most 7,281 Q4 or 12,945 DKT elements; larger problems fail with
 *     PG_EINVAL before any work is queued.
 *   - The first call on a device looks up that array's device address
 *     (cudaGetSymbolAddress) and keeps it; make that first call before any
 *     stream capture.  The kept address is not valid after a
 *     cudaDeviceReset of that device: do not use this entry point across a
 *     device reset.
 *   - x and y must not overlap (y is cleared before K x is summed into it):
 *     an overlapping call fails with PG_EINVAL.  color_offsets must start
 *     at 0, not decrease and end at element_count (PG_EINVAL otherwise).
 *   - Work is queued on `stream` (a cudaStream_t; NULL = legacy default
 *     stream) and the call returns without waiting.  All calls share the
 *     one array, so calls whose work overlaps on the GPU (other streams,
 *     other host threads) race; serialise them.
 *   - msg/msg_len (optional) receive the reason for a failure. */
int pg_apply_k_static(const pg_problem* prob, const double* x, double* y, void* stream, char* msg,
                      size_t msg_len);

/* Test hook: element stiffness matrices, [element_count * (3*npe)^2] FP64. */
int pg_element_stiffness(pg_ctx* ctx, const pg_problem* prob, double* ke_out);

/* Host-only test hook (no device needed): builds the partition plan the
 * solver would use with `ctas` blocks and checks its invariants (every
 * node owned by exactly one part, ghosts = the other nodes of the owned
 * nodes' elements, no two elements of one colour sharing a node, every (element, owned node)
 * incidence present once as a task of the owning part).  stats_out[8]:
 * parts, colours, recoloured (0/1), max local nodes, max owned nodes, max
 * tasks per part, total ghost nodes, invariant violations (0 when valid).
 * msg/msg_len (optional) receive the failure reason. */
int pg_plan_inspect(const pg_problem* prob, int ctas, int32_t* stats_out, char* msg,
                    size_t msg_len);

/* pg_plan_inspect for a plan with a ghost halo of `rings` element layers
 * (1, or 2 as the Chebyshev smoother uses: ring-1 nodes then carry tasks
 * too, and the invariants cover them). */
int pg_plan_inspect_halo(const pg_problem* prob, int ctas, int rings, int32_t* stats_out,
                         char* msg, size_t msg_len);

/* ---------------------------------------------------------------------------
 * Learned two-level preconditioner (no counterpart in the reference, whose
 * PCG applies only the 3x3 block Jacobi -- src/lib/plate/gpu/shaders/
 * index.ts:214-262, once per iteration of runGPUPCG, gpu/solver.ts:190-553;
 * the network's correction is added at that point of the iteration).
 *
 * pg_net: a 4-level U-Net over a height x width grid (multiples of 8):
 * 3 x 3 convolutions without bias, channels 16/32/64/128, ReLU, 2x2 average
 * pooling, nearest upsampling, skip connections by concatenation; 3 input
 * and 3 output channels (w, theta_x, theta_y of the node at each pixel).
 * BF16 weights and activations with FP32 accumulation on the tensor cores
 * (mma.sync), FP32 master weights and Adam state.  Parameters cross the ABI
 * in the real (unpadded) layout: per layer [cout][3][3][cin], layers in the
 * order e0a e0b e1a e1b e2a e2b e3a e3b d2a d2b d1a d1b d0a d0b out.
 * scales[6]: the input scales applied to the residual's three components
 * and the output scales applied to the network's three outputs.
 * ------------------------------------------------------------------------- */
typedef struct pg_net pg_net;
int pg_net_create(pg_ctx* ctx, int height, int width, uint64_t seed, pg_net** out);
void pg_net_destroy(pg_net* net);
int64_t pg_net_param_count(const pg_net* net);
/* params (may be NULL): [pg_net_param_count] floats; setting them resets the
 * Adam state.  scales (may be NULL): 6 floats > 0. */
int pg_net_set_params(pg_net* net, const float* params, const float* scales);
int pg_net_get_params(pg_net* net, float* params, float* scales);
/* Test hooks on device buffers: forward of `batch` images [batch][h][w][3]
 * (FP32 in and out); backward of the last forward from dL/d out (FP32
 * [batch][h][w][3]) into dL/d in (device, may be NULL) and the parameter
 * gradients (host, real layout, may be NULL); one Adam step (lr, betas 0.9
 * and 0.999, eps 1e-8) with given gradients (host, real layout). */
int pg_net_forward(pg_net* net, int batch, const float* in_dev, float* out_dev);
int pg_net_backward(pg_net* net, int batch, const float* gout_dev, float* gin_dev, float* gparams);
int pg_net_adam_step(pg_net* net, const float* grads, float lr);

/* The learned solver of one plan: the plan's operator and block Jacobi, the
 * network, and node_pixel [node_count] (host) mapping every node to a
 * distinct pixel y * width + x of the network's grid.  Neither the plan nor
 * the network may be destroyed before it. */
typedef struct pg_learned pg_learned;
int pg_learned_create(pg_plan* plan, pg_net* net, const int32_t* node_pixel, pg_learned** out);
void pg_learned_destroy(pg_learned* learned);

/* Residual/error pairs from solver output, on the device: for each of
 * `count` loads, r = F - K x_k (FP64 K) and e = x* - x_k, with x_k = 0 when
 * xk_dev is NULL.  F_dev [count][3n] float, xstar_dev / xk_dev [count][3n]
 * double, R_out / E_out [count][3n] float. */
int pg_learned_make_pairs(pg_learned* learned, int count, const float* F_dev, const double* xstar_dev,
                          const double* xk_dev, float* R_out, float* E_out);

#define PG_TRAIN_MAX_EPOCHS 256
typedef enum pg_loss {
    PG_LOSS_ENERGY = 0,    /* energy norm of the error after the correction:
                              (e1 - y)^T K (e1 - y) / e1^T K e1 */
    PG_LOSS_SCALED_L2 = 1, /* the same error in the network's output units:
                              |(e1 - y) / s_out|^2 / |e1 / s_out|^2 (its gradient is not
                              weighted by K, whose condition number makes the energy
                              loss's gradient descent slow on smooth errors) */
    PG_LOSS_SMOOTHED_ENERGY = 2 /* the energy norm of the error after the correction and the
                                   solve's two smoothing sweeps on it (w <- w + S (r1 - K w)):
                                   |M^2 (e1 - y)|_K^2 / |e1|_K^2, M = I - S K */
} pg_loss;
typedef struct pg_train_options {
    uint32_t struct_size;   /* sizeof(pg_train_options); set by pg_train_options_default */
    int32_t epochs;         /* default 20 */
    int32_t batch;          /* pairs per Adam step, default 32 */
    float lr;               /* Adam learning rate, default 1e-3 */
    int32_t cosine;         /* 1 (default): cosine decay of lr to 0 over the run */
    uint64_t seed;          /* shuffles */
    int32_t val_count;      /* the last val_count pairs are held out for the validation loss */
    int32_t set_scales;     /* 1 (default): set the network's scales from the pairs */
    int32_t loss;           /* pg_loss of the training steps, default PG_LOSS_ENERGY (the
                               validation loss is always PG_LOSS_SMOOTHED_ENERGY, the
                               quantity the solve depends on) */
} pg_train_options;

typedef struct pg_train_info {
    int32_t steps, batch;
    double loss_first_step, loss_last_step;   /* training loss of the first / last step */
    double val_loss_before, val_loss;         /* validation loss before / after training */
    double train_ms;                          /* device time of the training graphs */
    double total_ms;                          /* whole call, host clock */
    double epoch_loss[PG_TRAIN_MAX_EPOCHS];   /* mean training loss of each epoch */
    double epoch_val_loss[PG_TRAIN_MAX_EPOCHS];
} pg_train_info;

void pg_train_options_default(pg_train_options* opt);
/* Trains the network on `count` residual/error pairs (device, [count][3n]
 * float; A e = r): each pair is pre-smoothed (t = D^-1 r, r1 = r - K t,
 * e1 = e - t) and the network is trained with Adam to minimise the
 * energy-norm error after its correction, (e1 - y)^T K (e1 - y) / e1^T K e1
 * with y = N(r1), K applied by this library's own element kernels.  One
 * CUDA graph launch per epoch. */
int pg_learned_train(pg_learned* learned, int count, const float* R_dev, const float* E_dev,
                     const pg_train_options* opt, pg_train_info* info);
/* Test hook: the PG_LOSS_SMOOTHED_ENERGY loss of each of `count` pairs with
 * the current network (replaces the training set held by `learned`). */
int pg_learned_loss(pg_learned* learned, int count, const float* R_dev, const float* E_dev, double* loss_out);

typedef struct pg_learned_stats {
    int32_t mode;                /* as passed */
    int32_t network_iterations;  /* iterations whose network correction was used */
    int32_t network_off_at;      /* iteration after which the network was switched off, or -1 */
    int32_t replacements;        /* FP64 true-residual recomputations */
    int32_t pdl;                 /* 1 when the solve graph's kernels use programmatic dependent
                                    launch (each starts while its predecessor finishes) */
} pg_learned_stats;

/* Flexible PCG (Polak-Ribiere) with the two-level preconditioner
 * z = t + c y + S (r1 - c K y), t = S r, r1 = r - K t, y = N(r1),
 * S = omega D^-1 (omega = min(1, 1.5 / lambda_max(D^-1 K))) and
 * c = y.r1 / y.K y the step along the correction that most reduces the
 * energy norm of the error (mode 1); an iteration whose correction cannot
 * reduce it (y.r1 <= 0) uses z = D^-1 r, and after three such iterations in
 * a row the solve continues as plain block-Jacobi PCG.  mode 0: plain
 * block-Jacobi PCG in the same loop; mode 2: the smoothing steps without
 * the network (z = t + S r1).  FP32 vectors and BF16 network, FP64 x, dot products
 * and alpha/beta; the stop test (opt: tolerance, max_iterations,
 * stop_rule) is made on the FP64 true residual F - K x, which also
 * replaces the recursive residual every 50 iterations.  The whole solve is
 * one CUDA graph launch (a conditional WHILE node).
 * _device: F_dev / x_dev device [3n] float / double; otherwise host buffers
 * (copies included).  info->solve_ms is the graph's device time.  With
 * opt->phase_timing the iterations run without the graph, one launch at a
 * time with the host checking the stop flag after each, and
 * info->phase_us[0..7] receives the average device time per iteration of:
 * update; true residual; smoothing and network input; network; K y and the
 * sweeps; preconditioner; direction and K p; loop tick (a diagnostic mode:
 * profilers cannot look inside a graph with conditional nodes). */
int pg_learned_solve_device(pg_learned* learned, const pg_options* opt, int mode, const float* F_dev,
                            double* x_dev, pg_info* info, pg_learned_stats* stats);
int pg_learned_solve(pg_learned* learned, const pg_options* opt, int mode, const float* F, double* x_out,
                     pg_info* info, pg_learned_stats* stats);

/* y = K x by the FP32 operator the learned solver's flexible PCG applies
 * (the node-block form of K, summed in FP64 and rounded once, where every
 * node has at most 32 neighbours; else the element gather), constrained
 * rows replaced by the identity.  x, y: host [3n] float. */
int pg_learned_apply_k(pg_learned* learned, const float* x, float* y);

#ifdef __cplusplus
}
#endif

#endif /* PLATEGPU_H */
