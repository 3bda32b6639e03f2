/* pgc.h -- C ABI of the sm_100a cycle-search library (libpgc.so).
 *
 * One handle is one product_graph_generator of the reference (class
 * ProductGraphGenerators, product_graph_generators/product_graph_generators.hpp:21-91,
 * bound to Python at pythonbinding/bindings.cpp:32-48 and to MATLAB at
 * mex/product_graph_generator_mex.cpp:29-151).  Each entry point below names
 * the reference member it replaces.
 *
 * Conventions
 *  - Matrices are dense, row-major (C order); indices are 0-based int32.
 *  - Every function returns PGC_OK (0) or a negative PGC_ERR_* code; the
 *    message of the last failure of the calling thread is pgc_last_error().
 *    Nothing calls exit().  A null handle, or a null pointer where an array
 *    is read or written, returns PGC_ERR_ARG.
 *  - A handle is not thread-safe; distinct handles may be used from
 *    distinct threads.  All device work of a handle runs on one CUDA stream
 *    of the device that was current when the handle was created.
 *  - All solver names of the reference are accepted.  "lawlercpu" and
 *    "lawlergpu" both run the sm_100a ratio solver, "dijkstracpu" and
 *    "dijkstragpu" (and, as in the reference, any other name) the sm_100a
 *    minimum-cost solver; their results are identical by construction.
 *    "export" writes the inputs as CSV files, as the reference does.
 */
#ifndef PGC_H
#define PGC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGC_OK 0
#define PGC_ERR_ARG -1        /* bad shape, index or argument */
#define PGC_ERR_STATE -2      /* call not allowed in the current state */
#define PGC_ERR_MODE -3       /* unsupported (cost, time) mode */
#define PGC_ERR_SOLVER -4     /* unknown ratio-solver name */
#define PGC_ERR_CUDA -5       /* CUDA runtime error (message has details) */
#define PGC_ERR_INTERNAL -6   /* solver invariant broken (message has details) */
#define PGC_ERR_TIMEOUT -7    /* a bounded device wait ran out */

typedef struct pgc_graph pgc_graph;

/* ProductGraphGenerators(VX, EX, VY, EY, featDiff, conjugate, regulariser[, pruneIntralayer])
 * product_graph_generators.hpp:65-66, bindings.cpp:33-34.
 * VX [nvx x 3] f64, EX [nex x 2] i32 (both orientations of every mesh edge),
 * VY [nvy x 3] f64, EY [ney x 2] i32 (ordered closed curve),
 * feat_diff [nvx x nvy] f64.  Inputs are copied. */
int pgc_create(const double* VX, int64_t nvx, const int32_t* EX, int64_t nex, const double* VY, int64_t nvy,
               const int32_t* EY, int64_t ney, const double* feat_diff, int use_conjugate_graph,
               int use_regularising_cost_term, int prune_intralayer, pgc_graph** out);

/* ~ProductGraphGenerators (product_graph_generators.hpp:67). */
void pgc_destroy(pgc_graph* g);

/* setNormals(NX, NY) -- product_graph_generators.cpp:118-130, bindings.cpp:38.
 * NX [rows_x x cols_x], NY [rows_y x cols_y]; the shapes must be |VX| x 3 and |VY| x 3. */
int pgc_set_normals(pgc_graph* g, const double* NX, int64_t rows_x, int64_t cols_x, const double* NY,
                    int64_t rows_y, int64_t cols_y);

/* setMaxDepth(k) -- product_graph_generators.cpp:305-307, bindings.cpp:47. */
int pgc_set_max_depth(pgc_graph* g, int max_depth);

/* setCostTimeRatioMode(costName, timeName) -- product_graph_generators.cpp:309-312, bindings.cpp:48. */
int pgc_set_cost_time_ratio_mode(pgc_graph* g, const char* cost_name, const char* time_name);

/* updateRobustLossParams(alpha, c, pwr) -- product_graph_generators.cpp:259-270, bindings.cpp:37.
 * Ignored for the plain graph and after generate(), as in the reference. */
int pgc_update_robust_loss_params(pgc_graph* g, double alpha, double c, double pwr);

/* Runs all device work of the handle on the given cudaStream_t (passed as a
 * pointer; NULL restores the handle's own stream).  No reference counterpart:
 * lets a caller order the solver with its own work and time it with events. */
int pgc_set_stream(pgc_graph* g, void* cuda_stream);

/* generate() -- product_graph_generators.cpp:21-89, bindings.cpp:35.
 * Builds the product graph and its edge costs on the device. */
int pgc_generate(pgc_graph* g);

/* getCostVector() -- product_graph_generators.cpp:138-143, bindings.cpp:36.
 * Shape query, then copy of the [rows x cols] cost matrix in edge-id order.
 * A ratio solve rescales these costs in place, as the reference does. */
int pgc_cost_vector_shape(pgc_graph* g, int64_t* rows, int64_t* cols);
int pgc_get_cost_vector(pgc_graph* g, double* out);

/* No counterpart in the reference.  pgc_get_cost_vector for callers that
 * cannot let this library allocate device memory: processes whose GPU memory
 * is already reserved by their own allocator (a PyTorch job's caching
 * allocator, a serving engine that pre-reserves most of HBM), where a
 * cudaMalloc would fail or make that allocator release memory, and loops that
 * cannot afford the device-wide synchronization of cudaFree.  The export
 * kernel writes into a fixed device scratch -- a file-scope array of 2^21
 * doubles (16 MiB) that every GPU loading the library holds until exit --
 * which is then copied to `out`.  Nothing is allocated and nothing is
 * generated: the graph's costs must exist already (PGC_ERR_STATE otherwise)
 * and rows x cols must be at most 2^21 (PGC_ERR_ARG otherwise).  Nothing
 * needs clearing first: the export writes every value.  The first call on a
 * device takes the scratch's device address (cudaGetSymbolAddress, that
 * device current) and keeps it for the life of the process; make that first
 * call before any stream capture.  A device reset (cudaDeviceReset, or
 * anything else that destroys the device's primary context) invalidates that
 * address: do not call this entry point on a device after resetting it in the
 * same process.  Every call shares the one scratch of its device, so calls
 * that overlap on the GPU race on it. */
int pgc_get_cost_vector_noalloc(pgc_graph* g, double* out);

/* getProductSpace() -- product_graph_generators.cpp:173-178, bindings.cpp:39.
 * [rows x 4] (plain) or [rows x 6] (conjugate) int32 edge table. */
int pgc_product_space_shape(pgc_graph* g, int64_t* rows, int64_t* cols);
int pgc_get_product_space(pgc_graph* g, int32_t* out);

/* solveWithCostTimeRatio(name, k) -- product_graph_generators.cpp:284-303, bindings.cpp:41-42;
 * CostTimeRatioSolver::run, cost_time_ratio_solver.cpp:868-900.
 * max_depth < 1 uses the stored depth (the one-argument overload).
 * The result (passes_layers_just_once, final_objective, matching) is kept in
 * the handle and read with pgc_result_*. */
int pgc_solve_with_cost_time_ratio(pgc_graph* g, const char* solver_name, int max_depth);

/* solveWithDijkstra(name, k) -- product_graph_generators.cpp:314-333, bindings.cpp:44-45;
 * DijkstraSolver::run, dijkstra_solver.cpp:563-579. */
int pgc_solve_with_minimum_cost(pgc_graph* g, const char* solver_name, int max_depth);

/* No reference counterpart.  Adjoint of the last solve's objective with
 * respect to feat_diff: adds (accumulate != 0) or writes grad_objective *
 * d objective / d feat_diff into the DEVICE buffer grad_feat_diff
 * [|VX| x |VY|] f64 of the handle's device.  Ratio: d lambda* / d c_e =
 * 1[e in cycle] / T(cycle) over the rescaled costs; minimum cost:
 * 1[e in cycle].  The rescale factor is held fixed and its rounding passed
 * straight through; the energy's adjoint scatters every cycle edge into the
 * feat_diff entries its cost reads (plain graph: two; conjugate graph:
 * fd[x2, y2] in the ("vanilla", *) and ("feature", *) modes, none in the
 * others; a ratio whose time column reads feat_diff, ("*", "feature") with
 * t = max(0, maxFd - fd), adds its time part and puts the subgradient of
 * maxFd on the matrix maximum's first entry).  PGC_ERR_STATE without a
 * result. */
int pgc_backward_feat_diff(pgc_graph* g, double grad_objective, double* grad_feat_diff, int accumulate);

/* No reference counterpart.  pgc_backward_feat_diff for `count` distinct
 * graphs (grad_objectives[i], grad_feat_diffs[i] a device buffer of graph i):
 * the adjoint kernels are enqueued on the graphs' streams, then each stream
 * is waited for once. */
int pgc_backward_feat_diff_batch(pgc_graph* const* graphs, int64_t count, const double* grad_objectives,
                                 double* const* grad_feat_diffs, int accumulate);

/* No reference counterpart (the oracle's setCostVector).  Sets the edge costs
 * [rows x cols] (rows = nY * edges per layer block, in edge-id order, cols 1
 * or 2) in place of generate(); solves then use (and rescale) them. */
int pgc_set_cost_vector(pgc_graph* g, const double* costs, int64_t rows, int64_t cols);

/* No reference counterpart.  Replaces feat_diff [|VX| x |VY|]; the next solve
 * regenerates the costs.  Lets one handle serve many training steps. */
int pgc_set_feat_diff(pgc_graph* g, const double* feat_diff, int64_t rows, int64_t cols);

/* No reference counterpart.  pgc_set_feat_diff from DEVICE memory (row-major
 * float64 on the handle's GPU): one device-to-device copy on the handle's
 * stream, complete when the call returns, so the buffer may be freed then.
 * The caller orders the buffer's producer before the call (synchronize the
 * producing stream, or give the handle that stream with pgc_set_stream). */
int pgc_set_feat_diff_device(pgc_graph* g, const double* feat_diff, int64_t rows, int64_t cols);

/* No reference counterpart.  pgc_set_feat_diff_device for `count` distinct
 * graphs (feat_diffs[i] is graph i's |VX| x |VY| matrix on its device): the
 * copies are enqueued on the graphs' streams and waited for once each. */
int pgc_set_feat_diff_device_batch(pgc_graph* const* graphs, int64_t count, const double* const* feat_diffs);

/* No reference counterpart.  Most CTAs one Bellman-Ford launch of this graph
 * may use (0, the default: as many as shorten a step).  A small team is
 * slower per solve but leaves the rest of the GPU to other graphs. */
int pgc_set_team_cap(pgc_graph* g, int max_ctas);

/* No reference counterpart.  The Bellman-Ford team of this graph: ctas CTAs
 * of threads_per_cta threads (a multiple of 32 in [32, 640]); 0 leaves
 * either automatic.  Set by the autotuner (cyclic_product_graphs.autotune);
 * results do not depend on it. */
int pgc_set_team_shape(pgc_graph* g, int ctas, int threads_per_cta);

/* No reference counterpart.  Solves `count` graphs concurrently, each with
 * the result pgc_solve_with_cost_time_ratio (solver "lawlercpu"/"lawlergpu")
 * or pgc_solve_with_minimum_cost (any other name) would give it.
 * Ratio solvers: `workers` host threads (0: 64) generate and rescale every
 * graph's costs; then one persistent launch runs each graph's whole ratio
 * solve on the device, teams of `ctas_per_graph` CTAs (0: the environment's
 * PGC_BATCH_TEAM, else 8) taking the graphs largest first; a graph whose
 * first-branch cycle wraps is finished on the host with branch and bound.
 * PGC_BATCH_STREAMS=1 selects the route of the other solvers instead.
 * Other solvers: each graph on its own stream with a team of at most
 * `ctas_per_graph` CTAs (0: SMs / min(count, 32)); graphs run side by side
 * only as far as the device has host work queues, so start the process with
 * CUDA_DEVICE_MAX_CONNECTIONS=32 (CUDA's default of 8 runs such a batch about
 * 3x slower).  With `regenerate` != 0 each graph first recomputes its edge
 * costs (pgc_generate).  Each graph's result is read afterwards with
 * pgc_result*; status[i] receives its return code.  Returns PGC_OK when all
 * succeeded, else the first failure's code (with its message).  The handles
 * must be distinct. */
int pgc_solve_batch(pgc_graph* const* graphs, int64_t count, const char* solver_name, int max_depth,
                    int ctas_per_graph, int workers, int regenerate, int* status);

/* No reference counterpart.  Kernel launches the library has issued in this
 * process so far, on every device and thread (a counter that only grows). */
int pgc_kernel_launches(int64_t* out);

/* No reference counterpart.  Where the calling thread's last
 * pgc_solve_batch spent its time (host wall clock, ms) when it solved ratio
 * cycles in one launch: out8 = {costs generated and rescaled, teams
 * prepared; the launch and its results read back; results taken over or
 * finished on the host; graphs handed back to the host; graphs solved on the
 * device; CTAs launched; threads per CTA; dynamic shared memory per CTA}.
 * All zero after the per-graph-stream route. */
int pgc_batch_profile(double* out8);

/* The CTR_CYCLE_SOLVER_OUTPUT / DIJKSTRA_SOLVER_OUTPUT tuple
 * (cost_time_ratio_solver.hpp:70, dijkstra_solver.hpp:22) of the last solve. */
int pgc_result(pgc_graph* g, int* passes_layers_just_once, float* final_objective, int64_t* rows, int64_t* cols);
int pgc_result_matching(pgc_graph* g, int32_t* out);
/* Edge ids (rows of the product space) of the returned cycle, in matching order. */
int pgc_result_cycle_edges(pgc_graph* g, int64_t* out, int64_t capacity, int64_t* count);

/* Counters of the last solve: [bf_calls, sweeps, candidates, lawler_iterations,
 * branches, fallback_walks, device_ms_x1000, kernel_launches]. */
int pgc_result_stats(pgc_graph* g, int64_t* out8);

/* Profile of the last solve's Bellman-Ford launches (no reference
 * counterpart).  SM cycles seen by one thread of the first CTA:
 * [0] relaxation, [1] sweep bookkeeping, [2] step hand-offs and barriers,
 * [3] sweep tail (wrap-around and cycle detection); [4] (layer, depth) steps
 * run; team shape of the last launch: [5] CTAs, [6] threads per CTA,
 * [7] wait-list entries over all CTAs. */
int pgc_result_profile(pgc_graph* g, int64_t* out8);
/* No reference counterpart.  Parts of pgc_result_profile's counters (SM
 * cycles of CTA 0's thread 0, summed over the last solve): out4 = {waits
 * for staged streams (part of the relaxation), and the sweep tail's
 * wrap-around with lap function, candidate walks, and the lead's choice
 * with cycle extraction}. */
int pgc_result_profile_detail(pgc_graph* g, int64_t* out4);

/* utils::normals2d (helper/utils.cpp:93-157, bindings.cpp:27): outward
 * vertex normals of an ordered closed curve lying in a coordinate plane.
 * V [nv x 3], E [ne x 2] with ne == nv; out [nv x 3]. */
int pgc_compute_normals_2d(const double* V, int64_t nv, const int32_t* E, int64_t ne, double* out);

/* No reference counterpart.  Sizes of the product graph of X (EX [nex x 2],
 * |VX| = nvx) with a closed curve of ney edges, built on the host without a
 * GPU: out6 = {nodes per layer, edges per block (= per Y edge), interlayer
 * edges per block, intralayer edges per block, 32-node slices, sliced-ELL
 * rows of both parts}.  The product graph has ney * out6[1] edges, the rows
 * of the reference's productspace. */
int pgc_product_graph_sizes(const int32_t* EX, int64_t nex, int64_t nvx, int64_t ney, int conjugate,
                            int prune_intralayer_edges, int64_t* out6);

/* utils::normals3d (helper/utils.cpp:86-90, bindings.cpp:26): area-weighted
 * vertex normals of a triangle mesh (libigl per_vertex_normals with its
 * default weighting).  V [nv x 3], F [nf x 3]; out [nv x 3]. */
int pgc_compute_normals_3d(const double* V, int64_t nv, const int32_t* F, int64_t nf, double* out);

/* Sizes of the generated graph (no reference counterpart): [nodes per layer,
 * layers, edges per Y edge, interlayer edges per layer, intralayer edges per
 * layer, interlayer slots per layer, intralayer slots per layer (slots include
 * the sliced-ELL padding), cost columns]. */
int pgc_graph_info(pgc_graph* g, int64_t* out8);

/* No reference counterpart.  Name of the GPU the handle's device work runs
 * on (cudaDeviceProp::name), NUL-terminated and cut to capacity - 1 bytes.
 * The autotuner keys its cache by it, so a cache file written on one GPU type
 * is not applied on another. */
int pgc_device_name(pgc_graph* g, char* out, int64_t capacity);

/* Returns the device memory and the pinned host memory cached by the
 * library's allocators to CUDA (no reference counterpart; freed buffers are
 * otherwise kept for reuse). */
int pgc_release_cached_memory(void);

/* Message of the last failing call on this thread ("" if none). */
const char* pgc_last_error(void);

/* Library version string. */
const char* pgc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PGC_H */
