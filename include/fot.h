/*
 * fot.h -- C ABI of the B200 indirect-increment loop engine (libfot.so).
 *
 * The engine runs the reference's indirect-increment loops (an iteration set
 * of "cells" -- edges, faces or elements -- each computing an increment from
 * direct and indirectly-addressed data and adding it to the "points" it maps
 * to) on one GPU.  It is the drop-in for the reference's Problem / Mesh /
 * data_t host API (problem.hpp, mesh.hpp, data_t.hpp) and its loop drivers;
 * include/fot_problem.hpp rebuilds that C++ surface on top of this ABI.
 *
 * Conventions
 *   - Every entry point returns an int status: FOT_OK (0) or a negative
 *     FOT_ERR_* code; fot_last_error() gives the message of the last failure
 *     on the calling thread.  Nothing here calls exit() (the reference's
 *     checkCudaErrors does, helper_cuda.h).
 *   - Handles are opaque.  A problem and its plans are thread-compatible, not
 *     thread-safe: use one handle from one thread (or serialise).
 *   - Streams are passed as void* (a cudaStream_t; NULL = the legacy default
 *     stream).  Launching calls are asynchronous; fot_sync() waits and reports
 *     device-side errors.
 *   - Arrays are plain host pointers with explicit element counts.
 *   - Types: mappings are uint32 (the reference's MY_SIZE); point and cell
 *     datasets have the element types of the loop (double, float, int).
 *
 * Data layout (the reference's, data_t.hpp:104-114 and kernels/*.hpp):
 *   mapping k        n_cells x mesh_dim[k] uint32, AOS (cell-major)
 *   point dataset k  n_points[k] x dim: AOS (point-major) when the problem's
 *                    layout is FOT_AOS, SOA (component-major) for FOT_SOA
 *   cell dataset j   always SOA: dim x n_cells
 * Point dataset 0 is the incremented dataset (point_weights[0]).
 */
#ifndef FOT_H
#define FOT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FOT_OK 0
#define FOT_ERR_ARG -1        /* invalid argument / size mismatch */
#define FOT_ERR_CUDA -2       /* a CUDA runtime call failed */
#define FOT_ERR_STATE -3      /* stale plan, wrong problem, ... */
#define FOT_ERR_LIMIT -4      /* an engine limit was exceeded (colours, sizes) */
#define FOT_ERR_DEVICE -5     /* a kernel reported an error (wait limit hit) */
#define FOT_ERR_NOMEM -6      /* device allocation failed */

/* loops: the reference's five applications (kernels/*_func.hpp) */
#define FOT_LOOP_RES_CALC 0  /* Airfoil edge flux, FP64 (kernels/res_calc.hpp) */
#define FOT_LOOP_MINI_AERO 1 /* miniAero face flux, FP64 (kernels/mini_aero.hpp) */
#define FOT_LOOP_LULESH 2    /* LULESH hex stress -> node force, FP64 (kernels/lulesh.hpp) */
#define FOT_LOOP_VOLNA 3     /* Volna edge flux, FP32 (kernels/volna.hpp) */
#define FOT_LOOP_GETACC 4    /* BookLeaf getacc scatter, FP64 (kernels/getacc_scatter.hpp) */
#define FOT_NUM_LOOPS 5

/* point-data layout: the reference's Problem<SOA> template parameter */
#define FOT_AOS 0
#define FOT_SOA 1

/* executors */
#define FOT_EXEC_ATOMIC 0      /* one launch, native atomics (+ warp aggregation) */
#define FOT_EXEC_HIER 1        /* two-level colouring, one persistent launch */
#define FOT_EXEC_HIER_LAUNCH 2 /* two-level colouring, one launch per block colour */

/* orderings (fot_reorder) */
#define FOT_ORDER_NATURAL 0 /* keep the point numbering, sort cells by point tuple */
#define FOT_ORDER_RANDOM 1  /* seeded random point numbering */
#define FOT_ORDER_RCM 2     /* reverse Cuthill-McKee */
#define FOT_ORDER_GPS 3     /* Gibbs-Poole-Stockmeyer (in place of SCOTCH "g") */

/* plan flags */
#define FOT_PLAN_NO_AGGREGATE 1u /* atomic executor: no warp aggregation */
#define FOT_PLAN_USE_PARTITION 2u /* hierarchical: blocks from the partition */
#define FOT_PLAN_DIRECT_READS 4u  /* hierarchical: gather read rows from HBM/L2 instead of
                                     staging them in shared memory (persistent executor:
                                     the direct split write-back kernel, one CTA per block) */
#define FOT_PLAN_SIMPLE_TILES 8u  /* persistent hierarchical: one tile at a time with a
                                     barrier per thread colour (no pipelining) */
#define FOT_PLAN_BLOCK_FLAGS 16u  /* persistent hierarchical: the pipelined kernel whose tiles
                                     wait for the per-block completion flags of the blocks
                                     they conflict with, all iterations in one launch (the
                                     default is the split write-back kernel: no tile waits,
                                     points shared by several blocks are summed in colour
                                     order by the next launch, one launch per iteration
                                     and a combine-only launch at the end of a call) */

typedef struct fot_problem fot_problem;
typedef struct fot_plan fot_plan;
typedef struct fot_graph fot_graph;
typedef struct fot_batch fot_batch;

/* Shape of a loop's data: the bindings of the reference drivers' initProblem
 * (res_calc.cu:10-28, mini_aero.cu:10-24, lulesh.cu:10-24, volna.cu:11-27,
 * getacc.cu:11-26). */
typedef struct fot_loop_info {
  uint32_t n_mappings;
  uint32_t mesh_dim[4];
  uint32_t n_point_sets; /* == n_mappings: point dataset k lives on mapping k */
  uint32_t point_dim[4];
  uint32_t point_type_size[4];
  uint32_t n_cell_sets;
  uint32_t cell_dim[8];
  uint32_t cell_type_size[8];
  uint32_t cell_written_mask; /* bit j set: cell dataset j is written (lulesh determ) */
} fot_loop_info;

/* Describe a loop's bindings.  Replaces the per-driver initProblem. */
int fot_loop_describe(int loop, fot_loop_info *info);

const char *fot_last_error(void);
const char *fot_version(void);

/* ---- problem (Problem<SOA> + Mesh + data_t) ---------------------------- */

/* Create a problem on the current CUDA device from host mappings.
 * Replaces Problem<SOA>(mesh streams, mesh_dim, point_data_params,
 * cell_data_params, block_size) (problem.hpp:59-77) and the Mesh stream
 * constructor (mesh.hpp:67-98).  n_points has n_mappings entries, maps[k]
 * n_cells*mesh_dim[k] entries.  Mappings whose point set the loop reads
 * through mapping 0 (res_calc 2, 3; mini_aero, lulesh, volna 1) must equal
 * mapping 0, as in the reference's inputs; the engine then keeps them as one. */
int fot_problem_create(int loop, int layout, uint32_t n_cells,
                       const uint32_t *n_points, const uint32_t *const *maps,
                       fot_problem **out);
int fot_problem_destroy(fot_problem *p);

/* Upload / download datasets in the problem's CURRENT numbering.
 * Replace Problem::readPointData / readCellData (problem.hpp:583-632) and
 * data_t::flushToDevice / flushToHost (data_t.cu:38-56).  bytes must equal
 * the dataset size.  The stream variants are asynchronous on `stream`
 * (host memory should be pinned); the plain ones synchronise. */
int fot_set_point_data(fot_problem *p, uint32_t k, const void *host, size_t bytes);
int fot_get_point_data(fot_problem *p, uint32_t k, void *host, size_t bytes);
int fot_set_cell_data(fot_problem *p, uint32_t j, const void *host, size_t bytes);
int fot_get_cell_data(fot_problem *p, uint32_t j, void *host, size_t bytes);
int fot_set_point_data_async(fot_problem *p, uint32_t k, const void *host, size_t bytes, void *stream);
int fot_get_point_data_async(fot_problem *p, uint32_t k, void *host, size_t bytes, void *stream);
int fot_set_cell_data_async(fot_problem *p, uint32_t j, const void *host, size_t bytes, void *stream);

/* Convert the problem's point datasets to `layout` (FOT_AOS or FOT_SOA) on the
 * GPU, in place of the reference's host conversion AOStoSOA
 * (data_t.hpp:249-275), both directions.  Plans built before become stale
 * (fot_run then fails with FOT_ERR_STATE); device addresses of the point
 * datasets change.  Synchronous. */
int fot_set_layout(fot_problem *p, int layout);

/* Device address of a dataset (owned by the problem; valid until the problem
 * is destroyed).  data_t::getDeviceData (data_t.hpp:48-52). */
int fot_point_data_device(fot_problem *p, uint32_t k, void **dptr);
int fot_cell_data_device(fot_problem *p, uint32_t j, void **dptr);

/* Current mapping k (n_cells*mesh_dim[k]) and sizes. */
int fot_get_mapping(fot_problem *p, uint32_t k, uint32_t *host);
int fot_problem_sizes(const fot_problem *p, uint32_t *n_cells, uint32_t *n_points /* [n_mappings] */);

/* Permutations applied so far.  point_perm[k][orig] = current number of
 * point `orig` of set k (the reference's applied_permutation, problem.hpp:35,
 * for k = 0); cell_order[current] = original cell id. */
int fot_get_point_permutation(fot_problem *p, uint32_t k, uint32_t *host);
int fot_get_cell_order(fot_problem *p, uint32_t *host);

/* ---- orderings and partitions (GPU plan builders) ----------------------- */

/* Renumber the points of mapping 0 by `order` (seed used by FOT_ORDER_RANDOM),
 * then sort the cells lexicographically by their sorted point tuples; the
 * other mappings follow: one equal to mapping 0 takes the same numbering,
 * another (res_calc's edge->node) is renumbered by first touch in the new cell
 * order.  Datasets move with their points and cells.  Replaces
 * Problem::reorder<SameMapping> (problem.hpp:439-482) with Mesh::reorder
 * (mesh.hpp:199-225) and SCOTCH's GPS ordering (reorder.hpp:135-175). */
int fot_reorder(fot_problem *p, int order, uint64_t seed);

/* Partition the cells into ceil(n_cells / part_size) parts on the GPU; the
 * partition is stored on the problem (Problem::partition_vector).  Replaces
 * Problem::partition / partitionOurs (problem.hpp:484-515), METIS k-way
 * (partition.cu:11-31) and the heuristic block growth (partition.cu:42-215).
 * Methods:
 *   FOT_PARTITION_BISECT  recursive graph bisection of the cell-to-cell graph
 *                         (each cut along a BFS front of the segment from a
 *                         far cell); parts within one cell of the mean size;
 *   FOT_PARTITION_GROW    parts grown from seeds over the cell-to-cell graph,
 *                         at most part_size cells each (more, smaller parts).
 * tolerance (>= 1): the reference's load-balance bound (METIS ubvec): with
 * BISECT no part exceeds tolerance x the mean size by more than one cell
 * (checked; FOT_ERR_STATE otherwise). */
#define FOT_PARTITION_BISECT 0
#define FOT_PARTITION_GROW 1
int fot_partition_tol(fot_problem *p, uint32_t part_size, float tolerance, int method);
/* fot_partition_tol(p, part_size, 1.001, FOT_PARTITION_BISECT); seed unused
 * (both methods are deterministic). */
int fot_partition(fot_problem *p, uint32_t part_size, uint64_t seed);
/* Quality of the problem's partition against mapping 0, on the GPU:
 * out[0] parts, out[1] largest / mean part size, out[2] (part, point) pairs
 * per point touched -- the points a hierarchical block stages and writes per
 * point, 1 when no point is shared --, out[3] the fraction of points touched
 * by more than one part. */
#define FOT_PARTITION_QUALITY 4
int fot_partition_quality(fot_problem *p, double *out, int n_out);
/* Problem::reorderToPartition (problem.hpp:517-526): cells sorted by part. */
int fot_reorder_to_partition(fot_problem *p);
/* Problem::renumberPoints (problem.hpp:528-551): points renumbered by the
 * number of parts touching them (descending) and then by part. */
int fot_renumber_points(fot_problem *p);
/* Partition vector (n_cells, current cell order); FOT_ERR_STATE when none. */
int fot_get_partition(fot_problem *p, uint32_t *host);
int fot_set_partition(fot_problem *p, const uint32_t *host);

/* ---- plans ---------------------------------------------------------------- */

typedef struct fot_plan_desc {
  int exec;            /* FOT_EXEC_* */
  uint32_t block_size; /* cells per block (hierarchical) / threads per CTA (atomic) */
  uint32_t flags;      /* FOT_PLAN_* */
  uint32_t reserved;
} fot_plan_desc;

typedef struct fot_plan_stats {
  int exec;
  uint32_t block_size;
  uint32_t n_blocks;
  uint32_t n_colours;          /* block colours */
  uint32_t max_block_points;   /* written points of the largest block */
  uint32_t max_block_points1;  /* second (read) mapping class, 0 if none */
  uint32_t max_thread_colours;
  double avg_thread_colours;
  double avg_block_points;     /* written points per block */
  uint64_t plan_bytes;         /* device bytes held by the plan */
  uint32_t smem_bytes;         /* dynamic shared memory per CTA */
  uint32_t grid;               /* CTAs per launch */
  double build_ms;             /* wall time of fot_plan_build */
  uint32_t shared_points;      /* split write-back: points written by more than one block */
  uint32_t partial_slots;      /* split write-back: (shared point, block) partial-sum slots */
  char kernel[32];             /* the kernel form that runs the plan */
} fot_plan_stats;

/* Build an execution plan on the GPU.  For the hierarchical executors this
 * replaces HierarchicalColourMemory (colouring.hpp:44-147, colouring.cu:12-102)
 * and REORDERS THE PROBLEM'S CELLS into plan order (blocks by block colour,
 * cells of a block by thread colour), recorded in fot_get_cell_order, so that
 * direct data are read coalesced.  A later plan build or reorder makes older
 * plans stale (fot_run then fails with FOT_ERR_STATE). */
int fot_plan_build(fot_problem *p, const fot_plan_desc *desc, fot_plan **out);
int fot_plan_destroy(fot_plan *plan);
int fot_plan_get_stats(const fot_plan *plan, fot_plan_stats *stats);

/* Export a hierarchical plan into host arrays (for exact checks):
 * colour_offsets[n_colours+1], block_start[n_blocks+1], cell_id[n_cells]
 * (original cell of each position), tcol[n_cells], block_ntcol[n_blocks],
 * pts_off[n_blocks+1], pts[pts_off[n_blocks]], lidx[mesh_dim*n_cells].
 * Call with pts == NULL to get the sizes only. */
int fot_plan_export(const fot_plan *plan, uint32_t *n_blocks, uint32_t *n_colours,
                    uint32_t *n_pts, uint32_t *colour_offsets, uint32_t *block_start,
                    uint32_t *cell_id, uint8_t *tcol, uint8_t *block_ntcol,
                    uint32_t *pts_off, uint32_t *pts, uint16_t *lidx);

/* ---- execution ------------------------------------------------------------ */

/* Run `iterations` iterations of the loop, accumulating into point dataset 0
 * on the device.  Replaces Problem::loopGPUCellCentred (problem.hpp:90-194)
 * and loopGPUHierarchical (problem.hpp:198-339) without their per-colour
 * cudaDeviceSynchronize and the per-iteration copy-back.  Asynchronous. */
int fot_run(fot_problem *p, fot_plan *plan, uint32_t iterations, void *stream);
/* Wait for the problem's work on `stream` and report device-side errors. */
int fot_sync(fot_problem *p, void *stream);

/* Fault injection for tests of the failure path (no counterpart in the
 * reference).  Zeroes the completion flag of `block` (plan order) of a
 * block-flag hierarchical plan (FOT_PLAN_BLOCK_FLAGS; FOT_ERR_STATE for
 * other plans, whose kernels read no flags) that has run at least once, as if the block's
 * last completion had been lost.  In the next fot_run the tiles that depend
 * on the block wait for it until their time limit (about 2 s), the kernel
 * returns early, and fot_sync reports FOT_ERR_DEVICE and resets the plan's
 * queue and flags: the problem's data are then undefined, the plan and the
 * CUDA context stay usable.  Synchronous. */
int fot_plan_inject_lost_flag(fot_plan *plan, uint32_t block);

/* Capture `iterations` iterations of fot_run into a CUDA graph and replay it. */
int fot_graph_create(fot_problem *p, fot_plan *plan, uint32_t iterations,
                     void *stream, fot_graph **out);
/* A graph replays the device addresses it was captured with: once its
 * problem is renumbered (fot_reorder, another plan build, fot_set_layout,
 * ...) or destroyed, fot_graph_launch refuses it with FOT_ERR_STATE.  A
 * graph must be destroyed before the plan (and the Airfoil step) it was
 * captured from. */
int fot_graph_launch(fot_graph *g, void *stream);
int fot_graph_destroy(fot_graph *g);

/* ---- row lists: the device side of a partitioned (multi-GPU) run -------- */

/* The reference runs one mesh on one GPU.  A mesh split by cells into parts
 * (fot_partition) runs one part per GPU: each part's problem holds its cells
 * and every point they touch; a point touched by several parts is owned by
 * one, and the increments the others add to their copies travel to the owner
 * after the loop (cuda_fot_b200/halo.py does the split and the exchange over
 * torch.distributed).  A row list is a set of DISTINCT rows of point dataset
 * k (current numbering, checked, kept on the device): gather packs them into
 * `dst` (device, rows x dim elements, AOS, list order); scatter_add adds such
 * a packed buffer into the dataset.  Lists become stale
 * (FOT_ERR_STATE) when the problem is renumbered. */
typedef struct fot_rowlist fot_rowlist;
int fot_rowlist_create(fot_problem *p, uint32_t k, const uint32_t *rows, uint32_t n, fot_rowlist **out);
int fot_rowlist_gather(const fot_rowlist *l, void *dst, void *stream);
int fot_rowlist_scatter_add(const fot_rowlist *l, const void *src, void *stream);
int fot_rowlist_destroy(fot_rowlist *l);

/* ---- the Airfoil time step around res_calc ------------------------------ */

/* The reference drives res_calc alone (res_calc.cu: Problem::loop*(num)).  An
 * Airfoil solver iteration runs, on a res_calc problem's data (res = point set
 * 0, x = 1 (nodes), q = 2, adt = 3, current numbering and layout):
 *   save_soln  qold = q
 *   2 x { adt_calc   per cell: adt = sum over its four sides (node j to j+1)
 *                    of |u dy - v dx| + c |side|, divided by cfl
 *                    (u, v = velocity, c = sound speed, gamma 1.4);
 *         res_calc   one iteration of `plan` (atomic or hierarchical);
 *         bres_calc  per boundary edge, in edge order per cell: a wall adds
 *                    the pressure flux (res[1] += p dy, res[2] -= p dx), a
 *                    far-field edge the res_calc flux against qinf with
 *                    dissipation adt * 0.05;
 *         update     per cell: d = res / adt; q = qold - d; res = 0 }
 * and reports rms = sqrt(sum of d^2 / cells) of the second stage.  Boundary
 * edges are oriented like res_calc's edges: with dx = x1 - x2, dy = y1 - y2
 * the normal (dy, -dx) points out of the cell.  Every sum has a fixed order,
 * so with a hierarchical plan a run is bit-reproducible. */
typedef struct fot_airfoil fot_airfoil;
typedef struct fot_airfoil_desc {
  const uint32_t *cell_to_node;  /* cells x 4 nodes, counter-clockwise (original numbering) */
  uint32_t n_bedges;
  const uint32_t *bedge_to_node; /* n_bedges x 2: node 1, node 2 */
  const uint32_t *bedge_to_cell; /* n_bedges */
  const int32_t *bound;          /* n_bedges: 1 = solid wall, otherwise far field */
  double qinf[4];                /* free stream (rho, rho u, rho v, rho E) */
  double cfl;
} fot_airfoil_desc;
/* Checks every index against the problem's sizes; renumbers the maps whenever
 * the problem's numbering changes (fot_reorder, fot_renumber_points, ...). */
int fot_airfoil_create(fot_problem *p, const fot_airfoil_desc *desc, fot_airfoil **out);
/* `iterations` solver iterations on `stream`; rms (host, may be NULL) receives
 * the last iteration's rms after the stream is synchronised. */
int fot_airfoil_run(fot_airfoil *a, fot_plan *plan, uint32_t iterations, double *rms, void *stream);
/* The whole time loop as one CUDA graph: `iterations` solver iterations
 * captured from `stream` (the problem's numbering is brought up to date
 * first); fot_graph_launch replays them, fot_airfoil_get_rms then reads the
 * last iteration's rms (synchronising `stream`). */
int fot_airfoil_graph_create(fot_airfoil *a, fot_plan *plan, uint32_t iterations, void *stream,
                             fot_graph **out);
int fot_airfoil_get_rms(fot_airfoil *a, double *rms, void *stream);
int fot_airfoil_destroy(fot_airfoil *a);

/* ---- batches: many meshes, one persistent launch -------------------------- */

/* Group the plans of several problems into one launch per fot_batch_run.
 * Hierarchical plans: one persistent launch over a (mesh, block) tile queue
 * ordered by block colour per mesh; each mesh's result is that of its own
 * plan.  Atomic plans (all with or all without warp aggregation): one launch
 * over tiles of 1,024 cells of every mesh and every iteration.  A batch holds
 * one executor kind, one layout, and one loop kind or res_calc with volna.
 * No counterpart in the reference (one mesh per process). */
int fot_batch_create(fot_problem *const *problems, fot_plan *const *plans,
                     uint32_t n, fot_batch **out);
int fot_batch_run(fot_batch *b, uint32_t iterations, void *stream);
int fot_batch_sync(fot_batch *b, void *stream);
int fot_batch_destroy(fot_batch *b);

/* ---- mesh statistics: the sector model and the cost model's mesh features - */

/* Statistics of mapping 0 in the problem's CURRENT numbering, on the GPU:
 * out[0] the largest and out[1] the mean spread (max - min point number) of a
 * cell's row; out[2..5] the fractions of points of degree <= 2, 3-4, 5-6 and
 * >= 7.  n_out >= FOT_MESH_FEATURES.  No counterpart in the reference (its
 * orderings report bandwidth on the host, reorder.hpp). */
#define FOT_MESH_FEATURES 6
int fot_mesh_features(fot_problem *p, double *out, int n_out);

/* The reference's sector model, countCacheLinesForBlock (problem.hpp:654-672)
 * as its global-colouring loop applies it (problem.hpp:145-152): for blocks of
 * `cells_per_block` consecutive cells (current order), the distinct 32-byte
 * sectors of point dataset 0 that their points touch -- AOS: every element
 * of every row; SOA: distinct p / (32 / type size), times the dimension --
 * summed over the blocks.  layout: FOT_AOS, FOT_SOA, or -1 for the problem's.
 * The reference prints sectors * 32 * 2 per iteration as its "cache line"
 * bandwidth (problem.hpp:191-192). */
int fot_sector_count(fot_problem *p, uint32_t cells_per_block, int layout, uint64_t *sectors,
                     uint64_t *blocks);
/* The same over a hierarchical plan's blocks and their written points, as
 * loopGPUHierarchical applies it to points_to_be_cached (problem.hpp:233-240). */
int fot_plan_sector_count(const fot_plan *plan, int layout, uint64_t *sectors, uint64_t *blocks);

/* ---- the learned plan cost model ------------------------------------------- */

/* A 24 -> 64 -> 64 -> 1 ReLU MLP (FP32) predicting log(seconds per
 * iteration) of a candidate plan from its feature vector; trained with the
 * engine's own forward / backward / Adam kernels on timings the autotuner
 * measured.  No counterpart in the reference. */
#define FOT_MODEL_FEATURES 24
#define FOT_MODEL_HIDDEN 64

typedef struct fot_model fot_model;

int fot_model_create(uint64_t seed, fot_model **out);
int fot_model_destroy(fot_model *m);
int fot_model_num_params(void);
int fot_model_set_params(fot_model *m, const float *params);
int fot_model_get_params(const fot_model *m, float *params);
/* per-feature mean and standard deviation used to standardise inputs */
int fot_model_set_normalisation(fot_model *m, const float *mean, const float *stddev);
/* y[i] = model(X[i]) for n feature rows X (n x FOT_MODEL_FEATURES) */
int fot_model_predict(fot_model *m, const float *X, int n, float *y);

/* fot_model_predict without any device allocation (no counterpart in the
 * reference).  For callers that must not allocate device memory once they
 * are running: the inputs and outputs of the call are staged in a fixed
 * file-scope device array of FOT_MODEL_NOALLOC_MAX_ROWS rows (25 floats per
 * row, 409,600 bytes) instead of buffers allocated per call.  The array
 * exists on a device once the library's module is loaded there -- with
 * CUDA's lazy module loading, from the first use on that device -- and stays
 * until the process exits.  More rows than the maximum: FOT_ERR_LIMIT,
 * nothing is computed.  No part of the array has to start at zero (a call
 * writes every row it reads).  All calls on one device share the array, so
 * calls that overlap in time (from several host threads) race and must be
 * serialised by the caller.  The first call on a device does the setup
 * (looks up the array's address, sets the kernel's shared-memory limit) and
 * should come before any stream capture.  Same results as
 * fot_model_predict.  Synchronous: inputs and outputs move with cudaMemcpy
 * and the kernel runs on the legacy default stream. */
#define FOT_MODEL_NOALLOC_MAX_ROWS 4096
int fot_model_predict_noalloc(fot_model *m, const float *X, int n, float *y);
/* gradient of 0.5/n * sum (model(X) - t)^2 w.r.t. the parameters, and the loss */
int fot_model_grad(fot_model *m, const float *X, const float *t, int n, float *grad, float *loss);
/* `epochs` passes of Adam over contiguous minibatches of `batch` rows;
 * epoch_loss (optional) receives the full-set loss after each epoch */
int fot_model_train(fot_model *m, const float *X, const float *t, int n, int epochs, int batch,
                    float lr, float weight_decay, float *epoch_loss);

#ifdef __cplusplus
}
#endif
#endif /* FOT_H */
