// Host-side structures of libfot: problems, plans, the per-loop dispatch
// table and the helpers shared by the plan builders and the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "executors.cuh"

namespace fot {

// Shared-memory layout of a hierarchical tile kernel.
struct SmemLayout {
  uint32_t read_off[4] = {0, 0, 0, 0}; // read set rows (relative to a pipeline buffer)
  uint32_t pts_off = 0;                // point lists (non-pipelined kernels)
  uint32_t acc_off = 0;                // accumulator (non-pipelined kernels)
  // pipelined kernel: 4 record slots, 2 read-row slots, the increments,
  // 2 output-row slots
  uint32_t rec_slot = 0, rows_off = 0, rows_bytes = 0;
  uint32_t inc_off = 0, outbuf_off = 0, outbuf_bytes = 0;
  size_t total = 0;                    // bytes per CTA
};

// Per-loop entry points, one table per loop translation unit (loop_*.cu).
// `variant` selects the hierarchical tile kernel: bit 0 = stage the read rows
// in shared memory (else gather them straight from HBM/L2); bit 1 = the
// pipelined persistent kernel (warp-specialised: tile records by bulk copy,
// double-buffered staging, per-point gather of the increments), launched
// with 64 threads more than `threads` for its two control warps; bit 2 = that
// kernel with three tile-record slots (else two); bit 3 = split write-back
// (hier_split.cuh, one launch per iteration): with bit 1 the warp-specialised
// staged form (same control warps and slot counts), without it the direct
// form (one CTA per tile, rows gathered straight from HBM/L2).
constexpr uint32_t kVariantStage = 1u, kVariantPipe = 2u, kVariantSlots3 = 4u, kVariantSplit = 8u;

struct LoopOps {
  // launch one iteration of the atomic executor
  int (*run_atomic)(const LoopData &d, bool soa, bool aggregate, uint32_t threads,
                    uint32_t grid, cudaStream_t st);
  // persistent hierarchical launch over P.total_tiles tiles
  int (*run_hier)(const LoopData &d, const HierPlanDev &P, bool soa, uint32_t threads,
                  uint32_t variant, uint32_t grid, size_t smem, cudaStream_t st);
  // one launch per block colour: blocks [first, first + count)
  int (*run_hier_colour)(const LoopData &d, const HierPlanDev &P, bool soa,
                         uint32_t threads, uint32_t variant, uint32_t first, uint32_t count,
                         size_t smem, cudaStream_t st);
  // resident CTAs per SM of an executor configuration (0 if it cannot launch)
  int (*occupancy)(int exec, bool soa, uint32_t threads, uint32_t variant, size_t smem,
                   int *per_sm);
  // shared-memory layout of a hierarchical tile for at most cap0 / cap1
  // points per block and tile records of at most rec_cap bytes
  void (*smem_layout)(uint32_t cap0, uint32_t cap1, uint32_t variant, uint32_t rec_cap,
                      uint32_t threads, SmemLayout *out);
};

const LoopOps *loop_ops(int loop);

// threads per CTA of the hierarchical kernels for a block size
inline uint32_t hier_threads(uint32_t block_size) {
  if (block_size <= 128) return 128;
  if (block_size <= 256) return 256;
  if (block_size <= 512) return 512;
  return 1024;
}

// mapping class of point set k: 1 only for res_calc's edge->node set
inline int set_class(int loop, uint32_t k) {
  return (loop == FOT_LOOP_RES_CALC && k == 1) ? 1 : 0;
}

int device_sm_count();

} // namespace fot

struct fot_problem {
  int loop = 0;
  int layout = FOT_AOS;
  fot_loop_info info{};
  uint32_t n_cells = 0;
  uint32_t n_points[4] = {0, 0, 0, 0};
  bool has_class1 = false;
  fot::DevBuf map[2];   // class 0 (mapping 0) and class 1, AOS u32, current order
  fot::DevBuf point[4]; // point datasets, current point numbering
  fot::DevBuf cell[8];  // cell datasets, SOA, current cell order
  std::vector<uint32_t> point_perm[2]; // per class: original point -> current
  std::vector<uint32_t> cell_order;    // current cell -> original cell
  std::vector<uint32_t> partition;     // part of each cell (current order), may be empty
  uint64_t version = 1; // bumped whenever cells or points are renumbered
  int device = 0;
  // plans with a device control block run since the last fot_sync
  std::vector<struct fot_plan *> pending;
  // live plans built on this problem (told when the problem is destroyed)
  std::vector<struct fot_plan *> plans;
  // live Airfoil steps on this problem (told when the problem is destroyed)
  std::vector<struct fot_airfoil *> airfoils;
  // live row lists of this problem's datasets (told when it is destroyed)
  std::vector<struct fot_rowlist *> rowlists;

  size_t point_bytes(uint32_t k) const {
    return (size_t)n_points[k] * info.point_dim[k] * info.point_type_size[k];
  }
  size_t cell_bytes(uint32_t j) const {
    return (size_t)n_cells * info.cell_dim[j] * info.cell_type_size[j];
  }
  uint32_t class_points(int c) const { return c == 0 ? n_points[0] : n_points[1]; }
  uint32_t mesh_dim() const { return info.mesh_dim[0]; }
  fot::LoopData loop_data() const;
};

// An Airfoil step whose problem is being destroyed (fails from now on).
void fot_airfoil_detach(struct fot_airfoil *a);
// A row list whose problem is being destroyed (fails from now on).
void fot_rowlist_detach(struct fot_rowlist *l);

namespace fot {
// Capture into a new fot_graph what enqueue(ctx, stream) launches (on a
// private non-blocking stream when st is the legacy default stream).
int capture_graph(cudaStream_t st, int (*enqueue)(void *ctx, cudaStream_t st), void *ctx,
                  fot_graph **out);
} // namespace fot

struct fot_plan {
  fot_problem *prob = nullptr;
  uint64_t version = 0;
  fot_plan_desc desc{};
  fot_plan_stats stats{};
  uint32_t variant = 0; // hierarchical tile kernel variant (see LoopOps)
  int point_layout = FOT_AOS; // the problem's point layout when the plan was built
  // hierarchical plans
  uint32_t n_blocks = 0, n_colours = 0;
  std::vector<uint32_t> colour_offsets; // host copy (n_colours + 1)
  fot::DevBuf block_start, block_wait, block_ntcol, tcol;
  fot::DevBuf pts_off[2], pts[2], lidx[2];
  fot::DevBuf build_perm; // position -> cell index before the build
  fot::DevBuf rec, rec_off; // tile records (see plan.cu)
  fot::DevBuf block_done;   // per block: completed iterations (pipelined executor)
  // split write-back kernels: two partial-sum buffers, the shared points and
  // their slot ranges, the tiles' launch order
  fot::DevBuf partial, comb_point, comb_base, launch, tile_hdr, wslot;
  uint32_t n_slots = 0, n_shared_points = 0;
  uint32_t rec_cap = 0;
  uint32_t cap[2] = {0, 0};
  fot::SmemLayout layout;
  size_t smem = 0;
  uint32_t threads = 0;
  int per_sm = 0;
  fot::DevBuf ctl;
  fot::HierPlanDev dev(uint32_t iterations) const;
};

struct fot_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  fot_problem *prob = nullptr;
  fot_plan *plan = nullptr;
  // the problem's numbering at capture: the graph holds its buffers' addresses
  uint64_t version = 0;
  fot::Ctl *ctl = nullptr;
  ~fot_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};
