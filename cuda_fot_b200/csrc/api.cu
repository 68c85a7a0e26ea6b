// extern "C" entry points of libfot (declared in include/fot.h).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>

#include "engine.hpp"

namespace fot {

static thread_local std::string g_error;

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
}

int fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
  return code;
}

extern const LoopOps k_ops_res_calc, k_ops_mini_aero, k_ops_lulesh, k_ops_volna, k_ops_getacc;

const LoopOps *loop_ops(int loop) {
  switch (loop) {
  case FOT_LOOP_RES_CALC: return &k_ops_res_calc;
  case FOT_LOOP_MINI_AERO: return &k_ops_mini_aero;
  case FOT_LOOP_LULESH: return &k_ops_lulesh;
  case FOT_LOOP_VOLNA: return &k_ops_volna;
  case FOT_LOOP_GETACC: return &k_ops_getacc;
  }
  return nullptr;
}

int device_sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

// The data bindings of the reference drivers' initProblem.
int describe(int loop, fot_loop_info *info) {
  fot_loop_info z{};
  const uint32_t d = sizeof(double), f = sizeof(float), i32 = sizeof(int);
  switch (loop) {
  case FOT_LOOP_RES_CALC: // res_calc.cu:17-27: res, x, q, adt; all mappings dim 2
    z.n_mappings = 4;
    for (int k = 0; k < 4; ++k) z.mesh_dim[k] = 2;
    z.n_point_sets = 4;
    z.point_dim[0] = 4; z.point_dim[1] = 2; z.point_dim[2] = 4; z.point_dim[3] = 1;
    for (int k = 0; k < 4; ++k) z.point_type_size[k] = d;
    z.n_cell_sets = 0;
    break;
  case FOT_LOOP_MINI_AERO: // mini_aero.cu:15-23: flux (5), cell record (28); face (12)
    z.n_mappings = 2;
    z.mesh_dim[0] = z.mesh_dim[1] = 2;
    z.n_point_sets = 2;
    z.point_dim[0] = 5; z.point_dim[1] = 28;
    z.point_type_size[0] = z.point_type_size[1] = d;
    z.n_cell_sets = 1;
    z.cell_dim[0] = 12; z.cell_type_size[0] = d;
    break;
  case FOT_LOOP_LULESH: // lulesh.cu:15-23: f (3), xyz (3); sig (3), determ (1, written)
    z.n_mappings = 2;
    z.mesh_dim[0] = z.mesh_dim[1] = 8;
    z.n_point_sets = 2;
    z.point_dim[0] = 3; z.point_dim[1] = 3;
    z.point_type_size[0] = z.point_type_size[1] = d;
    z.n_cell_sets = 2;
    z.cell_dim[0] = 3; z.cell_type_size[0] = d;
    z.cell_dim[1] = 1; z.cell_type_size[1] = d;
    z.cell_written_mask = 2u;
    break;
  case FOT_LOOP_VOLNA: // volna.cu:16-25: out (4 f32), vol (1 f32); flux 3, bathy 2, normals 2, isBoundary
    z.n_mappings = 2;
    z.mesh_dim[0] = z.mesh_dim[1] = 2;
    z.n_point_sets = 2;
    z.point_dim[0] = 4; z.point_dim[1] = 1;
    z.point_type_size[0] = z.point_type_size[1] = f;
    z.n_cell_sets = 4;
    z.cell_dim[0] = 3; z.cell_type_size[0] = f;
    z.cell_dim[1] = 2; z.cell_type_size[1] = f;
    z.cell_dim[2] = 2; z.cell_type_size[2] = f;
    z.cell_dim[3] = 1; z.cell_type_size[3] = i32;
    break;
  case FOT_LOOP_GETACC: // getacc.cu:15-25: out (4); cnmass 4, rho 1, cnwt 4, cnfx 4, cnfy 4
    z.n_mappings = 1;
    z.mesh_dim[0] = 4;
    z.n_point_sets = 1;
    z.point_dim[0] = 4;
    z.point_type_size[0] = d;
    z.n_cell_sets = 5;
    const uint32_t dims[5] = {4, 1, 4, 4, 4};
    for (int j = 0; j < 5; ++j) {
      z.cell_dim[j] = dims[j];
      z.cell_type_size[j] = d;
    }
    break;
  }
  if (z.n_mappings == 0) return fail(FOT_ERR_ARG, "unknown loop %d", loop);
  *info = z;
  return FOT_OK;
}

} // namespace fot

using namespace fot;

fot::LoopData fot_problem::loop_data() const {
  LoopData d{};
  d.map[0] = map[0].as<uint32_t>();
  d.map[1] = has_class1 ? map[1].as<uint32_t>() : nullptr;
  for (uint32_t k = 0; k < info.n_point_sets; ++k) {
    d.point[k] = point[k].ptr;
    d.n_points[k] = n_points[k];
  }
  d.out = point[0].ptr;
  for (uint32_t j = 0; j < info.n_cell_sets; ++j) {
    d.cell[j] = cell[j].ptr;
    d.cell_dim[j] = info.cell_dim[j];
    d.cell_size[j] = info.cell_type_size[j];
  }
  d.n_cell_sets = info.n_cell_sets;
  d.n_cells = n_cells;
  return d;
}

fot::HierPlanDev fot_plan::dev(uint32_t iterations) const {
  HierPlanDev P{};
  P.block_start = block_start.as<uint32_t>();
  P.block_wait = block_wait.as<uint32_t>();
  P.block_ntcol = block_ntcol.as<uint8_t>();
  P.tcol = tcol.as<uint8_t>();
  for (int c = 0; c < 2; ++c) {
    P.pts_off[c] = pts_off[c].as<uint32_t>();
    P.pts[c] = pts[c].as<uint32_t>();
    P.lidx[c] = lidx[c].as<uint16_t>();
  }
  P.n_blocks = n_blocks;
  P.total_tiles = iterations * n_blocks;
  for (int r = 0; r < 4; ++r) P.read_off[r] = layout.read_off[r];
  P.acc_off = layout.acc_off;
  P.pts_smem_off = layout.pts_off;
  P.rec = rec.as<unsigned char>();
  P.rec_off = rec_off.as<uint32_t>();
  P.rec_slot = layout.rec_slot;
  P.rows_off = layout.rows_off;
  P.rows_bytes = layout.rows_bytes;
  P.inc_off = layout.inc_off;
  P.outbuf_off = layout.outbuf_off;
  P.outbuf_bytes = layout.outbuf_bytes;
  P.block_done = block_done.as<unsigned int>();
  P.launch = launch.as<uint32_t>();
  P.partial = partial.ptr;
  P.comb_point = comb_point.as<uint32_t>();
  P.tile_hdr = tile_hdr.as<uint4>();
  P.wslot = wslot.as<uint32_t>();
  P.comb_base = comb_base.as<uint32_t>();
  P.n_slots = n_slots;
  P.n_shared = n_shared_points;
  P.tiles_on = 1;
  P.ctl = ctl.as<Ctl>();
  return P;
}

namespace fot {
int build_hier_plan(fot_problem *p, fot_plan *plan);
}

extern "C" {

const char *fot_last_error(void) { return g_error.c_str(); }
const char *fot_version(void) { return "fot-b200 0.1 (sm_100a)"; }

int fot_loop_describe(int loop, fot_loop_info *info) {
  if (!info) return fail(FOT_ERR_ARG, "null info");
  return describe(loop, info);
}

int fot_problem_create(int loop, int layout, uint32_t n_cells, const uint32_t *n_points,
                       const uint32_t *const *maps, fot_problem **out) {
  if (!out || !n_points || !maps) return fail(FOT_ERR_ARG, "null argument");
  *out = nullptr;
  fot_loop_info info;
  FOT_TRY(describe(loop, &info));
  if (layout != FOT_AOS && layout != FOT_SOA) return fail(FOT_ERR_ARG, "bad layout %d", layout);
  if (n_cells == 0) return fail(FOT_ERR_ARG, "a problem needs at least one cell");
  for (uint32_t k = 0; k < info.n_mappings; ++k) {
    if (!maps[k]) return fail(FOT_ERR_ARG, "mapping %u is null", k);
    if (n_points[k] == 0) return fail(FOT_ERR_ARG, "point set %u is empty", k);
    const uint32_t D = info.mesh_dim[k];
    for (size_t e = 0; e < (size_t)n_cells * D; ++e)
      if (maps[k][e] >= n_points[k])
        return fail(FOT_ERR_ARG, "mapping %u entry %zu = %u out of range (%u points)", k, e,
                    maps[k][e], n_points[k]);
  }
  // point sets read through mapping 0 must be the same mapping
  for (uint32_t k = 1; k < info.n_mappings; ++k) {
    if (set_class(loop, k) != 0) continue;
    if (n_points[k] != n_points[0] ||
        std::memcmp(maps[k], maps[0], (size_t)n_cells * info.mesh_dim[0] * 4) != 0)
      return fail(FOT_ERR_ARG,
                  "mapping %u must equal mapping 0 for this loop (its data are read through "
                  "mapping 0)", k);
  }
  auto *p = new fot_problem();
  p->loop = loop;
  p->layout = layout;
  p->info = info;
  p->n_cells = n_cells;
  for (uint32_t k = 0; k < info.n_mappings; ++k) p->n_points[k] = n_points[k];
  p->has_class1 = loop == FOT_LOOP_RES_CALC;
  cudaGetDevice(&p->device);
  int rc = FOT_OK;
  auto up = [&](DevBuf &b, const void *src, size_t bytes) {
    if (rc != FOT_OK) return;
    rc = b.alloc(bytes);
    if (rc != FOT_OK) return;
    cudaError_t e = cudaMemcpy(b.ptr, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = fail(FOT_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
  };
  up(p->map[0], maps[0], (size_t)n_cells * info.mesh_dim[0] * 4);
  if (p->has_class1) up(p->map[1], maps[1], (size_t)n_cells * info.mesh_dim[1] * 4);
  for (uint32_t k = 0; k < info.n_point_sets && rc == FOT_OK; ++k) {
    rc = p->point[k].alloc(p->point_bytes(k));
    if (rc == FOT_OK && cudaMemset(p->point[k].ptr, 0, p->point_bytes(k)) != cudaSuccess)
      rc = fail(FOT_ERR_CUDA, "memset failed");
  }
  for (uint32_t j = 0; j < info.n_cell_sets && rc == FOT_OK; ++j) {
    rc = p->cell[j].alloc(p->cell_bytes(j));
    if (rc == FOT_OK && cudaMemset(p->cell[j].ptr, 0, p->cell_bytes(j)) != cudaSuccess)
      rc = fail(FOT_ERR_CUDA, "memset failed");
  }
  if (rc != FOT_OK) {
    delete p;
    return rc;
  }
  for (int c = 0; c < (p->has_class1 ? 2 : 1); ++c) {
    p->point_perm[c].resize(p->class_points(c));
    std::iota(p->point_perm[c].begin(), p->point_perm[c].end(), 0u);
  }
  p->cell_order.resize(n_cells);
  std::iota(p->cell_order.begin(), p->cell_order.end(), 0u);
  *out = p;
  return FOT_OK;
}

int fot_problem_destroy(fot_problem *p) {
  // plans outliving their problem fail with FOT_ERR_STATE from now on
  if (p) {
    for (fot_plan *plan : p->plans) plan->prob = nullptr;
    for (fot_airfoil *a : p->airfoils) fot_airfoil_detach(a);
    for (fot_rowlist *l : p->rowlists) fot_rowlist_detach(l);
  }
  delete p;
  return FOT_OK;
}

static int check_set(fot_problem *p, uint32_t k, size_t bytes, bool point) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  if (point) {
    if (k >= p->info.n_point_sets) return fail(FOT_ERR_ARG, "point set %u out of range", k);
    if (bytes != p->point_bytes(k))
      return fail(FOT_ERR_ARG, "point set %u holds %zu bytes, got %zu", k, p->point_bytes(k), bytes);
  } else {
    if (k >= p->info.n_cell_sets) return fail(FOT_ERR_ARG, "cell set %u out of range", k);
    if (bytes != p->cell_bytes(k))
      return fail(FOT_ERR_ARG, "cell set %u holds %zu bytes, got %zu", k, p->cell_bytes(k), bytes);
  }
  return FOT_OK;
}

int fot_set_point_data(fot_problem *p, uint32_t k, const void *host, size_t bytes) {
  FOT_TRY(check_set(p, k, bytes, true));
  FOT_CUDA(cudaMemcpy(p->point[k].ptr, host, bytes, cudaMemcpyHostToDevice));
  return FOT_OK;
}
int fot_get_point_data(fot_problem *p, uint32_t k, void *host, size_t bytes) {
  FOT_TRY(check_set(p, k, bytes, true));
  FOT_CUDA(cudaMemcpy(host, p->point[k].ptr, bytes, cudaMemcpyDeviceToHost));
  return FOT_OK;
}
int fot_set_cell_data(fot_problem *p, uint32_t j, const void *host, size_t bytes) {
  FOT_TRY(check_set(p, j, bytes, false));
  FOT_CUDA(cudaMemcpy(p->cell[j].ptr, host, bytes, cudaMemcpyHostToDevice));
  return FOT_OK;
}
int fot_get_cell_data(fot_problem *p, uint32_t j, void *host, size_t bytes) {
  FOT_TRY(check_set(p, j, bytes, false));
  FOT_CUDA(cudaMemcpy(host, p->cell[j].ptr, bytes, cudaMemcpyDeviceToHost));
  return FOT_OK;
}
int fot_set_point_data_async(fot_problem *p, uint32_t k, const void *host, size_t bytes,
                             void *stream) {
  FOT_TRY(check_set(p, k, bytes, true));
  FOT_CUDA(cudaMemcpyAsync(p->point[k].ptr, host, bytes, cudaMemcpyHostToDevice,
                           static_cast<cudaStream_t>(stream)));
  return FOT_OK;
}
int fot_get_point_data_async(fot_problem *p, uint32_t k, void *host, size_t bytes, void *stream) {
  FOT_TRY(check_set(p, k, bytes, true));
  FOT_CUDA(cudaMemcpyAsync(host, p->point[k].ptr, bytes, cudaMemcpyDeviceToHost,
                           static_cast<cudaStream_t>(stream)));
  return FOT_OK;
}
int fot_set_cell_data_async(fot_problem *p, uint32_t j, const void *host, size_t bytes,
                            void *stream) {
  FOT_TRY(check_set(p, j, bytes, false));
  FOT_CUDA(cudaMemcpyAsync(p->cell[j].ptr, host, bytes, cudaMemcpyHostToDevice,
                           static_cast<cudaStream_t>(stream)));
  return FOT_OK;
}

int fot_point_data_device(fot_problem *p, uint32_t k, void **dptr) {
  if (!p || !dptr || k >= p->info.n_point_sets) return fail(FOT_ERR_ARG, "bad argument");
  *dptr = p->point[k].ptr;
  return FOT_OK;
}
int fot_cell_data_device(fot_problem *p, uint32_t j, void **dptr) {
  if (!p || !dptr || j >= p->info.n_cell_sets) return fail(FOT_ERR_ARG, "bad argument");
  *dptr = p->cell[j].ptr;
  return FOT_OK;
}

int fot_get_mapping(fot_problem *p, uint32_t k, uint32_t *host) {
  if (!p || !host || k >= p->info.n_mappings) return fail(FOT_ERR_ARG, "bad argument");
  const int c = set_class(p->loop, k);
  FOT_CUDA(cudaMemcpy(host, p->map[c].ptr, (size_t)p->n_cells * p->info.mesh_dim[k] * 4,
                      cudaMemcpyDeviceToHost));
  return FOT_OK;
}

int fot_problem_sizes(const fot_problem *p, uint32_t *n_cells, uint32_t *n_points) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  if (n_cells) *n_cells = p->n_cells;
  if (n_points)
    for (uint32_t k = 0; k < p->info.n_mappings; ++k) n_points[k] = p->n_points[k];
  return FOT_OK;
}

int fot_get_point_permutation(fot_problem *p, uint32_t k, uint32_t *host) {
  if (!p || !host || k >= p->info.n_mappings) return fail(FOT_ERR_ARG, "bad argument");
  const auto &v = p->point_perm[set_class(p->loop, k)];
  std::copy(v.begin(), v.end(), host);
  return FOT_OK;
}

int fot_get_cell_order(fot_problem *p, uint32_t *host) {
  if (!p || !host) return fail(FOT_ERR_ARG, "bad argument");
  std::copy(p->cell_order.begin(), p->cell_order.end(), host);
  return FOT_OK;
}

int fot_get_partition(fot_problem *p, uint32_t *host) {
  if (!p || !host) return fail(FOT_ERR_ARG, "bad argument");
  if (p->partition.size() != p->n_cells) return fail(FOT_ERR_STATE, "problem has no partition");
  std::copy(p->partition.begin(), p->partition.end(), host);
  return FOT_OK;
}

int fot_set_partition(fot_problem *p, const uint32_t *host) {
  if (!p || !host) return fail(FOT_ERR_ARG, "bad argument");
  p->partition.assign(host, host + p->n_cells);
  return FOT_OK;
}

// ---- plans ------------------------------------------------------------------

int fot_plan_build(fot_problem *p, const fot_plan_desc *desc, fot_plan **out) {
  if (!p || !desc || !out) return fail(FOT_ERR_ARG, "null argument");
  *out = nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  auto *plan = new fot_plan();
  plan->prob = p;
  plan->desc = *desc;
  plan->point_layout = p->layout;
  const LoopOps *ops = loop_ops(p->loop);
  int rc = FOT_OK;
  if (desc->exec == FOT_EXEC_ATOMIC) {
    plan->threads = 256;
    const uint32_t agg = (desc->flags & FOT_PLAN_NO_AGGREGATE) ? 0u : 1u;
    rc = ops->occupancy(FOT_EXEC_ATOMIC, p->layout == FOT_SOA, 256, agg, 0, &plan->per_sm);
  } else if (desc->exec == FOT_EXEC_HIER || desc->exec == FOT_EXEC_HIER_LAUNCH) {
    // Persistent executor (blocks of at most 512 cells): the staged split
    // write-back kernel by default, the direct split write-back kernel with
    // FOT_PLAN_DIRECT_READS, the pipelined kernel with per-block completion
    // flags with FOT_PLAN_BLOCK_FLAGS; FOT_PLAN_SIMPLE_TILES (or larger
    // blocks) selects the simple persistent kernel, staged or direct.
    const bool direct = desc->flags & FOT_PLAN_DIRECT_READS;
    plan->variant = direct ? 0u : kVariantStage;
    if (desc->exec == FOT_EXEC_HIER && desc->block_size <= 512 &&
        !(desc->flags & FOT_PLAN_SIMPLE_TILES)) {
      if (direct) plan->variant |= kVariantSplit;
      else plan->variant |= kVariantPipe | ((desc->flags & FOT_PLAN_BLOCK_FLAGS) ? 0u : kVariantSplit);
    }
    rc = build_hier_plan(p, plan);
    if (rc == FOT_OK) {
      plan->threads = hier_threads(desc->block_size);
      ops->smem_layout(plan->cap[0], plan->cap[1], plan->variant, plan->rec_cap, plan->threads,
                       &plan->layout);
      // a third tile-record slot deepens the pipelined kernel's look-ahead;
      // keep it only when it costs no resident CTA
      if ((plan->variant & kVariantPipe) && plan->layout.total <= 227 * 1024) {
        SmemLayout l3;
        const uint32_t v3 = plan->variant | kVariantSlots3;
        ops->smem_layout(plan->cap[0], plan->cap[1], v3, plan->rec_cap, plan->threads, &l3);
        int per2 = 0, per3 = 0;
        const bool soa = p->layout == FOT_SOA;
        rc = ops->occupancy(desc->exec, soa, plan->threads, plan->variant, plan->layout.total, &per2);
        if (rc == FOT_OK && l3.total <= 227 * 1024)
          rc = ops->occupancy(desc->exec, soa, plan->threads, v3, l3.total, &per3);
        if (rc == FOT_OK && per3 >= per2 && per3 > 0) {
          plan->variant = v3;
          plan->layout = l3;
        }
      }
      // the pipelined kernel holds two tiles' rows; when they do not fit,
      // the single-buffer persistent kernel runs the plan instead
      if ((plan->variant & kVariantPipe) && plan->layout.total > 227 * 1024) {
        plan->variant &= ~(kVariantPipe | kVariantSplit);
        ops->smem_layout(plan->cap[0], plan->cap[1], plan->variant, plan->rec_cap,
                         plan->threads, &plan->layout);
      }
      plan->smem = plan->layout.total;
      if (plan->smem > 227 * 1024)
        rc = fail(FOT_ERR_LIMIT,
                  "a block needs %zu bytes of shared memory (limit 227 KB): use a smaller block "
                  "size or a locality-improving ordering",
                  plan->smem);
    }
    if (rc == FOT_OK)
      rc = ops->occupancy(desc->exec, p->layout == FOT_SOA, plan->threads, plan->variant,
                          plan->smem, &plan->per_sm);
    if (rc == FOT_OK && plan->per_sm == 0 && (plan->variant & kVariantPipe)) {
      // the two-tile layout fits the limit but not beside the kernel's own
      // shared memory: the single-buffer persistent kernel runs the plan
      plan->variant &= ~(kVariantPipe | kVariantSplit);
      ops->smem_layout(plan->cap[0], plan->cap[1], plan->variant, plan->rec_cap, plan->threads,
                       &plan->layout);
      plan->smem = plan->layout.total;
      rc = ops->occupancy(desc->exec, p->layout == FOT_SOA, plan->threads, plan->variant,
                          plan->smem, &plan->per_sm);
    }
    if (rc == FOT_OK && plan->per_sm == 0)
      rc = fail(FOT_ERR_LIMIT, "hierarchical kernel cannot be resident (%zu B smem, %u threads)",
                plan->smem, plan->threads);
    if (rc == FOT_OK) {
      rc = plan->ctl.alloc(sizeof(Ctl));
      if (rc == FOT_OK && cudaMemset(plan->ctl.ptr, 0, sizeof(Ctl)) != cudaSuccess)
        rc = fail(FOT_ERR_CUDA, "memset failed");
    }
  } else {
    rc = fail(FOT_ERR_ARG, "unknown executor %d", desc->exec);
  }
  if (rc == FOT_OK) {
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = fail(FOT_ERR_CUDA, "plan build: %s", cudaGetErrorString(e));
  }
  if (rc != FOT_OK) {
    delete plan;
    return rc;
  }
  fot_plan_stats &s = plan->stats;
  s.exec = desc->exec;
  s.block_size = desc->block_size;
  s.smem_bytes = (uint32_t)plan->smem;
  s.grid = (uint32_t)(plan->per_sm * device_sm_count());
  s.plan_bytes = plan->block_start.bytes + plan->block_wait.bytes + plan->block_ntcol.bytes +
                 plan->tcol.bytes + plan->pts_off[0].bytes + plan->pts_off[1].bytes +
                 plan->pts[0].bytes + plan->pts[1].bytes + plan->lidx[0].bytes +
                 plan->lidx[1].bytes;
  s.build_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  s.shared_points = plan->n_shared_points;
  s.partial_slots = plan->n_slots;
  const char *kname = "atomic";
  if (desc->exec == FOT_EXEC_HIER_LAUNCH) kname = "per-colour launches";
  else if (desc->exec == FOT_EXEC_HIER)
    kname = (plan->variant & kVariantSplit)
                ? ((plan->variant & kVariantPipe) ? "split write-back" : "split write-back, direct")
            : (plan->variant & kVariantPipe) ? "pipelined, block flags"
            : (plan->variant & kVariantStage) ? "simple persistent"
                                               : "simple persistent, direct reads";
  std::snprintf(s.kernel, sizeof(s.kernel), "%s", kname);
  p->plans.push_back(plan);
  *out = plan;
  return FOT_OK;
}

int fot_plan_destroy(fot_plan *plan) {
  if (plan && plan->prob) {
    auto &v = plan->prob->pending;
    v.erase(std::remove(v.begin(), v.end(), plan), v.end());
    auto &w = plan->prob->plans;
    w.erase(std::remove(w.begin(), w.end(), plan), w.end());
  }
  delete plan;
  return FOT_OK;
}

// Remember every plan with a device control block that ran since the last
// fot_sync, so that fot_sync reports (and clears) the device-side errors of
// all of them, not only of the last one.
static void note_run(fot_problem *p, fot_plan *plan) {
  if (!plan->ctl.ptr) return;
  if (std::find(p->pending.begin(), p->pending.end(), plan) == p->pending.end())
    p->pending.push_back(plan);
}

int fot_plan_get_stats(const fot_plan *plan, fot_plan_stats *stats) {
  if (!plan || !stats) return fail(FOT_ERR_ARG, "null argument");
  *stats = plan->stats;
  return FOT_OK;
}

int fot_plan_export(const fot_plan *plan, uint32_t *n_blocks, uint32_t *n_colours, uint32_t *n_pts,
                    uint32_t *colour_offsets, uint32_t *block_start, uint32_t *cell_id,
                    uint8_t *tcol, uint8_t *block_ntcol, uint32_t *pts_off, uint32_t *pts,
                    uint16_t *lidx) {
  if (!plan) return fail(FOT_ERR_ARG, "null plan");
  if (plan->desc.exec == FOT_EXEC_ATOMIC) return fail(FOT_ERR_STATE, "atomic plans hold no arrays");
  if (!plan->prob) return fail(FOT_ERR_STATE, "the plan's problem was destroyed");
  const fot_problem *p = plan->prob;
  const uint32_t nb = plan->n_blocks, n = p->n_cells;
  uint32_t total = 0;
  FOT_CUDA(cudaMemcpy(&total, plan->pts_off[0].as<uint32_t>() + nb, 4, cudaMemcpyDeviceToHost));
  if (n_blocks) *n_blocks = nb;
  if (n_colours) *n_colours = plan->n_colours;
  if (n_pts) *n_pts = total;
  if (!pts) return FOT_OK;
  std::copy(plan->colour_offsets.begin(), plan->colour_offsets.end(), colour_offsets);
  FOT_CUDA(cudaMemcpy(block_start, plan->block_start.ptr, (size_t)(nb + 1) * 4, cudaMemcpyDeviceToHost));
  FOT_CUDA(cudaMemcpy(cell_id, plan->build_perm.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost));
  FOT_CUDA(cudaMemcpy(tcol, plan->tcol.ptr, n, cudaMemcpyDeviceToHost));
  FOT_CUDA(cudaMemcpy(block_ntcol, plan->block_ntcol.ptr, nb, cudaMemcpyDeviceToHost));
  FOT_CUDA(cudaMemcpy(pts_off, plan->pts_off[0].ptr, (size_t)(nb + 1) * 4, cudaMemcpyDeviceToHost));
  FOT_CUDA(cudaMemcpy(pts, plan->pts[0].ptr, (size_t)total * 4, cudaMemcpyDeviceToHost));
  FOT_CUDA(cudaMemcpy(lidx, plan->lidx[0].ptr, (size_t)p->mesh_dim() * n * 2, cudaMemcpyDeviceToHost));
  return FOT_OK;
}

// ---- execution ------------------------------------------------------------

static int run_plan(fot_problem *p, fot_plan *plan, uint32_t iterations, cudaStream_t st) {
  if (!p || !plan) return fail(FOT_ERR_ARG, "null argument");
  if (plan->prob != p) return fail(FOT_ERR_STATE, "plan belongs to another (or a destroyed) problem");
  if (iterations == 0) return FOT_OK;
  const LoopOps *ops = loop_ops(p->loop);
  const LoopData d = p->loop_data();
  const bool soa = p->layout == FOT_SOA;
  const int sms = device_sm_count();
  if (plan->point_layout != p->layout)
    return fail(FOT_ERR_STATE, "plan is stale: the problem's point layout changed after the plan was built");
  if (plan->desc.exec == FOT_EXEC_ATOMIC) {
    const bool agg = !(plan->desc.flags & FOT_PLAN_NO_AGGREGATE);
    const uint32_t need = (p->n_cells + 255) / 256;
    const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(need, (uint32_t)(plan->per_sm * sms)));
    for (uint32_t it = 0; it < iterations; ++it) FOT_TRY(ops->run_atomic(d, soa, agg, 256, grid, st));
    return FOT_OK;
  }
  if (plan->version != p->version)
    return fail(FOT_ERR_STATE, "plan is stale: the problem was reordered after the plan was built");
  if (plan->desc.exec == FOT_EXEC_HIER) {
    if ((uint64_t)iterations * plan->n_blocks + (uint64_t)plan->per_sm * sms >= 0xFFFFFFFFull)
      return fail(FOT_ERR_LIMIT, "too many tiles in one launch");
    const HierPlanDev P = plan->dev(iterations);
    // the split kernels run one iteration per launch over the plan's blocks:
    // persistent CTAs (staged form) or one CTA per block (direct form)
    const bool split = plan->variant & kVariantSplit;
    const uint32_t tiles = split ? plan->n_blocks : P.total_tiles;
    const uint32_t grid = (split && !(plan->variant & kVariantPipe))
                              ? plan->n_blocks
                              : std::min<uint32_t>(tiles, (uint32_t)(plan->per_sm * sms));
    return ops->run_hier(d, P, soa, plan->threads, plan->variant, grid, plan->smem, st);
  }
  const HierPlanDev P = plan->dev(1);
  for (uint32_t it = 0; it < iterations; ++it)
    for (uint32_t c = 0; c < plan->n_colours; ++c) {
      const uint32_t first = plan->colour_offsets[c];
      const uint32_t count = plan->colour_offsets[c + 1] - first;
      if (count)
        FOT_TRY(ops->run_hier_colour(d, P, soa, plan->threads, plan->variant, first, count,
                                     plan->smem, st));
    }
  return FOT_OK;
}

int fot_run(fot_problem *p, fot_plan *plan, uint32_t iterations, void *stream) {
  FOT_TRY(run_plan(p, plan, iterations, static_cast<cudaStream_t>(stream)));
  note_run(p, plan);
  return FOT_OK;
}

int fot_sync(fot_problem *p, void *stream) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  FOT_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  std::vector<fot_plan *> pending;
  pending.swap(p->pending);
  int failed = 0;
  for (fot_plan *plan : pending) {
    Ctl c{};
    FOT_CUDA(cudaMemcpy(&c, plan->ctl.ptr, sizeof(Ctl), cudaMemcpyDeviceToHost));
    if (!c.error) continue;
    // the run stopped early: restart the plan's queue and flags from zero
    ++failed;
    FOT_CUDA(cudaMemset(plan->ctl.ptr, 0, sizeof(Ctl)));
    if (plan->block_done.ptr) FOT_CUDA(cudaMemset(plan->block_done.ptr, 0, (size_t)plan->n_blocks * 4));
  }
  if (failed)
    return fail(FOT_ERR_DEVICE, "%d hierarchical plan(s) stopped early: a wait of the persistent "
                "executor hit its limit (the problem's data are undefined)", failed);
  return FOT_OK;
}

int fot_plan_inject_lost_flag(fot_plan *plan, uint32_t block) {
  if (!plan) return fail(FOT_ERR_ARG, "null plan");
  if (!(plan->variant & kVariantPipe) || (plan->variant & kVariantSplit) || !plan->block_done.ptr)
    return fail(FOT_ERR_STATE, "the plan does not run the block-flag hierarchical kernel");
  if (block >= plan->n_blocks) return fail(FOT_ERR_ARG, "block %u out of range (%u blocks)", block, plan->n_blocks);
  FOT_CUDA(cudaDeviceSynchronize());
  Ctl c{};
  FOT_CUDA(cudaMemcpy(&c, plan->ctl.ptr, sizeof(Ctl), cudaMemcpyDeviceToHost));
  if (c.base == 0) return fail(FOT_ERR_STATE, "run the plan at least once before injecting");
  FOT_CUDA(cudaMemset(plan->block_done.as<unsigned int>() + block, 0, sizeof(unsigned int)));
  FOT_CUDA(cudaDeviceSynchronize());
  return FOT_OK;
}

int fot_graph_create(fot_problem *p, fot_plan *plan, uint32_t iterations, void *stream,
                     fot_graph **out) {
  if (!p || !plan || !out) return fail(FOT_ERR_ARG, "null argument");
  *out = nullptr;
  struct Ctx {
    fot_problem *p;
    fot_plan *plan;
    uint32_t iterations;
  } ctx{p, plan, iterations};
  auto enqueue = [](void *c, cudaStream_t st) {
    const Ctx *x = static_cast<const Ctx *>(c);
    return run_plan(x->p, x->plan, x->iterations, st);
  };
  FOT_TRY(capture_graph(static_cast<cudaStream_t>(stream), enqueue, &ctx, out));
  (*out)->prob = p;
  (*out)->plan = plan;
  (*out)->ctl = plan->ctl.as<Ctl>();
  (*out)->version = p->version;
  return FOT_OK;
}

int fot_graph_launch(fot_graph *g, void *stream) {
  if (!g) return fail(FOT_ERR_ARG, "null graph");
  // the graph replays the device addresses it was captured with: refuse it
  // once its problem is gone or its buffers were replaced (renumbering,
  // another plan's cell order, a layout change)
  if (g->plan) {
    if (!g->plan->prob) return fail(FOT_ERR_STATE, "the graph's problem was destroyed");
    if (g->plan->prob->version != g->version)
      return fail(FOT_ERR_STATE, "graph is stale: the problem was renumbered after the capture");
  }
  FOT_CUDA(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
  if (g->plan) note_run(g->plan->prob, g->plan);
  return FOT_OK;
}

int fot_graph_destroy(fot_graph *g) {
  delete g;
  return FOT_OK;
}

} // extern "C"

namespace fot {

int capture_graph(cudaStream_t st, int (*enqueue)(void *ctx, cudaStream_t st), void *ctx,
                  fot_graph **out) {
  *out = nullptr;
  cudaStream_t cap = st;
  bool own = false;
  if (!cap) {
    FOT_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    own = true;
  }
  const cudaError_t b = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (b != cudaSuccess) {
    if (own) cudaStreamDestroy(cap);
    return fail(FOT_ERR_CUDA, "begin capture: %s", cudaGetErrorString(b));
  }
  const int rc = enqueue(ctx, cap);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cap, &graph);
  if (own) cudaStreamDestroy(cap);
  if (rc != FOT_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return fail(FOT_ERR_CUDA, "stream capture: %s", cudaGetErrorString(e));
  auto *g = new fot_graph();
  g->graph = graph;
  const cudaError_t e2 = cudaGraphInstantiate(&g->exec, graph, 0);
  if (e2 != cudaSuccess) {
    delete g;
    return fail(FOT_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e2));
  }
  *out = g;
  return FOT_OK;
}

} // namespace fot
