// Batched executors: many meshes in ONE launch.
//   * hierarchical plans: CTAs claim tiles from one queue ordered by
//     (iteration, block colour, mesh, block); a tile waits only for its own
//     mesh's earlier colours, on a per-mesh counter, so meshes of very
//     different sizes share the GPU without a launch per mesh and colour;
//   * atomic plans: tiles of 1,024 consecutive cells of one mesh, for every
//     mesh and every iteration, in one grid-stride launch (iterations need no
//     ordering: the loops never read the dataset they increment); that
//     kernel lives in atomic_batch.cu.
// The reference has no counterpart (one mesh per process, one launch per
// colour).
#define FOT_ADAPTER_ALL 1
#include <algorithm>
#include <numeric>

#include "devutil.cuh"
#include "batch.cuh"
#include "engine.hpp"
#include "loops.cuh"

namespace fot {

template <bool SOA, int T, class L>
__device__ __forceinline__ void batch_tile(const BatchMesh &m, unsigned char *smem, uint32_t b,
                                           uint32_t iter, unsigned int *done, unsigned int *err) {
  unsigned int seen = 0;  // counters differ per mesh: no cached value
  hier_tile_waiting<L, SOA, T>(m.d, m.P, smem, b, iter, done, err, seen);
}

template <bool SOA, int T, class... Ls>
__global__ void __launch_bounds__(T) k_batch(BatchDev B) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint32_t s_ticket;
  const uint32_t tid = threadIdx.x;
  for (;;) {
    if (tid == 0) {
      uint32_t t = atomicAdd(&B.ctl->ticket, 1u);
      if (*(volatile unsigned int *)&B.ctl->error) t = B.total_tiles;
      s_ticket = t;
    }
    __syncthreads();
    const uint32_t t = s_ticket;
    if (t >= B.total_tiles) break;
    const uint32_t iter = t / B.tiles_per_iter;
    const uint32_t r = t - iter * B.tiles_per_iter;
    const uint32_t mi = B.tile_mesh[r];
    const uint32_t b = B.tile_block[r];
    const BatchMesh &m = B.mesh[mi];
    ((m.loop == Ls::kLoop ? (batch_tile<SOA, T, Ls>(m, smem, b, iter, &B.done[mi], &B.ctl->error), 0)
                          : 0),
     ...);
    if (tid == 0) red_release_add(&B.done[mi], 1u);
  }
  if (tid == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(&B.ctl->exited, 1u);
    if (prev == gridDim.x - 1) {
      for (uint32_t i = 0; i < B.n_mesh; ++i) atomicExch(&B.done[i], 0u);
      atomicExch(&B.ctl->ticket, 0u);
      atomicExch(&B.ctl->exited, 0u);
      __threadfence();
    }
  }
}

// Kernel variants: one loop kind, or the res_calc + volna pair.
template <bool SOA, int T> const void *batch_kernel(uint32_t loop_mask) {
  using RC = res_calc::Loop;
  using MA = mini_aero::Loop;
  using LU = lulesh::Loop;
  using VO = volna::Loop;
  using GA = getacc::Loop;
  switch (loop_mask) {
  case 1u << FOT_LOOP_RES_CALC: return (const void *)&k_batch<SOA, T, RC>;
  case 1u << FOT_LOOP_MINI_AERO: return (const void *)&k_batch<SOA, T, MA>;
  case 1u << FOT_LOOP_LULESH: return (const void *)&k_batch<SOA, T, LU>;
  case 1u << FOT_LOOP_VOLNA: return (const void *)&k_batch<SOA, T, VO>;
  case 1u << FOT_LOOP_GETACC: return (const void *)&k_batch<SOA, T, GA>;
  case (1u << FOT_LOOP_RES_CALC) | (1u << FOT_LOOP_VOLNA): return (const void *)&k_batch<SOA, T, RC, VO>;
  }
  return nullptr;
}

const void *batch_kernel_for(bool soa, uint32_t threads, uint32_t loop_mask) {
  if (soa) {
    switch (threads) {
    case 128: return batch_kernel<true, 128>(loop_mask);
    case 256: return batch_kernel<true, 256>(loop_mask);
    case 512: return batch_kernel<true, 512>(loop_mask);
    }
  } else {
    switch (threads) {
    case 128: return batch_kernel<false, 128>(loop_mask);
    case 256: return batch_kernel<false, 256>(loop_mask);
    case 512: return batch_kernel<false, 512>(loop_mask);
    }
  }
  return nullptr;
}

} // namespace fot

using namespace fot;

struct fot_batch {
  std::vector<fot_problem *> probs;
  std::vector<fot_plan *> plans;
  std::vector<uint64_t> versions;
  DevBuf mesh, tile_mesh, tile_block, done, ctl;
  uint32_t tiles_per_iter = 0;
  uint32_t threads = 0;
  size_t smem = 0;
  int per_sm = 0;
  bool soa = false;
  bool atomic = false;  // atomic plans (else hierarchical)
  const void *kernel = nullptr;
};

extern "C" {

int fot_batch_create(fot_problem *const *problems, fot_plan *const *plans, uint32_t n,
                     fot_batch **out) {
  if (!problems || !plans || !out || n == 0) return fail(FOT_ERR_ARG, "bad argument");
  *out = nullptr;
  auto *B = new fot_batch();
  std::vector<BatchMesh> meshes(n);
  uint32_t mask = 0;
  int rc = FOT_OK;
  B->atomic = plans[0] && plans[0]->desc.exec == FOT_EXEC_ATOMIC;
  const bool agg = plans[0] && !(plans[0]->desc.flags & FOT_PLAN_NO_AGGREGATE);
  for (uint32_t i = 0; i < n && rc == FOT_OK; ++i) {
    fot_problem *p = problems[i];
    fot_plan *pl = plans[i];
    if (!p || !pl || pl->prob != p) rc = fail(FOT_ERR_ARG, "batch entry %u: plan/problem mismatch", i);
    else if ((pl->desc.exec == FOT_EXEC_ATOMIC) != B->atomic)
      rc = fail(FOT_ERR_ARG, "batch entry %u: a batch holds atomic plans only or hierarchical plans only", i);
    else if (B->atomic && agg != !(pl->desc.flags & FOT_PLAN_NO_AGGREGATE))
      rc = fail(FOT_ERR_ARG, "batch entry %u: atomic plans of a batch all aggregate or none does", i);
    else if (!B->atomic && pl->version != p->version)
      rc = fail(FOT_ERR_STATE, "batch entry %u: stale plan", i);
    else if (i > 0 && (p->layout == FOT_SOA) != B->soa) rc = fail(FOT_ERR_ARG, "batch mixes layouts");
    if (rc != FOT_OK) break;
    B->soa = p->layout == FOT_SOA;
    mask |= 1u << p->loop;
    meshes[i].d = p->loop_data();
    meshes[i].loop = p->loop;
    B->probs.push_back(p);
    B->plans.push_back(pl);
    B->versions.push_back(p->version);
    if (B->atomic) {
      B->threads = 256;
      continue;
    }
    meshes[i].P = pl->dev(1);
    // the batched tiles use the staged one-tile-at-a-time layout
    SmemLayout lay;
    loop_ops(p->loop)->smem_layout(pl->cap[0], pl->cap[1], kVariantStage, 0, pl->threads, &lay);
    for (int r = 0; r < 4; ++r) meshes[i].P.read_off[r] = lay.read_off[r];
    meshes[i].P.acc_off = lay.acc_off;
    meshes[i].P.pts_smem_off = lay.pts_off;
    B->threads = std::max(B->threads, pl->threads);
    B->smem = std::max(B->smem, lay.total);
  }
  if (rc == FOT_OK && B->threads > 512)
    rc = fail(FOT_ERR_ARG, "batched plans must use block sizes of at most 512");
  if (rc == FOT_OK) {
    B->kernel = B->atomic ? batch_atomic_kernel_for(B->soa, agg, mask)
                          : batch_kernel_for(B->soa, B->threads, mask);
    if (!B->kernel)
      rc = fail(FOT_ERR_ARG, "a batch holds one loop kind, or res_calc with volna");
  }
  if (rc == FOT_OK) {
    // tile order: colour-major across meshes, then mesh, then block (atomic
    // plans: mesh after mesh, kAtomicTile cells per tile)
    uint32_t max_col = 0;
    for (auto *pl : B->plans) max_col = std::max(max_col, pl->n_colours);
    std::vector<uint32_t> tm, tb;
    if (B->atomic) {
      for (uint32_t i = 0; i < n; ++i)
        for (uint32_t c0 = 0; c0 < B->probs[i]->n_cells; c0 += kAtomicTile) {
          tm.push_back(i);
          tb.push_back(c0);
        }
      max_col = 0;
    }
    for (uint32_t c = 0; c < max_col; ++c)
      for (uint32_t i = 0; i < n; ++i) {
        const fot_plan *pl = B->plans[i];
        if (c >= pl->n_colours) continue;
        for (uint32_t b = pl->colour_offsets[c]; b < pl->colour_offsets[c + 1]; ++b) {
          tm.push_back(i);
          tb.push_back(b);
        }
      }
    B->tiles_per_iter = (uint32_t)tm.size();
    rc = upload(B->tile_mesh, tm);
    if (rc == FOT_OK) rc = upload(B->tile_block, tb);
    if (rc == FOT_OK) rc = upload(B->mesh, meshes);
    if (rc == FOT_OK) rc = B->done.alloc((size_t)n * 4);
    if (rc == FOT_OK) rc = B->ctl.alloc(sizeof(Ctl));
    if (rc == FOT_OK && (cudaMemset(B->done.ptr, 0, (size_t)n * 4) != cudaSuccess ||
                         cudaMemset(B->ctl.ptr, 0, sizeof(Ctl)) != cudaSuccess))
      rc = fail(FOT_ERR_CUDA, "memset failed");
  }
  if (rc == FOT_OK) {
    const cudaError_t e1 = cudaFuncSetAttribute(B->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)B->smem);
    const cudaError_t e2 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B->per_sm, B->kernel,
                                                                         (int)B->threads, B->smem);
    if (e1 != cudaSuccess || e2 != cudaSuccess || B->per_sm == 0)
      rc = fail(FOT_ERR_LIMIT, "batched kernel cannot be resident (%zu B smem)", B->smem);
  }
  if (rc != FOT_OK) {
    delete B;
    return rc;
  }
  *out = B;
  return FOT_OK;
}

int fot_batch_run(fot_batch *B, uint32_t iterations, void *stream) {
  if (!B) return fail(FOT_ERR_ARG, "null batch");
  if (iterations == 0) return FOT_OK;
  for (size_t i = 0; i < B->probs.size(); ++i)
    // the batch holds device views of each problem's data (and of each
    // hierarchical plan): a reorder after creation invalidates them
    if (B->probs[i]->version != B->versions[i] ||
        (!B->atomic && B->plans[i]->version != B->versions[i]))
      return fail(FOT_ERR_STATE, "batch entry %zu changed since the batch was created", i);
  const uint64_t total = (uint64_t)iterations * B->tiles_per_iter;
  const uint32_t grid_max = (uint32_t)(B->per_sm * device_sm_count());
  if (total + grid_max >= 0xFFFFFFFFull) return fail(FOT_ERR_LIMIT, "too many tiles in one launch");
  BatchDev d{};
  d.mesh = B->mesh.as<BatchMesh>();
  d.tile_mesh = B->tile_mesh.as<uint32_t>();
  d.tile_block = B->tile_block.as<uint32_t>();
  d.tiles_per_iter = B->tiles_per_iter;
  d.total_tiles = (uint32_t)total;
  d.n_mesh = (uint32_t)B->probs.size();
  d.done = B->done.as<unsigned int>();
  d.ctl = B->ctl.as<Ctl>();
  const uint32_t grid = (uint32_t)std::min<uint64_t>(total, grid_max);
  void *args[] = {&d};
  FOT_CUDA(cudaLaunchKernel(B->kernel, dim3(grid), dim3(B->threads), args, B->smem,
                            static_cast<cudaStream_t>(stream)));
  return FOT_OK;
}

int fot_batch_sync(fot_batch *B, void *stream) {
  if (!B) return fail(FOT_ERR_ARG, "null batch");
  FOT_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  Ctl c{};
  FOT_CUDA(cudaMemcpy(&c, B->ctl.ptr, sizeof(Ctl), cudaMemcpyDeviceToHost));
  if (c.error) {
    FOT_CUDA(cudaMemset(B->ctl.ptr, 0, sizeof(Ctl)));
    return fail(FOT_ERR_DEVICE, "a dependency wait of the batched executor hit its limit");
  }
  return FOT_OK;
}

int fot_batch_destroy(fot_batch *B) {
  delete B;
  return FOT_OK;
}

} // extern "C"
