// Mesh statistics computed on the GPU, for the learned cost model's features
// and for the bandwidth reports:
//   fot_mesh_features      the spread of mapping 0's rows in the current
//                          numbering (largest and mean max - min of a cell's
//                          points) and the histogram of point degrees;
//   fot_sector_count       the reference's sector model
//   fot_plan_sector_count  (countCacheLinesForBlock, problem.hpp:654-672, as
//                          loopGPUCellCentred / loopGPUHierarchical use it,
//                          problem.hpp:145-152, :233-240): per block, the
//                          distinct 32-byte sectors of point dataset 0 its
//                          points touch -- AOS: every element of every row;
//                          SOA: distinct p / (32 / type size), times the
//                          dimension -- summed over blocks.  Blocks are runs
//                          of consecutive cells (fot_sector_count) or a
//                          hierarchical plan's blocks with their written
//                          points (fot_plan_sector_count).
// Counting uses (block, sector) keys, one radix sort and a distinct count,
// all on the device; only the totals come back.
//   fot_set_layout         point data AOS <-> SOA on the GPU (the reference
//                          converts on the host, AOStoSOA, data_t.hpp:249-275)
#include <algorithm>

#include "devutil.cuh"
#include "engine.hpp"

namespace fot {
namespace {

__global__ void k_row_span(const uint32_t *__restrict__ map, uint32_t n, int D,
                           unsigned long long *sum, unsigned int *mx) {
  unsigned long long s = 0;
  unsigned int m = 0;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    uint32_t lo = 0xFFFFFFFFu, hi = 0;
    for (int q = 0; q < D; ++q) {
      const uint32_t v = map[(size_t)c * D + q];
      lo = min(lo, v);
      hi = max(hi, v);
    }
    s += hi - lo;
    m = max(m, hi - lo);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
  m = __reduce_max_sync(0xFFFFFFFFu, m);
  if ((threadIdx.x & 31u) == 0) {
    atomicAdd(sum, s);
    atomicMax(mx, m);
  }
}

__global__ void k_point_degree(const uint32_t *__restrict__ map, size_t ne, uint32_t *deg) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ne; e += (size_t)gridDim.x * blockDim.x)
    atomicAdd(&deg[map[e]], 1u);
}

// bins: degree <= 2, 3-4, 5-6, >= 7
__global__ void k_degree_bins(const uint32_t *__restrict__ deg, uint32_t np, unsigned long long *bins) {
  unsigned int c[4] = {0, 0, 0, 0};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const uint32_t d = deg[i];
    c[d <= 2 ? 0 : d <= 4 ? 1 : d <= 6 ? 2 : 3]++;
  }
  for (int b = 0; b < 4; ++b) {
    const unsigned int t = __reduce_add_sync(0xFFFFFFFFu, c[b]);
    if ((threadIdx.x & 31u) == 0 && t) atomicAdd(&bins[b], (unsigned long long)t);
  }
}

// Sectors touched by one point: AOS rows of row_bytes from p * row_bytes
// (at most E sectors; the last one repeats to fill E keys), SOA element p of
// component 0 (one key; the caller multiplies by the dimension).
struct SectorRule {
  uint32_t row_bytes, type_size, E;
  int soa;
  __device__ __forceinline__ void keys(uint32_t block, uint32_t p, uint64_t *out) const {
    const uint64_t hi = (uint64_t)block << 32;
    if (soa) {
      const uint32_t s = (uint32_t)(((uint64_t)p * type_size) / 32u);
      for (uint32_t e = 0; e < E; ++e) out[e] = hi | s;
      return;
    }
    const uint64_t b0 = (uint64_t)p * row_bytes;
    const uint32_t s0 = (uint32_t)(b0 / 32u), s1 = (uint32_t)((b0 + row_bytes - 1) / 32u);
    for (uint32_t e = 0; e < E; ++e) out[e] = hi | min(s0 + e, s1);
  }
};

__global__ void k_sector_keys_cells(const uint32_t *__restrict__ map, uint32_t n, int D,
                                    uint32_t cells_per_block, SectorRule r, uint64_t *keys) {
  const size_t ne = (size_t)n * D;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ne; e += (size_t)gridDim.x * blockDim.x)
    r.keys((uint32_t)(e / D) / cells_per_block, map[e], keys + e * r.E);
}

__global__ void k_sector_keys_plan(const uint32_t *__restrict__ pts_off, const uint32_t *__restrict__ pts,
                                   uint32_t n_blocks, SectorRule r, uint64_t *keys) {
  const uint32_t b = blockIdx.x;
  if (b >= n_blocks) return;
  for (uint32_t j = pts_off[b] + threadIdx.x; j < pts_off[b + 1]; j += blockDim.x)
    r.keys(b, pts[j], keys + (size_t)j * r.E);
}

__global__ void k_count_distinct(const uint64_t *__restrict__ k, size_t n, unsigned long long *count) {
  unsigned int c = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    c += (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
  const unsigned int t = __reduce_add_sync(0xFFFFFFFFu, c);
  if ((threadIdx.x & 31u) == 0 && t) atomicAdd(count, (unsigned long long)t);
}

// Point-data layout conversion: tiles of kLayoutTile points staged in
// shared memory so that both the AOS rows and the SOA component runs are
// read and written coalesced.
constexpr uint32_t kLayoutTile = 128;

template <class T>
__global__ void k_aos_to_soa(const T *__restrict__ src, T *__restrict__ dst, uint32_t n, uint32_t dim) {
  extern __shared__ __align__(16) unsigned char tile_raw[];
  T *tile = reinterpret_cast<T *>(tile_raw);
  const uint32_t p0 = blockIdx.x * kLayoutTile;
  const uint32_t np = min(kLayoutTile, n - p0);
  for (uint32_t e = threadIdx.x; e < np * dim; e += blockDim.x) tile[e] = src[(size_t)p0 * dim + e];
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < np * dim; e += blockDim.x) {
    const uint32_t k = e / np, i = e - k * np;
    dst[(size_t)k * n + p0 + i] = tile[i * dim + k];
  }
}

template <class T>
__global__ void k_soa_to_aos(const T *__restrict__ src, T *__restrict__ dst, uint32_t n, uint32_t dim) {
  extern __shared__ __align__(16) unsigned char tile_raw[];
  T *tile = reinterpret_cast<T *>(tile_raw);
  const uint32_t p0 = blockIdx.x * kLayoutTile;
  const uint32_t np = min(kLayoutTile, n - p0);
  for (uint32_t e = threadIdx.x; e < np * dim; e += blockDim.x) {
    const uint32_t k = e / np, i = e - k * np;
    tile[i * dim + k] = src[(size_t)k * n + p0 + i];
  }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < np * dim; e += blockDim.x) dst[(size_t)p0 * dim + e] = tile[e];
}

template <class T>
int convert_layout(const void *src, void *dst, uint32_t n, uint32_t dim, bool to_soa) {
  const size_t smem = (size_t)kLayoutTile * dim * sizeof(T);
  const void *k = to_soa ? reinterpret_cast<const void *>(&k_aos_to_soa<T>)
                         : reinterpret_cast<const void *>(&k_soa_to_aos<T>);
  FOT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const T *s = static_cast<const T *>(src);
  T *d = static_cast<T *>(dst);
  void *args[] = {&s, &d, &n, &dim};
  FOT_CUDA(cudaLaunchKernel(k, dim3((n + kLayoutTile - 1) / kLayoutTile), dim3(256), args, smem, 0));
  return FOT_OK;
}

__global__ void k_point_part_keys(const uint32_t *__restrict__ map, uint32_t n, int D,
                                  const uint32_t *__restrict__ part, uint64_t *keys) {
  const size_t ne = (size_t)n * D;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ne; e += (size_t)gridDim.x * blockDim.x)
    keys[e] = ((uint64_t)map[e] << 32) | part[e / D];
}

// over distinct sorted (point, part) keys: points touched, and points
// touched by at least two parts
__global__ void k_point_sharing(const uint64_t *__restrict__ k, size_t n, unsigned long long *acc) {
  unsigned int first = 0, second = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t q = (uint32_t)(k[i] >> 32);
    const bool f = i == 0 || (uint32_t)(k[i - 1] >> 32) != q;
    first += f;
    second += !f && (i < 2 || (uint32_t)(k[i - 2] >> 32) != q);
  }
  const unsigned int a = __reduce_add_sync(0xFFFFFFFFu, first), b = __reduce_add_sync(0xFFFFFFFFu, second);
  if ((threadIdx.x & 31u) == 0) {
    atomicAdd(&acc[0], (unsigned long long)a);
    atomicAdd(&acc[1], (unsigned long long)b);
  }
}

SectorRule sector_rule(const fot_problem *p, int layout) {
  SectorRule r;
  r.type_size = p->info.point_type_size[0];
  r.row_bytes = p->info.point_dim[0] * r.type_size;
  r.soa = layout == FOT_SOA;
  r.E = r.soa ? 1u : (r.row_bytes + 31u) / 32u + 1u;
  return r;
}

// distinct keys of n_keys keys, the keys buffer holding 2 * n_keys entries
int count_distinct(DevBuf &keys, size_t n_keys, uint64_t *count) {
  *count = 0;
  if (n_keys == 0) return FOT_OK;
  if (n_keys > 0x7FFFFFFFull) return fail(FOT_ERR_LIMIT, "too many sector keys (%zu)", n_keys);
  uint64_t *k = keys.as<uint64_t>();
  FOT_TRY(sort_keys(k, k + n_keys, n_keys));
  DevBuf c;
  FOT_TRY(c.alloc(8));
  FOT_CUDA(cudaMemset(c.ptr, 0, 8));
  k_count_distinct<<<std::min<uint32_t>(blocks_for(n_keys), 4096), 256>>>(k + n_keys, n_keys,
                                                                            c.as<unsigned long long>());
  FOT_CUDA(cudaGetLastError());
  unsigned long long h = 0;
  FOT_CUDA(cudaMemcpy(&h, c.ptr, 8, cudaMemcpyDeviceToHost));
  *count = h;
  return FOT_OK;
}

} // namespace
} // namespace fot

using namespace fot;

extern "C" {

int fot_mesh_features(fot_problem *p, double *out, int n_out) {
  if (!p || !out || n_out < FOT_MESH_FEATURES) return fail(FOT_ERR_ARG, "bad argument");
  const uint32_t n = p->n_cells, np = p->n_points[0];
  const int D = (int)p->mesh_dim();
  DevBuf acc, deg;
  FOT_TRY(acc.alloc(64));
  FOT_TRY(deg.alloc((size_t)np * 4));
  FOT_CUDA(cudaMemset(acc.ptr, 0, 64));
  FOT_CUDA(cudaMemset(deg.ptr, 0, (size_t)np * 4));
  unsigned long long *a = acc.as<unsigned long long>();
  const uint32_t *map = p->map[0].as<uint32_t>();
  k_row_span<<<std::min<uint32_t>(blocks_for(n), 4096), 256>>>(map, n, D, a,
                                                                reinterpret_cast<unsigned int *>(a + 1));
  k_point_degree<<<std::min<uint32_t>(blocks_for((size_t)n * D), 8192), 256>>>(map, (size_t)n * D,
                                                                               deg.as<uint32_t>());
  k_degree_bins<<<std::min<uint32_t>(blocks_for(np), 4096), 256>>>(deg.as<uint32_t>(), np, a + 2);
  FOT_CUDA(cudaGetLastError());
  unsigned long long h[8];
  FOT_CUDA(cudaMemcpy(h, acc.ptr, 64, cudaMemcpyDeviceToHost));
  const unsigned int mx = (unsigned int)(h[1] & 0xFFFFFFFFull);
  out[0] = (double)mx;
  out[1] = (double)h[0] / n;
  for (int b = 0; b < 4; ++b) out[2 + b] = (double)h[2 + b] / np;
  return FOT_OK;
}

int fot_partition_quality(fot_problem *p, double *out, int n_out) {
  if (!p || !out || n_out < FOT_PARTITION_QUALITY) return fail(FOT_ERR_ARG, "bad argument");
  if (p->partition.size() != p->n_cells) return fail(FOT_ERR_STATE, "problem has no partition");
  const uint32_t n = p->n_cells;
  const int D = (int)p->mesh_dim();
  std::vector<uint32_t> size;
  for (uint32_t q : p->partition) {
    if (q >= size.size()) size.resize(q + 1, 0);
    ++size[q];
  }
  uint32_t parts = 0, largest = 0;
  for (uint32_t sz : size)
    if (sz) {
      ++parts;
      largest = std::max(largest, sz);
    }
  DevBuf part, keys, uniq, acc;
  FOT_TRY(upload(part, p->partition));
  const size_t ne = (size_t)n * D;
  FOT_TRY(keys.alloc(2 * ne * 8));
  FOT_TRY(uniq.alloc(ne * 8));
  FOT_TRY(acc.alloc(16));
  FOT_CUDA(cudaMemset(acc.ptr, 0, 16));
  k_point_part_keys<<<std::min<uint32_t>(blocks_for(ne), 8192), 256>>>(p->map[0].as<uint32_t>(), n, D,
                                                                        part.as<uint32_t>(),
                                                                        keys.as<uint64_t>());
  FOT_CUDA(cudaGetLastError());
  uint64_t *k = keys.as<uint64_t>();
  FOT_TRY(sort_keys(k, k + ne, ne));
  uint32_t m = 0;
  FOT_TRY(unique_keys(k + ne, uniq.as<uint64_t>(), ne, &m));
  k_point_sharing<<<std::min<uint32_t>(blocks_for(m), 4096), 256>>>(uniq.as<uint64_t>(), m,
                                                                     acc.as<unsigned long long>());
  FOT_CUDA(cudaGetLastError());
  unsigned long long h[2];
  FOT_CUDA(cudaMemcpy(h, acc.ptr, 16, cudaMemcpyDeviceToHost));
  out[0] = parts;
  out[1] = parts ? largest / ((double)n / parts) : 0.0;
  out[2] = h[0] ? (double)m / h[0] : 0.0;
  out[3] = h[0] ? (double)h[1] / h[0] : 0.0;
  return FOT_OK;
}

int fot_set_layout(fot_problem *p, int layout) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  if (layout != FOT_AOS && layout != FOT_SOA) return fail(FOT_ERR_ARG, "bad layout %d", layout);
  if (layout == p->layout) return FOT_OK;
  for (uint32_t k = 0; k < p->info.n_point_sets; ++k) {
    const uint32_t dim = p->info.point_dim[k], ts = p->info.point_type_size[k];
    if (dim == 1) continue;  // one component: both layouts are the same bytes
    DevBuf nb;
    FOT_TRY(nb.alloc(p->point_bytes(k)));
    if (ts == 8) FOT_TRY(convert_layout<uint64_t>(p->point[k].ptr, nb.ptr, p->n_points[k], dim, layout == FOT_SOA));
    else FOT_TRY(convert_layout<uint32_t>(p->point[k].ptr, nb.ptr, p->n_points[k], dim, layout == FOT_SOA));
    FOT_CUDA(cudaDeviceSynchronize());
    p->point[k] = std::move(nb);
  }
  p->layout = layout;
  p->version++;  // plans built for the other layout are stale
  return FOT_OK;
}

int fot_sector_count(fot_problem *p, uint32_t cells_per_block, int layout, uint64_t *sectors,
                     uint64_t *blocks) {
  if (!p || !sectors || cells_per_block == 0) return fail(FOT_ERR_ARG, "bad argument");
  if (layout < 0) layout = p->layout;
  if (layout != FOT_AOS && layout != FOT_SOA) return fail(FOT_ERR_ARG, "bad layout %d", layout);
  const SectorRule r = sector_rule(p, layout);
  const uint32_t n = p->n_cells;
  const int D = (int)p->mesh_dim();
  const size_t nk = (size_t)n * D * r.E;
  DevBuf keys;
  FOT_TRY(keys.alloc(2 * nk * 8));
  k_sector_keys_cells<<<std::min<uint32_t>(blocks_for((size_t)n * D), 8192), 256>>>(
      p->map[0].as<uint32_t>(), n, D, cells_per_block, r, keys.as<uint64_t>());
  FOT_CUDA(cudaGetLastError());
  uint64_t c = 0;
  FOT_TRY(count_distinct(keys, nk, &c));
  *sectors = c * (r.soa ? p->info.point_dim[0] : 1u);
  if (blocks) *blocks = (n + cells_per_block - 1) / cells_per_block;
  return FOT_OK;
}

int fot_plan_sector_count(const fot_plan *plan, int layout, uint64_t *sectors, uint64_t *blocks) {
  if (!plan || !sectors) return fail(FOT_ERR_ARG, "bad argument");
  if (plan->desc.exec == FOT_EXEC_ATOMIC) return fail(FOT_ERR_STATE, "atomic plans hold no blocks");
  if (!plan->prob) return fail(FOT_ERR_STATE, "the plan's problem was destroyed");
  const fot_problem *p = plan->prob;
  if (layout < 0) layout = p->layout;
  if (layout != FOT_AOS && layout != FOT_SOA) return fail(FOT_ERR_ARG, "bad layout %d", layout);
  const SectorRule r = sector_rule(p, layout);
  uint32_t total = 0;
  FOT_CUDA(cudaMemcpy(&total, plan->pts_off[0].as<uint32_t>() + plan->n_blocks, 4, cudaMemcpyDeviceToHost));
  const size_t nk = (size_t)total * r.E;
  DevBuf keys;
  FOT_TRY(keys.alloc(2 * nk * 8 + 16));
  if (plan->n_blocks) {
    k_sector_keys_plan<<<plan->n_blocks, 128>>>(plan->pts_off[0].as<uint32_t>(), plan->pts[0].as<uint32_t>(),
                                                 plan->n_blocks, r, keys.as<uint64_t>());
    FOT_CUDA(cudaGetLastError());
  }
  uint64_t c = 0;
  FOT_TRY(count_distinct(keys, nk, &c));
  *sectors = c * (r.soa ? p->info.point_dim[0] : 1u);
  if (blocks) *blocks = plan->n_blocks;
  return FOT_OK;
}

} // extern "C"
