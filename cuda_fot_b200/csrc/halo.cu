// Row lists of a point dataset: the device side of a partitioned (multi-GPU)
// run.  A mesh split into parts by cells runs one part per GPU; a point
// touched by several parts is owned by one of them, and the increments the
// others add to their copies (halo rows) travel to the owner after the loop.
// A row list is a validated, device-resident list of distinct point rows of
// one dataset: gather packs those rows (AOS, list order) into a device
// buffer for the exchange, scatter_add adds received rows into the dataset.
// Distinct rows make scatter_add race-free and its result independent of the
// thread order; successive calls (one per sending part, in part order) give
// a fixed summation order.
#include <algorithm>
#include <vector>

#include "engine.hpp"

namespace fot {
namespace {

constexpr uint32_t kThreads = 256;

template <class T>
__global__ void __launch_bounds__(kThreads) k_gather_rows(const T *__restrict__ data, uint32_t np,
                                                          uint32_t dim, int soa,
                                                          const uint32_t *__restrict__ rows,
                                                          uint32_t n, T *__restrict__ dst) {
  const size_t total = (size_t)n * dim;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(e / dim), k = (uint32_t)(e % dim);
    const uint32_t p = rows[i];
    dst[e] = data[soa ? (size_t)k * np + p : (size_t)p * dim + k];
  }
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_scatter_add_rows(T *__restrict__ data, uint32_t np,
                                                               uint32_t dim, int soa,
                                                               const uint32_t *__restrict__ rows,
                                                               uint32_t n, const T *__restrict__ src) {
  const size_t total = (size_t)n * dim;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(e / dim), k = (uint32_t)(e % dim);
    const uint32_t p = rows[i];
    const size_t o = soa ? (size_t)k * np + p : (size_t)p * dim + k;
    data[o] = data[o] + src[e];
  }
}

uint32_t grid_for(size_t n) {
  return (uint32_t)std::max<size_t>(1, std::min<size_t>((n + kThreads - 1) / kThreads, 4096));
}

} // namespace
} // namespace fot

using namespace fot;

struct fot_rowlist {
  fot_problem *prob = nullptr;
  uint64_t version = 0; // the problem's numbering the rows refer to
  uint32_t set = 0, n = 0;
  DevBuf rows;
};

void fot_rowlist_detach(fot_rowlist *l) {
  if (l) l->prob = nullptr;
}

namespace {

int rowlist_check(const fot_rowlist *l) {
  if (!l) return fail(FOT_ERR_ARG, "null row list");
  if (!l->prob) return fail(FOT_ERR_STATE, "the row list's problem was destroyed");
  if (l->version != l->prob->version)
    return fail(FOT_ERR_STATE, "row list is stale: the problem was renumbered after it was made");
  return FOT_OK;
}

template <class T> int launch_gather(const fot_rowlist *l, void *dst, cudaStream_t st) {
  const fot_problem *p = l->prob;
  const uint32_t dim = p->info.point_dim[l->set];
  k_gather_rows<T><<<grid_for((size_t)l->n * dim), kThreads, 0, st>>>(
      static_cast<const T *>(p->point[l->set].ptr), p->n_points[l->set], dim, p->layout == FOT_SOA,
      l->rows.as<uint32_t>(), l->n, static_cast<T *>(dst));
  FOT_CUDA(cudaGetLastError());
  return FOT_OK;
}

template <class T> int launch_scatter_add(const fot_rowlist *l, const void *src, cudaStream_t st) {
  const fot_problem *p = l->prob;
  const uint32_t dim = p->info.point_dim[l->set];
  k_scatter_add_rows<T><<<grid_for((size_t)l->n * dim), kThreads, 0, st>>>(
      static_cast<T *>(p->point[l->set].ptr), p->n_points[l->set], dim, p->layout == FOT_SOA,
      l->rows.as<uint32_t>(), l->n, static_cast<const T *>(src));
  FOT_CUDA(cudaGetLastError());
  return FOT_OK;
}

} // namespace

extern "C" {

int fot_rowlist_create(fot_problem *p, uint32_t k, const uint32_t *rows, uint32_t n, fot_rowlist **out) {
  if (!p || !out || (n && !rows)) return fail(FOT_ERR_ARG, "null argument");
  *out = nullptr;
  if (k >= p->info.n_point_sets) return fail(FOT_ERR_ARG, "point set %u out of range", k);
  const uint32_t ts = p->info.point_type_size[k];
  if (ts != 4 && ts != 8) return fail(FOT_ERR_ARG, "point set %u has %u-byte elements", k, ts);
  std::vector<uint32_t> sorted(rows, rows + n);
  std::sort(sorted.begin(), sorted.end());
  for (uint32_t i = 0; i < n; ++i) {
    if (sorted[i] >= p->n_points[k]) return fail(FOT_ERR_ARG, "row %u out of range (%u points)", sorted[i], p->n_points[k]);
    if (i && sorted[i] == sorted[i - 1]) return fail(FOT_ERR_ARG, "row %u listed twice", sorted[i]);
  }
  auto *l = new fot_rowlist;
  l->prob = p;
  l->version = p->version;
  l->set = k;
  l->n = n;
  int rc = l->rows.alloc((size_t)n * sizeof(uint32_t));
  if (rc == FOT_OK && n && cudaMemcpy(l->rows.ptr, rows, (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(FOT_ERR_CUDA, "cudaMemcpy failed");
  if (rc != FOT_OK) {
    delete l;
    return rc;
  }
  p->rowlists.push_back(l);
  *out = l;
  return FOT_OK;
}

int fot_rowlist_gather(const fot_rowlist *l, void *dst, void *stream) {
  FOT_TRY(rowlist_check(l));
  if (l->n == 0) return FOT_OK;
  if (!dst) return fail(FOT_ERR_ARG, "null buffer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return l->prob->info.point_type_size[l->set] == 8 ? launch_gather<double>(l, dst, st)
                                                    : launch_gather<float>(l, dst, st);
}

int fot_rowlist_scatter_add(const fot_rowlist *l, const void *src, void *stream) {
  FOT_TRY(rowlist_check(l));
  if (l->n == 0) return FOT_OK;
  if (!src) return fail(FOT_ERR_ARG, "null buffer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // point datasets are double or float (4-byte ones are float in every loop)
  return l->prob->info.point_type_size[l->set] == 8 ? launch_scatter_add<double>(l, src, st)
                                                    : launch_scatter_add<float>(l, src, st);
}

int fot_rowlist_destroy(fot_rowlist *l) {
  if (!l) return FOT_OK;
  if (l->prob) {
    auto &v = l->prob->rowlists;
    v.erase(std::remove(v.begin(), v.end(), l), v.end());
  }
  delete l;
  return FOT_OK;
}

} // extern "C"
