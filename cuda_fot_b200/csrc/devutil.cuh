// Device-wide helpers of the plan and ordering builders (CUB sorts and scans
// with their own temporary storage, host<->device vector copies).
#pragma once

#include <cub/cub.cuh>

#include <vector>

#include "common.cuh"

namespace fot {

inline uint32_t blocks_for(size_t n, uint32_t t = 256) { return (uint32_t)((n + t - 1) / t); }

// Grow-only temporary storage of the CUB calls below (one per host thread,
// per device), so that the many small sorts of the level-by-level orderings
// do not allocate and free device memory every time.
inline int cub_scratch(size_t bytes, void **ptr) {
  struct Scratch {
    DevBuf buf[16];
  };
  static thread_local Scratch s;
  int dev = 0;
  cudaGetDevice(&dev);
  DevBuf &b = s.buf[dev & 15];
  if (b.bytes < bytes) FOT_TRY(b.alloc(bytes + bytes / 2 + 4096));
  *ptr = b.ptr;
  return FOT_OK;
}

template <class K, class V>
int sort_pairs(const K *kin, K *kout, const V *vin, V *vout, size_t n, cudaStream_t st = 0,
               int end_bit = sizeof(K) * 8) {
  if (n == 0) return FOT_OK;
  size_t tb = 0;
  FOT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, (int)n, 0, end_bit, st));
  void *tmp = nullptr;
  FOT_TRY(cub_scratch(tb, &tmp));
  FOT_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, vin, vout, (int)n, 0, end_bit, st));
  return FOT_OK;
}

template <class K> int sort_keys(const K *kin, K *kout, size_t n, cudaStream_t st = 0) {
  if (n == 0) return FOT_OK;
  size_t tb = 0;
  FOT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, kin, kout, (int)n, 0, sizeof(K) * 8, st));
  void *tmp = nullptr;
  FOT_TRY(cub_scratch(tb, &tmp));
  FOT_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tb, kin, kout, (int)n, 0, sizeof(K) * 8, st));
  return FOT_OK;
}

// unique of sorted keys; returns the count
template <class K> int unique_keys(const K *in, K *out, size_t n, uint32_t *count, cudaStream_t st = 0) {
  *count = 0;
  if (n == 0) return FOT_OK;
  DevBuf nsel;
  FOT_TRY(nsel.alloc(4));
  size_t tb = 0;
  FOT_CUDA(cub::DeviceSelect::Unique(nullptr, tb, in, out, nsel.as<uint32_t>(), (int)n, st));
  void *tmp = nullptr;
  FOT_TRY(cub_scratch(tb, &tmp));
  FOT_CUDA(cub::DeviceSelect::Unique(tmp, tb, in, out, nsel.as<uint32_t>(), (int)n, st));
  FOT_CUDA(cudaMemcpyAsync(count, nsel.ptr, 4, cudaMemcpyDeviceToHost, st));
  FOT_CUDA(cudaStreamSynchronize(st));
  return FOT_OK;
}

template <class T> int excl_sum(const T *in, T *out, size_t n, cudaStream_t st = 0) {
  if (n == 0) return FOT_OK;
  size_t tb = 0;
  FOT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, st));
  void *tmp = nullptr;
  FOT_TRY(cub_scratch(tb, &tmp));
  FOT_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, (int)n, st));
  return FOT_OK;
}

template <class T> int upload(DevBuf &b, const std::vector<T> &v) {
  FOT_TRY(b.alloc(v.size() * sizeof(T)));
  if (!v.empty()) FOT_CUDA(cudaMemcpy(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return FOT_OK;
}

template <class T> int download(std::vector<T> &v, const DevBuf &b, size_t n) {
  v.resize(n);
  if (n) FOT_CUDA(cudaMemcpy(v.data(), b.ptr, n * sizeof(T), cudaMemcpyDeviceToHost));
  return FOT_OK;
}

template <class T> int download(std::vector<T> &v, const T *d, size_t n) {
  v.resize(n);
  if (n) FOT_CUDA(cudaMemcpy(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
  return FOT_OK;
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

} // namespace fot
