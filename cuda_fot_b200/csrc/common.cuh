// Shared internals of libfot: error reporting, device buffers, the device
// control block of the persistent executors, and small PTX helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "fot.h"

#ifndef MY_SIZE
#define MY_SIZE unsigned
#endif

namespace fot {

// ---- error reporting ------------------------------------------------------
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);

#define FOT_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      return ::fot::fail(e_ == cudaErrorMemoryAllocation ? FOT_ERR_NOMEM        \
                                                         : FOT_ERR_CUDA,        \
                         "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                         __FILE__, __LINE__);                                  \
    }                                                                          \
  } while (0)

#define FOT_TRY(expr)                                                          \
  do {                                                                         \
    int rc_ = (expr);                                                          \
    if (rc_ != FOT_OK) return rc_;                                             \
  } while (0)

// ---- device buffer ----------------------------------------------------------
struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  int alloc(size_t n) {
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
      ptr = nullptr;
      return fail(FOT_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
    }
    bytes = n;
    return FOT_OK;
  }
  template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// ---- device control block of the persistent executors --------------------
// One per plan (and per batch).  ticket: next tile to claim; done: tiles whose
// write-back finished; exited: CTAs that left the claim loop (the last one
// resets the three counters so the next launch starts from zero); error:
// bit 0 = a dependency wait hit its limit.
// base: iterations completed by all earlier launches (the per-block
// completion flags of the pipelined executor count from it); the last CTA
// advances it.
struct Ctl {
  unsigned int ticket;
  unsigned int done;
  unsigned int exited;
  unsigned int error;
  unsigned int base;
  unsigned int pad[3];
};

__device__ __forceinline__ void st_release_gpu(unsigned int *p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr unsigned int kErrWaitLimit = 1u;
// Upper bound of the dependency-wait polls (each followed by a ~256 ns
// sleep): about 2-4 s before the kernel gives up and flags kErrWaitLimit.
constexpr unsigned int kWaitPollLimit = 8u * 1000u * 1000u;

// ---- loop descriptions ------------------------------------------------------
int describe(int loop, fot_loop_info *info);

// ---- PTX helpers ------------------------------------------------------------
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned int smem_addr(const void *p) {
  return static_cast<unsigned int>(__cvta_generic_to_shared(p));
}

// asynchronous global -> shared copies (LDGSTS); 16-byte copies bypass L1
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// mbarrier + 1D bulk copy (TMA engine, no tensor map, no multicast) of a
// 16-byte aligned segment of this GPU's global memory into shared memory.
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for an mbarrier phase: gives up (returns false) after about
// two seconds of wall time.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase) {
  if (mbar_try_wait(bar, phase)) return true;
  const uint64_t t0 = global_timer_ns();
  for (unsigned i = 1;; ++i) {
    if (mbar_try_wait(bar, phase)) return true;
    if ((i & 63u) == 0 && global_timer_ns() - t0 > 2000000000ull) return false;
  }
}

} // namespace fot
