// The pipelined persistent hierarchical-colour kernel (variant kVariantPipe).
//
// Each CTA runs a two-deep software pipeline over the tiles it claims (tiles
// = blocks in block-colour order, iteration after iteration):
//   * a tile's RECORD (header, point lists, local indices, per-point
//     contribution lists; built by plan.cu) arrives by one bulk copy on the
//     TMA engine, completing an mbarrier, one tile ahead;
//   * the tile's READ ROWS are staged with cp.async into the same pipeline
//     buffer while the previous tile computes and writes back;
//   * if the tile's dependency (all tiles of the earlier block colours
//     written back) already holds when the tile starts, its OUTPUT ROWS are
//     prefetched too, so the write-back is a plain store;
//   * compute: each thread computes its cell's per-slot increments into a
//     shared buffer; one barrier; then each thread owns written points and
//     sums their contributions in thread-colour order -- the order of the
//     reference's colour-by-colour shared accumulation, so results stay
//     bit-identical to the CPU replay -- and writes out[p] += sum.
// Three CTA barriers per tile instead of one per thread colour; every wait is
// bounded (mbarrier waits by wall time, the dependency wait by polls).
#pragma once

#include <cstdint>
#include <type_traits>

#include "common.cuh"

namespace fot {

// View of a tile record in shared memory (layout: plan.cu, step 4b).
template <class L> struct RecView {
  uint32_t start, ncell, n0, n1, ntcol, wait, ndep, block;
  const uint32_t *pts0, *pts1;
  const uint16_t *lidx0, *lidx1;
  const uint16_t *pc_off, *pc_idx;
  const uint32_t *dep;
  __device__ __forceinline__ explicit RecView(const unsigned char *r) {
    const uint32_t *h = reinterpret_cast<const uint32_t *>(r);
    start = h[0];
    ncell = h[1];
    n0 = h[2];
    n1 = h[3];
    ntcol = h[4];
    wait = h[5];
    ndep = h[6];
    block = h[7];
    pts0 = h + 8;
    pts1 = pts0 + n0;
    const uint16_t *l = reinterpret_cast<const uint16_t *>(pts1 + n1);
    lidx0 = l;
    l += L::kDim * ncell;
    lidx1 = l;
    if (L::kHasClass1) l += L::kDim * ncell;
    pc_off = l;
    pc_idx = l + n0 + 1;
    const uintptr_t e = reinterpret_cast<uintptr_t>(pc_idx + L::kDim * ncell);
    dep = reinterpret_cast<const uint32_t *>((e + 3) & ~uintptr_t(3));
  }
};

__device__ __forceinline__ unsigned int ld_relaxed_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Dependency flags of a tile, read by the lanes of one warp: every block
// conflicting with the tile must have completed what precedes it -- blocks
// of an earlier colour iteration `it` (flag >= it + 1), the others and the
// block itself iteration it - 1 (flag >= it); `it` counts from the launch's
// base.  Lane l holds entries l, l + 32, ... (up to kDepPerLane of them);
// the block's own flag is the entry after the list.
constexpr int kDepPerLane = 4;

template <class L> struct DepProbe {
  unsigned int have[kDepPerLane];
  unsigned int need[kDepPerLane];
  const unsigned int *ptr[kDepPerLane];
  bool overflow;

  // issue relaxed loads (non-blocking until evaluated)
  __device__ __forceinline__ void issue(const RecView<L> &m, uint32_t it, const unsigned int *flags) {
    const uint32_t lane = threadIdx.x & 31u;
    overflow = m.ndep + 1 > 32u * kDepPerLane;
#pragma unroll
    for (int q = 0; q < kDepPerLane; ++q) {
      const uint32_t e = lane + 32u * q;
      ptr[q] = nullptr;
      need[q] = 0;
      have[q] = 0;
      if (e <= m.ndep) {
        uint32_t blk;
        if (e == m.ndep) {
          blk = m.block;
          need[q] = it;
        } else {
          const uint32_t v = m.dep[e];
          blk = v & 0x7FFFFFFFu;
          need[q] = it + (v >> 31);
        }
        ptr[q] = flags + blk;
        have[q] = ld_relaxed_gpu(ptr[q]);
      }
    }
  }
  // all satisfied (warp-uniform)
  __device__ __forceinline__ bool ready() const {
    bool ok = !overflow;
#pragma unroll
    for (int q = 0; q < kDepPerLane; ++q) ok = ok && have[q] >= need[q];
    return __all_sync(0xFFFFFFFFu, ok);
  }
  // re-read the flags not yet satisfied
  __device__ __forceinline__ void reload() {
#pragma unroll
    for (int q = 0; q < kDepPerLane; ++q)
      if (ptr[q] && have[q] < need[q]) have[q] = ld_relaxed_gpu(ptr[q]);
  }
};

// Blocking bounded check for a tile whose list is too long for a probe.
template <class L>
__device__ __forceinline__ bool deps_ready_slow(const RecView<L> &m, uint32_t it,
                                                const unsigned int *flags) {
  const uint32_t lane = threadIdx.x & 31u;
  bool ok = true;
  for (uint32_t e = lane; e <= m.ndep; e += 32) {
    uint32_t blk, need;
    if (e == m.ndep) {
      blk = m.block;
      need = it;
    } else {
      const uint32_t v = m.dep[e];
      blk = v & 0x7FFFFFFFu;
      need = it + (v >> 31);
    }
    if (ld_acquire_gpu(flags + blk) < need) ok = false;
  }
  return __all_sync(0xFFFFFFFFu, ok);
}

// Stage the read rows of a tile (points from its record) into buffer `buf`.
template <class L, bool SOA, int THREADS>
__device__ __forceinline__ void pipe_stage_rows(const LoopData &d, const HierPlanDev &P,
                                                unsigned char *buf, const RecView<L> &m) {
  using read_t = typename L::read_t;
  const uint32_t tid = threadIdx.x;
  static_for_read<L>([&](auto r) {
    constexpr int R = decltype(r)::value;
    constexpr int DIM = L::read_dim(R);
    constexpr int ROW = DIM * (int)sizeof(read_t);
    const bool c0 = L::read_class(R) == 0;
    const uint32_t n = c0 ? m.n0 : m.n1;
    const uint32_t *pts = c0 ? m.pts0 : m.pts1;
    const char *src = static_cast<const char *>(d.point[L::read_set(R)]);
    char *dst = reinterpret_cast<char *>(buf + P.read_off[R]);
    if constexpr (!SOA) {
      constexpr int CS = ROW % 16 == 0 ? 16 : (ROW % 8 == 0 ? 8 : 4);
      constexpr int CH = ROW / CS;
      for (uint32_t e = tid; e < n * CH; e += THREADS) {
        const uint32_t i = e / CH, c = e - i * CH;
        const char *g = src + (size_t)pts[i] * ROW + c * CS;
        char *s = dst + (size_t)i * ROW + c * CS;
        if constexpr (CS == 16) cp_async16(s, g);
        else if constexpr (CS == 8) cp_async8(s, g);
        else cp_async4(s, g);
      }
    } else {
      const uint32_t np = d.n_points[L::read_set(R)];
      for (uint32_t e = tid; e < n * DIM; e += THREADS) {
        const uint32_t k = e / n, i = e - k * n;
        const char *g = src + ((size_t)k * np + pts[i]) * sizeof(read_t);
        char *s = dst + ((size_t)i * DIM + k) * sizeof(read_t);
        if constexpr (sizeof(read_t) == 8) cp_async8(s, g);
        else cp_async4(s, g);
      }
    }
  });
}

template <class L, bool SOA, int THREADS>
__global__ void __launch_bounds__(THREADS, hier_min_blocks<L, THREADS>())
    k_hier_pipe(LoopData d, HierPlanDev P) {
  using out_t = typename L::out_t;
  using read_t = typename L::read_t;
  constexpr int D = L::kDim, K = L::kOut;
  constexpr int ROW_OUT = K * (int)sizeof(out_t);
  constexpr bool kPrefetchOut = !SOA && ROW_OUT % 16 == 0;
  constexpr uint32_t NONE = 0xFFFFFFFFu;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ uint32_t s_iter[2];
  __shared__ uint32_t s_valid[2];
  __shared__ int s_dep[2];  // the dependencies of the tile in each buffer already held
  __shared__ int s_abort;
  const uint32_t tid = threadIdx.x;
  out_t *inc = reinterpret_cast<out_t *>(smem + P.inc_off);
  out_t *outbuf = reinterpret_cast<out_t *>(smem + P.outbuf_off);
  out_t *__restrict__ out = static_cast<out_t *>(d.out);
  const uint32_t base = *(volatile unsigned int *)&P.ctl->base;

  // thread 0's pipeline state
  uint32_t t_claim = NONE;                     // ticket for the next buffer refill
  uint32_t pre_off = 0, pre_bytes = 0, pre_iter = 0;  // its record
  bool pre_ok = false;

  auto claim = [&]() {  // thread 0
    t_claim = atomicAdd(&P.ctl->ticket, 1u);
  };
  auto prefetch_record_info = [&]() {  // thread 0, after claim()
    pre_ok = t_claim < P.total_tiles && !(*(volatile unsigned int *)&P.ctl->error);
    if (pre_ok) {
      const uint32_t it = t_claim / P.n_blocks, b = t_claim - it * P.n_blocks;
      pre_off = P.rec_off[b];
      pre_bytes = P.rec_off[b + 1] - pre_off;
      pre_iter = it;
    }
  };
  auto issue_record = [&](int c) {  // thread 0: refill buffer c with the claimed tile
    if (pre_ok) {
      s_iter[c] = pre_iter;
      s_valid[c] = 1;
      // the buffer was last read through the generic proxy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&s_bar[c], pre_bytes);
      bulk_copy_g2s(smem + c * P.buf_bytes, P.rec + pre_off, pre_bytes, &s_bar[c]);
    } else {
      s_valid[c] = 0;
    }
  };

  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0) {
    claim();
    prefetch_record_info();
    issue_record(0);
    claim();
    prefetch_record_info();
    issue_record(1);
    claim();
  }
  __syncthreads();
  {
    const bool first = s_valid[0];
    const bool ok = !first || mbar_wait(&s_bar[0], 0);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(&P.ctl->error, kErrWaitLimit);
        s_valid[0] = 0;
      }
      __syncthreads();
    } else if (first) {
      const RecView<L> m0(smem);
      pipe_stage_rows<L, SOA, THREADS>(d, P, smem, m0);
      if (tid < 32) {
        const bool r = deps_ready_slow(m0, base + s_iter[0], P.block_done);
        if (tid == 0) s_dep[0] = r;
      }
    }
  }
  cp_async_commit();

  for (uint32_t k = 0;; ++k) {
    const int c = k & 1, n = c ^ 1;
    if (!s_valid[c]) break;
    unsigned char *buf = smem + c * P.buf_bytes;
    const RecView<L> m(buf);
    const uint32_t iter = s_iter[c];
    const uint32_t it_abs = base + iter;
    // 1. the claimed tile's record offsets
    if (tid == 0) prefetch_record_info();
    // 2. this tile's rows have landed
    cp_async_wait_group<0>();
    __syncthreads();
    // 3. prefetch this tile's output rows when its dependencies already held
    //    (checked when its record arrived)
    const bool dep = s_dep[c];
    if constexpr (kPrefetchOut) {
      if (dep) {
        constexpr int CH = ROW_OUT / 16;
        char *ob = reinterpret_cast<char *>(outbuf);
        const char *og = reinterpret_cast<const char *>(out);
        for (uint32_t e = tid; e < m.n0 * CH; e += THREADS) {
          const uint32_t i = e / CH, q = e - i * CH;
          cp_async16(ob + (size_t)i * ROW_OUT + q * 16, og + (size_t)m.pts0[i] * ROW_OUT + q * 16);
        }
      }
    }
    cp_async_commit();
    // 4. the next tile's record, then its rows (a record that did not arrive
    //    in time ends this CTA's queue after the current tile)
    {
      const bool next = s_valid[n];
      const bool ok = !next || mbar_wait(&s_bar[n], ((k + 1) >> 1) & 1u);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicOr(&P.ctl->error, kErrWaitLimit);
          s_valid[n] = 0;
        }
      } else if (next) {
        const RecView<L> mn(smem + n * P.buf_bytes);
        pipe_stage_rows<L, SOA, THREADS>(d, P, smem + n * P.buf_bytes, mn);
        // the next tile's dependencies (read now, used when it starts)
        if (tid < 32) {
          const bool r = deps_ready_slow(mn, base + s_iter[n], P.block_done);
          if (tid == 0) s_dep[n] = r;
        }
      }
    }
    cp_async_commit();
    // 5. compute: per-slot increments of each cell into the shared buffer
    if (tid < m.ncell) {
      SmemRows<L> rows;
#pragma unroll
      for (int s = 0; s < D; ++s) {
        rows.l[0][s] = m.lidx0[s * m.ncell + tid];
        rows.l[1][s] = L::kHasClass1 ? m.lidx1[s * m.ncell + tid] : 0;
      }
      static_for_read<L>([&](auto r) {
        constexpr int R = decltype(r)::value;
        rows.base[R] = reinterpret_cast<const read_t *>(buf + P.read_off[R]);
      });
      out_t v[D][K];
      Direct dir{d.cell, m.start + tid, d.n_cells};
      L::cell(rows, dir, v);
#pragma unroll
      for (int s = 0; s < D; ++s)
#pragma unroll
        for (int q = 0; q < K; ++q) inc[(q * D + s) * THREADS + tid] = v[s][q];
    }
    // 6. output rows (if prefetched) landed; otherwise wait (bounded) for the
    //    dependencies
    cp_async_wait_group<1>();
    if (tid < 32) {
      int ab = 0;
      if (!dep) {
        unsigned int polls = 0;
        while (!deps_ready_slow(m, it_abs, P.block_done)) {
          if (++polls > kWaitPollLimit) {
            if (tid == 0) atomicOr(&P.ctl->error, kErrWaitLimit);
            ab = 1;
            break;
          }
          __nanosleep(128);
        }
      }
      if (tid == 0) s_abort = ab;
    }
    __syncthreads();
    // 7. per written point: sum its contributions in thread-colour order and
    //    add to the output row
    if (!s_abort) {
      for (uint32_t j = tid; j < m.n0; j += THREADS) {
        out_t acc[K];
#pragma unroll
        for (int q = 0; q < K; ++q) acc[q] = out_t(0);
        const uint32_t e0 = m.pc_off[j], e1 = m.pc_off[j + 1];
        for (uint32_t e = e0; e < e1; ++e) {
          const uint32_t ie = m.pc_idx[e];
#pragma unroll
          for (int q = 0; q < K; ++q) acc[q] += inc[q * D * THREADS + ie];
        }
        const uint32_t p = m.pts0[j];
        if constexpr (kPrefetchOut) {
          using vec_t = typename std::conditional<sizeof(out_t) == 8, double2, float4>::type;
          constexpr int CH = ROW_OUT / 16;
          constexpr int PER = 16 / sizeof(out_t);
          vec_t *og = reinterpret_cast<vec_t *>(out) + (size_t)p * CH;
          const vec_t *ob = reinterpret_cast<const vec_t *>(outbuf) + (size_t)j * CH;
#pragma unroll
          for (int q = 0; q < CH; ++q) {
            vec_t w = dep ? ob[q] : __ldcg(og + q);
            if constexpr (PER == 2) {
              w.x += acc[q * 2];
              w.y += acc[q * 2 + 1];
            } else {
              w.x += acc[q * 4];
              w.y += acc[q * 4 + 1];
              w.z += acc[q * 4 + 2];
              w.w += acc[q * 4 + 3];
            }
            __stcg(og + q, w);
          }
        } else {
          out_t o[K];
#pragma unroll
          for (int q = 0; q < K; ++q) o[q] = __ldcg(out + out_index(SOA, d.n_points[0], p, K, q));
#pragma unroll
          for (int q = 0; q < K; ++q) __stcg(out + out_index(SOA, d.n_points[0], p, K, q), o[q] + acc[q]);
        }
      }
    }
    __syncthreads();
    // 8. signal; refill this buffer with the claimed tile; claim the next
    if (tid == 0) {
      st_release_gpu(P.block_done + m.block, it_abs + 1);
      issue_record(c);
      if (pre_ok) claim();
    }
  }
  // after an error, let any record copy still in flight land (bounded)
  if (tid == 0 && *(volatile unsigned int *)&P.ctl->error)
    for (int c = 0; c < 2; ++c)
      if (!mbar_try_wait(&s_bar[c], 0) || !mbar_try_wait(&s_bar[c], 1))
        (void)(mbar_wait(&s_bar[c], 0) && mbar_wait(&s_bar[c], 1));
  // the last CTA to leave resets the queue and advances the flags' base by
  // the iterations of this launch
  if (tid == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(&P.ctl->exited, 1u);
    if (prev == gridDim.x - 1) {
      atomicAdd(&P.ctl->base, P.total_tiles / P.n_blocks);
      atomicExch(&P.ctl->ticket, 0u);
      atomicExch(&P.ctl->done, 0u);
      atomicExch(&P.ctl->exited, 0u);
      __threadfence();
    }
  }
}

} // namespace fot
