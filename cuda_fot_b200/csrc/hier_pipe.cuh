// The pipelined persistent hierarchical-colour kernel (variant kVariantPipe),
// warp-specialised.
//
// A CTA runs T compute threads and two control warps over the tiles it
// claims (tiles = blocks in block-colour order, iteration after iteration):
//   * the RECORD warp claims tiles from the plan's queue and copies each
//     tile's record (header, point lists, local indices, per-point
//     contribution lists, dependency list; built by plan.cu) into one of
//     kRecSlots record slots with a bulk copy on the TMA engine (no
//     multicast).  Once the compute threads have written a tile back it
//     refills the tile's slot with the tile kRecSlots places ahead and
//     publishes the tile's completion flag (per block: iterations completed,
//     counted from Ctl::base);
//   * the STAGING warp gathers a tile's read rows into one of two row slots
//     with cp.async, then polls the completion flags of the blocks the tile
//     conflicts with and, once they hold, prefetches the tile's output rows;
//   * the COMPUTE threads compute each cell's per-slot increments into
//     shared memory, then, per written point, sum its contributions in
//     thread-colour order -- the order of the reference's colour-by-colour
//     shared accumulation, so results stay bit-identical to the CPU replay --
//     and store out[p] + sum.
// The roles hand over through mbarriers (record landed, rows landed, rows
// consumed, output rows landed / dependencies held, tile written back): a
// row slot is refilled as soon as the compute phase that read it ends, so the
// next-but-one tile's rows load during a tile's write-back; the compute threads
// also meet at a named barrier three times per tile.  The claim, the record
// copy and the flag release therefore stay off the compute threads' path.
// Every wait is bounded: after about two seconds the kernel sets
// kErrWaitLimit in Ctl::error, drains its copies in flight and returns.
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

// ---- small PTX helpers of the warp-specialised kernel -------------------------
__device__ __forceinline__ unsigned int ld_relaxed_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// arrive once every cp.async this thread issued so far has landed
__device__ __forceinline__ void mbar_arrive_cp_async(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
template <int T> __device__ __forceinline__ void named_bar_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(T) : "memory");
}
// named barrier 1 over T threads that also ANDs a predicate
template <int T> __device__ __forceinline__ bool named_bar_and(bool v) {
  unsigned r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}"
      : "=r"(r)
      : "r"((unsigned)v), "n"(T)
      : "memory");
  return r != 0;
}
// Bounded mbarrier wait that also gives up once *stop is set.
__device__ __forceinline__ bool mbar_wait_or_stop(uint64_t *bar, unsigned phase,
                                                  const volatile uint32_t *stop) {
  if (mbar_try_wait(bar, phase)) return true;
  const uint64_t t0 = global_timer_ns();
  for (unsigned i = 1;; ++i) {
    if (mbar_try_wait(bar, phase)) return true;
    if ((i & 15u) == 0 && (*stop || global_timer_ns() - t0 > 2000000000ull)) return false;
  }
}

// Dependency flags of a tile, read by the 32 lanes of one warp: every block
// conflicting with the tile must have completed what precedes it -- blocks of
// an earlier colour iteration `it` (flag >= it + 1), the others and the block
// itself iteration it - 1 (flag >= it); `it` counts from Ctl::base.  Lane l
// holds entries l, l + 32, ...; the block's own flag is the entry after the
// list.  Loads are relaxed; the caller issues one acquire fence once all hold.
constexpr int kDepPerLane = 4;

struct DepProbe {
  unsigned int have[kDepPerLane];
  unsigned int need[kDepPerLane];
  const unsigned int *ptr[kDepPerLane];

  template <class L>
  __device__ __forceinline__ void issue(const RecView<L> &m, uint32_t it, const unsigned int *flags,
                                        uint32_t round) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int q = 0; q < kDepPerLane; ++q) {
      const uint32_t e = lane + 32u * (q + kDepPerLane * round);
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
  __device__ __forceinline__ bool ready() const {  // warp-uniform
    bool ok = true;
#pragma unroll
    for (int q = 0; q < kDepPerLane; ++q) ok = ok && have[q] >= need[q];
    return __all_sync(0xFFFFFFFFu, ok);
  }
  __device__ __forceinline__ void reload() {
#pragma unroll
    for (int q = 0; q < kDepPerLane; ++q)
      if (ptr[q] && have[q] < need[q]) have[q] = ld_relaxed_gpu(ptr[q]);
  }
};

// Wait (bounded by wall time) until every dependency of a tile holds; all
// 32 lanes of the warp call it.  Returns false on timeout or stop.
template <class L>
__device__ __forceinline__ bool wait_deps(const RecView<L> &m, uint32_t it, const unsigned int *flags,
                                          const volatile uint32_t *stop) {
  const uint32_t rounds = (m.ndep + 1 + 32u * kDepPerLane - 1) / (32u * kDepPerLane);
  uint64_t t0 = 0;
  for (uint32_t r = 0; r < rounds; ++r) {
    DepProbe pr;
    pr.issue(m, it, flags, r);
    for (unsigned i = 0; !pr.ready(); ++i) {
      if ((i & 15u) == 0) {
        const uint64_t t = global_timer_ns();
        if (t0 == 0) t0 = t;
        if (*stop || t - t0 > 2000000000ull) return false;
      }
      __nanosleep(64);
      pr.reload();
    }
  }
  return true;
}

// Stage the read rows of a tile into a row slot: the 32 lanes of one warp.
template <class L, bool SOA>
__device__ __forceinline__ void ws_stage_rows(const LoopData &d, const HierPlanDev &P,
                                              unsigned char *slot, const RecView<L> &m) {
  using read_t = typename L::read_t;
  const uint32_t lane = threadIdx.x & 31u;
  static_for_read<L>([&](auto r) {
    constexpr int R = decltype(r)::value;
    constexpr int DIM = L::read_dim(R);
    constexpr int ROW = DIM * (int)sizeof(read_t);
    const bool c0 = L::read_class(R) == 0;
    const uint32_t n = c0 ? m.n0 : m.n1;
    const uint32_t *pts = c0 ? m.pts0 : m.pts1;
    const char *src = static_cast<const char *>(d.point[L::read_set(R)]);
    char *dst = reinterpret_cast<char *>(slot + P.read_off[R]);
    if constexpr (!SOA) {
      constexpr int CS = ROW % 16 == 0 ? 16 : (ROW % 8 == 0 ? 8 : 4);
      constexpr int CH = ROW / CS;
      for (uint32_t e = lane; e < n * CH; e += 32) {
        const uint32_t i = e / CH, c = e - i * CH;
        const char *g = src + (size_t)pts[i] * ROW + c * CS;
        char *s = dst + (size_t)i * ROW + c * CS;
        if constexpr (CS == 16) cp_async16(s, g);
        else if constexpr (CS == 8) cp_async8(s, g);
        else cp_async4(s, g);
      }
    } else {
      const uint32_t np = d.n_points[L::read_set(R)];
      for (uint32_t e = lane; e < n * DIM; e += 32) {
        const uint32_t k = e / n, i = e - k * n;
        const char *g = src + ((size_t)k * np + pts[i]) * sizeof(read_t);
        char *s = dst + ((size_t)i * DIM + k) * sizeof(read_t);
        if constexpr (sizeof(read_t) == 8) cp_async8(s, g);
        else cp_async4(s, g);
      }
    }
  });
}

// kRecSlots: tile-record slots (2 or 3; the plan picks 3 when the extra slot
// costs no resident CTA).  Registers are capped at the loop's kRegCap for
// every thread of the CTA.
template <class L, bool SOA, int T, uint32_t kRecSlots>
__global__ void __launch_bounds__(T + 64) __maxnreg__(L::kRegCap)
    k_hier_pipe(LoopData d, HierPlanDev P) {
  using out_t = typename L::out_t;
  using read_t = typename L::read_t;
  constexpr int D = L::kDim, K = L::kOut;
  constexpr int ROW_OUT = K * (int)sizeof(out_t);
  constexpr bool kPrefetchOut = !SOA && ROW_OUT % 16 == 0;
  constexpr uint32_t kRecordWarp = T / 32, kStagingWarp = T / 32 + 1;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t s_rec_full[kRecSlots];
  __shared__ __align__(8) uint64_t s_tile_done[kRecSlots];
  __shared__ __align__(8) uint64_t s_rows_full[2];
  __shared__ __align__(8) uint64_t s_out_full[2];
  __shared__ __align__(8) uint64_t s_rows_empty[2];
  __shared__ uint32_t s_iter[kRecSlots];   // iteration of the tile in each record slot
  __shared__ uint32_t s_valid[kRecSlots];  // 0: no tile (end of this CTA's queue)
  __shared__ uint32_t s_abort[2];          // per row slot: skip the write-back
  __shared__ uint32_t s_tile_abort[kRecSlots];  // per record slot: the tile was not written back
  __shared__ volatile uint32_t s_stop;     // a role gave up (error path)
  const uint32_t tid = threadIdx.x;
  const uint32_t warp = tid >> 5, lane = tid & 31u;
  unsigned char *const rec_base = smem;
  unsigned char *const rows_base = smem + P.rows_off;
  out_t *const inc = reinterpret_cast<out_t *>(smem + P.inc_off);
  out_t *__restrict__ out = static_cast<out_t *>(d.out);

  if (tid == 0) {
    for (uint32_t s = 0; s < kRecSlots; ++s) {
      mbar_init(&s_rec_full[s], 1);
      mbar_init(&s_tile_done[s], T / 32);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&s_rows_full[b], 33);
      mbar_init(&s_rows_empty[b], 1);
      mbar_init(&s_out_full[b], 33);
    }
    mbar_fence_init();
    s_stop = 0;
  }
  __syncthreads();
  const uint32_t base = *(volatile unsigned int *)&P.ctl->base;

  if (warp == kRecordWarp) {
    // ---------------------------------------------------------------- record
    if (lane == 0) {
      uint32_t uses[kRecSlots] = {};  // copies issued per slot
      bool valid[kRecSlots] = {};
      uint32_t blk[kRecSlots] = {};
      // a slot is refilled with a freshly claimed tile: claiming only when a
      // slot frees keeps few tiles claimed ahead of their dependencies
      bool more = true;
      auto refill = [&](uint32_t s) {
        const uint32_t t = more ? atomicAdd(&P.ctl->ticket, 1u) : P.total_tiles;
        const bool ok = more && t < P.total_tiles && *(volatile unsigned int *)&P.ctl->error == 0;
        const uint32_t it = ok ? t / P.n_blocks : 0;
        const uint32_t b = ok ? t - it * P.n_blocks : 0;
        s_iter[s] = it;
        s_valid[s] = ok;
        valid[s] = ok;
        blk[s] = b;
        if (ok) {
          const uint32_t off = P.rec_off[b], end = P.rec_off[b + 1];
          // the slot was last read through the generic proxy
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_expect_tx(&s_rec_full[s], end - off);
          bulk_copy_g2s(rec_base + s * P.rec_slot, P.rec + off, end - off, &s_rec_full[s]);
        } else {
          mbar_arrive(&s_rec_full[s]);
          more = false;
        }
        ++uses[s];
      };
      for (uint32_t s = 0; s < kRecSlots && more; ++s) refill(s);
      for (uint32_t j = 0;; ++j) {
        const uint32_t s = j % kRecSlots;
        if (!valid[s]) break;
        if (!mbar_wait_or_stop(&s_tile_done[s], (j / kRecSlots) & 1u, &s_stop)) {
          atomicOr(&P.ctl->error, kErrWaitLimit);
          s_stop = 1;
          break;
        }
        // a tile that skipped its write-back publishes no completion: its
        // dependents time out instead of adding on top of missing sums
        if (s_tile_abort[s]) {
          s_stop = 1;
          break;
        }
        // the compute threads' stores (ordered before this thread by the
        // mbarrier) become visible before the flag
        st_release_gpu(P.block_done + blk[s], base + s_iter[s] + 1);
        if (more) refill(s);
        else valid[s] = false;
      }
      // let every record copy still in flight land (bounded)
      for (uint32_t s = 0; s < kRecSlots; ++s)
        if (uses[s] > 0) (void)mbar_wait(&s_rec_full[s], (uses[s] - 1) & 1u);
    }
    __syncwarp();
  } else if (warp == kStagingWarp) {
    // --------------------------------------------------------------- staging
    bool err = false;
    for (uint32_t j = 0;; ++j) {
      const uint32_t s = j % kRecSlots, b = j & 1u;
      bool ok = mbar_wait_or_stop(&s_rec_full[s], (j / kRecSlots) & 1u, &s_stop);
      // the row slot of tile j - 2 is free once that tile's compute phase ended
      if (ok && j >= 2) ok = mbar_wait_or_stop(&s_rows_empty[b], ((j - 2) >> 1) & 1u, &s_stop);
      ok = __all_sync(0xFFFFFFFFu, ok);
      if (!ok || err || !s_valid[s]) {
        if (!ok && !err) {
          err = true;
          if (lane == 0) atomicOr(&P.ctl->error, kErrWaitLimit);
        }
        if (lane == 0) {
          s_valid[s] = 0;
          if (err) s_stop = 1;
          mbar_arrive(&s_rows_full[b]);
        }
        mbar_arrive(&s_rows_full[b]);
        break;
      }
      const RecView<L> m(rec_base + s * P.rec_slot);
      ws_stage_rows<L, SOA>(d, P, rows_base + b * P.rows_bytes, m);
      mbar_arrive_cp_async(&s_rows_full[b]);
      if (lane == 0) mbar_arrive(&s_rows_full[b]);
      // dependencies, then the output rows (into the output slot of tile
      // j - 2, free once that tile is written back)
      bool dep_ok = wait_deps(m, base + s_iter[s], P.block_done, &s_stop);
      fence_acq_rel_gpu();
      if (dep_ok && j >= 2)
        dep_ok = __all_sync(0xFFFFFFFFu, mbar_wait_or_stop(&s_tile_done[(j - 2) % kRecSlots],
                                                           ((j - 2) / kRecSlots) & 1u, &s_stop));
      if (kPrefetchOut && dep_ok) {
        constexpr int CH = ROW_OUT / 16;
        char *ob = reinterpret_cast<char *>(smem + P.outbuf_off + b * P.outbuf_bytes);
        const char *og = reinterpret_cast<const char *>(out);
        for (uint32_t e = lane; e < m.n0 * CH; e += 32) {
          const uint32_t i = e / CH, q = e - i * CH;
          cp_async16(ob + (size_t)i * ROW_OUT + q * 16, og + (size_t)m.pts0[i] * ROW_OUT + q * 16);
        }
      }
      if (lane == 0) {
        s_abort[b] = dep_ok ? 0u : 1u;
        if (!dep_ok) atomicOr(&P.ctl->error, kErrWaitLimit);
      }
      mbar_arrive_cp_async(&s_out_full[b]);
      if (lane == 0) mbar_arrive(&s_out_full[b]);
      if (!dep_ok) err = true;  // later tiles are dropped
    }
    cp_async_wait_all();
  } else {
    // --------------------------------------------------------------- compute
    for (uint32_t j = 0;; ++j) {
      const uint32_t s = j % kRecSlots, b = j & 1u, ph = (j >> 1) & 1u;
      const bool ok_rows = mbar_wait_or_stop(&s_rows_full[b], ph, &s_stop);
      if (!named_bar_and<T>(ok_rows)) {
        if (tid == 0) {
          atomicOr(&P.ctl->error, kErrWaitLimit);
          s_stop = 1;
        }
        break;
      }
      if (!s_valid[s]) break;
      // the record landed through the async proxy
      (void)mbar_try_wait(&s_rec_full[s], (j / kRecSlots) & 1u);
      const RecView<L> m(rec_base + s * P.rec_slot);
      const unsigned char *rows = rows_base + b * P.rows_bytes;
      if (tid < m.ncell) {
        SmemRows<L> rv;
#pragma unroll
        for (int q = 0; q < D; ++q) {
          rv.l[0][q] = m.lidx0[q * m.ncell + tid];
          rv.l[1][q] = L::kHasClass1 ? m.lidx1[q * m.ncell + tid] : 0;
        }
        static_for_read<L>([&](auto r) {
          constexpr int R = decltype(r)::value;
          rv.base[R] = reinterpret_cast<const read_t *>(rows + P.read_off[R]);
        });
        out_t v[D][K];
        Direct dir{d.cell, m.start + tid, d.n_cells};
        L::cell(rv, dir, v);
#pragma unroll
        for (int q = 0; q < D; ++q)
#pragma unroll
          for (int k = 0; k < K; ++k) inc[(k * D + q) * T + tid] = v[q][k];
      }
      named_bar_sync<T>();
      if (tid == 0) mbar_arrive(&s_rows_empty[b]);  // the row slot may be refilled
      const bool ok_out = mbar_wait_or_stop(&s_out_full[b], ph, &s_stop);
      if (ok_out && !s_abort[b]) {
        const out_t *ob = reinterpret_cast<const out_t *>(smem + P.outbuf_off + b * P.outbuf_bytes);
        for (uint32_t i = tid; i < m.n0; i += T) {
          out_t acc[K];
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = out_t(0);
          const uint32_t e0 = m.pc_off[i], e1 = m.pc_off[i + 1];
          for (uint32_t e = e0; e < e1; ++e) {
            const uint32_t ie = m.pc_idx[e];
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] += inc[k * D * T + ie];
          }
          const uint32_t p = m.pts0[i];
          if constexpr (kPrefetchOut) {
            using vec_t = typename std::conditional<sizeof(out_t) == 8, double2, float4>::type;
            constexpr int CH = ROW_OUT / 16;
            constexpr int PER = 16 / sizeof(out_t);
            vec_t *og = reinterpret_cast<vec_t *>(out) + (size_t)p * CH;
            const vec_t *obv = reinterpret_cast<const vec_t *>(ob) + (size_t)i * CH;
#pragma unroll
            for (int q = 0; q < CH; ++q) {
              vec_t w = obv[q];
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
            for (int k = 0; k < K; ++k) o[k] = __ldcg(out + out_index(SOA, d.n_points[0], p, K, k));
#pragma unroll
            for (int k = 0; k < K; ++k)
              __stcg(out + out_index(SOA, d.n_points[0], p, K, k), o[k] + acc[k]);
          }
        }
      }
      if (tid == 0) s_tile_abort[s] = (ok_out && !s_abort[b]) ? 0u : 1u;
      __syncwarp();
      if (lane == 0) mbar_arrive(&s_tile_done[s]);
      // the increments buffer is reused by the next tile
      if (!named_bar_and<T>(ok_out)) {
        if (tid == 0) {
          atomicOr(&P.ctl->error, kErrWaitLimit);
          s_stop = 1;
        }
        break;
      }
    }
  }
  __syncthreads();
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
