// The split write-back hierarchical-colour kernels (variant kVariantSplit).
//
// The coloured replay of a plan (blocks in block-colour order; in a block,
// cells in thread-colour order accumulate into a zeroed per-block sum; then
// out[p] += sum for each written point) fixes, for every point p, the order
// out[p] = ((out[p] + S_b1) + S_b2) + ... over the blocks b1 < b2 < ... (plan
// order) that write p.  These kernels reproduce that order without making
// any tile wait for another:
//   * a point written by ONE block (private) gets out[p] += S_b as soon as
//     the block's sum is ready -- a fire-and-forget L2 reduction (RED.F64) for
//     FP64 data, whose single rounding equals the replay's add; FP32 data
//     (atomics there flush subnormals) take a load-add-store;
//   * a point written by several blocks (shared) gets S_b stored into the
//     point's slot for that block (plain stores, one buffer per iteration
//     parity); the NEXT launch -- the next iteration's, or the flush launch
//     that ends a run -- adds out[p] + S_b1 + S_b2 ... in plan order while its
//     own tiles fill the other buffer.  Private and shared points are
//     disjoint, so the combine never races with the tiles.
// Block colours therefore fix the summation order but never stall a tile.
// One launch runs ONE iteration; consecutive launches are chained with
// programmatic dependent launch: every CTA lets the next grid launch at once,
// and the next grid's tiles gather and compute (they only read datasets the
// loop never writes) before they wait (griddepcontrol.wait) for this grid to
// complete and only then write.  Loops that write cell data wait before
// computing.
//
// Two forms:
//   * k_hier_dsplit (direct): one CTA per tile, one thread per cell; each
//     thread gathers its cell's rows straight from HBM/L2 through the
//     plan-ordered mapping (like the atomic executor: thousands of
//     independent gathers in flight per SM), adds its increments into a
//     shared-memory sum one thread colour after another, and the block's
//     sums go out as above.  Extra CTAs at the end of the grid do the
//     combine.
//   * k_hier_split (staged): persistent CTAs of T compute threads and two
//     control warps; the RECORD warp bulk-copies each tile's record (plan.cu,
//     step 4b) into one of kRecSlots slots (TMA engine, no multicast), the
//     STAGING warp gathers the tile's read rows into one of two row slots
//     with cp.async, the compute threads compute from shared memory.  Tile i
//     of CTA c is launch[c + i * gridDim.x]; every CTA's compute threads
//     combine one chunk of the shared points after their wait.  Every wait
//     between the roles is bounded (about two seconds); on a timeout the
//     kernel sets kErrWaitLimit in Ctl::error and returns.
#pragma once

#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "hier_pipe.cuh"

namespace fot {

// Programmatic dependent launch (sm_90+): let the dependent grid launch /
// wait for the prerequisite grid to complete with its memory visible.  Both
// are no-ops when the grid was launched without the programmatic attribute.
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void griddep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Shared points [g0, g1) of the previous launch's buffer: out[p] plus the
// blocks' sums in plan order (thread t of nt).
template <class L, bool SOA>
__device__ __forceinline__ void combine_shared(const LoopData &d, const HierPlanDev &P, uint32_t g0,
                                               uint32_t g1, uint32_t t, uint32_t nt) {
  using out_t = typename L::out_t;
  constexpr int K = L::kOut;
  const out_t *part = static_cast<const out_t *>(P.partial) + (size_t)(P.put_buf ^ 1u) * P.n_slots * K;
  out_t *out = static_cast<out_t *>(d.out);
  for (uint32_t g = g0 + t; g < g1; g += nt) {
    const uint32_t p = P.comb_point[g], e0 = P.comb_base[g], e1 = P.comb_base[g + 1];
    out_t o[K];
#pragma unroll
    for (int k = 0; k < K; ++k) o[k] = __ldcg(out + out_index(SOA, d.n_points[0], p, K, k));
    for (uint32_t e = e0; e < e1; ++e)
#pragma unroll
      for (int k = 0; k < K; ++k) o[k] += __ldcg(part + (size_t)e * K + k);
#pragma unroll
    for (int k = 0; k < K; ++k) __stcg(out + out_index(SOA, d.n_points[0], p, K, k), o[k]);
  }
}

__device__ __forceinline__ void comb_chunk(uint32_t n, uint32_t c, uint32_t parts, uint32_t &g0,
                                           uint32_t &g1) {
  g0 = (uint32_t)((uint64_t)n * c / parts);
  g1 = (uint32_t)((uint64_t)n * (c + 1) / parts);
}

// Written point j of a tile (threads j = t, t + T, ...): sum its contributions
// in thread-colour order from the increments in shared memory, then add it
// (private) or store it into its slot of this launch's buffer (shared).
template <class L, bool SOA, int T>
__device__ __forceinline__ void split_writeback(const LoopData &d, const HierPlanDev &P,
                                                const RecView<L> &m, const typename L::out_t *inc,
                                                uint32_t t) {
  using out_t = typename L::out_t;
  constexpr int D = L::kDim, K = L::kOut;
  out_t *out = static_cast<out_t *>(d.out);
  out_t *put = static_cast<out_t *>(P.partial) + (size_t)P.put_buf * P.n_slots * K;
  const uint32_t *wslot = m.dep;  // split plans: the record's slot list
  for (uint32_t j = t; j < m.n0; j += T) {
    out_t acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = out_t(0);
    const uint32_t e0 = m.pc_off[j], e1 = m.pc_off[j + 1];
    for (uint32_t e = e0; e < e1; ++e) {
      const uint32_t ie = m.pc_idx[e];
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] += inc[k * D * T + ie];
    }
    const uint32_t p = m.pts0[j];
    const uint32_t ws = wslot[j];
    if (ws == 0xFFFFFFFFu) {
      // private point: this block alone writes it in this iteration
      if constexpr (sizeof(out_t) == 8) {
#pragma unroll
        for (int k = 0; k < K; ++k) atomicAdd(out + out_index(SOA, d.n_points[0], p, K, k), acc[k]);
      } else {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          out_t *o = out + out_index(SOA, d.n_points[0], p, K, k);
          __stcg(o, __ldcg(o) + acc[k]);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) __stcg(put + (size_t)ws * K + k, acc[k]);
    }
  }
}

// Direct form: CTAs [0, n_blocks) run one tile each, the comb_ctas after
// them combine the previous buffer (hardware CTA scheduling keeps several tiles per SM in
// different phases; a persistent form with one tile in flight per CTA and
// the next tile's plan data prefetched measured slower).  A tile is the
// reference's block step with HBM/L2 gathers: one thread per cell gathers its
// rows through the plan-ordered mapping and computes its increments in
// registers; the increments go into a zeroed shared-memory sum one thread
// colour after another (cells of one colour write disjoint points: the
// replay's order, bit for bit); then each written point's sum goes out (RED
// for private points, the slot for shared ones).  The tile header (start,
// cells | colours << 16, written points, their offset) is one 16-byte load.
template <class L, int T> constexpr int dsplit_min_blocks() {
  return (65536 / (T * L::kDirectRegCap)) > 0 ? 65536 / (T * L::kDirectRegCap) : 1;
}

template <class L, bool SOA, int T>
__global__ void __launch_bounds__(T, dsplit_min_blocks<L, T>()) k_hier_dsplit(LoopData d, HierPlanDev P) {
  using out_t = typename L::out_t;
  using read_t = typename L::read_t;
  constexpr int D = L::kDim, K = L::kOut;
  extern __shared__ __align__(16) unsigned char smem[];
  out_t *const acc = reinterpret_cast<out_t *>(smem);
  const uint32_t tid = threadIdx.x;
  griddep_launch_dependents();
  const uint32_t n_tiles = P.tiles_on ? P.n_blocks : 0u;
  if (blockIdx.x >= n_tiles) {
    // the combine CTAs come last, so that the tiles are scheduled first
    // (they gather and compute before their wait; these only wait)
    griddep_wait();
    if (P.comb_on) {
      uint32_t g0, g1;
      comb_chunk(P.n_shared, blockIdx.x - n_tiles, P.comb_ctas, g0, g1);
      combine_shared<L, SOA>(d, P, g0, g1, tid, T);
    }
    return;
  }
  const uint4 h = __ldg(P.tile_hdr + blockIdx.x);
  const uint32_t start = h.x, ncell = h.y & 0xFFFFu, ntcol = h.y >> 16, n0 = h.z, poff = h.w;
  for (uint32_t e = tid; e < n0 * K; e += T) acc[e] = out_t(0);
  // this thread's first written point (issued early; used after the sums)
  uint32_t p_first = 0, ws_first = 0;
  if (tid < n0) {
    p_first = __ldg(P.pts[0] + poff + tid);
    ws_first = __ldg(P.wslot + poff + tid);
  }
  if constexpr (L::kWritesCell) griddep_wait();  // the previous iteration may still write cell data
  const bool active = tid < ncell;
  const uint32_t pos = start + tid;
  uint32_t my_col = 0xFFFFFFFFu;
  uint16_t l0[D];
  out_t v[D][K];
  if (active) {
    GlobalRows<L, SOA> rows;
    load_row<D>(d.map[0], pos, rows.p[0]);
    if constexpr (L::kHasClass1) load_row<D>(d.map[1], pos, rows.p[1]);
#pragma unroll
    for (int q = 0; q < D; ++q) l0[q] = __ldg(P.lidx[0] + (size_t)q * d.n_cells + pos);
    my_col = __ldg(P.tcol + pos);
    static_for_read<L>([&](auto r) {
      constexpr int R = decltype(r)::value;
      rows.base[R] = static_cast<const read_t *>(d.point[L::read_set(R)]);
      rows.np[R] = d.n_points[L::read_set(R)];
    });
    Direct dir{d.cell, pos, d.n_cells};
    L::cell(rows, dir, v);
  }
  __syncthreads();  // the sums are zeroed
  for (uint32_t col = 0; col < ntcol; ++col) {
    if (my_col == col) {
#pragma unroll
      for (int q = 0; q < D; ++q)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[(uint32_t)l0[q] * K + k] += v[q][k];
    }
    __syncthreads();
  }
  if constexpr (!L::kWritesCell) griddep_wait();  // the previous iteration's writes are visible
  out_t *out = static_cast<out_t *>(d.out);
  out_t *put = static_cast<out_t *>(P.partial) + (size_t)P.put_buf * P.n_slots * K;
  for (uint32_t j = tid; j < n0; j += T) {
    const uint32_t p = j == tid ? p_first : __ldg(P.pts[0] + poff + j);
    const uint32_t ws = j == tid ? ws_first : __ldg(P.wslot + poff + j);
    const out_t *a = acc + (size_t)j * K;
    if (ws == 0xFFFFFFFFu) {
      // private point: this block alone writes it in this iteration
      if constexpr (sizeof(out_t) == 8) {
#pragma unroll
        for (int k = 0; k < K; ++k) atomicAdd(out + out_index(SOA, d.n_points[0], p, K, k), a[k]);
      } else {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          out_t *o = out + out_index(SOA, d.n_points[0], p, K, k);
          __stcg(o, __ldcg(o) + a[k]);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) __stcg(put + (size_t)ws * K + k, a[k]);
    }
  }
}

template <class L, bool SOA, int T, uint32_t kRecSlots>
__global__ void __launch_bounds__(T + 64) __maxnreg__(L::kRegCap)
    k_hier_split(LoopData d, HierPlanDev P) {
  using out_t = typename L::out_t;
  using read_t = typename L::read_t;
  constexpr int D = L::kDim, K = L::kOut;
  constexpr uint32_t kRecordWarp = T / 32, kStagingWarp = T / 32 + 1;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t s_rec_full[kRecSlots];
  __shared__ __align__(8) uint64_t s_tile_done[kRecSlots];
  __shared__ __align__(8) uint64_t s_rows_full[2];
  __shared__ __align__(8) uint64_t s_rows_empty[2];
  __shared__ uint32_t s_valid[kRecSlots];  // 0: no tile (end of this CTA's tiles)
  __shared__ volatile uint32_t s_stop;     // a role gave up (error path)
  const uint32_t tid = threadIdx.x;
  const uint32_t warp = tid >> 5, lane = tid & 31u;
  unsigned char *const rec_base = smem;
  unsigned char *const rows_base = smem + P.rows_off;
  out_t *const inc = reinterpret_cast<out_t *>(smem + P.inc_off);

  griddep_launch_dependents();
  if (tid == 0) {
    for (uint32_t s = 0; s < kRecSlots; ++s) {
      mbar_init(&s_rec_full[s], 1);
      mbar_init(&s_tile_done[s], T / 32);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&s_rows_full[b], 33);
      mbar_init(&s_rows_empty[b], 1);
    }
    mbar_fence_init();
    s_stop = 0;
  }
  __syncthreads();

  if (warp == kRecordWarp) {
    // ---------------------------------------------------------------- record
    if (lane == 0) {
      uint32_t uses[kRecSlots] = {};
      bool valid[kRecSlots] = {};
      auto refill = [&](uint32_t s, uint32_t i) {
        const uint32_t t = blockIdx.x + i * gridDim.x;
        const bool ok = t < P.n_blocks;
        s_valid[s] = ok;
        valid[s] = ok;
        if (ok) {
          const uint32_t b = P.launch[t];
          const uint32_t off = P.rec_off[b], end = P.rec_off[b + 1];
          // the slot was last read through the generic proxy
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_expect_tx(&s_rec_full[s], end - off);
          bulk_copy_g2s(rec_base + s * P.rec_slot, P.rec + off, end - off, &s_rec_full[s]);
        } else {
          mbar_arrive(&s_rec_full[s]);
        }
        ++uses[s];
      };
      for (uint32_t s = 0; s < kRecSlots; ++s) refill(s, s);
      for (uint32_t i = 0;; ++i) {
        const uint32_t s = i % kRecSlots;
        if (!valid[s]) break;
        if (!mbar_wait_or_stop(&s_tile_done[s], (i / kRecSlots) & 1u, &s_stop)) {
          atomicOr(&P.ctl->error, kErrWaitLimit);
          s_stop = 1;
          break;
        }
        refill(s, i + kRecSlots);
      }
      // let every record copy still in flight land (bounded)
      for (uint32_t s = 0; s < kRecSlots; ++s)
        if (uses[s] > 0) (void)mbar_wait(&s_rec_full[s], (uses[s] - 1) & 1u);
    }
    __syncwarp();
  } else if (warp == kStagingWarp) {
    // --------------------------------------------------------------- staging
    for (uint32_t i = 0;; ++i) {
      const uint32_t s = i % kRecSlots, b = i & 1u;
      bool ok = mbar_wait_or_stop(&s_rec_full[s], (i / kRecSlots) & 1u, &s_stop);
      // the row slot of tile i - 2 is free once that tile's compute phase ended
      if (ok && i >= 2) ok = mbar_wait_or_stop(&s_rows_empty[b], ((i - 2) >> 1) & 1u, &s_stop);
      ok = __all_sync(0xFFFFFFFFu, ok);
      if (!ok || !s_valid[s]) {
        if (lane == 0) {
          if (!ok) {
            atomicOr(&P.ctl->error, kErrWaitLimit);
            s_stop = 1;
          }
          s_valid[s] = 0;
          mbar_arrive(&s_rows_full[b]);
        }
        mbar_arrive(&s_rows_full[b]);
        break;
      }
      const RecView<L> m(rec_base + s * P.rec_slot);
      ws_stage_rows<L, SOA>(d, P, rows_base + b * P.rows_bytes, m);
      mbar_arrive_cp_async(&s_rows_full[b]);
      if (lane == 0) mbar_arrive(&s_rows_full[b]);
    }
    cp_async_wait_all();
  } else {
    // --------------------------------------------------------------- compute
    bool waited = false;    // griddepcontrol.wait done
    bool combined = false;  // this CTA's combine chunk done
    for (uint32_t i = 0;; ++i) {
      const uint32_t s = i % kRecSlots, b = i & 1u, ph = (i >> 1) & 1u;
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
      (void)mbar_try_wait(&s_rec_full[s], (i / kRecSlots) & 1u);
      const RecView<L> m(rec_base + s * P.rec_slot);
      const unsigned char *rows = rows_base + b * P.rows_bytes;
      if constexpr (L::kWritesCell) {
        // the previous iteration may still write these cells' data
        if (!waited) {
          griddep_wait();
          waited = true;
        }
      }
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
      if (!waited) {
        // the previous iteration's writes must be complete and visible
        griddep_wait();
        waited = true;
      }
      if (!combined) {
        // this CTA's share of the previous buffer's shared points
        combined = true;
        if (P.comb_on) {
          uint32_t g0, g1;
          comb_chunk(P.n_shared, blockIdx.x, gridDim.x, g0, g1);
          combine_shared<L, SOA>(d, P, g0, g1, tid, T);
        }
      }
      split_writeback<L, SOA, T>(d, P, m, inc, tid);
      __syncwarp();
      if (lane == 0) mbar_arrive(&s_tile_done[s]);
      // the increments buffer is reused by the next tile
      named_bar_sync<T>();
    }
  }
  __syncthreads();
}

} // namespace fot
