// The split write-back hierarchical-colour kernel (variant kVariantSplit).
//
// The coloured replay of a plan (blocks in block-colour order; in a block,
// cells in thread-colour order accumulate into a zeroed per-block sum; then
// out[p] += sum for each written point) fixes, for every point p, the order
// out[p] = ((out[p] + S_b1) + S_b2) + ... over the blocks b1 < b2 < ... (plan
// order) that write p.  This kernel reproduces that order without making any
// tile wait for another:
//   * a point written by ONE block (private) gets out[p] += S_b as soon as
//     the block's sum is ready -- a fire-and-forget L2 reduction (RED.F64) for
//     FP64 data, whose single rounding equals the replay's add; FP32 data
//     (atomics there flush subnormals) take a load-add-store;
//   * a point written by several blocks (shared) gets each block's S_b stored
//     into the block's partial-sum slot; the block that arrives LAST at the
//     point's counter (acquire-release atomic) adds out[p] + S_b1 + S_b2 ...
//     in plan order and resets the counter.
// Block colours therefore fix the summation order but never stall a tile.
// One launch runs ONE iteration (the partial slots and counters are reused
// by the next one); consecutive iterations are chained with programmatic
// dependent launch: every CTA allows the next grid to launch at once, and the
// next grid's tiles stage and compute (they only read datasets the loop never
// writes) before they wait (griddepcontrol.wait) for this grid to complete
// and only then write.  Loops that write cell data wait before computing.
//
// A CTA runs T compute threads and two control warps over its tiles (tile i
// of CTA c is launch[c + i * gridDim.x]: at any moment the GPU works on a
// window of consecutive tiles in formation order, so blocks sharing points
// run close together and their partial sums meet in L2):
//   * the RECORD warp bulk-copies each tile's record (plan.cu, step 4b) into
//     one of kRecSlots record slots (TMA engine, no multicast) and refills a
//     slot once the compute threads are done with its tile;
//   * the STAGING warp gathers a tile's read rows into one of two row slots
//     with cp.async as soon as the compute phase that used the slot ends;
//   * the COMPUTE threads compute each cell's per-slot increments into
//     shared memory, then, per written point, sum its contributions in
//     thread-colour order (bit-identical to the replay) and write it back.
// Every wait between the roles is bounded (about two seconds); on a timeout
// the kernel sets kErrWaitLimit in Ctl::error and returns.
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

__device__ __forceinline__ unsigned int atom_add_acq_rel_gpu(unsigned int *p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// The split part of a tile record (plan.cu, build_split), at the record's
// dependency offset (split plans have no dependency list).
struct SplitView {
  uint32_t n_sh, sh_off;
  const uint16_t *sh_of;   // per written point: index among the shared points, 0xFFFF private
  const uint16_t *sl_off;  // n_sh + 1
  const uint32_t *sl;      // slots of each shared point's blocks, plan order
  __device__ __forceinline__ SplitView(const uint32_t *at, uint32_t n0) {
    n_sh = at[0];
    sh_off = at[1];
    sh_of = reinterpret_cast<const uint16_t *>(at + 2);
    sl_off = sh_of + n0;
    const uintptr_t e = reinterpret_cast<uintptr_t>(sl_off + n_sh + 1);
    sl = reinterpret_cast<const uint32_t *>((e + 3) & ~uintptr_t(3));
  }
};

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
  out_t *__restrict__ out = static_cast<out_t *>(d.out);
  out_t *__restrict__ partial = static_cast<out_t *>(P.partial);

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
    bool waited = false;  // griddepcontrol.wait done
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
      const SplitView sv(m.dep, m.n0);
      for (uint32_t j = tid; j < m.n0; j += T) {
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
        const uint32_t sh = sv.sh_of[j];
        if (sh == 0xFFFFu) {
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
          // shared point: publish the block's sum; the last block to arrive
          // adds all sums to out[p] in plan order
          const uint32_t slot = sv.sh_off + sh;
#pragma unroll
          for (int k = 0; k < K; ++k) __stcg(partial + (size_t)slot * K + k, acc[k]);
          const uint32_t l0 = sv.sl_off[sh], l1 = sv.sl_off[sh + 1];
          unsigned int *cnt = P.counter + sv.sl[l0];
          const unsigned int prev = atom_add_acq_rel_gpu(cnt, 1u);
          if (prev + 1 == l1 - l0) {
            out_t o[K];
#pragma unroll
            for (int k = 0; k < K; ++k) o[k] = __ldcg(out + out_index(SOA, d.n_points[0], p, K, k));
            for (uint32_t e = l0; e < l1; ++e) {
              const out_t *q = partial + (size_t)sv.sl[e] * K;
#pragma unroll
              for (int k = 0; k < K; ++k) o[k] += __ldcg(q + k);
            }
#pragma unroll
            for (int k = 0; k < K; ++k) __stcg(out + out_index(SOA, d.n_points[0], p, K, k), o[k]);
            // every block of this point has arrived: ready for the next launch
            *cnt = 0u;
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&s_tile_done[s]);
      // the increments buffer is reused by the next tile
      named_bar_sync<T>();
    }
  }
  __syncthreads();
}

} // namespace fot
