// (b) The hierarchical-colour executor (see executors.cuh for the overview).
//
// A tile is one block of cells run by one CTA, in phases:
//   stage    the block's written-point list to shared memory (cp.async), the
//            accumulator zeroed; with STAGE, also the rows of every read set
//            for the block's unique points (cp.async), so the cells read
//            their indirect data from shared memory;
//   compute  each thread computes its cell's increments (reading staged rows,
//            or -- without STAGE -- gathering straight from HBM/L2 through the
//            problem's mapping, which the plan build put in plan order) and
//            adds them into the accumulator, one thread colour after another;
//   write    out[p] += acc[p] for the block's written points.
// The persistent kernel claims tiles from a queue in block-colour order; a
// tile's write phase waits until the tiles of the earlier colours have
// written back.  Thread 0 claims the next ticket and loads its metadata while
// the current tile runs.
#pragma once

#include <cstdint>
#include <type_traits>

#include "common.cuh"

namespace fot {

// Per-tile metadata, staged in shared memory by one thread.
struct TileMeta {
  uint32_t b;      // block index in the plan (0xFFFFFFFF: no more tiles)
  uint32_t iter;   // iteration of the tile
  uint32_t start;  // first position of the block
  uint32_t ncell;  // cells of the block
  uint32_t off0, n0, off1, n1; // point lists of the two mapping classes
  uint32_t ntcol;  // thread colours of the block
  uint32_t wait;   // write-back waits for done >= wait (iteration-relative)
};

__device__ __forceinline__ void red_release_add(unsigned int *p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <bool HAS1>
__device__ __forceinline__ TileMeta load_meta(const HierPlanDev &P, uint32_t b, uint32_t iter) {
  TileMeta m;
  m.b = b;
  m.iter = iter;
  m.start = P.block_start[b];
  m.ncell = P.block_start[b + 1] - m.start;
  m.off0 = P.pts_off[0][b];
  m.n0 = P.pts_off[0][b + 1] - m.off0;
  if constexpr (HAS1) {
    m.off1 = P.pts_off[1][b];
    m.n1 = P.pts_off[1][b + 1] - m.off1;
  } else {
    m.off1 = 0;
    m.n1 = 0;
  }
  m.ntcol = P.block_ntcol[b];
  m.wait = P.block_wait[b];
  return m;
}

__device__ __forceinline__ uint32_t *smem_pts(unsigned char *smem, const HierPlanDev &P) {
  return reinterpret_cast<uint32_t *>(smem + P.pts_smem_off);
}

template <class L, bool SOA, int THREADS, bool STAGE>
__device__ __forceinline__ void tile_stage(const LoopData &d, const HierPlanDev &P,
                                           unsigned char *smem, const TileMeta &m) {
  using out_t = typename L::out_t;
  using read_t = typename L::read_t;
  constexpr int K = L::kOut;
  const uint32_t tid = threadIdx.x;
  uint32_t *spts = smem_pts(smem, P);
  {
    const uint32_t *g0 = P.pts[0] + m.off0;
    for (uint32_t i = tid; i < m.n0; i += THREADS) cp_async4(spts + i, g0 + i);
    if constexpr (STAGE && L::kHasClass1) {
      const uint32_t *g1 = P.pts[1] + m.off1;
      for (uint32_t i = tid; i < m.n1; i += THREADS) cp_async4(spts + m.n0 + i, g1 + i);
    }
  }
  out_t *acc = reinterpret_cast<out_t *>(smem + P.acc_off);
  for (uint32_t e = tid; e < m.n0 * K; e += THREADS) acc[e] = out_t(0);
  if constexpr (STAGE) {
    cp_async_wait_all();
    __syncthreads();
    static_for_read<L>([&](auto r) {
      constexpr int R = decltype(r)::value;
      constexpr int DIM = L::read_dim(R);
      constexpr int ROW = DIM * (int)sizeof(read_t);
      const bool c0 = L::read_class(R) == 0;
      const uint32_t n = c0 ? m.n0 : m.n1;
      const uint32_t *pts = c0 ? spts : spts + m.n0;
      const char *src = static_cast<const char *>(d.point[L::read_set(R)]);
      char *dst = reinterpret_cast<char *>(smem + P.read_off[R]);
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
}

template <class L, bool SOA, int THREADS, bool STAGE>
__device__ __forceinline__ void tile_compute(const LoopData &d, const HierPlanDev &P,
                                             unsigned char *smem, const TileMeta &m) {
  using out_t = typename L::out_t;
  using read_t = typename L::read_t;
  constexpr int D = L::kDim, K = L::kOut;
  const uint32_t tid = threadIdx.x;
  const bool active = tid < m.ncell;
  const uint32_t pos = m.start + tid;
  out_t inc[D][K];
  uint16_t l0[D];
  uint32_t my_col = 0xFFFFFFFFu;
  if constexpr (STAGE) {
    SmemRows<L> rows;
    if (active) {
#pragma unroll
      for (int s = 0; s < D; ++s) {
        rows.l[0][s] = P.lidx[0][(size_t)s * d.n_cells + pos];
        rows.l[1][s] = L::kHasClass1 ? P.lidx[1][(size_t)s * d.n_cells + pos] : 0;
        l0[s] = rows.l[0][s];
      }
      my_col = P.tcol[pos];
    }
    static_for_read<L>([&](auto r) {
      constexpr int R = decltype(r)::value;
      rows.base[R] = reinterpret_cast<const read_t *>(smem + P.read_off[R]);
    });
    cp_async_wait_all();
    __syncthreads();
    if (active) {
      Direct dir{d.cell, pos, d.n_cells};
      L::cell(rows, dir, inc);
    }
  } else {
    GlobalRows<L, SOA> rows;
    if (active) {
      load_row<D>(d.map[0], pos, rows.p[0]);
      if constexpr (L::kHasClass1) load_row<D>(d.map[1], pos, rows.p[1]);
#pragma unroll
      for (int s = 0; s < D; ++s) l0[s] = P.lidx[0][(size_t)s * d.n_cells + pos];
      my_col = P.tcol[pos];
      static_for_read<L>([&](auto r) {
        constexpr int R = decltype(r)::value;
        rows.base[R] = static_cast<const read_t *>(d.point[L::read_set(R)]);
        rows.np[R] = d.n_points[L::read_set(R)];
      });
      Direct dir{d.cell, pos, d.n_cells};
      L::cell(rows, dir, inc);
    }
    cp_async_wait_all();  // the point list
    __syncthreads();
  }
  out_t *acc = reinterpret_cast<out_t *>(smem + P.acc_off);
  for (uint32_t col = 0; col < m.ntcol; ++col) {
    if (my_col == col) {
#pragma unroll
      for (int s = 0; s < D; ++s)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[(uint32_t)l0[s] * K + k] += inc[s][k];
    }
    __syncthreads();
  }
}

// out[p] += acc for the tile's written points (L2 loads/stores: L1 may hold
// stale lines of rows another SM wrote).  Loads of a batch are issued before
// any of its stores so their latencies overlap.
template <class L, bool SOA, int THREADS>
__device__ __forceinline__ void tile_writeback(const LoopData &d, const HierPlanDev &P,
                                               unsigned char *smem, const TileMeta &m) {
  using out_t = typename L::out_t;
  constexpr int K = L::kOut;
  constexpr int BATCH = 2;
  const uint32_t tid = threadIdx.x;
  const uint32_t *spts = smem_pts(smem, P);
  const out_t *acc = reinterpret_cast<const out_t *>(smem + P.acc_off);
  out_t *__restrict__ out = static_cast<out_t *>(d.out);
  if constexpr (!SOA && (K * sizeof(out_t)) % 16 == 0) {
    constexpr int CH = K * sizeof(out_t) / 16;
    using vec_t = typename std::conditional<sizeof(out_t) == 8, double2, float4>::type;
    vec_t *o = reinterpret_cast<vec_t *>(out);
    const vec_t *a = reinterpret_cast<const vec_t *>(acc);
    const uint32_t total = m.n0 * CH;
    for (uint32_t base = 0; base < total; base += BATCH * THREADS) {
      vec_t v[BATCH];
      size_t gi[BATCH];
#pragma unroll
      for (int j = 0; j < BATCH; ++j) {
        const uint32_t e = base + j * THREADS + tid;
        if (e < total) {
          const uint32_t i = e / CH, c = e - i * CH;
          gi[j] = (size_t)spts[i] * CH + c;
          v[j] = __ldcg(o + gi[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < BATCH; ++j) {
        const uint32_t e = base + j * THREADS + tid;
        if (e < total) {
          const vec_t w = a[e];
          if constexpr (sizeof(out_t) == 8) {
            v[j].x += w.x;
            v[j].y += w.y;
          } else {
            v[j].x += w.x;
            v[j].y += w.y;
            v[j].z += w.z;
            v[j].w += w.w;
          }
          __stcg(o + gi[j], v[j]);
        }
      }
    }
  } else {
    const uint32_t total = m.n0 * K;
    for (uint32_t base = 0; base < total; base += BATCH * THREADS) {
      out_t v[BATCH];
      size_t gi[BATCH];
#pragma unroll
      for (int j = 0; j < BATCH; ++j) {
        const uint32_t e = base + j * THREADS + tid;
        if (e < total) {
          const uint32_t i = e / K, k = e - i * K;
          gi[j] = out_index(SOA, d.n_points[0], spts[i], K, k);
          v[j] = __ldcg(out + gi[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < BATCH; ++j) {
        const uint32_t e = base + j * THREADS + tid;
        if (e < total) __stcg(out + gi[j], v[j] + acc[e]);
      }
    }
  }
}

// Thread 0 waits (bounded) until *done >= target; `seen` caches the last value
// read.  Returns 1 if the wait gave up (and flags *err).
__device__ __forceinline__ int wait_done(unsigned int *done, unsigned int target,
                                         unsigned int *err, unsigned int &seen) {
  if (seen >= target) return 0;
  unsigned int polls = 0;
  for (;;) {
    seen = ld_acquire_gpu(done);
    if (seen >= target) return 0;
    if (++polls > kWaitPollLimit) {
      atomicOr(err, kErrWaitLimit);
      return 1;
    }
    __nanosleep(128);
  }
}

template <class L, int THREADS>
constexpr int hier_min_blocks() {
  return (65536 / (THREADS * L::kRegCap)) > 0 ? 65536 / (THREADS * L::kRegCap) : 1;
}

// Persistent form: CTAs claim tiles in colour order until the queue is empty.
template <class L, bool SOA, int THREADS, bool STAGE>
__global__ void __launch_bounds__(THREADS, hier_min_blocks<L, THREADS>())
    k_hier(LoopData d, HierPlanDev P) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ TileMeta s_meta;
  __shared__ int s_abort;
  const uint32_t tid = threadIdx.x;
  constexpr uint32_t NONE = 0xFFFFFFFFu;
  unsigned int seen = 0;  // thread 0: last value of done read
  uint32_t t_next = 0;    // thread 0: prefetched ticket
  if (tid == 0) {
    uint32_t t = atomicAdd(&P.ctl->ticket, 1u);
    if (t < P.total_tiles) {
      const uint32_t it = t / P.n_blocks;
      s_meta = load_meta<L::kHasClass1>(P, t - it * P.n_blocks, it);
    } else {
      s_meta.b = NONE;
    }
    t_next = atomicAdd(&P.ctl->ticket, 1u);
  }
  __syncthreads();
  for (;;) {
    const TileMeta m = s_meta;
    if (m.b == NONE) break;
    tile_stage<L, SOA, THREADS, STAGE>(d, P, smem, m);
    tile_compute<L, SOA, THREADS, STAGE>(d, P, smem, m);
    // prefetch the next tile's metadata (consumed after the write-back)
    TileMeta nm;
    nm.b = NONE;
    if (tid == 0 && t_next < P.total_tiles && !(*(volatile unsigned int *)&P.ctl->error)) {
      const uint32_t it = t_next / P.n_blocks;
      nm = load_meta<L::kHasClass1>(P, t_next - it * P.n_blocks, it);
    }
    if (tid == 0) s_abort = wait_done(&P.ctl->done, m.iter * P.n_blocks + m.wait, &P.ctl->error, seen);
    __syncthreads();
    if (!s_abort) tile_writeback<L, SOA, THREADS>(d, P, smem, m);
    __syncthreads();
    if (tid == 0) {
      red_release_add(&P.ctl->done, 1u);
      s_meta = nm;
      if (nm.b != NONE) t_next = atomicAdd(&P.ctl->ticket, 1u);
    }
    __syncthreads();
  }
  // the last CTA to leave resets the queue for the next launch
  if (tid == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(&P.ctl->exited, 1u);
    if (prev == gridDim.x - 1) {
      atomicExch(&P.ctl->ticket, 0u);
      atomicExch(&P.ctl->done, 0u);
      atomicExch(&P.ctl->exited, 0u);
      __threadfence();
    }
  }
}

// One launch per block colour: CTA x handles block first + x, no waiting.
template <class L, bool SOA, int THREADS, bool STAGE>
__global__ void __launch_bounds__(THREADS, hier_min_blocks<L, THREADS>())
    k_hier_colour(LoopData d, HierPlanDev P, uint32_t first) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ TileMeta s_meta;
  if (threadIdx.x == 0) s_meta = load_meta<L::kHasClass1>(P, first + blockIdx.x, 0);
  __syncthreads();
  const TileMeta m = s_meta;
  tile_stage<L, SOA, THREADS, STAGE>(d, P, smem, m);
  tile_compute<L, SOA, THREADS, STAGE>(d, P, smem, m);
  tile_writeback<L, SOA, THREADS>(d, P, smem, m);
}

// One tile with its dependency wait, for the batched executor.
template <class L, bool SOA, int THREADS>
__device__ __forceinline__ void hier_tile_waiting(const LoopData &d, const HierPlanDev &P,
                                                  unsigned char *smem, uint32_t b, uint32_t iter,
                                                  unsigned int *done, unsigned int *err,
                                                  unsigned int &seen) {
  __shared__ TileMeta s_m;
  __shared__ int s_ab;
  if (threadIdx.x == 0) s_m = load_meta<L::kHasClass1>(P, b, iter);
  __syncthreads();
  const TileMeta m = s_m;
  tile_stage<L, SOA, THREADS, true>(d, P, smem, m);
  tile_compute<L, SOA, THREADS, true>(d, P, smem, m);
  if (threadIdx.x == 0) s_ab = wait_done(done, iter * P.n_blocks + m.wait, err, seen);
  __syncthreads();
  if (!s_ab) tile_writeback<L, SOA, THREADS>(d, P, smem, m);
  __syncthreads();
}

} // namespace fot
