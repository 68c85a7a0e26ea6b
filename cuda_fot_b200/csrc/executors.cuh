// The two executors, templated on a loop adapter (loops.cuh).
//
// (a) Global atomics (FOT_EXEC_ATOMIC) -- replaces the reference's
//     global-colouring executor (problem.hpp:90-194, one launch and one
//     cudaDeviceSynchronize per colour).  One launch per iteration, one thread
//     per cell, mapping rows read as vectors, read sets gathered straight from
//     HBM/L2, increments added with native atomics (f64 RED; one 16-byte f32x4
//     RED per row for the FP32 loop).  With warp aggregation, lanes whose
//     slot targets the same point are grouped with __match_any_sync and summed
//     in registers by a segmented shuffle tree before one lane issues the
//     atomics.
//
// (b) Hierarchical colouring (FOT_EXEC_HIER / _HIER_LAUNCH) -- replaces
//     loopGPUHierarchical (problem.hpp:198-339) and its kernels
//     (e.g. res_calc.hpp:218-383).  A block of cells is one CTA tile.  The
//     CTA stages the read rows of the block's unique points into shared memory
//     with cp.async, computes every cell's increments, adds them into a
//     zeroed shared accumulator in thread-colour order (one __syncthreads per
//     thread colour) and finally adds the accumulator to point dataset 0 in
//     HBM.  Blocks of one block colour write disjoint points.  In the
//     persistent forms (FOT_EXEC_HIER) CTAs claim tiles from a queue stored
//     in block-colour order (and iteration after iteration); a tile computes
//     immediately -- the loops never read the dataset they increment -- and
//     only its write-back waits, with a bounded spin, until what it conflicts
//     with has been written back: every tile of the earlier colours for the
//     simple kernel (k_hier, hier.cuh), the conflicting blocks' completion
//     flags for the pipelined warp-specialised kernel (k_hier_pipe,
//     hier_pipe.cuh).  The split write-back kernel (k_hier_split,
//     hier_split.cuh, the default) makes no tile wait: points written by one
//     block are added at once, points shared by several blocks through
//     per-block partial sums that the next launch (or a final combine-only
//     launch) adds in colour order.  The result is therefore deterministic
//     and equal to replaying the colours in order on the CPU.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace fot {

// Device view of a problem's data for one run (current cell order).
struct LoopData {
  const uint32_t *map[2]; // class 0 = mapping 0; class 1 = a second distinct mapping
  const void *point[4];   // point datasets by set index
  void *out;              // point dataset 0
  void *cell[8];          // cell datasets (SOA, stride n_cells)
  uint32_t n_points[4];
  uint32_t n_cells;
  uint32_t n_cell_sets;
  uint32_t cell_dim[8];   // components of each cell dataset
  uint32_t cell_size[8];  // bytes of one component
};

// Device view of a hierarchical plan.
struct HierPlanDev {
  const uint32_t *block_start; // n_blocks+1 positions
  const uint32_t *block_wait;  // tiles of earlier colours (per block)
  const uint8_t *block_ntcol;  // thread colours per block
  const uint8_t *tcol;         // thread colour per position
  const uint32_t *pts_off[2];  // per class: n_blocks+1 offsets
  const uint32_t *pts[2];      // per class: unique points of each block
  const uint16_t *lidx[2];     // per class: kDim x n_cells local indices (SOA)
  uint32_t n_blocks;
  uint32_t total_tiles;        // iterations * n_blocks (persistent form)
  uint32_t read_off[4];        // shared-memory byte offset of each read set
  uint32_t acc_off;            // shared-memory byte offset of the accumulator
  uint32_t pts_smem_off;       // shared-memory byte offset of the tile's point lists
  Ctl *ctl;
  // pipelined kernel
  const unsigned char *rec;    // tile records
  const uint32_t *rec_off;     // n_blocks+1 byte offsets of the records
  uint32_t rec_slot;           // bytes of one tile-record slot (slots start at offset 0)
  uint32_t rows_off;           // first read-row slot (read_off[] are relative to a slot)
  uint32_t rows_bytes;         // bytes of one read-row slot
  uint32_t inc_off;            // per-slot increments
  uint32_t outbuf_off;         // first prefetched-output-row slot
  uint32_t outbuf_bytes;       // bytes of one output-row slot
  unsigned int *block_done;    // per block: completed iterations (relative to ctl->base)
  // split write-back kernels
  const uint32_t *launch;      // tile -> block (formation order)
  void *partial;               // 2 x n_slots partial-sum rows (AOS, point dataset 0's type)
  const uint32_t *comb_point;  // shared point g -> point number
  const uint32_t *comb_base;   // shared point g -> its slots [base[g], base[g+1])
  uint32_t n_slots, n_shared;
  const uint4 *tile_hdr;       // per tile (launch order): start, cells | colours << 16,
                               // written points, their offset in pts[0]
  const uint32_t *wslot;       // per pts[0] entry: its slot, 0xFFFFFFFF private
  // per launch: tiles run (0: combine only), the buffer they fill, whether
  // the other buffer (previous iteration) is combined, CTAs doing that
  uint32_t tiles_on, put_buf, comb_on, comb_ctas;
};

// Direct (cell) data of one cell: SOA with stride n_cells.
struct Direct {
  void *const *base;
  uint32_t idx;
  unsigned stride;
  template <class T> __device__ __forceinline__ const T *ptr(int j) const {
    return static_cast<const T *>(base[j]) + idx;
  }
  template <class T> __device__ __forceinline__ T *wptr(int j) const {
    return static_cast<T *>(base[j]) + idx;
  }
};

// Read rows straight from global memory (problem layout AOS or SOA).
template <class L, bool SOA> struct GlobalRows {
  using T = typename L::read_t;
  const T *base[L::kNumRead > 0 ? L::kNumRead : 1];
  unsigned np[L::kNumRead > 0 ? L::kNumRead : 1];
  uint32_t p[2][L::kDim];
  template <int R> __device__ __forceinline__ const T *ptr(int s) const {
    const uint32_t q = p[L::read_class(R)][s];
    const T *r = base[R] + (SOA ? (size_t)q : (size_t)q * L::read_dim(R));
    // AOS rows of a multiple of 16 bytes start 16-byte aligned: the compiler
    // may then merge neighbouring element loads into vector loads
    if constexpr (!SOA && (L::read_dim(R) * sizeof(T)) % 16 == 0)
      return static_cast<const T *>(__builtin_assume_aligned(r, 16));
    return r;
  }
  template <int R> __device__ __forceinline__ unsigned stride() const {
    return SOA ? np[R] : 1u;
  }
};

// Read rows staged in shared memory (AOS rows, stride 1).
template <class L> struct SmemRows {
  using T = typename L::read_t;
  const T *base[L::kNumRead > 0 ? L::kNumRead : 1];
  uint16_t l[2][L::kDim];
  template <int R> __device__ __forceinline__ const T *ptr(int s) const {
    const T *r = base[R] + (uint32_t)l[L::read_class(R)][s] * L::read_dim(R);
    if constexpr ((L::read_dim(R) * sizeof(T)) % 16 == 0)
      return static_cast<const T *>(__builtin_assume_aligned(r, 16));
    return r;
  }
  template <int R> __device__ __forceinline__ unsigned stride() const { return 1u; }
};

template <class L, int I = 0, class F>
__device__ __forceinline__ void static_for_read(F &&f) {
  if constexpr (I < L::kNumRead) {
    f(std::integral_constant<int, I>{});
    static_for_read<L, I + 1>(f);
  }
}

__device__ __forceinline__ size_t out_index(bool soa, uint32_t np0, uint32_t p,
                                            int dim, int k) {
  return soa ? (size_t)k * np0 + p : (size_t)p * dim + k;
}

// Load mapping row `c` of a class into q[kDim] with vector loads.
template <int D>
__device__ __forceinline__ void load_row(const uint32_t *__restrict__ map, uint32_t c,
                                         uint32_t (&q)[D]) {
  if constexpr (D == 2) {
    const uint2 v = __ldg(reinterpret_cast<const uint2 *>(map) + c);
    q[0] = v.x;
    q[1] = v.y;
  } else if constexpr (D == 4) {
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(map) + c);
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
  } else if constexpr (D == 8) {
    const uint4 a = __ldg(reinterpret_cast<const uint4 *>(map) + 2 * (size_t)c);
    const uint4 b = __ldg(reinterpret_cast<const uint4 *>(map) + 2 * (size_t)c + 1);
    q[0] = a.x; q[1] = a.y; q[2] = a.z; q[3] = a.w;
    q[4] = b.x; q[5] = b.y; q[6] = b.z; q[7] = b.w;
  } else {
#pragma unroll
    for (int s = 0; s < D; ++s) q[s] = __ldg(map + (size_t)c * D + s);
  }
}

// ===========================================================================
// (a) atomic executor
// ===========================================================================

template <class T> __device__ __forceinline__ void atomic_add(T *a, T v) { atomicAdd(a, v); }

// Cells [base, base + 32) of one mesh, one per lane of the calling warp
// (cells past n_cells are masked): compute, optionally aggregate by target
// point, add with atomics.
template <class L, bool SOA, bool AGG>
__device__ __forceinline__ void atomic_warp(const LoopData &d, uint32_t base) {
  using out_t = typename L::out_t;
  constexpr int D = L::kDim, K = L::kOut;
  const uint32_t lane = threadIdx.x & 31u;
  out_t *__restrict__ out = static_cast<out_t *>(d.out);
  const uint32_t c = base + lane;
  const bool valid = c < d.n_cells;
  GlobalRows<L, SOA> rows;
  out_t inc[D][K];
#pragma unroll
  for (int s = 0; s < D; ++s) {
    rows.p[0][s] = 0;
    rows.p[1][s] = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) inc[s][k] = out_t(0);
  }
  if (valid) {
    load_row<D>(d.map[0], c, rows.p[0]);
    if constexpr (L::kHasClass1) load_row<D>(d.map[1], c, rows.p[1]);
    static_for_read<L>([&](auto r) {
      constexpr int R = decltype(r)::value;
      rows.base[R] = static_cast<const typename L::read_t *>(d.point[L::read_set(R)]);
      rows.np[R] = d.n_points[L::read_set(R)];
    });
    Direct dir{d.cell, c, d.n_cells};
    L::cell(rows, dir, inc);
  }
#pragma unroll
  for (int s = 0; s < D; ++s) {
    const uint32_t key = valid ? rows.p[0][s] : 0xFFFFFFFFu;
    bool leader = valid;
    if constexpr (AGG) {
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
      const unsigned lt = (1u << lane) - 1u;
      const int rank = __popc(peers & lt);
      const int cnt = __popc(peers);
      const int maxcnt = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)cnt);
      for (int off = 1; off < maxcnt; off <<= 1) {
        const bool has = rank + off < cnt;
        const int src = has ? (int)__fns(peers, 0, rank + off + 1) : (int)lane;
        const bool take = has && (rank % (2 * off)) == 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const out_t v = __shfl_sync(0xFFFFFFFFu, inc[s][k], src);
          if (take) inc[s][k] += v;
        }
      }
      leader = valid && rank == 0;
    }
    if (leader) {
      if constexpr (!SOA && sizeof(out_t) == 4 && K == 4) {
        float4 v = make_float4(inc[s][0], inc[s][1], inc[s][2], inc[s][3]);
        atomicAdd(reinterpret_cast<float4 *>(out) + key, v);
      } else {
#pragma unroll
        for (int k = 0; k < K; ++k)
          atomic_add(out + out_index(SOA, d.n_points[0], key, K, k), inc[s][k]);
      }
    }
  }
}

__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Prefetch cell c's mapping rows and direct data (every component of every
// cell dataset, SOA) into L2; one instruction per array covers a warp's 32
// consecutive cells.  Straight-line code: the loops over the loop's cell
// datasets and their (at most kMaxPrefetchDim) components are unrolled.
constexpr uint32_t kMaxPrefetchDim = 12;
template <class L> __device__ __forceinline__ void prefetch_cell(const LoopData &d, uint32_t c) {
  prefetch_l2(d.map[0] + (size_t)c * L::kDim);
  if constexpr (L::kHasClass1) prefetch_l2(d.map[1] + (size_t)c * L::kDim);
#pragma unroll
  for (int j = 0; j < L::kNumDirect; ++j) {
    const char *b = static_cast<const char *>(d.cell[j]) + (size_t)c * d.cell_size[j];
    const size_t stride = (size_t)d.n_cells * d.cell_size[j];
#pragma unroll
    for (uint32_t k = 0; k < kMaxPrefetchDim; ++k)
      if (k < d.cell_dim[j]) prefetch_l2(b + k * stride);
  }
}

// Persistent grid-stride loop over 32-cell chunks, one chunk per warp at a
// time; with L::kAtomicPrefetch, in the SOA form, each warp first prefetches
// the chunk it will take next, so that its mapping rows and direct data come
// from L2 then.
template <class L, bool SOA, bool AGG>
__global__ void __launch_bounds__(256, L::kAtomicMinBlocks) k_atomic(LoopData d) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = warp * 32u; base < d.n_cells; base += n_warps * 32u) {
    if constexpr (L::kAtomicPrefetch && SOA) {
      const uint32_t next = base + n_warps * 32u + lane;
      if (next < d.n_cells) prefetch_cell<L>(d, next);
    }
    atomic_warp<L, SOA, AGG>(d, base);
  }
}

} // namespace fot

#include "hier.cuh"
#include "hier_pipe.cuh"
#include "hier_split.cuh"
