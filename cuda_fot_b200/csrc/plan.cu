// GPU plan builder of the hierarchical-colour executor.
//
// Replaces the reference's host builder HierarchicalColourMemory
// (colouring.hpp:44-147, colourBlock :169-235, sortCellsByColours :246-272)
// and its per-block thread colouring (colouring.cu:12-102).  Steps:
//   1. blocks: contiguous runs of block_size cells, or runs of one part of the
//      problem's partition split at block_size (colouring.hpp:70-115);
//   2. one CTA per block: unique written points (ascending) and each slot's
//      local index, the same for the second mapping class; greedy first-fit
//      thread colouring over the written points; cells sorted by thread colour
//      (k_block_local);
//   3. the block conflict graph (blocks sharing a written point) and its
//      colouring by Jones-Plassmann rounds with first-fit colours (the
//      reference colours blocks greedily in block order, :117-144);
//   4. blocks ordered by colour; all per-block data gathered into that order
//      (k_gather_plan);
//   5. the problem's cells are permuted into plan order so that direct data
//      are read coalesced (the reference copies them per colour instead,
//      copyCellWeights :310-335).
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>

#include "devutil.cuh"
#include "engine.hpp"

namespace fot {
namespace {

constexpr int kPlanThreads = 256;
constexpr int kMaxThreadColours = 64;
constexpr int kMaxBlockColours = 256;

// ---------------------------------------------------------------------------
// step 2: per-block unique points, local indices, thread colours
// ---------------------------------------------------------------------------
struct LocalOut {
  const uint32_t *map[2];
  int n_class;
  int D;
  const uint32_t *fstart;     // nfb+1
  const uint32_t *form_cells; // formation position -> cell, or null (identity)
  uint32_t cap;               // padded points per block (block_size * D)
  uint32_t *pad_pts[2];
  uint32_t *cnt[2];
  uint32_t *out_cell;         // formation position -> cell, sorted by thread colour
  uint16_t *out_lidx[2];      // D x n_cells by formation position
  uint8_t *out_tcol;
  uint8_t *ntcol;
  uint32_t n_cells;
  int *err;
};

template <int ITEMS>
__global__ void __launch_bounds__(kPlanThreads) k_block_local(LocalOut o) {
  using Sort = cub::BlockRadixSort<uint32_t, kPlanThreads, ITEMS, uint16_t>;
  using Scan = cub::BlockScan<uint32_t, kPlanThreads>;
  __shared__ union {
    typename Sort::TempStorage sort;
    typename Scan::TempStorage scan;
  } tmp;
  __shared__ uint32_t s_last[kPlanThreads];
  __shared__ uint32_t s_count;
  __shared__ uint8_t s_col[1024];
  __shared__ uint16_t s_order[1024];
  __shared__ uint32_t s_ncol;
  extern __shared__ __align__(16) unsigned char dyn[];
  uint16_t *lidx[2] = {reinterpret_cast<uint16_t *>(dyn),
                       reinterpret_cast<uint16_t *>(dyn) + o.cap};
  uint64_t *masks = reinterpret_cast<uint64_t *>(dyn + ((4 * o.cap * sizeof(uint16_t) + 15) & ~15u));

  const uint32_t b = blockIdx.x, t = threadIdx.x;
  const uint32_t s0 = o.fstart[b];
  const uint32_t n = o.fstart[b + 1] - s0;
  const int D = o.D;
  const uint32_t E = n * D;

  for (int c = 0; c < o.n_class; ++c) {
    uint32_t keys[ITEMS];
    uint16_t vals[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const uint32_t e = t * ITEMS + j;
      if (e < E) {
        const uint32_t i = e / D, s = e - i * D;
        const uint32_t cell = o.form_cells ? o.form_cells[s0 + i] : s0 + i;
        keys[j] = o.map[c][(size_t)cell * D + s];
      } else {
        keys[j] = 0xFFFFFFFFu;
      }
      vals[j] = (uint16_t)e;
    }
    Sort(tmp.sort).Sort(keys, vals);
    __syncthreads();
    s_last[t] = keys[ITEMS - 1];
    __syncthreads();
    uint32_t flags[ITEMS];
    uint32_t prev = t > 0 ? s_last[t - 1] : 0xFFFFFFFFu;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const bool valid = t * ITEMS + j < E;
      flags[j] = (valid && (j == 0 ? (t == 0 || keys[j] != prev) : keys[j] != keys[j - 1])) ? 1u : 0u;
    }
    uint32_t excl[ITEMS];
    uint32_t total;
    Scan(tmp.scan).ExclusiveSum(flags, excl, total);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      if (t * ITEMS + j < E) {
        const uint32_t u = excl[j] + flags[j] - 1u;
        lidx[c][vals[j]] = (uint16_t)u;
        if (flags[j]) o.pad_pts[c][(size_t)b * o.cap + u] = keys[j];
      }
    }
    if (t == 0) {
      o.cnt[c][b] = total;
      if (c == 0) s_count = total;
    }
    __syncthreads();
  }

  // greedy first-fit thread colouring over the written points, cells in
  // block order (one thread: a block holds at most 1024 cells)
  for (uint32_t i = t; i < s_count; i += kPlanThreads) masks[i] = 0;
  __syncthreads();
  if (t == 0) {
    uint32_t ncol = 0;
    for (uint32_t i = 0; i < n; ++i) {
      uint64_t m = 0;
      for (int s = 0; s < D; ++s) m |= masks[lidx[0][i * D + s]];
      if (m == ~0ull) {
        atomicOr(o.err, 1);
        break;
      }
      const uint32_t col = __ffsll(~m) - 1;
      s_col[i] = (uint8_t)col;
      for (int s = 0; s < D; ++s) masks[lidx[0][i * D + s]] |= 1ull << col;
      ncol = max(ncol, col + 1);
    }
    // stable counting sort of the cells by colour
    uint32_t start[kMaxThreadColours + 1];
    for (uint32_t c = 0; c <= ncol; ++c) start[c] = 0;
    for (uint32_t i = 0; i < n; ++i) start[s_col[i] + 1]++;
    for (uint32_t c = 0; c < ncol; ++c) start[c + 1] += start[c];
    for (uint32_t i = 0; i < n; ++i) s_order[start[s_col[i]]++] = (uint16_t)i;
    s_ncol = ncol;
    o.ntcol[b] = (uint8_t)ncol;
  }
  __syncthreads();
  for (uint32_t pos = t; pos < n; pos += kPlanThreads) {
    const uint32_t i = s_order[pos];
    const uint32_t cell = o.form_cells ? o.form_cells[s0 + i] : s0 + i;
    o.out_cell[s0 + pos] = cell;
    o.out_tcol[s0 + pos] = s_col[i];
    for (int c = 0; c < o.n_class; ++c)
      for (int s = 0; s < D; ++s)
        o.out_lidx[c][(size_t)s * o.n_cells + s0 + pos] = lidx[c][i * D + s];
  }
}

// ---------------------------------------------------------------------------
// step 3: block conflict graph and Jones-Plassmann colouring
// ---------------------------------------------------------------------------
__global__ void k_compact_pairs(const uint32_t *pad, const uint32_t *cnt, const uint32_t *off,
                                uint32_t cap, uint32_t nfb, uint32_t *keys, uint32_t *vals) {
  const uint32_t b = blockIdx.x;
  if (b >= nfb) return;
  for (uint32_t i = threadIdx.x; i < cnt[b]; i += blockDim.x) {
    keys[off[b] + i] = pad[(size_t)b * cap + i];
    vals[off[b] + i] = b;
  }
}

__global__ void k_count_edges(const uint32_t *keys, uint32_t n, uint32_t *count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = 0;
  if (i == 0 || keys[i] != keys[i - 1]) {
    uint32_t m = 1;
    while (i + m < n && keys[i + m] == keys[i]) ++m;
    c = m * (m - 1);
  }
  count[i] = c;
}

__global__ void k_emit_edges(const uint32_t *keys, const uint32_t *vals, uint32_t n,
                             const uint32_t *off, uint64_t *edges) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(i == 0 || keys[i] != keys[i - 1])) return;
  uint32_t m = 1;
  while (i + m < n && keys[i + m] == keys[i]) ++m;
  uint32_t w = off[i];
  for (uint32_t a = 0; a < m; ++a)
    for (uint32_t c = 0; c < m; ++c)
      if (a != c) edges[w++] = ((uint64_t)vals[i + a] << 32) | vals[i + c];
}

__global__ void k_degree(const uint64_t *edges, uint32_t ne, uint32_t *deg) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < ne) atomicAdd(&deg[edges[e] >> 32], 1u);
}

__global__ void k_jp_round(const uint32_t *row, const uint64_t *edges, uint32_t nv,
                           int *colour, uint32_t *n_done, int *err) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv || colour[v] >= 0) return;
  const uint32_t wv = hash32(v);
  uint64_t used[kMaxBlockColours / 64] = {0, 0, 0, 0};
  for (uint32_t e = row[v]; e < row[v + 1]; ++e) {
    const uint32_t u = (uint32_t)edges[e];
    const int cu = colour[u];
    if (cu < 0) {
      const uint32_t wu = hash32(u);
      if (wu > wv || (wu == wv && u > v)) return;
    } else {
      used[cu >> 6] |= 1ull << (cu & 63);
    }
  }
  for (int w = 0; w < kMaxBlockColours / 64; ++w) {
    if (~used[w]) {
      colour[v] = w * 64 + __ffsll(~used[w]) - 1;
      atomicAdd(n_done, 1u);
      return;
    }
  }
  atomicOr(err, 2);
  colour[v] = kMaxBlockColours - 1;
  atomicAdd(n_done, 1u);
}

// ---------------------------------------------------------------------------
// step 4: gather per-block data into colour order
// ---------------------------------------------------------------------------
struct GatherArgs {
  const uint32_t *order;       // final block -> formation block
  const uint32_t *fstart;      // formation offsets
  const uint32_t *block_start; // final offsets
  const uint32_t *f_cell;
  const uint8_t *f_tcol;
  const uint16_t *f_lidx[2];
  const uint32_t *pad_pts[2];
  const uint32_t *cnt[2];
  const uint32_t *pts_off[2];
  const uint8_t *f_ntcol;
  const int *colour;
  const uint32_t *colour_first; // block index where each colour starts
  uint32_t *cell;               // final position -> cell (pre-build order)
  uint8_t *tcol;
  uint16_t *lidx[2];
  uint32_t *pts[2];
  uint8_t *ntcol;
  uint32_t *block_wait;
  uint32_t cap, n_cells;
  int n_class, D;
};

__global__ void k_gather_plan(GatherArgs g) {
  const uint32_t b = blockIdx.x;
  const uint32_t fb = g.order[b];
  const uint32_t fs = g.fstart[fb], n = g.fstart[fb + 1] - fs;
  const uint32_t ds = g.block_start[b];
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    g.cell[ds + i] = g.f_cell[fs + i];
    g.tcol[ds + i] = g.f_tcol[fs + i];
    for (int c = 0; c < g.n_class; ++c)
      for (int s = 0; s < g.D; ++s)
        g.lidx[c][(size_t)s * g.n_cells + ds + i] = g.f_lidx[c][(size_t)s * g.n_cells + fs + i];
  }
  for (int c = 0; c < g.n_class; ++c) {
    const uint32_t m = g.cnt[c][fb];
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x)
      g.pts[c][g.pts_off[c][b] + i] = g.pad_pts[c][(size_t)fb * g.cap + i];
  }
  if (threadIdx.x == 0) {
    g.ntcol[b] = g.f_ntcol[fb];
    g.block_wait[b] = g.colour_first[g.colour[fb]];
  }
}

// ---------------------------------------------------------------------------
// step 4b: tile records -- everything a tile needs besides the read rows, in
// one 16-byte aligned segment per block so one bulk copy brings it in:
//   u32 header[8] = {start, ncell, n0, n1, ntcol, wait, ndep, block}
//   u32 pts0[n0], u32 pts1[n1], u16 lidx0[D][ncell], u16 lidx1[D][ncell],
//   u16 pc_off[n0 + 1], u16 pc_idx[D * ncell], (pad to 4 bytes),
//   u32 dep[ndep], zero padding to 16 bytes
// pc_off / pc_idx list, for each written point j of the block, its
// contributions e = s * T + i (slot s of the block's i-th cell; T = threads
// per CTA) in increasing (i, s) order -- cells are sorted by thread colour, so
// this is the thread-colour order of the reference's shared-memory
// accumulation (res_calc.hpp:328-339).
// dep lists the blocks sharing a written point with this one (the conflict
// graph); bit 31 marks those of an earlier block colour.
// Plans of the split write-back kernels (hier_split.cuh) have no dep list;
// in its place, at the same offset, comes u32 wslot[n0] (build_split below),
// then zero padding to 16 bytes.
// ---------------------------------------------------------------------------
struct RecordArgs {
  const uint32_t *block_start, *block_wait, *pts_off[2], *pts[2], *rec_off;
  const uint16_t *lidx[2];
  const uint8_t *ntcol;
  const uint32_t *dep_off, *dep;
  const uint32_t *wslot;           // split plans: per written point (pts_off order), or null
  unsigned char *rec;
  uint32_t n_cells, threads;
  int n_class, D;
};

__host__ __device__ inline uint32_t record_dep_offset(uint32_t ncell, uint32_t n0, uint32_t n1,
                                                      int D, int n_class) {
  const uint32_t b = 32 + 4 * (n0 + n1) + 2 * D * ncell * n_class + 2 * (n0 + 1) + 2 * D * ncell;
  return (b + 3) & ~3u;
}

__host__ __device__ inline uint32_t record_bytes(uint32_t ncell, uint32_t n0, uint32_t n1, int D,
                                                 int n_class, uint32_t ndep) {
  return (record_dep_offset(ncell, n0, n1, D, n_class) + 4 * ndep + 15) & ~15u;
}

__global__ void k_build_records(RecordArgs a) {
  const uint32_t b = blockIdx.x;
  const uint32_t start = a.block_start[b], ncell = a.block_start[b + 1] - start;
  uint32_t n[2] = {a.pts_off[0][b + 1] - a.pts_off[0][b], 0};
  if (a.n_class > 1) n[1] = a.pts_off[1][b + 1] - a.pts_off[1][b];
  unsigned char *r = a.rec + a.rec_off[b];
  uint32_t *h = reinterpret_cast<uint32_t *>(r);
  if (threadIdx.x == 0) {
    h[0] = start;
    h[1] = ncell;
    h[2] = n[0];
    h[3] = n[1];
    h[4] = a.ntcol[b];
    h[5] = a.block_wait[b];
    h[6] = a.dep_off[b + 1] - a.dep_off[b];
    h[7] = b;
  }
  uint32_t *pts = h + 8;
  for (int c = 0; c < a.n_class; ++c) {
    for (uint32_t i = threadIdx.x; i < n[c]; i += blockDim.x) pts[i] = a.pts[c][a.pts_off[c][b] + i];
    pts += n[c];
  }
  uint16_t *l = reinterpret_cast<uint16_t *>(pts);
  for (int c = 0; c < a.n_class; ++c)
    for (int s = 0; s < a.D; ++s) {
      for (uint32_t i = threadIdx.x; i < ncell; i += blockDim.x)
        l[i] = a.lidx[c][(size_t)s * a.n_cells + start + i];
      l += ncell;
    }
  // contributions per written point: counts, offsets, then each thread
  // collects the entries of its own points by scanning all of them in order
  uint16_t *pc_off = l;
  uint16_t *pc_idx = l + n[0] + 1;
  const uint16_t *l0 = reinterpret_cast<const uint16_t *>(h + 8 + n[0] + n[1]);
  const uint32_t E = a.D * ncell;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t j = 0; j <= n[0]; ++j) pc_off[j] = 0;
    for (uint32_t i = 0; i < ncell; ++i)
      for (int s = 0; s < a.D; ++s) pc_off[l0[s * ncell + i] + 1]++;
    for (uint32_t j = 0; j < n[0]; ++j) pc_off[j + 1] += pc_off[j];
  }
  __syncthreads();
  for (uint32_t j0 = 0; j0 < n[0]; j0 += blockDim.x) {
    const uint32_t j = j0 + threadIdx.x;
    uint32_t w = j < n[0] ? pc_off[j] : 0;
    for (uint32_t i = 0; i < ncell; ++i)
      for (int s = 0; s < a.D; ++s)
        if (j < n[0] && l0[s * ncell + i] == j) pc_idx[w++] = (uint16_t)(s * a.threads + i);
  }
  const uint32_t dep_at = record_dep_offset(ncell, n[0], n[1], a.D, a.n_class);
  const uint32_t ndep = a.dep_off[b + 1] - a.dep_off[b];
  for (uint32_t i = (uint32_t)(reinterpret_cast<unsigned char *>(pc_idx + E) - r) + threadIdx.x;
       i < dep_at; i += blockDim.x)
    r[i] = 0;
  uint32_t *dep = reinterpret_cast<uint32_t *>(r + dep_at);
  for (uint32_t i = threadIdx.x; i < ndep; i += blockDim.x) dep[i] = a.dep[a.dep_off[b] + i];
  uint32_t used = dep_at + 4 * ndep;
  if (a.wslot) {
    uint32_t *w = reinterpret_cast<uint32_t *>(r + used);
    const uint32_t *src = a.wslot + a.pts_off[0][b];
    for (uint32_t i = threadIdx.x; i < n[0]; i += blockDim.x) w[i] = src[i];
    used += 4 * n[0];
  }
  for (uint32_t i = used + threadIdx.x; i < a.rec_off[b + 1] - a.rec_off[b]; i += blockDim.x) r[i] = 0;
}

// ---------------------------------------------------------------------------
// step 5: permute the problem's cells (rows of the mappings, cell datasets)
// ---------------------------------------------------------------------------
__global__ void k_gather_rows_u32(const uint32_t *src, uint32_t *dst, const uint32_t *perm,
                                  uint32_t n, int D) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i];
  for (int s = 0; s < D; ++s) dst[(size_t)i * D + s] = src[(size_t)c * D + s];
}

template <class T>
__global__ void k_gather_soa(const T *src, T *dst, const uint32_t *perm, uint32_t n, int dim) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i];
  for (int k = 0; k < dim; ++k) dst[(size_t)k * n + i] = src[(size_t)k * n + c];
}

template <int ITEMS> int launch_local(const LocalOut &o, uint32_t nfb, size_t dyn) {
  FOT_CUDA(cudaFuncSetAttribute(k_block_local<ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dyn));
  k_block_local<ITEMS><<<nfb, kPlanThreads, dyn>>>(o);
  FOT_CUDA(cudaGetLastError());
  return FOT_OK;
}

} // namespace

// Colour the blocks; returns per-formation-block colours on the host.
static int colour_blocks(const DevBuf &pad0, const DevBuf &cnt0, uint32_t nfb, uint32_t cap,
                         std::vector<int> &colours, DevBuf &d_err, std::vector<uint32_t> &g_row,
                         std::vector<uint32_t> &g_col) {
  std::vector<uint32_t> h_cnt;
  FOT_TRY(download(h_cnt, cnt0, nfb));
  std::vector<uint32_t> h_off(nfb);
  size_t n_pairs = 0;
  for (uint32_t b = 0; b < nfb; ++b) {
    h_off[b] = (uint32_t)n_pairs;
    n_pairs += h_cnt[b];
  }
  DevBuf off, k0, v0, k1, v1;
  FOT_TRY(upload(off, h_off));
  FOT_TRY(k0.alloc(n_pairs * 4));
  FOT_TRY(v0.alloc(n_pairs * 4));
  FOT_TRY(k1.alloc(n_pairs * 4));
  FOT_TRY(v1.alloc(n_pairs * 4));
  k_compact_pairs<<<nfb, 128>>>(pad0.as<uint32_t>(), cnt0.as<uint32_t>(), off.as<uint32_t>(), cap,
                                nfb, k0.as<uint32_t>(), v0.as<uint32_t>());
  FOT_CUDA(cudaGetLastError());
  FOT_TRY(sort_pairs(k0.as<uint32_t>(), k1.as<uint32_t>(), v0.as<uint32_t>(), v1.as<uint32_t>(),
                     n_pairs, 0));
  DevBuf ecnt, eoff;
  FOT_TRY(ecnt.alloc((n_pairs + 1) * 4));
  FOT_TRY(eoff.alloc((n_pairs + 1) * 4));
  FOT_CUDA(cudaMemset(ecnt.ptr, 0, (n_pairs + 1) * 4));
  if (n_pairs) {
    k_count_edges<<<blocks_for(n_pairs), 256>>>(k1.as<uint32_t>(), (uint32_t)n_pairs, ecnt.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
  }
  FOT_TRY(excl_sum(ecnt.as<uint32_t>(), eoff.as<uint32_t>(), n_pairs + 1, 0));
  uint32_t n_edges = 0;
  FOT_CUDA(cudaMemcpy(&n_edges, eoff.as<uint32_t>() + n_pairs, 4, cudaMemcpyDeviceToHost));
  DevBuf e0, e1;
  FOT_TRY(e0.alloc((size_t)n_edges * 8));
  FOT_TRY(e1.alloc((size_t)n_edges * 8));
  if (n_pairs) {
    k_emit_edges<<<blocks_for(n_pairs), 256>>>(k1.as<uint32_t>(), v1.as<uint32_t>(), (uint32_t)n_pairs,
                                               eoff.as<uint32_t>(), e0.as<uint64_t>());
    FOT_CUDA(cudaGetLastError());
  }
  uint32_t n_unique = 0;
  if (n_edges) {
    size_t tb = 0;
    FOT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, e0.as<uint64_t>(), e1.as<uint64_t>(),
                                            (int)n_edges));
    DevBuf tmp;
    FOT_TRY(tmp.alloc(tb));
    FOT_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, e0.as<uint64_t>(), e1.as<uint64_t>(),
                                            (int)n_edges));
    DevBuf nsel;
    FOT_TRY(nsel.alloc(4));
    size_t tb2 = 0;
    FOT_CUDA(cub::DeviceSelect::Unique(nullptr, tb2, e1.as<uint64_t>(), e0.as<uint64_t>(),
                                       nsel.as<uint32_t>(), (int)n_edges));
    DevBuf tmp2;
    FOT_TRY(tmp2.alloc(tb2));
    FOT_CUDA(cub::DeviceSelect::Unique(tmp2.ptr, tb2, e1.as<uint64_t>(), e0.as<uint64_t>(),
                                       nsel.as<uint32_t>(), (int)n_edges));
    FOT_CUDA(cudaMemcpy(&n_unique, nsel.ptr, 4, cudaMemcpyDeviceToHost));
  }
  DevBuf deg, row;
  FOT_TRY(deg.alloc((size_t)(nfb + 1) * 4));
  FOT_TRY(row.alloc((size_t)(nfb + 1) * 4));
  FOT_CUDA(cudaMemset(deg.ptr, 0, (size_t)(nfb + 1) * 4));
  if (n_unique) {
    k_degree<<<blocks_for(n_unique), 256>>>(e0.as<uint64_t>(), n_unique, deg.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
  }
  FOT_TRY(excl_sum(deg.as<uint32_t>(), row.as<uint32_t>(), nfb + 1, 0));
  DevBuf col, done;
  FOT_TRY(col.alloc((size_t)nfb * 4));
  FOT_TRY(done.alloc(4));
  FOT_CUDA(cudaMemset(col.ptr, 0xFF, (size_t)nfb * 4));
  FOT_CUDA(cudaMemset(done.ptr, 0, 4));
  uint32_t n_done = 0;
  for (int round = 0; n_done < nfb; ++round) {
    if (round > 100000) return fail(FOT_ERR_LIMIT, "block colouring did not converge");
    k_jp_round<<<blocks_for(nfb), 256>>>(row.as<uint32_t>(), e0.as<uint64_t>(), nfb, col.as<int>(),
                                         done.as<uint32_t>(), d_err.as<int>());
    FOT_CUDA(cudaGetLastError());
    FOT_CUDA(cudaMemcpy(&n_done, done.ptr, 4, cudaMemcpyDeviceToHost));
  }
  // the conflict graph (CSR over formation blocks) for the per-block
  // dependencies of the pipelined executor
  FOT_TRY(download(g_row, row, nfb + 1));
  std::vector<uint64_t> edges;
  FOT_TRY(download(edges, e0.as<uint64_t>(), n_unique));
  g_col.resize(n_unique);
  for (uint32_t e = 0; e < n_unique; ++e) g_col[e] = (uint32_t)edges[e];
  return download(colours, col, nfb);
}

// Split write-back data of a plan (hier_split.cuh).  A written point of a
// block is PRIVATE when no other block writes it, else SHARED.  Shared points
// are numbered g = 0, 1, ... in point order; shared point g owns the
// partial-sum slots [base[g], base[g + 1]), one per block writing it, in
// plan order -- block-colour order, the order in which the coloured replay
// adds the blocks' sums.  Per block, wslot[j] is the slot of its j-th written
// point (0xFFFFFFFF: private); per shared point, its point number and base.
struct SplitRecords {
  std::vector<uint32_t> wslot;            // per (block, written point), plan order
  std::vector<uint32_t> point, base;      // n_shared, n_shared + 1
  uint32_t n_slots = 0;
};

static int build_split(const std::vector<uint32_t> &pts0, const std::vector<uint32_t> &off0,
                       uint32_t n_points, SplitRecords &out) {
  const uint32_t nfb = (uint32_t)off0.size() - 1;
  const size_t n_pairs = pts0.size();
  std::vector<uint32_t> deg(n_points, 0);
  for (size_t j = 0; j < n_pairs; ++j) {
    if (pts0[j] >= n_points) return fail(FOT_ERR_STATE, "plan point %u out of range", pts0[j]);
    ++deg[pts0[j]];
  }
  std::vector<uint32_t> g_of(n_points, 0xFFFFFFFFu);
  out.point.clear();
  out.base.assign(1, 0);
  for (uint32_t q = 0; q < n_points; ++q)
    if (deg[q] > 1) {
      g_of[q] = (uint32_t)out.point.size();
      out.point.push_back(q);
      out.base.push_back(out.base.back() + deg[q]);
    }
  std::vector<uint32_t> fill(out.base.begin(), out.base.end() - 1);
  out.wslot.assign(n_pairs, 0xFFFFFFFFu);
  for (uint32_t b = 0; b < nfb; ++b)  // plan order: each point's slots in colour order
    for (uint32_t j = off0[b]; j < off0[b + 1]; ++j) {
      const uint32_t g = g_of[pts0[j]];
      if (g != 0xFFFFFFFFu) out.wslot[j] = fill[g]++;
    }
  out.n_slots = out.base.back();
  return FOT_OK;
}

int build_hier_plan(fot_problem *p, fot_plan *plan) {
  const uint32_t B = plan->desc.block_size;
  const int D = (int)p->mesh_dim();
  const uint32_t n = p->n_cells;
  const int n_class = p->has_class1 ? 2 : 1;
  if (B == 0 || B > 1024) return fail(FOT_ERR_ARG, "block size must be in [1, 1024]");
  if ((uint64_t)B * D > 8192) return fail(FOT_ERR_LIMIT, "block_size * mesh_dim must be <= 8192");
  if (n == 0) return fail(FOT_ERR_ARG, "empty problem");
  const uint32_t cap = B * D;

  // 1. blocks
  std::vector<uint32_t> fstart;
  DevBuf form_cells;
  if (plan->desc.flags & FOT_PLAN_USE_PARTITION) {
    if (p->partition.size() != n) return fail(FOT_ERR_STATE, "problem has no partition");
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(),
                     [&](uint32_t a, uint32_t b) { return p->partition[a] < p->partition[b]; });
    fstart.push_back(0);
    uint32_t run = 0;
    for (uint32_t i = 1; i < n; ++i) {
      ++run;
      if (run == B || p->partition[idx[i]] != p->partition[idx[i - 1]]) {
        fstart.push_back(i);
        run = 0;
      }
    }
    fstart.push_back(n);
    FOT_TRY(upload(form_cells, idx));
  } else {
    for (uint32_t i = 0; i < n; i += B) fstart.push_back(i);
    fstart.push_back(n);
  }
  const uint32_t nfb = (uint32_t)fstart.size() - 1;

  // 2. per-block local data
  DevBuf d_fstart, pad[2], cnt[2], f_cell, f_tcol, f_lidx[2], f_ntcol, d_err;
  FOT_TRY(upload(d_fstart, fstart));
  for (int c = 0; c < n_class; ++c) {
    FOT_TRY(pad[c].alloc((size_t)nfb * cap * 4));
    FOT_TRY(cnt[c].alloc((size_t)nfb * 4));
    FOT_TRY(f_lidx[c].alloc((size_t)D * n * 2));
  }
  FOT_TRY(f_cell.alloc((size_t)n * 4));
  FOT_TRY(f_tcol.alloc(n));
  FOT_TRY(f_ntcol.alloc(nfb));
  FOT_TRY(d_err.alloc(4));
  FOT_CUDA(cudaMemset(d_err.ptr, 0, 4));
  LocalOut o{};
  o.map[0] = p->map[0].as<uint32_t>();
  o.map[1] = n_class > 1 ? p->map[1].as<uint32_t>() : nullptr;
  o.n_class = n_class;
  o.D = D;
  o.fstart = d_fstart.as<uint32_t>();
  o.form_cells = form_cells.ptr ? form_cells.as<uint32_t>() : nullptr;
  o.cap = cap;
  for (int c = 0; c < 2; ++c) {
    o.pad_pts[c] = c < n_class ? pad[c].as<uint32_t>() : nullptr;
    o.cnt[c] = c < n_class ? cnt[c].as<uint32_t>() : nullptr;
    o.out_lidx[c] = c < n_class ? f_lidx[c].as<uint16_t>() : nullptr;
  }
  o.out_cell = f_cell.as<uint32_t>();
  o.out_tcol = f_tcol.as<uint8_t>();
  o.ntcol = f_ntcol.as<uint8_t>();
  o.n_cells = n;
  o.err = d_err.as<int>();
  const size_t dyn = ((4 * (size_t)cap * sizeof(uint16_t) + 15) & ~size_t(15)) + (size_t)cap * 8;
  const uint32_t items = (cap + kPlanThreads - 1) / kPlanThreads;
  if (items <= 1) FOT_TRY(launch_local<1>(o, nfb, dyn));
  else if (items <= 2) FOT_TRY(launch_local<2>(o, nfb, dyn));
  else if (items <= 4) FOT_TRY(launch_local<4>(o, nfb, dyn));
  else if (items <= 8) FOT_TRY(launch_local<8>(o, nfb, dyn));
  else if (items <= 16) FOT_TRY(launch_local<16>(o, nfb, dyn));
  else FOT_TRY(launch_local<32>(o, nfb, dyn));

  // 3. block colours
  std::vector<int> colours;
  std::vector<uint32_t> g_row, g_col;
  FOT_TRY(colour_blocks(pad[0], cnt[0], nfb, cap, colours, d_err, g_row, g_col));
  int h_err = 0;
  FOT_CUDA(cudaMemcpy(&h_err, d_err.ptr, 4, cudaMemcpyDeviceToHost));
  if (h_err & 1) return fail(FOT_ERR_LIMIT, "a block needs more than %d thread colours", kMaxThreadColours);
  if (h_err & 2) return fail(FOT_ERR_LIMIT, "more than %d block colours", kMaxBlockColours);

  // 4. order blocks by colour (stable) and gather
  const int n_col = *std::max_element(colours.begin(), colours.end()) + 1;
  std::vector<uint32_t> colour_first(n_col + 1, 0);
  for (uint32_t b = 0; b < nfb; ++b) colour_first[colours[b] + 1]++;
  for (int c = 0; c < n_col; ++c) colour_first[c + 1] += colour_first[c];
  std::vector<uint32_t> order(nfb);
  {
    std::vector<uint32_t> fill(colour_first.begin(), colour_first.end() - 1);
    for (uint32_t b = 0; b < nfb; ++b) order[fill[colours[b]]++] = b;
  }
  std::vector<uint32_t> block_start(nfb + 1, 0);
  for (uint32_t b = 0; b < nfb; ++b)
    block_start[b + 1] = block_start[b] + (fstart[order[b] + 1] - fstart[order[b]]);
  std::vector<uint32_t> h_cnt[2], h_off[2];
  for (int c = 0; c < n_class; ++c) {
    FOT_TRY(download(h_cnt[c], cnt[c], nfb));
    h_off[c].assign(nfb + 1, 0);
    for (uint32_t b = 0; b < nfb; ++b) h_off[c][b + 1] = h_off[c][b] + h_cnt[c][order[b]];
    plan->cap[c] = *std::max_element(h_cnt[c].begin(), h_cnt[c].end());
  }
  std::vector<uint8_t> h_ntcol;
  FOT_TRY(download(h_ntcol, f_ntcol, nfb));

  DevBuf d_order, d_colour, d_colour_first;
  FOT_TRY(upload(d_order, order));
  FOT_TRY(upload(d_colour, colours));
  FOT_TRY(upload(d_colour_first, colour_first));
  FOT_TRY(upload(plan->block_start, block_start));
  FOT_TRY(plan->block_wait.alloc((size_t)nfb * 4));
  FOT_TRY(plan->block_ntcol.alloc(nfb));
  FOT_TRY(plan->tcol.alloc(n));
  FOT_TRY(plan->build_perm.alloc((size_t)n * 4));
  for (int c = 0; c < n_class; ++c) {
    FOT_TRY(upload(plan->pts_off[c], h_off[c]));
    FOT_TRY(plan->pts[c].alloc((size_t)h_off[c][nfb] * 4));
    FOT_TRY(plan->lidx[c].alloc((size_t)D * n * 2));
  }
  GatherArgs g{};
  g.order = d_order.as<uint32_t>();
  g.fstart = d_fstart.as<uint32_t>();
  g.block_start = plan->block_start.as<uint32_t>();
  g.f_cell = f_cell.as<uint32_t>();
  g.f_tcol = f_tcol.as<uint8_t>();
  g.f_ntcol = f_ntcol.as<uint8_t>();
  g.colour = d_colour.as<int>();
  g.colour_first = d_colour_first.as<uint32_t>();
  g.cell = plan->build_perm.as<uint32_t>();
  g.tcol = plan->tcol.as<uint8_t>();
  g.ntcol = plan->block_ntcol.as<uint8_t>();
  g.block_wait = plan->block_wait.as<uint32_t>();
  g.cap = cap;
  g.n_cells = n;
  g.n_class = n_class;
  g.D = D;
  for (int c = 0; c < n_class; ++c) {
    g.f_lidx[c] = f_lidx[c].as<uint16_t>();
    g.pad_pts[c] = pad[c].as<uint32_t>();
    g.cnt[c] = cnt[c].as<uint32_t>();
    g.pts_off[c] = plan->pts_off[c].as<uint32_t>();
    g.lidx[c] = plan->lidx[c].as<uint16_t>();
    g.pts[c] = plan->pts[c].as<uint32_t>();
  }
  k_gather_plan<<<nfb, 256>>>(g);
  FOT_CUDA(cudaGetLastError());

  // 4b. tile records
  {
    const bool split = plan->variant & kVariantSplit;
    std::vector<uint32_t> final_of(nfb);
    for (uint32_t b = 0; b < nfb; ++b) final_of[order[b]] = b;
    // conflict neighbours of each block in final order; bit 31: earlier
    // colour (the pipelined kernel's dependencies; the split kernel has none)
    std::vector<uint32_t> dep_off(nfb + 1, 0), dep;
    for (uint32_t b = 0; b < nfb && !split; ++b) {
      const uint32_t fb = order[b];
      for (uint32_t e = g_row[fb]; e < g_row[fb + 1]; ++e) {
        const uint32_t fn = g_col[e];
        dep.push_back(final_of[fn] | (colours[fn] < colours[fb] ? 0x80000000u : 0u));
      }
      dep_off[b + 1] = (uint32_t)dep.size();
    }
    DevBuf d_dep_off, d_dep, d_split;
    FOT_TRY(upload(d_dep_off, dep_off));
    FOT_TRY(upload(d_dep, dep));
    SplitRecords sr;
    if (split) {
      std::vector<uint32_t> h_pts0;
      FOT_TRY(download(h_pts0, plan->pts[0], h_off[0][nfb]));
      FOT_TRY(build_split(h_pts0, h_off[0], p->n_points[0], sr));
      FOT_TRY(upload(d_split, sr.wslot));
      // two buffers of partial sums (AOS rows of the incremented dataset's
      // element type; a launch fills one while it combines the other), the
      // shared points with their slot ranges, and the launch order of the
      // tiles: formation order, so that neighbouring blocks run together
      const size_t row = (size_t)p->info.point_dim[0] * p->info.point_type_size[0];
      FOT_TRY(plan->partial.alloc(2 * (size_t)sr.n_slots * row));
      FOT_TRY(upload(plan->comb_point, sr.point));
      FOT_TRY(upload(plan->comb_base, sr.base));
      FOT_TRY(upload(plan->launch, final_of));
      FOT_TRY(upload(plan->wslot, sr.wslot));
      // direct form: one 16-byte header per tile, in launch order
      std::vector<uint32_t> hdr((size_t)4 * nfb);
      for (uint32_t t = 0; t < nfb; ++t) {
        const uint32_t b = final_of[t], fb = order[b];
        hdr[4 * t + 0] = block_start[b];
        hdr[4 * t + 1] = (block_start[b + 1] - block_start[b]) | ((uint32_t)h_ntcol[fb] << 16);
        hdr[4 * t + 2] = h_off[0][b + 1] - h_off[0][b];
        hdr[4 * t + 3] = h_off[0][b];
      }
      FOT_TRY(upload(plan->tile_hdr, hdr));
      plan->n_slots = sr.n_slots;
      plan->n_shared_points = (uint32_t)sr.point.size();
    }
    std::vector<uint32_t> rec_off(nfb + 1, 0);
    uint32_t rec_cap = 0;
    for (uint32_t b = 0; b < nfb; ++b) {
      const uint32_t ncell = block_start[b + 1] - block_start[b];
      const uint32_t n0 = h_off[0][b + 1] - h_off[0][b];
      const uint32_t n1 = n_class > 1 ? h_off[1][b + 1] - h_off[1][b] : 0;
      uint32_t padded = record_bytes(ncell, n0, n1, D, n_class, dep_off[b + 1] - dep_off[b]);
      if (split) padded = (record_dep_offset(ncell, n0, n1, D, n_class) + 4 * n0 + 15) & ~15u;
      rec_cap = std::max(rec_cap, padded);
      rec_off[b + 1] = rec_off[b] + padded;
    }
    FOT_TRY(upload(plan->rec_off, rec_off));
    FOT_TRY(plan->rec.alloc(rec_off[nfb]));
    plan->rec_cap = rec_cap;
    // completed iterations of each block (the dependency flags)
    FOT_TRY(plan->block_done.alloc((size_t)nfb * 4));
    FOT_CUDA(cudaMemset(plan->block_done.ptr, 0, (size_t)nfb * 4));
    RecordArgs ra{};
    ra.block_start = plan->block_start.as<uint32_t>();
    ra.block_wait = plan->block_wait.as<uint32_t>();
    ra.rec_off = plan->rec_off.as<uint32_t>();
    ra.threads = hier_threads(B);
    ra.dep_off = d_dep_off.as<uint32_t>();
    ra.dep = d_dep.as<uint32_t>();
    ra.wslot = split ? d_split.as<uint32_t>() : nullptr;
    ra.ntcol = plan->block_ntcol.as<uint8_t>();
    ra.rec = plan->rec.as<unsigned char>();
    ra.n_cells = n;
    ra.n_class = n_class;
    ra.D = D;
    for (int c = 0; c < n_class; ++c) {
      ra.pts_off[c] = plan->pts_off[c].as<uint32_t>();
      ra.pts[c] = plan->pts[c].as<uint32_t>();
      ra.lidx[c] = plan->lidx[c].as<uint16_t>();
    }
    k_build_records<<<nfb, 128>>>(ra);
    FOT_CUDA(cudaGetLastError());
  }

  // 5. permute the problem's cells into plan order
  const uint32_t *perm = plan->build_perm.as<uint32_t>();
  for (int c = 0; c < n_class; ++c) {
    DevBuf nm;
    FOT_TRY(nm.alloc((size_t)n * D * 4));
    k_gather_rows_u32<<<blocks_for(n), 256>>>(p->map[c].as<uint32_t>(), nm.as<uint32_t>(), perm, n, D);
    FOT_CUDA(cudaGetLastError());
    p->map[c] = std::move(nm);
  }
  for (uint32_t j = 0; j < p->info.n_cell_sets; ++j) {
    DevBuf nc;
    FOT_TRY(nc.alloc(p->cell_bytes(j)));
    if (p->info.cell_type_size[j] == 8)
      k_gather_soa<uint64_t><<<blocks_for(n), 256>>>(p->cell[j].as<uint64_t>(), nc.as<uint64_t>(), perm, n,
                                                     p->info.cell_dim[j]);
    else
      k_gather_soa<uint32_t><<<blocks_for(n), 256>>>(p->cell[j].as<uint32_t>(), nc.as<uint32_t>(), perm, n,
                                                     p->info.cell_dim[j]);
    FOT_CUDA(cudaGetLastError());
    p->cell[j] = std::move(nc);
  }
  std::vector<uint32_t> h_perm;
  FOT_TRY(download(h_perm, plan->build_perm, n));
  {
    std::vector<uint32_t> co(n);
    for (uint32_t i = 0; i < n; ++i) co[i] = p->cell_order[h_perm[i]];
    p->cell_order.swap(co);
    if (p->partition.size() == n) {
      std::vector<uint32_t> pv(n);
      for (uint32_t i = 0; i < n; ++i) pv[i] = p->partition[h_perm[i]];
      p->partition.swap(pv);
    }
  }
  p->version++;
  plan->version = p->version;
  plan->n_blocks = nfb;
  plan->n_colours = (uint32_t)n_col;
  plan->colour_offsets = colour_first;

  // statistics
  fot_plan_stats &s = plan->stats;
  s.n_blocks = nfb;
  s.n_colours = (uint32_t)n_col;
  s.max_block_points = plan->cap[0];
  s.max_block_points1 = n_class > 1 ? plan->cap[1] : 0;
  double tc = 0, pts_sum = 0;
  uint32_t tmax = 0;
  for (uint32_t b = 0; b < nfb; ++b) {
    tc += h_ntcol[b];
    tmax = std::max<uint32_t>(tmax, h_ntcol[b]);
    pts_sum += h_cnt[0][b];
  }
  s.avg_thread_colours = tc / nfb;
  s.max_thread_colours = tmax;
  s.avg_block_points = pts_sum / nfb;
  return FOT_OK;
}

} // namespace fot
