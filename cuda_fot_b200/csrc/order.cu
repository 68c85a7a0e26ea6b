// GPU orderings and partitions of a problem.
//
// Replaces the reference's ordering calls and the external libraries behind
// them:
//   fot_reorder             Problem::reorder<SameMapping> (problem.hpp:439-482)
//                           with Mesh::reorder (mesh.hpp:199-225) and
//                           SCOTCH's "g" (Gibbs-Poole-Stockmeyer) ordering
//                           (reorder.hpp:135-175), here RCM / GPS / random
//                           computed on the GPU;
//   fot_partition           Problem::partition / partitionOurs
//                           (problem.hpp:484-515), METIS k-way plus the
//                           heuristic block growth (partition.cu:42-215), here
//                           a deterministic GPU region growing;
//   fot_reorder_to_partition Problem::reorderToPartition (problem.hpp:517-526);
//   fot_renumber_points     Problem::renumberPoints (problem.hpp:528-551) with
//                           getPointRenumberingPermutation2 (mesh.hpp:346-388).
#include <algorithm>
#include <numeric>

#include "devutil.cuh"
#include "engine.hpp"

namespace fot {
namespace {

constexpr uint32_t INF = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------
// graphs: point-to-point (points sharing a cell) and cell-to-cell (cells
// sharing a point), as CSR with sorted unique neighbour lists
// ---------------------------------------------------------------------------
struct Csr {
  uint32_t n = 0;
  uint32_t nnz = 0;
  DevBuf row, col, deg;
};

__global__ void k_point_pairs(const uint32_t *map, uint32_t n_cells, int D, uint64_t *out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  uint32_t w = c * D * (D - 1);
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j)
      if (i != j) {
        const uint32_t a = map[(size_t)c * D + i], b = map[(size_t)c * D + j];
        out[w++] = a == b ? ~0ull : ((uint64_t)a << 32) | b;
      }
}

__global__ void k_csr_degree(const uint64_t *edges, uint32_t ne, uint32_t *deg) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < ne && edges[e] != ~0ull) atomicAdd(&deg[edges[e] >> 32], 1u);
}

__global__ void k_csr_col(const uint64_t *edges, uint32_t ne, uint32_t *col) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < ne) col[e] = (uint32_t)edges[e];
}

// CSR from a list of 64-bit (src << 32 | dst) edges (sentinel ~0 dropped).
int csr_from_edges(DevBuf &edges, size_t ne, uint32_t n, Csr &g) {
  DevBuf sorted;
  FOT_TRY(sorted.alloc(ne * 8));
  FOT_TRY(sort_keys(edges.as<uint64_t>(), sorted.as<uint64_t>(), ne));
  uint32_t nu = 0;
  FOT_TRY(unique_keys(sorted.as<uint64_t>(), edges.as<uint64_t>(), ne, &nu));
  // drop the sentinel (sorts last)
  if (nu) {
    uint64_t last = 0;
    FOT_CUDA(cudaMemcpy(&last, edges.as<uint64_t>() + nu - 1, 8, cudaMemcpyDeviceToHost));
    if (last == ~0ull) --nu;
  }
  g.n = n;
  g.nnz = nu;
  FOT_TRY(g.deg.alloc((size_t)(n + 1) * 4));
  FOT_TRY(g.row.alloc((size_t)(n + 1) * 4));
  FOT_TRY(g.col.alloc((size_t)nu * 4 + 4));
  FOT_CUDA(cudaMemset(g.deg.ptr, 0, (size_t)(n + 1) * 4));
  if (nu) {
    k_csr_degree<<<blocks_for(nu), 256>>>(edges.as<uint64_t>(), nu, g.deg.as<uint32_t>());
    k_csr_col<<<blocks_for(nu), 256>>>(edges.as<uint64_t>(), nu, g.col.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
  }
  FOT_TRY(excl_sum(g.deg.as<uint32_t>(), g.row.as<uint32_t>(), n + 1));
  return FOT_OK;
}

int point_graph(const fot_problem *p, int cls, Csr &g) {
  const int D = (int)p->info.mesh_dim[cls == 0 ? 0 : 1];
  const size_t ne = (size_t)p->n_cells * D * (D - 1);
  DevBuf edges;
  FOT_TRY(edges.alloc(ne * 8 + 8));
  k_point_pairs<<<blocks_for(p->n_cells), 256>>>(p->map[cls].as<uint32_t>(), p->n_cells, D,
                                                 edges.as<uint64_t>());
  FOT_CUDA(cudaGetLastError());
  return csr_from_edges(edges, ne, p->class_points(cls), g);
}

__global__ void k_incidence(const uint32_t *map, uint32_t n_cells, int D, uint32_t *keys,
                            uint32_t *vals) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_cells * D) return;
  keys[e] = map[e];
  vals[e] = e / D;
}

__global__ void k_cell_pairs_count(const uint32_t *keys, uint32_t n, uint32_t *cnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = 0;
  if (i == 0 || keys[i] != keys[i - 1]) {
    uint32_t m = 1;
    while (i + m < n && keys[i + m] == keys[i]) ++m;
    c = m * (m - 1);
  }
  cnt[i] = c;
}

__global__ void k_cell_pairs_emit(const uint32_t *keys, const uint32_t *vals, uint32_t n,
                                  const uint32_t *off, uint64_t *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(i == 0 || keys[i] != keys[i - 1])) return;
  uint32_t m = 1;
  while (i + m < n && keys[i + m] == keys[i]) ++m;
  uint32_t w = off[i];
  for (uint32_t a = 0; a < m; ++a)
    for (uint32_t b = 0; b < m; ++b)
      if (a != b) out[w++] = vals[i + a] == vals[i + b] ? ~0ull : ((uint64_t)vals[i + a] << 32) | vals[i + b];
}

// cells adjacent when they share a point of mapping 0 (Mesh::getCellToCellGraph, mesh.hpp:317-344)
int cell_graph(const fot_problem *p, Csr &g) {
  const int D = (int)p->mesh_dim();
  const uint32_t ne = p->n_cells * D;
  DevBuf k0, v0, k1, v1, cnt, off;
  FOT_TRY(k0.alloc((size_t)ne * 4));
  FOT_TRY(v0.alloc((size_t)ne * 4));
  FOT_TRY(k1.alloc((size_t)ne * 4));
  FOT_TRY(v1.alloc((size_t)ne * 4));
  k_incidence<<<blocks_for(ne), 256>>>(p->map[0].as<uint32_t>(), p->n_cells, D, k0.as<uint32_t>(),
                                       v0.as<uint32_t>());
  FOT_CUDA(cudaGetLastError());
  FOT_TRY(sort_pairs(k0.as<uint32_t>(), k1.as<uint32_t>(), v0.as<uint32_t>(), v1.as<uint32_t>(), ne));
  FOT_TRY(cnt.alloc((size_t)(ne + 1) * 4));
  FOT_TRY(off.alloc((size_t)(ne + 1) * 4));
  FOT_CUDA(cudaMemset(cnt.ptr, 0, (size_t)(ne + 1) * 4));
  k_cell_pairs_count<<<blocks_for(ne), 256>>>(k1.as<uint32_t>(), ne, cnt.as<uint32_t>());
  FOT_CUDA(cudaGetLastError());
  FOT_TRY(excl_sum(cnt.as<uint32_t>(), off.as<uint32_t>(), ne + 1));
  uint32_t total = 0;
  FOT_CUDA(cudaMemcpy(&total, off.as<uint32_t>() + ne, 4, cudaMemcpyDeviceToHost));
  DevBuf edges;
  FOT_TRY(edges.alloc((size_t)total * 8 + 8));
  k_cell_pairs_emit<<<blocks_for(ne), 256>>>(k1.as<uint32_t>(), v1.as<uint32_t>(), ne,
                                             off.as<uint32_t>(), edges.as<uint64_t>());
  FOT_CUDA(cudaGetLastError());
  return csr_from_edges(edges, total, p->n_cells, g);
}

// ---------------------------------------------------------------------------
// level-synchronous BFS
// ---------------------------------------------------------------------------
// Expand one level.  lvl[v] == INF: unvisited.  Every frontier node u offers
// its order position to each not-yet-levelled neighbour v (atomicMin on
// parent[v]); the first to claim v appends it to the next frontier.
__global__ void k_bfs_expand(const uint32_t *row, const uint32_t *col, const uint32_t *frontier,
                             uint32_t nf, const uint32_t *pos, uint32_t next_level, uint32_t *lvl,
                             uint32_t *parent, uint32_t *next, uint32_t *n_next) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const uint32_t u = frontier[i];
  const uint32_t pu = pos ? pos[u] : 0;
  for (uint32_t e = row[u]; e < row[u + 1]; ++e) {
    const uint32_t v = col[e];
    if (lvl[v] >= next_level) {
      if (parent) atomicMin(&parent[v], pu);
      if (atomicCAS(&lvl[v], INF, next_level) == INF) next[atomicAdd(n_next, 1u)] = v;
    }
  }
}

__global__ void k_set_u32(uint32_t *a, uint32_t n, uint32_t v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

__global__ void k_sort_key(const uint32_t *nodes, uint32_t n, const uint32_t *parent,
                           const uint32_t *deg, uint64_t *key) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t v = nodes[i];
  key[i] = ((uint64_t)parent[v] << 24) | min(deg[v], 0xFFFFFFu);
}

__global__ void k_assign_pos(const uint32_t *nodes, uint32_t n, uint32_t base, uint32_t *pos,
                             uint32_t *order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pos[nodes[i]] = base + i;
  order[base + i] = nodes[i];
}

// Plain BFS from `src`: levels of every reached node; returns the depth, the
// number of reached nodes and a node of the last level of minimum degree.
int bfs_levels(const Csr &g, uint32_t src, DevBuf &lvl, uint32_t *depth, uint32_t *reached,
               uint32_t *far_node) {
  const uint32_t n = g.n;
  DevBuf fa, fb, cnt;
  FOT_TRY(fa.alloc((size_t)n * 4));
  FOT_TRY(fb.alloc((size_t)n * 4));
  FOT_TRY(cnt.alloc(4));
  k_set_u32<<<blocks_for(n), 256>>>(lvl.as<uint32_t>(), n, INF);
  FOT_CUDA(cudaMemcpy(fa.ptr, &src, 4, cudaMemcpyHostToDevice));
  const uint32_t zero = 0;
  FOT_CUDA(cudaMemcpy(lvl.as<uint32_t>() + src, &zero, 4, cudaMemcpyHostToDevice));
  uint32_t nf = 1, level = 0, total = 1;
  std::vector<uint32_t> last;
  for (;;) {
    FOT_CUDA(cudaMemsetAsync(cnt.ptr, 0, 4));
    k_bfs_expand<<<blocks_for(nf), 256>>>(g.row.as<uint32_t>(), g.col.as<uint32_t>(),
                                          fa.as<uint32_t>(), nf, nullptr, level + 1,
                                          lvl.as<uint32_t>(), nullptr, fb.as<uint32_t>(),
                                          cnt.as<uint32_t>());
    uint32_t nn = 0;
    FOT_CUDA(cudaMemcpy(&nn, cnt.ptr, 4, cudaMemcpyDeviceToHost));
    if (nn == 0) break;
    std::swap(fa, fb);
    nf = nn;
    total += nn;
    ++level;
  }
  // the last frontier is in fa (nf nodes): pick the minimum degree, then id
  std::vector<uint32_t> h_last, h_deg;
  FOT_TRY(download(h_last, fa.as<uint32_t>(), nf));
  FOT_TRY(download(h_deg, g.deg, n));
  uint32_t best = h_last[0];
  for (uint32_t v : h_last)
    if (h_deg[v] < h_deg[best] || (h_deg[v] == h_deg[best] && v < best)) best = v;
  *depth = level;
  *reached = total;
  *far_node = best;
  return FOT_OK;
}

// George-Liu pseudo-peripheral node of the component of `start`.
int pseudo_peripheral(const Csr &g, uint32_t start, uint32_t *out, uint32_t *out_far,
                      uint32_t *out_depth) {
  DevBuf lvl;
  FOT_TRY(lvl.alloc((size_t)g.n * 4));
  uint32_t x = start, depth = 0, reached = 0, far = start;
  FOT_TRY(bfs_levels(g, x, lvl, &depth, &reached, &far));
  for (int it = 0; it < 8; ++it) {
    uint32_t d2 = 0, r2 = 0, f2 = 0;
    FOT_TRY(bfs_levels(g, far, lvl, &d2, &r2, &f2));
    if (d2 <= depth) break;
    x = far;
    depth = d2;
    far = f2;
  }
  *out = x;
  *out_far = far;
  *out_depth = depth;
  return FOT_OK;
}

// Cuthill-McKee order of the whole graph (components one after another, each
// from a pseudo-peripheral node of minimum degree): within a level, nodes are
// sorted by the position of their earliest-ordered neighbour in the previous
// level, then degree, then id.  order[i] = i-th node.
int cuthill_mckee(const Csr &g, std::vector<uint32_t> &order) {
  const uint32_t n = g.n;
  DevBuf lvl, parent, pos, d_order, fa, fb, cnt, keys, keys2, vals2;
  FOT_TRY(lvl.alloc((size_t)n * 4));
  FOT_TRY(parent.alloc((size_t)n * 4));
  FOT_TRY(pos.alloc((size_t)n * 4));
  FOT_TRY(d_order.alloc((size_t)n * 4));
  FOT_TRY(fa.alloc((size_t)n * 4));
  FOT_TRY(fb.alloc((size_t)n * 4));
  FOT_TRY(cnt.alloc(4));
  FOT_TRY(keys.alloc((size_t)n * 8));
  FOT_TRY(keys2.alloc((size_t)n * 8));
  FOT_TRY(vals2.alloc((size_t)n * 4));
  k_set_u32<<<blocks_for(n), 256>>>(lvl.as<uint32_t>(), n, INF);
  k_set_u32<<<blocks_for(n), 256>>>(parent.as<uint32_t>(), n, INF);
  std::vector<uint32_t> h_deg;
  FOT_TRY(download(h_deg, g.deg, n));
  std::vector<uint8_t> seen(n, 0);
  uint32_t placed = 0, scan_from = 0;
  while (placed < n) {
    // next component: an unplaced node of minimum degree (first by id)
    std::vector<uint32_t> h_lvl;
    FOT_TRY(download(h_lvl, lvl, n));
    uint32_t start = INF;
    for (uint32_t v = scan_from; v < n; ++v)
      if (h_lvl[v] == INF && (start == INF || h_deg[v] < h_deg[start])) start = v;
    while (scan_from < n && h_lvl[scan_from] != INF) ++scan_from;
    // pseudo-peripheral start within the component: BFS levels on a scratch
    // copy so that placed components stay marked
    uint32_t pp = start, far = start, depth = 0;
    {
      Csr sub;  // the BFS helpers work on the whole graph; components are disjoint
      (void)sub;
      FOT_TRY(pseudo_peripheral(g, start, &pp, &far, &depth));
    }
    const uint32_t lev0 = placed == 0 ? 0 : 0;
    FOT_CUDA(cudaMemcpy(fa.ptr, &pp, 4, cudaMemcpyHostToDevice));
    FOT_CUDA(cudaMemcpy(lvl.as<uint32_t>() + pp, &lev0, 4, cudaMemcpyHostToDevice));
    k_assign_pos<<<1, 1>>>(fa.as<uint32_t>(), 1, placed, pos.as<uint32_t>(), d_order.as<uint32_t>());
    uint32_t nf = 1, level = 0;
    placed += 1;
    for (;;) {
      FOT_CUDA(cudaMemsetAsync(cnt.ptr, 0, 4));
      // levels of different components never meet; the level counter only
      // needs to exceed every level already assigned in this component
      k_bfs_expand<<<blocks_for(nf), 256>>>(g.row.as<uint32_t>(), g.col.as<uint32_t>(),
                                            fa.as<uint32_t>(), nf, pos.as<uint32_t>(), level + 1,
                                            lvl.as<uint32_t>(), parent.as<uint32_t>(),
                                            fb.as<uint32_t>(), cnt.as<uint32_t>());
      uint32_t nn = 0;
      FOT_CUDA(cudaMemcpy(&nn, cnt.ptr, 4, cudaMemcpyDeviceToHost));
      if (nn == 0) break;
      // deterministic order: by id, then stably by (parent position, degree)
      FOT_TRY(sort_keys(fb.as<uint32_t>(), fa.as<uint32_t>(), nn));
      k_sort_key<<<blocks_for(nn), 256>>>(fa.as<uint32_t>(), nn, parent.as<uint32_t>(),
                                          g.deg.as<uint32_t>(), keys.as<uint64_t>());
      FOT_TRY(sort_pairs(keys.as<uint64_t>(), keys2.as<uint64_t>(), fa.as<uint32_t>(),
                         fb.as<uint32_t>(), nn, 0, 56));
      k_assign_pos<<<blocks_for(nn), 256>>>(fb.as<uint32_t>(), nn, placed, pos.as<uint32_t>(),
                                            d_order.as<uint32_t>());
      FOT_CUDA(cudaGetLastError());
      std::swap(fa, fb);
      nf = nn;
      placed += nn;
      ++level;
    }
    (void)seen;
  }
  return download(order, d_order, n);
}

// ---------------------------------------------------------------------------
// applying permutations
// ---------------------------------------------------------------------------
__global__ void k_renumber(uint32_t *map, size_t n, const uint32_t *perm) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) map[i] = perm[map[i]];
}

template <class T>
__global__ void k_scatter_rows(const T *src, T *dst, const uint32_t *perm, uint32_t n, int dim,
                               bool soa) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = perm[i];
  for (int k = 0; k < dim; ++k) {
    if (soa) dst[(size_t)k * n + j] = src[(size_t)k * n + i];
    else dst[(size_t)j * dim + k] = src[(size_t)i * dim + k];
  }
}

__global__ void k_gather_rows(const uint32_t *src, uint32_t *dst, const uint32_t *perm, uint32_t n, int D) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i];
  for (int s = 0; s < D; ++s) dst[(size_t)i * D + s] = src[(size_t)c * D + s];
}

template <class T>
__global__ void k_gather_cols(const T *src, T *dst, const uint32_t *perm, uint32_t n, int dim) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i];
  for (int k = 0; k < dim; ++k) dst[(size_t)k * n + i] = src[(size_t)k * n + c];
}

} // namespace

// Renumber the points of class `cls`: old point i becomes perm[i]; the point
// datasets on that class move with them.
int apply_point_perm(fot_problem *p, int cls, const std::vector<uint32_t> &perm) {
  const uint32_t np = p->class_points(cls);
  DevBuf d_perm;
  FOT_TRY(upload(d_perm, perm));
  const int D = (int)p->info.mesh_dim[cls == 0 ? 0 : 1];
  const size_t ne = (size_t)p->n_cells * D;
  k_renumber<<<blocks_for(ne), 256>>>(p->map[cls].as<uint32_t>(), ne, d_perm.as<uint32_t>());
  FOT_CUDA(cudaGetLastError());
  for (uint32_t k = 0; k < p->info.n_point_sets; ++k) {
    if (set_class(p->loop, k) != cls) continue;
    DevBuf nb;
    FOT_TRY(nb.alloc(p->point_bytes(k)));
    const int dim = p->info.point_dim[k];
    const bool soa = p->layout == FOT_SOA;
    if (p->info.point_type_size[k] == 8)
      k_scatter_rows<uint64_t><<<blocks_for(np), 256>>>(p->point[k].as<uint64_t>(), nb.as<uint64_t>(),
                                                        d_perm.as<uint32_t>(), np, dim, soa);
    else
      k_scatter_rows<uint32_t><<<blocks_for(np), 256>>>(p->point[k].as<uint32_t>(), nb.as<uint32_t>(),
                                                        d_perm.as<uint32_t>(), np, dim, soa);
    FOT_CUDA(cudaGetLastError());
    p->point[k] = std::move(nb);
  }
  auto &pp = p->point_perm[cls];
  for (auto &v : pp) v = perm[v];
  p->version++;
  return FOT_OK;
}

// Reorder the cells: new cell i is old cell order[i].
int apply_cell_order(fot_problem *p, const std::vector<uint32_t> &order) {
  const uint32_t n = p->n_cells;
  DevBuf d_ord;
  FOT_TRY(upload(d_ord, order));
  for (int c = 0; c < (p->has_class1 ? 2 : 1); ++c) {
    const int D = (int)p->info.mesh_dim[c == 0 ? 0 : 1];
    DevBuf nm;
    FOT_TRY(nm.alloc((size_t)n * D * 4));
    k_gather_rows<<<blocks_for(n), 256>>>(p->map[c].as<uint32_t>(), nm.as<uint32_t>(),
                                          d_ord.as<uint32_t>(), n, D);
    FOT_CUDA(cudaGetLastError());
    p->map[c] = std::move(nm);
  }
  for (uint32_t j = 0; j < p->info.n_cell_sets; ++j) {
    DevBuf nc;
    FOT_TRY(nc.alloc(p->cell_bytes(j)));
    if (p->info.cell_type_size[j] == 8)
      k_gather_cols<uint64_t><<<blocks_for(n), 256>>>(p->cell[j].as<uint64_t>(), nc.as<uint64_t>(),
                                                      d_ord.as<uint32_t>(), n, p->info.cell_dim[j]);
    else
      k_gather_cols<uint32_t><<<blocks_for(n), 256>>>(p->cell[j].as<uint32_t>(), nc.as<uint32_t>(),
                                                      d_ord.as<uint32_t>(), n, p->info.cell_dim[j]);
    FOT_CUDA(cudaGetLastError());
    p->cell[j] = std::move(nc);
  }
  std::vector<uint32_t> co(n);
  for (uint32_t i = 0; i < n; ++i) co[i] = p->cell_order[order[i]];
  p->cell_order.swap(co);
  if (p->partition.size() == n) {
    std::vector<uint32_t> pv(n);
    for (uint32_t i = 0; i < n; ++i) pv[i] = p->partition[order[i]];
    p->partition.swap(pv);
  }
  p->version++;
  return FOT_OK;
}

namespace {

// ---------------------------------------------------------------------------
// GPS: levels from both ends of a pseudo-diameter, ambiguous nodes assigned
// per connected component to the end that keeps the widest level narrow,
// numbered level by level in Cuthill-McKee fashion.
// ---------------------------------------------------------------------------
__global__ void k_gps_pair(const uint32_t *lu, const uint32_t *lv, uint32_t n, uint32_t depth,
                           uint32_t *lvl, uint32_t *amb) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  const uint32_t i = lu[x];
  const uint32_t j = lv[x] == INF ? INF : depth - min(lv[x], depth);
  if (i == INF) {
    lvl[x] = INF;
    amb[x] = 0;
  } else if (i == j) {
    lvl[x] = i;
    amb[x] = 0;
  } else {
    lvl[x] = INF;
    amb[x] = 1;
  }
}

__global__ void k_cc_init(const uint32_t *amb, uint32_t n, uint32_t *label) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < n) label[x] = amb[x] ? x : INF;
}

__global__ void k_cc_step(const uint32_t *row, const uint32_t *col, uint32_t n, uint32_t *label,
                          uint32_t *changed) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n || label[x] == INF) return;
  uint32_t m = label[x];
  for (uint32_t e = row[x]; e < row[x + 1]; ++e) {
    const uint32_t l = label[col[e]];
    if (l < m) m = l;
  }
  if (m < label[x]) {
    atomicMin(&label[x], m);
    *changed = 1;
  }
}

} // namespace

int gps_levels(const Csr &g, std::vector<uint32_t> &level_of, uint32_t *n_levels) {
  const uint32_t n = g.n;
  std::vector<uint32_t> h_deg;
  FOT_TRY(download(h_deg, g.deg, n));
  DevBuf lu, lv, lvl, amb, label, changed;
  FOT_TRY(lu.alloc((size_t)n * 4));
  FOT_TRY(lv.alloc((size_t)n * 4));
  FOT_TRY(lvl.alloc((size_t)n * 4));
  FOT_TRY(amb.alloc((size_t)n * 4));
  FOT_TRY(label.alloc((size_t)n * 4));
  FOT_TRY(changed.alloc(4));
  level_of.assign(n, INF);
  uint32_t level_base = 0;
  std::vector<uint32_t> h_lvl_all(n, INF);
  for (;;) {
    // next component from an unlevelled node of minimum degree
    uint32_t start = INF;
    for (uint32_t v = 0; v < n; ++v)
      if (level_of[v] == INF && (start == INF || h_deg[v] < h_deg[start])) start = v;
    if (start == INF) break;
    uint32_t u = start, v = start, depth = 0, reached = 0, far2 = 0;
    FOT_TRY(pseudo_peripheral(g, start, &u, &v, &depth));
    uint32_t d1 = 0, d2 = 0, f = 0;
    FOT_TRY(bfs_levels(g, u, lu, &d1, &reached, &f));
    FOT_TRY(bfs_levels(g, v, lv, &d2, &reached, &far2));
    depth = d1;
    k_gps_pair<<<blocks_for(n), 256>>>(lu.as<uint32_t>(), lv.as<uint32_t>(), n, depth,
                                       lvl.as<uint32_t>(), amb.as<uint32_t>());
    k_cc_init<<<blocks_for(n), 256>>>(amb.as<uint32_t>(), n, label.as<uint32_t>());
    // components of the ambiguous nodes: min-label propagation restricted to them
    for (int it = 0; it < 100000; ++it) {
      FOT_CUDA(cudaMemset(changed.ptr, 0, 4));
      k_cc_step<<<blocks_for(n), 256>>>(g.row.as<uint32_t>(), g.col.as<uint32_t>(), n,
                                        label.as<uint32_t>(), changed.as<uint32_t>());
      uint32_t ch = 0;
      FOT_CUDA(cudaMemcpy(&ch, changed.ptr, 4, cudaMemcpyDeviceToHost));
      if (!ch) break;
    }
    std::vector<uint32_t> h_lu, h_lv, h_lvl, h_lab;
    FOT_TRY(download(h_lu, lu, n));
    FOT_TRY(download(h_lv, lv, n));
    FOT_TRY(download(h_lvl, lvl, n));
    FOT_TRY(download(h_lab, label, n));
    // width of each level from the fixed nodes
    std::vector<uint32_t> width(depth + 1, 0);
    std::vector<std::vector<uint32_t>> comps;
    std::vector<uint32_t> comp_id(n, INF);
    for (uint32_t x = 0; x < n; ++x) {
      if (h_lu[x] == INF) continue;  // another component of the graph
      if (h_lab[x] == INF) {
        width[h_lvl[x]]++;
      } else {
        if (comp_id[h_lab[x]] == INF) {
          comp_id[h_lab[x]] = (uint32_t)comps.size();
          comps.emplace_back();
        }
        comps[comp_id[h_lab[x]]].push_back(x);
      }
    }
    // larger components first; each goes to the structure (from u or from v)
    // whose resulting widest level is narrower (ties: from u)
    std::sort(comps.begin(), comps.end(), [](const auto &a, const auto &b) {
      return a.size() != b.size() ? a.size() > b.size() : a[0] < b[0];
    });
    for (const auto &cc : comps) {
      std::vector<uint32_t> wu = width, wv = width;
      for (uint32_t x : cc) {
        wu[h_lu[x]]++;
        wv[depth - std::min(h_lv[x], depth)]++;
      }
      uint32_t mu = 0, mv = 0;
      for (uint32_t l = 0; l <= depth; ++l) {
        if (wu[l] > width[l]) mu = std::max(mu, wu[l]);
        if (wv[l] > width[l]) mv = std::max(mv, wv[l]);
      }
      const bool use_u = mu <= mv;
      for (uint32_t x : cc) h_lvl[x] = use_u ? h_lu[x] : depth - std::min(h_lv[x], depth);
      width = use_u ? wu : wv;
    }
    for (uint32_t x = 0; x < n; ++x)
      if (h_lu[x] != INF) level_of[x] = level_base + h_lvl[x];
    level_base += depth + 1;
  }
  *n_levels = level_base;
  return FOT_OK;
}

namespace {
__global__ void k_level_expand(const uint32_t *row, const uint32_t *col, const uint32_t *frontier,
                               uint32_t nf, const uint32_t *pos, const uint32_t *level_of,
                               uint32_t next_level, uint32_t *parent) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const uint32_t u = frontier[i];
  for (uint32_t e = row[u]; e < row[u + 1]; ++e) {
    const uint32_t v = col[e];
    if (level_of[v] == next_level) atomicMin(&parent[v], pos[u]);
  }
}
} // namespace

// Number the nodes level by level; inside a level by (position of the
// earliest-numbered neighbour in the previous level, degree, id).
int number_by_levels(const Csr &g, const std::vector<uint32_t> &level_of, uint32_t n_levels,
                     std::vector<uint32_t> &order) {
  const uint32_t n = g.n;
  std::vector<std::vector<uint32_t>> members(n_levels);
  for (uint32_t x = 0; x < n; ++x) members[level_of[x]].push_back(x);
  DevBuf d_level, parent, pos, d_order, fa, fb, keys, keys2;
  FOT_TRY(upload(d_level, level_of));
  FOT_TRY(parent.alloc((size_t)n * 4));
  FOT_TRY(pos.alloc((size_t)n * 4));
  FOT_TRY(d_order.alloc((size_t)n * 4));
  FOT_TRY(fa.alloc((size_t)n * 4 + 4));
  FOT_TRY(fb.alloc((size_t)n * 4 + 4));
  FOT_TRY(keys.alloc((size_t)n * 8 + 8));
  FOT_TRY(keys2.alloc((size_t)n * 8 + 8));
  k_set_u32<<<blocks_for(n), 256>>>(parent.as<uint32_t>(), n, INF);
  uint32_t placed = 0, nf = 0;
  for (uint32_t l = 0; l < n_levels; ++l) {
    const uint32_t m = (uint32_t)members[l].size();
    if (m == 0) {
      nf = 0;
      continue;
    }
    if (l > 0 && nf > 0) {
      k_level_expand<<<blocks_for(nf), 256>>>(g.row.as<uint32_t>(), g.col.as<uint32_t>(),
                                              fa.as<uint32_t>(), nf, pos.as<uint32_t>(),
                                              d_level.as<uint32_t>(), l, parent.as<uint32_t>());
      FOT_CUDA(cudaGetLastError());
    }
    FOT_CUDA(cudaMemcpy(fb.ptr, members[l].data(), (size_t)m * 4, cudaMemcpyHostToDevice));
    k_sort_key<<<blocks_for(m), 256>>>(fb.as<uint32_t>(), m, parent.as<uint32_t>(),
                                       g.deg.as<uint32_t>(), keys.as<uint64_t>());
    FOT_TRY(sort_pairs(keys.as<uint64_t>(), keys2.as<uint64_t>(), fb.as<uint32_t>(),
                       fa.as<uint32_t>(), m, 0, 56));
    k_assign_pos<<<blocks_for(m), 256>>>(fa.as<uint32_t>(), m, placed, pos.as<uint32_t>(),
                                         d_order.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
    placed += m;
    nf = m;
  }
  return download(order, d_order, n);
}

namespace {

__global__ void k_first_touch(const uint32_t *map, size_t ne, uint32_t *first) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < ne) atomicMin(&first[map[e]], (uint32_t)e);
}

__global__ void k_cell_keys(const uint32_t *map, uint32_t n, int D, int slot, uint32_t *keys,
                            const uint32_t *order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = order[i];
  uint32_t t[8];
  for (int s = 0; s < D; ++s) t[s] = map[(size_t)c * D + s];
  // insertion sort of the tuple (D <= 8)
  for (int a = 1; a < D; ++a) {
    const uint32_t v = t[a];
    int b = a - 1;
    while (b >= 0 && t[b] > v) {
      t[b + 1] = t[b];
      --b;
    }
    t[b + 1] = v;
  }
  keys[i] = t[slot];
}

__global__ void k_random_keys(uint32_t n, uint64_t seed, uint64_t *keys, uint32_t *vals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = splitmix64(seed * 0x100000001b3ull + i);
  vals[i] = i;
}

} // namespace

// Cells sorted lexicographically by their sorted class-0 point tuples, ties
// by current index (Mesh::reorder, mesh.hpp:199-225): LSD passes of a stable
// radix sort, last tuple slot first.
int lexicographic_cell_order(fot_problem *p, std::vector<uint32_t> &order) {
  const uint32_t n = p->n_cells;
  const int D = (int)p->mesh_dim();
  std::vector<uint32_t> iota(n);
  std::iota(iota.begin(), iota.end(), 0u);
  DevBuf ord, ord2, keys, keys2;
  FOT_TRY(upload(ord, iota));
  FOT_TRY(ord2.alloc((size_t)n * 4));
  FOT_TRY(keys.alloc((size_t)n * 4));
  FOT_TRY(keys2.alloc((size_t)n * 4));
  for (int s = D - 1; s >= 0; --s) {
    k_cell_keys<<<blocks_for(n), 256>>>(p->map[0].as<uint32_t>(), n, D, s, keys.as<uint32_t>(),
                                        ord.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
    FOT_TRY(sort_pairs(keys.as<uint32_t>(), keys2.as<uint32_t>(), ord.as<uint32_t>(),
                       ord2.as<uint32_t>(), n));
    std::swap(ord, ord2);
  }
  return download(order, ord, n);
}

// First-touch numbering of class `cls` in the current cell order
// (Mesh::getPointRenumberingPermutation, mesh.hpp:247-270): unreferenced
// points follow in index order.
int first_touch_perm(fot_problem *p, int cls, std::vector<uint32_t> &perm) {
  const uint32_t np = p->class_points(cls);
  const int D = (int)p->info.mesh_dim[cls == 0 ? 0 : 1];
  const size_t ne = (size_t)p->n_cells * D;
  DevBuf first;
  FOT_TRY(first.alloc((size_t)np * 4));
  k_set_u32<<<blocks_for(np), 256>>>(first.as<uint32_t>(), np, INF);
  k_first_touch<<<blocks_for(ne), 256>>>(p->map[cls].as<uint32_t>(), ne, first.as<uint32_t>());
  FOT_CUDA(cudaGetLastError());
  std::vector<uint32_t> h_first;
  FOT_TRY(download(h_first, first, np));
  std::vector<uint32_t> idx(np);
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return h_first[a] < h_first[b]; });
  perm.resize(np);
  for (uint32_t r = 0; r < np; ++r) perm[idx[r]] = r;
  return FOT_OK;
}

// ---------------------------------------------------------------------------
// partitioning: deterministic region growing over the cell-to-cell graph
// ---------------------------------------------------------------------------
namespace {
__global__ void k_grow_candidates(const uint32_t *row, const uint32_t *col, uint32_t n,
                                  const uint32_t *part, const uint32_t *size, uint32_t cap,
                                  uint64_t *cand, uint32_t *n_cand) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || part[c] != INF) return;
  uint32_t best = INF;
  for (uint32_t e = row[c]; e < row[c + 1]; ++e) {
    const uint32_t q = part[col[e]];
    if (q != INF && size[q] < cap && q < best) best = q;
  }
  if (best != INF) cand[atomicAdd(n_cand, 1u)] = ((uint64_t)best << 32) | c;
}

__global__ void k_grow_accept(const uint64_t *cand, uint32_t m, const uint32_t *size, uint32_t cap,
                              uint32_t *part, uint32_t *size_out, uint32_t *accepted) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t q = (uint32_t)(cand[i] >> 32), c = (uint32_t)cand[i];
  // rank within the part's run (runs are contiguous after sorting)
  uint32_t first = i;
  while (first > 0 && (uint32_t)(cand[first - 1] >> 32) == q) --first;
  if (i - first < cap - size[q]) {
    part[c] = q;
    atomicAdd(&size_out[q], 1u);
    atomicAdd(accepted, 1u);
  }
}

__global__ void k_new_seeds(const uint32_t *row, const uint32_t *col, uint32_t n, const uint32_t *part,
                            uint32_t *seed_flag) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  uint32_t f = 0;
  if (part[c] == INF) {
    f = 1;
    for (uint32_t e = row[c]; e < row[c + 1]; ++e)
      if (part[col[e]] == INF && col[e] < c) {
        f = 0;
        break;
      }
  }
  seed_flag[c] = f;
}
} // namespace

int grow_partition(fot_problem *p, uint32_t part_size, std::vector<uint32_t> &part_out) {
  const uint32_t n = p->n_cells;
  Csr g;
  FOT_TRY(cell_graph(p, g));
  std::vector<uint32_t> h_part(n, INF);
  uint32_t n_parts = 0;
  for (uint32_t i = 0; i < n; i += part_size) h_part[i] = n_parts++;
  std::vector<uint32_t> h_size(n_parts, 1);
  DevBuf part, size, size2, cand, cand2, cnt, acc, flags;
  FOT_TRY(upload(part, h_part));
  FOT_TRY(cand.alloc((size_t)n * 8 + 8));
  FOT_TRY(cand2.alloc((size_t)n * 8 + 8));
  FOT_TRY(cnt.alloc(4));
  FOT_TRY(acc.alloc(4));
  FOT_TRY(flags.alloc((size_t)n * 4));
  uint32_t assigned = n_parts;
  for (int outer = 0; assigned < n; ++outer) {
    if (outer > 100000) return fail(FOT_ERR_LIMIT, "partitioning did not converge");
    FOT_TRY(upload(size, h_size));
    FOT_TRY(size2.alloc(h_size.size() * 4));
    FOT_CUDA(cudaMemcpy(size2.ptr, size.ptr, h_size.size() * 4, cudaMemcpyDeviceToDevice));
    // grow until no part can take a neighbour
    for (;;) {
      FOT_CUDA(cudaMemset(cnt.ptr, 0, 4));
      FOT_CUDA(cudaMemset(acc.ptr, 0, 4));
      k_grow_candidates<<<blocks_for(n), 256>>>(g.row.as<uint32_t>(), g.col.as<uint32_t>(), n,
                                                part.as<uint32_t>(), size.as<uint32_t>(), part_size,
                                                cand.as<uint64_t>(), cnt.as<uint32_t>());
      uint32_t m = 0;
      FOT_CUDA(cudaMemcpy(&m, cnt.ptr, 4, cudaMemcpyDeviceToHost));
      if (m == 0) break;
      FOT_TRY(sort_keys(cand.as<uint64_t>(), cand2.as<uint64_t>(), m));
      k_grow_accept<<<blocks_for(m), 256>>>(cand2.as<uint64_t>(), m, size.as<uint32_t>(), part_size,
                                            part.as<uint32_t>(), size2.as<uint32_t>(),
                                            acc.as<uint32_t>());
      FOT_CUDA(cudaGetLastError());
      FOT_CUDA(cudaMemcpy(size.ptr, size2.ptr, h_size.size() * 4, cudaMemcpyDeviceToDevice));
      uint32_t a = 0;
      FOT_CUDA(cudaMemcpy(&a, acc.ptr, 4, cudaMemcpyDeviceToHost));
      assigned += a;
      if (a == 0) break;
    }
    if (assigned >= n) break;
    // seed new parts at unassigned cells that are local minima among
    // unassigned neighbours
    FOT_TRY(download(h_size, size, h_size.size()));
    k_new_seeds<<<blocks_for(n), 256>>>(g.row.as<uint32_t>(), g.col.as<uint32_t>(), n,
                                        part.as<uint32_t>(), flags.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
    std::vector<uint32_t> h_flags;
    FOT_TRY(download(h_flags, flags, n));
    FOT_TRY(download(h_part, part, n));
    for (uint32_t c = 0; c < n; ++c)
      if (h_flags[c]) {
        h_part[c] = n_parts++;
        h_size.push_back(1);
        ++assigned;
      }
    FOT_TRY(upload(part, h_part));
  }
  return download(part_out, part, n);
}

// ---------------------------------------------------------------------------
// partitioning: recursive graph bisection over the cell-to-cell graph
// ---------------------------------------------------------------------------
// Every round, each segment that still holds k > 1 parts is cut in two: a
// BFS restricted to the segment from its first cell finds a far cell (the
// largest level, then the smallest id), a second restricted BFS from there
// levels the segment along its longest extent, a stable sort by (segment,
// level) orders its cells, and the first round(size * floor(k/2) / k) cells
// form the part range [first, first + k/2), the rest [first + k/2, first +
// k).  Parts end up within one cell of n / nparts, compact (each cut follows
// a BFS front), and numbered so that neighbouring parts have nearby numbers.
namespace {
__global__ void k_seg_bfs_expand(const uint32_t *row, const uint32_t *col, const uint32_t *frontier,
                                 uint32_t nf, const uint32_t *seg, uint32_t next_level, uint32_t *lvl,
                                 uint32_t *next, uint32_t *n_next) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const uint32_t u = frontier[i], su = seg[u];
  for (uint32_t e = row[u]; e < row[u + 1]; ++e) {
    const uint32_t v = col[e];
    if (seg[v] == su && lvl[v] == INF && atomicCAS(&lvl[v], INF, next_level) == INF)
      next[atomicAdd(n_next, 1u)] = v;
  }
}

__global__ void k_gather_seeds(const uint32_t *perm, const uint32_t *pos, uint32_t m, uint32_t *seeds,
                               uint32_t *lvl) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint32_t c = pos ? perm[pos[j]] : perm[j];
  seeds[j] = c;
  lvl[c] = 0;
}

__global__ void k_seg_far(const uint32_t *lvl, const uint32_t *seg, uint32_t n, unsigned long long *best) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || lvl[c] == INF) return;
  atomicMax(&best[seg[c]], ((unsigned long long)lvl[c] << 32) | (INF - c));
}

__global__ void k_seg_keys(const uint32_t *perm, uint32_t n, const uint32_t *seg, const uint32_t *lvl,
                           uint64_t *keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i];
  keys[i] = ((uint64_t)seg[c] << 32) | lvl[c];
}

__global__ void k_seg_split(const uint32_t *perm, uint32_t n, uint32_t *seg, const uint32_t *start_of,
                            const uint32_t *nleft_of, const uint32_t *k_of) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i], s = seg[c], k = k_of[s];
  if (k > 1 && i - start_of[s] >= nleft_of[s]) seg[c] = s + k / 2;
}

// multi-source BFS restricted to segments; lvl[seeds] must be 0, the rest INF
int seg_bfs(const Csr &g, const DevBuf &seg, DevBuf &lvl, DevBuf &fa, DevBuf &fb, DevBuf &cnt,
            uint32_t n_seeds) {
  uint32_t nf = n_seeds, level = 0;
  while (nf) {
    FOT_CUDA(cudaMemsetAsync(cnt.ptr, 0, 4));
    k_seg_bfs_expand<<<blocks_for(nf), 256>>>(g.row.as<uint32_t>(), g.col.as<uint32_t>(),
                                              fa.as<uint32_t>(), nf, seg.as<uint32_t>(), level + 1,
                                              lvl.as<uint32_t>(), fb.as<uint32_t>(), cnt.as<uint32_t>());
    FOT_CUDA(cudaMemcpy(&nf, cnt.ptr, 4, cudaMemcpyDeviceToHost));
    std::swap(fa, fb);
    ++level;
  }
  return FOT_OK;
}
} // namespace

int bisect_partition(fot_problem *p, uint32_t part_size, std::vector<uint32_t> &part_out) {
  const uint32_t n = p->n_cells;
  const uint32_t nparts = (n + part_size - 1) / part_size;
  Csr g;
  FOT_TRY(cell_graph(p, g));
  struct Seg {
    uint32_t first, k, start, size;
  };
  std::vector<Seg> segs{{0, nparts, 0, n}};
  std::vector<uint32_t> iota(n);
  std::iota(iota.begin(), iota.end(), 0u);
  DevBuf seg, perm, perm2, keys, keys2, lvl, fa, fb, cnt, best, d_start, d_nleft, d_k, d_pos;
  FOT_TRY(seg.alloc((size_t)n * 4));
  FOT_CUDA(cudaMemset(seg.ptr, 0, (size_t)n * 4));
  FOT_TRY(upload(perm, iota));
  FOT_TRY(perm2.alloc((size_t)n * 4));
  FOT_TRY(keys.alloc((size_t)n * 8));
  FOT_TRY(keys2.alloc((size_t)n * 8));
  FOT_TRY(lvl.alloc((size_t)n * 4));
  FOT_TRY(fa.alloc((size_t)n * 4));
  FOT_TRY(fb.alloc((size_t)n * 4));
  FOT_TRY(cnt.alloc(4));
  FOT_TRY(best.alloc((size_t)nparts * 8));
  for (int round = 0;; ++round) {
    std::vector<uint32_t> act;  // indices into segs of segments still to cut
    for (uint32_t i = 0; i < segs.size(); ++i)
      if (segs[i].k > 1) act.push_back(i);
    if (act.empty()) break;
    if (round > 64) return fail(FOT_ERR_LIMIT, "partitioning did not converge");
    const uint32_t m = (uint32_t)act.size();
    std::vector<uint32_t> pos(m);
    for (uint32_t j = 0; j < m; ++j) pos[j] = segs[act[j]].start;
    FOT_TRY(upload(d_pos, pos));
    // pass 1: from each segment's first cell, find a far cell
    k_set_u32<<<blocks_for(n), 256>>>(lvl.as<uint32_t>(), n, INF);
    k_gather_seeds<<<blocks_for(m), 256>>>(perm.as<uint32_t>(), d_pos.as<uint32_t>(), m,
                                           fa.as<uint32_t>(), lvl.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
    FOT_TRY(seg_bfs(g, seg, lvl, fa, fb, cnt, m));
    FOT_CUDA(cudaMemset(best.ptr, 0, (size_t)nparts * 8));
    k_seg_far<<<blocks_for(n), 256>>>(lvl.as<uint32_t>(), seg.as<uint32_t>(), n,
                                      best.as<unsigned long long>());
    FOT_CUDA(cudaGetLastError());
    std::vector<unsigned long long> h_best;
    FOT_TRY(download(h_best, best.as<unsigned long long>(), nparts));
    std::vector<uint32_t> far(m);
    for (uint32_t j = 0; j < m; ++j) far[j] = INF - (uint32_t)(h_best[segs[act[j]].first] & 0xFFFFFFFFull);
    // pass 2: level each segment from its far cell
    DevBuf d_far;
    FOT_TRY(upload(d_far, far));
    k_set_u32<<<blocks_for(n), 256>>>(lvl.as<uint32_t>(), n, INF);
    k_gather_seeds<<<blocks_for(m), 256>>>(d_far.as<uint32_t>(), nullptr, m, fa.as<uint32_t>(),
                                           lvl.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
    FOT_TRY(seg_bfs(g, seg, lvl, fa, fb, cnt, m));
    // order every segment by level (stable: ties keep the previous order)
    k_seg_keys<<<blocks_for(n), 256>>>(perm.as<uint32_t>(), n, seg.as<uint32_t>(), lvl.as<uint32_t>(),
                                       keys.as<uint64_t>());
    FOT_CUDA(cudaGetLastError());
    FOT_TRY(sort_pairs(keys.as<uint64_t>(), keys2.as<uint64_t>(), perm.as<uint32_t>(),
                       perm2.as<uint32_t>(), n));
    std::swap(perm, perm2);
    // cut
    std::vector<uint32_t> start_of(nparts, 0), nleft_of(nparts, 0), k_of(nparts, 1);
    std::vector<Seg> next;
    for (const Seg &sg : segs) {
      start_of[sg.first] = sg.start;
      k_of[sg.first] = sg.k;
      nleft_of[sg.first] = sg.size;
      if (sg.k == 1) {
        next.push_back(sg);
        continue;
      }
      const uint32_t kl = sg.k / 2;
      const uint32_t nl = (uint32_t)(((uint64_t)2 * sg.size * kl + sg.k) / (2 * (uint64_t)sg.k));
      nleft_of[sg.first] = nl;
      next.push_back({sg.first, kl, sg.start, nl});
      next.push_back({sg.first + kl, sg.k - kl, sg.start + nl, sg.size - nl});
    }
    FOT_TRY(upload(d_start, start_of));
    FOT_TRY(upload(d_nleft, nleft_of));
    FOT_TRY(upload(d_k, k_of));
    k_seg_split<<<blocks_for(n), 256>>>(perm.as<uint32_t>(), n, seg.as<uint32_t>(), d_start.as<uint32_t>(),
                                        d_nleft.as<uint32_t>(), d_k.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
    segs.swap(next);
  }
  return download(part_out, seg, n);
}

} // namespace fot

using namespace fot;

extern "C" {

int fot_reorder(fot_problem *p, int order, uint64_t seed) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  const uint32_t np = p->n_points[0];
  std::vector<uint32_t> perm(np);
  if (order == FOT_ORDER_NATURAL) {
    std::iota(perm.begin(), perm.end(), 0u);
  } else if (order == FOT_ORDER_RANDOM) {
    DevBuf k0, k1, v0, v1;
    FOT_TRY(k0.alloc((size_t)np * 8));
    FOT_TRY(k1.alloc((size_t)np * 8));
    FOT_TRY(v0.alloc((size_t)np * 4));
    FOT_TRY(v1.alloc((size_t)np * 4));
    k_random_keys<<<blocks_for(np), 256>>>(np, seed, k0.as<uint64_t>(), v0.as<uint32_t>());
    FOT_CUDA(cudaGetLastError());
    FOT_TRY(sort_pairs(k0.as<uint64_t>(), k1.as<uint64_t>(), v0.as<uint32_t>(), v1.as<uint32_t>(), np));
    std::vector<uint32_t> inv;
    FOT_TRY(download(inv, v1, np));
    for (uint32_t r = 0; r < np; ++r) perm[inv[r]] = r;
  } else if (order == FOT_ORDER_RCM || order == FOT_ORDER_GPS) {
    Csr g;
    FOT_TRY(point_graph(p, 0, g));
    std::vector<uint32_t> ord;
    if (order == FOT_ORDER_RCM) {
      FOT_TRY(cuthill_mckee(g, ord));
      for (uint32_t i = 0; i < np; ++i) perm[ord[i]] = np - 1 - i;
    } else {
      std::vector<uint32_t> level_of;
      uint32_t n_levels = 0;
      FOT_TRY(gps_levels(g, level_of, &n_levels));
      FOT_TRY(number_by_levels(g, level_of, n_levels, ord));
      for (uint32_t i = 0; i < np; ++i) perm[ord[i]] = i;
    }
  } else {
    return fail(FOT_ERR_ARG, "unknown ordering %d", order);
  }
  FOT_TRY(apply_point_perm(p, 0, perm));
  std::vector<uint32_t> cell_ord;
  FOT_TRY(lexicographic_cell_order(p, cell_ord));
  FOT_TRY(apply_cell_order(p, cell_ord));
  if (p->has_class1) {
    std::vector<uint32_t> perm1;
    FOT_TRY(first_touch_perm(p, 1, perm1));
    FOT_TRY(apply_point_perm(p, 1, perm1));
  }
  FOT_CUDA(cudaDeviceSynchronize());
  return FOT_OK;
}

int fot_partition_tol(fot_problem *p, uint32_t part_size, float tolerance, int method) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  if (part_size == 0) return fail(FOT_ERR_ARG, "part size must be positive");
  if (!(tolerance >= 1.0f)) return fail(FOT_ERR_ARG, "tolerance must be at least 1 (got %g)", tolerance);
  std::vector<uint32_t> part;
  if (method == FOT_PARTITION_BISECT) {
    FOT_TRY(bisect_partition(p, part_size, part));
  } else if (method == FOT_PARTITION_GROW) {
    FOT_TRY(grow_partition(p, part_size, part));
  } else {
    return fail(FOT_ERR_ARG, "unknown partitioning method %d", method);
  }
  if (method == FOT_PARTITION_BISECT) {
    // the load-balance bound of the reference's METIS call (ubvec =
    // tolerance, partition.cu:18-29): parts of at most tolerance x the mean,
    // up to the one cell that integral sizes need
    std::vector<uint32_t> size;
    for (uint32_t q : part) {
      if (q >= size.size()) size.resize(q + 1, 0);
      ++size[q];
    }
    const double mean = (double)p->n_cells / size.size();
    for (uint32_t sz : size)
      if (sz > tolerance * mean + 1.0)
        return fail(FOT_ERR_STATE, "part of %u cells exceeds the tolerance bound %.1f", sz, tolerance * mean);
  }
  p->partition.swap(part);
  FOT_CUDA(cudaDeviceSynchronize());
  return FOT_OK;
}

int fot_partition(fot_problem *p, uint32_t part_size, uint64_t seed) {
  (void)seed;  // both methods are deterministic
  return fot_partition_tol(p, part_size, 1.001f, FOT_PARTITION_BISECT);
}

int fot_reorder_to_partition(fot_problem *p) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  if (p->partition.size() != p->n_cells) return fail(FOT_ERR_STATE, "problem has no partition");
  std::vector<uint32_t> order(p->n_cells);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return p->partition[a] < p->partition[b]; });
  FOT_TRY(apply_cell_order(p, order));
  FOT_CUDA(cudaDeviceSynchronize());
  return FOT_OK;
}

int fot_renumber_points(fot_problem *p) {
  if (!p) return fail(FOT_ERR_ARG, "null problem");
  if (p->partition.size() != p->n_cells) return fail(FOT_ERR_STATE, "problem has no partition");
  for (int cls = 0; cls < (p->has_class1 ? 2 : 1); ++cls) {
    const uint32_t np = p->class_points(cls);
    const int D = (int)p->info.mesh_dim[cls == 0 ? 0 : 1];
    std::vector<uint32_t> map;
    FOT_TRY(download(map, p->map[cls].as<uint32_t>(), (size_t)p->n_cells * D));
    // the sorted set of parts touching each point (getPointToPartition)
    std::vector<std::vector<uint32_t>> parts(np);
    for (uint32_t c = 0; c < p->n_cells; ++c)
      for (int s = 0; s < D; ++s) {
        auto &v = parts[map[(size_t)c * D + s]];
        const uint32_t q = p->partition[c];
        if (std::find(v.begin(), v.end(), q) == v.end()) v.push_back(q);
      }
    for (auto &v : parts) std::sort(v.begin(), v.end());
    // points touched by more parts first, then by part set descending,
    // points touched by none last (getPointRenumberingPermutation2)
    std::vector<uint32_t> idx(np);
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
      if (parts[a].size() != parts[b].size()) return parts[a].size() > parts[b].size();
      if (parts[a].empty() || parts[b].empty()) return false;  // both untouched: keep order
      return parts[a] > parts[b];
    });
    std::vector<uint32_t> perm(np);
    for (uint32_t r = 0; r < np; ++r) perm[idx[r]] = r;
    FOT_TRY(apply_point_perm(p, cls, perm));
  }
  FOT_CUDA(cudaDeviceSynchronize());
  return FOT_OK;
}

} // extern "C"
