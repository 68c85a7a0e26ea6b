// The Airfoil time step around the res_calc loop.
//
// The reference drives res_calc alone (res_calc.cu, Problem::loop*(num)).
// An Airfoil solver step also needs the loops on each side of it, which the
// reference does not contain; they restate the Airfoil finite-volume scheme
// (explicit two-stage update with local time steps, Roe-type edge fluxes
// with scalar dissipation) on the res_calc problem's own data:
//
//   per iteration:  save_soln  qold = q
//                   2 x { adt_calc   per cell: adt = sum over its 4 sides of
//                                    (|u dy - v dx| + c |side|), over cfl
//                         res_calc   per edge (the engine's plan: atomic or
//                                    coloured)
//                         bres_calc  per boundary edge: wall pressure, or the
//                                    res_calc flux against the free stream
//                         update     per cell: q = qold - res / adt, res = 0,
//                                    rms += |q change|^2 }
//                   rms = sqrt(rms / cells) of the second stage
//
// Data: the res_calc problem's point sets res (0), x (1, nodes), q (2),
// adt (3) in its current numbering and layout, plus the airfoil's own qold,
// cell -> 4 nodes, boundary edge -> 2 nodes / 1 cell / bound flag (given in
// the original numbering and renumbered here whenever the problem's
// numbering changes).  The per-cell loops run fused, each cell's values
// unchanged: update + the next stage's adt_calc in one pass (and between
// iterations + save_soln), so an iteration is two res_calc runs, two
// bres_calc launches, two cell passes and the rms reduction.
// Every kernel is compiled without multiply-add
// contraction, and every sum has a fixed order: boundary edges are added per
// cell in increasing edge order (one thread per boundary cell), the rms is a
// fixed-shape tree.  With a coloured res_calc plan a step is therefore
// bit-identical to its CPU restatement replaying the same plan.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.hpp"

namespace fot {
namespace {

constexpr double kGam = 1.4, kGm1 = 0.4, kEps = 0.05; // gm1 and eps as res_calc_func.hpp
constexpr uint32_t kThreads = 256;
#ifndef FOT_AIRFOIL_MAX_CTAS
#define FOT_AIRFOIL_MAX_CTAS 1184
#endif
// CTAs of a cell pass (grid-stride beyond); the rms sums one partial per CTA
constexpr uint32_t kMaxUpdateCtas = FOT_AIRFOIL_MAX_CTAS;

struct AirfoilDev {
  const double *x;
  double *q, *qold, *adt, *res;
  uint32_t n_nodes, n_cells;
  int soa;
  const uint4 *cell_nodes;      // per cell: its 4 nodes, counter-clockwise
  const uint32_t *bcell;        // boundary cells
  const uint32_t *bcell_off;    // their boundary edges [off[i], off[i+1]) in bedge order
  const uint2 *bedge_nodes;     // per boundary edge (grouped by cell): node 1, node 2
  const int *bedge_bound;       // 1: solid wall, else far field
  uint32_t n_bcells;
  double qinf[4];
  double cfl;
};

__device__ __forceinline__ size_t at(int soa, uint32_t n, uint32_t i, int dim, int k) {
  return soa ? (size_t)k * n + i : (size_t)i * dim + k;
}

// adt_calc of cell c from its state q.
__device__ __forceinline__ double cell_adt(const AirfoilDev &a, uint32_t c, const double (&q)[4]) {
  const uint4 nd = a.cell_nodes[c];
  const uint32_t node[4] = {nd.x, nd.y, nd.z, nd.w};
  double px[4], py[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    px[j] = a.x[at(a.soa, a.n_nodes, node[j], 2, 0)];
    py[j] = a.x[at(a.soa, a.n_nodes, node[j], 2, 1)];
  }
  const double ri = 1.0 / q[0];
  const double u = ri * q[1], v = ri * q[2];
  const double snd = sqrt(kGam * kGm1 * (ri * q[3] - 0.5 * (u * u + v * v)));
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double dx = px[(j + 1) & 3] - px[j];
    const double dy = py[(j + 1) & 3] - py[j];
    s += fabs(u * dy - v * dx) + snd * sqrt(dx * dx + dy * dy);
  }
  return s / a.cfl;
}

// One thread per boundary cell: its boundary edges in increasing edge order.
__global__ void __launch_bounds__(kThreads) k_bres_calc(AirfoilDev a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_bcells) return;
  const uint32_t c = a.bcell[i];
  double q[4], r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    q[k] = a.q[at(a.soa, a.n_cells, c, 4, k)];
    r[k] = a.res[at(a.soa, a.n_cells, c, 4, k)];
  }
  const double adt1 = a.adt[c];
  for (uint32_t e = a.bcell_off[i]; e < a.bcell_off[i + 1]; ++e) {
    const uint2 nd = a.bedge_nodes[e];
    const double dx = a.x[at(a.soa, a.n_nodes, nd.x, 2, 0)] - a.x[at(a.soa, a.n_nodes, nd.y, 2, 0)];
    const double dy = a.x[at(a.soa, a.n_nodes, nd.x, 2, 1)] - a.x[at(a.soa, a.n_nodes, nd.y, 2, 1)];
    const double ri = 1.0 / q[0];
    const double p1 = kGm1 * (q[3] - 0.5 * ri * (q[1] * q[1] + q[2] * q[2]));
    if (a.bedge_bound[e] == 1) {
      r[1] += p1 * dy;
      r[2] += -p1 * dx;
    } else {
      const double vol1 = ri * (q[1] * dy - q[2] * dx);
      const double *qi = a.qinf;
      const double ri2 = 1.0 / qi[0];
      const double p2 = kGm1 * (qi[3] - 0.5 * ri2 * (qi[1] * qi[1] + qi[2] * qi[2]));
      const double vol2 = ri2 * (qi[1] * dy - qi[2] * dx);
      const double mu = adt1 * kEps;
      r[0] += 0.5 * (vol1 * q[0] + vol2 * qi[0]) + mu * (q[0] - qi[0]);
      r[1] += 0.5 * (vol1 * q[1] + p1 * dy + vol2 * qi[1] + p2 * dy) + mu * (q[1] - qi[1]);
      r[2] += 0.5 * (vol1 * q[2] - p1 * dx + vol2 * qi[2] - p2 * dx) + mu * (q[2] - qi[2]);
      r[3] += 0.5 * (vol1 * (q[3] + p1) + vol2 * (qi[3] + p2)) + mu * (q[3] - qi[3]);
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) a.res[at(a.soa, a.n_cells, c, 4, k)] = r[k];
}

// Sum of the block's values in a fixed order (warp trees, then the warps'
// sums in warp order); the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) s += smem[w];
  return s;
}

// The per-cell loops of the iteration, fused (each cell's values are the
// same as loop by loop): UPDATE (q = qold - res / adt, res = 0, squared
// updates summed per CTA in a fixed order into partial[]), then SAVE
// (qold = q: save_soln of the next iteration) and ADT (adt_calc on the new q).
template <bool UPDATE, bool SAVE, bool ADT>
__global__ void __launch_bounds__(kThreads) k_cells(AirfoilDev a, double *partial) {
  __shared__ double smem[kThreads / 32];
  double sum = 0.0;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < a.n_cells; c += stride) {
    double q[4];
    if constexpr (UPDATE) {
      const double adti = 1.0 / a.adt[c];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const size_t o = at(a.soa, a.n_cells, c, 4, k);
        const double del = adti * a.res[o];
        q[k] = a.qold[o] - del;
        a.q[o] = q[k];
        a.res[o] = 0.0;
        sum += del * del;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) q[k] = a.q[at(a.soa, a.n_cells, c, 4, k)];
    }
    if constexpr (SAVE) {
#pragma unroll
      for (int k = 0; k < 4; ++k) a.qold[at(a.soa, a.n_cells, c, 4, k)] = q[k];
    }
    if constexpr (ADT) a.adt[c] = cell_adt(a, c, q);
  }
  if constexpr (UPDATE) {
    const double s = block_sum(sum, smem);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(kThreads) k_rms(const double *partial, uint32_t n_partial,
                                                 uint32_t n_cells, double *rms) {
  __shared__ double smem[kThreads / 32];
  double v = 0.0;
  for (uint32_t i = threadIdx.x; i < n_partial; i += blockDim.x) v += partial[i];
  const double s = block_sum(v, smem);
  if (threadIdx.x == 0) *rms = sqrt(s / (double)n_cells);
}

uint32_t update_ctas(uint32_t n_cells) {
  return std::max<uint32_t>(1, std::min<uint32_t>((n_cells + kThreads - 1) / kThreads, kMaxUpdateCtas));
}

} // namespace
} // namespace fot

using namespace fot;

struct fot_airfoil {
  fot_problem *prob = nullptr;
  uint64_t version = 0; // problem numbering the device maps were built for
  uint32_t n_cells = 0, n_nodes = 0, n_bedges = 0;
  // original numbering (host)
  std::vector<uint32_t> cell_nodes, bedge_nodes, bedge_cell;
  std::vector<int32_t> bound;
  double qinf[4] = {0, 0, 0, 0};
  double cfl = 0.0;
  // device, current numbering
  DevBuf d_cell_nodes, d_bcell, d_bcell_off, d_bedge_nodes, d_bedge_bound;
  uint32_t n_bcells = 0;
  DevBuf qold, partial, rms;
};

namespace {

int upload(DevBuf &b, const void *host, size_t bytes) {
  FOT_TRY(b.alloc(bytes));
  if (bytes) FOT_CUDA(cudaMemcpy(b.ptr, host, bytes, cudaMemcpyHostToDevice));
  return FOT_OK;
}

// Rebuild the device maps for the problem's current numbering.
int airfoil_renumber(fot_airfoil *a) {
  fot_problem *p = a->prob;
  const std::vector<uint32_t> &cperm = p->point_perm[0], &nperm = p->point_perm[1];
  if (cperm.size() != a->n_cells || nperm.size() != a->n_nodes)
    return fail(FOT_ERR_STATE, "res_calc problem has no point permutation of the expected size");
  // cell -> nodes, rows moved to the cells' current numbers
  std::vector<uint32_t> cn((size_t)a->n_cells * 4);
  for (uint32_t c = 0; c < a->n_cells; ++c)
    for (int j = 0; j < 4; ++j) cn[(size_t)cperm[c] * 4 + j] = nperm[a->cell_nodes[(size_t)c * 4 + j]];
  // boundary edges grouped by (current) cell, increasing edge order inside a cell
  std::vector<uint32_t> idx(a->n_bedges);
  for (uint32_t e = 0; e < a->n_bedges; ++e) idx[e] = e;
  std::stable_sort(idx.begin(), idx.end(),
                   [&](uint32_t x, uint32_t y) { return cperm[a->bedge_cell[x]] < cperm[a->bedge_cell[y]]; });
  std::vector<uint32_t> bcell, boff, bnodes((size_t)a->n_bedges * 2);
  std::vector<int32_t> bb(a->n_bedges);
  for (uint32_t i = 0; i < a->n_bedges; ++i) {
    const uint32_t e = idx[i], c = cperm[a->bedge_cell[e]];
    if (bcell.empty() || bcell.back() != c) {
      bcell.push_back(c);
      boff.push_back(i);
    }
    bnodes[2 * (size_t)i] = nperm[a->bedge_nodes[2 * (size_t)e]];
    bnodes[2 * (size_t)i + 1] = nperm[a->bedge_nodes[2 * (size_t)e + 1]];
    bb[i] = a->bound[e];
  }
  boff.push_back(a->n_bedges);
  a->n_bcells = (uint32_t)bcell.size();
  FOT_TRY(upload(a->d_cell_nodes, cn.data(), cn.size() * sizeof(uint32_t)));
  FOT_TRY(upload(a->d_bcell, bcell.data(), bcell.size() * sizeof(uint32_t)));
  FOT_TRY(upload(a->d_bcell_off, boff.data(), boff.size() * sizeof(uint32_t)));
  FOT_TRY(upload(a->d_bedge_nodes, bnodes.data(), bnodes.size() * sizeof(uint32_t)));
  FOT_TRY(upload(a->d_bedge_bound, bb.data(), bb.size() * sizeof(int32_t)));
  a->version = p->version;
  return FOT_OK;
}

} // namespace

void fot_airfoil_detach(fot_airfoil *a) {
  if (a) a->prob = nullptr;
}

extern "C" {

int fot_airfoil_create(fot_problem *p, const fot_airfoil_desc *desc, fot_airfoil **out) {
  if (!p || !desc || !out) return fail(FOT_ERR_ARG, "null argument");
  *out = nullptr;
  if (p->loop != FOT_LOOP_RES_CALC) return fail(FOT_ERR_ARG, "the Airfoil step runs on a res_calc problem");
  if (!desc->cell_to_node || (desc->n_bedges && (!desc->bedge_to_node || !desc->bedge_to_cell || !desc->bound)))
    return fail(FOT_ERR_ARG, "null mapping");
  if (!(desc->cfl > 0.0) || !(desc->qinf[0] > 0.0)) return fail(FOT_ERR_ARG, "cfl and qinf[0] must be positive");
  const uint32_t n_cells = p->n_points[0], n_nodes = p->n_points[1];
  for (size_t i = 0; i < (size_t)n_cells * 4; ++i)
    if (desc->cell_to_node[i] >= n_nodes) return fail(FOT_ERR_ARG, "cell_to_node[%zu] = %u out of range", i, desc->cell_to_node[i]);
  for (uint32_t e = 0; e < desc->n_bedges; ++e) {
    if (desc->bedge_to_cell[e] >= n_cells) return fail(FOT_ERR_ARG, "bedge_to_cell[%u] out of range", e);
    if (desc->bedge_to_node[2 * (size_t)e] >= n_nodes || desc->bedge_to_node[2 * (size_t)e + 1] >= n_nodes)
      return fail(FOT_ERR_ARG, "bedge_to_node[%u] out of range", e);
  }
  auto *a = new fot_airfoil;
  a->prob = p;
  a->n_cells = n_cells;
  a->n_nodes = n_nodes;
  a->n_bedges = desc->n_bedges;
  a->cell_nodes.assign(desc->cell_to_node, desc->cell_to_node + (size_t)n_cells * 4);
  a->bedge_nodes.assign(desc->bedge_to_node, desc->bedge_to_node + (size_t)desc->n_bedges * 2);
  a->bedge_cell.assign(desc->bedge_to_cell, desc->bedge_to_cell + desc->n_bedges);
  a->bound.assign(desc->bound, desc->bound + desc->n_bedges);
  std::memcpy(a->qinf, desc->qinf, sizeof(a->qinf));
  a->cfl = desc->cfl;
  int rc = airfoil_renumber(a);
  if (rc == FOT_OK) rc = a->qold.alloc((size_t)n_cells * 4 * sizeof(double));
  if (rc == FOT_OK) rc = a->partial.alloc(update_ctas(n_cells) * sizeof(double));
  if (rc == FOT_OK) rc = a->rms.alloc(sizeof(double));
  if (rc == FOT_OK && cudaMemset(a->rms.ptr, 0, sizeof(double)) != cudaSuccess)
    rc = fail(FOT_ERR_CUDA, "cudaMemset failed");
  if (rc != FOT_OK) {
    delete a;
    return rc;
  }
  p->airfoils.push_back(a);
  *out = a;
  return FOT_OK;
}

int fot_airfoil_destroy(fot_airfoil *a) {
  if (!a) return FOT_OK;
  if (a->prob) {
    auto &v = a->prob->airfoils;
    v.erase(std::remove(v.begin(), v.end(), a), v.end());
  }
  delete a;
  return FOT_OK;
}

} // extern "C"

namespace {

// Launch `iterations` solver iterations on st (no synchronisation).
int airfoil_enqueue(fot_airfoil *a, fot_plan *plan, uint32_t iterations, cudaStream_t st) {
  fot_problem *p = a->prob;
  AirfoilDev d{};
  d.x = static_cast<const double *>(p->point[1].ptr);
  d.q = static_cast<double *>(p->point[2].ptr);
  d.adt = static_cast<double *>(p->point[3].ptr);
  d.res = static_cast<double *>(p->point[0].ptr);
  d.qold = static_cast<double *>(a->qold.ptr);
  d.n_nodes = a->n_nodes;
  d.n_cells = a->n_cells;
  d.soa = p->layout == FOT_SOA;
  d.cell_nodes = a->d_cell_nodes.as<uint4>();
  d.bcell = a->d_bcell.as<uint32_t>();
  d.bcell_off = a->d_bcell_off.as<uint32_t>();
  d.bedge_nodes = a->d_bedge_nodes.as<uint2>();
  d.bedge_bound = a->d_bedge_bound.as<int>();
  d.n_bcells = a->n_bcells;
  std::memcpy(d.qinf, a->qinf, sizeof(d.qinf));
  d.cfl = a->cfl;
  const uint32_t ctas = update_ctas(a->n_cells);
  const uint32_t bctas = (a->n_bcells + kThreads - 1) / kThreads;
  double *part = a->partial.as<double>();
  // save_soln + adt_calc of the first stage; afterwards each update carries
  // the next stage's adt_calc (and, between iterations, save_soln)
  k_cells<false, true, true><<<ctas, kThreads, 0, st>>>(d, part);
  FOT_CUDA(cudaGetLastError());
  for (uint32_t it = 0; it < iterations; ++it) {
    for (int stage = 0; stage < 2; ++stage) {
      FOT_TRY(fot_run(p, plan, 1, st));
      if (bctas) {
        k_bres_calc<<<bctas, kThreads, 0, st>>>(d);
        FOT_CUDA(cudaGetLastError());
      }
      if (stage == 0)
        k_cells<true, false, true><<<ctas, kThreads, 0, st>>>(d, part);
      else if (it + 1 < iterations)
        k_cells<true, true, true><<<ctas, kThreads, 0, st>>>(d, part);
      else
        k_cells<true, false, false><<<ctas, kThreads, 0, st>>>(d, part);
      FOT_CUDA(cudaGetLastError());
    }
    k_rms<<<1, kThreads, 0, st>>>(part, ctas, a->n_cells, a->rms.as<double>());
    FOT_CUDA(cudaGetLastError());
  }
  return FOT_OK;
}

int airfoil_ready(fot_airfoil *a, fot_plan *plan) {
  if (!a || !plan) return fail(FOT_ERR_ARG, "null argument");
  if (!a->prob) return fail(FOT_ERR_STATE, "the airfoil's problem was destroyed");
  if (plan->prob != a->prob) return fail(FOT_ERR_STATE, "plan belongs to another (or a destroyed) problem");
  if (a->version != a->prob->version) FOT_TRY(airfoil_renumber(a));
  return FOT_OK;
}

} // namespace

extern "C" {

int fot_airfoil_run(fot_airfoil *a, fot_plan *plan, uint32_t iterations, double *rms, void *stream) {
  FOT_TRY(airfoil_ready(a, plan));
  if (iterations == 0) return FOT_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  FOT_TRY(airfoil_enqueue(a, plan, iterations, st));
  if (rms) {
    FOT_CUDA(cudaMemcpyAsync(rms, a->rms.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
    FOT_CUDA(cudaStreamSynchronize(st));
  }
  return FOT_OK;
}

int fot_airfoil_graph_create(fot_airfoil *a, fot_plan *plan, uint32_t iterations, void *stream,
                             fot_graph **out) {
  if (!out) return fail(FOT_ERR_ARG, "null argument");
  *out = nullptr;
  FOT_TRY(airfoil_ready(a, plan));
  if (iterations == 0) return fail(FOT_ERR_ARG, "a graph of zero iterations");
  struct Ctx {
    fot_airfoil *a;
    fot_plan *plan;
    uint32_t iterations;
  } ctx{a, plan, iterations};
  auto enqueue = [](void *c, cudaStream_t st) {
    const Ctx *x = static_cast<const Ctx *>(c);
    return airfoil_enqueue(x->a, x->plan, x->iterations, st);
  };
  FOT_TRY(capture_graph(static_cast<cudaStream_t>(stream), enqueue, &ctx, out));
  (*out)->prob = a->prob;
  (*out)->plan = plan;
  (*out)->ctl = plan->ctl.as<Ctl>();
  (*out)->version = a->prob->version;
  return FOT_OK;
}

int fot_airfoil_get_rms(fot_airfoil *a, double *rms, void *stream) {
  if (!a || !rms) return fail(FOT_ERR_ARG, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  FOT_CUDA(cudaMemcpyAsync(rms, a->rms.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
  FOT_CUDA(cudaStreamSynchronize(st));
  return FOT_OK;
}

} // extern "C"
