/*
 * ref_wrapper.cu -- extern "C" entry points over the reference's own CPU loop
 * drivers, compiled from the reference sources where they lie (see
 * oracle/Makefile, target `ref`).  TEST INFRASTRUCTURE ONLY: the compiled
 * library (oracle/_ref/libref.so) pins the oracle (tests/golden) and is the
 * timed CPU baseline of bench.py's reference arm.
 *
 * Nothing of the reference is copied here: this file includes the reference's
 * headers and calls
 *   Problem<SOA>::loopCPUCellCentred<StepSeq>     problem.hpp:362-380
 *   Problem<SOA>::loopCPUCellCentredOMP<StepOMP>  problem.hpp:405-437
 *   Mesh::colourCells                              mesh.hpp:117-162
 *   HierarchicalColourMemory<SOA>                  colouring.hpp:44-147
 *   countCacheLinesForBlock<SOA>                   problem.hpp:654-672
 * with the data bindings of each driver's initProblem (res_calc.cu:10-28,
 * mini_aero.cu:10-24, lulesh.cu:10-24, volna.cu:11-27, getacc.cu:11-26).
 */
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <utility>
#include <vector>

#include "colouring.hpp"
#include "kernels/getacc_scatter.hpp"
#include "kernels/lulesh.hpp"
#include "kernels/mini_aero.hpp"
#include "kernels/res_calc.hpp"
#include "kernels/volna.hpp"

namespace {

using params_t = std::vector<std::pair<MY_SIZE, unsigned>>;

struct LoopBinding {
  std::vector<unsigned> mesh_dim;
  params_t point, cell;
};

bool binding(int loop, LoopBinding &b) {
  switch (loop) {
  case 0: /* res_calc.cu:17-27 */
    b = {{2, 2, 2, 2},
         {{4, sizeof(double)}, {2, sizeof(double)}, {4, sizeof(double)}, {1, sizeof(double)}},
         {}};
    return true;
  case 1: /* mini_aero.cu:15-23 */
    b = {{2, 2}, {{5, sizeof(double)}, {28, sizeof(double)}}, {{12, sizeof(double)}}};
    return true;
  case 2: /* lulesh.cu:15-23 */
    b = {{8, 8},
         {{3, sizeof(double)}, {3, sizeof(double)}},
         {{3, sizeof(double)}, {1, sizeof(double)}}};
    return true;
  case 3: /* volna.cu:16-25 */
    b = {{2, 2},
         {{4, sizeof(float)}, {1, sizeof(float)}},
         {{3, sizeof(float)}, {2, sizeof(float)}, {2, sizeof(float)}, {1, sizeof(int)}}};
    return true;
  case 4: /* getacc.cu:15-25 */
    b = {{4},
         {{4, sizeof(double)}},
         {{4, sizeof(double)}, {1, sizeof(double)}, {4, sizeof(double)},
          {4, sizeof(double)}, {4, sizeof(double)}}};
    return true;
  }
  return false;
}

/* Mesh's and Problem's array constructors are protected; these subclasses
 * reach them the way the reference's own StructuredProblem does
 * (structured_problem.hpp). */
struct ArrayMesh : Mesh {
  ArrayMesh(const std::vector<MY_SIZE> &np, MY_SIZE nc,
            const std::vector<unsigned> &dims,
            const std::vector<const MY_SIZE *> &maps)
      : Mesh(np, nc, dims, maps) {}
};

template <bool SOA> struct ArrayProblem : Problem<SOA> {
  ArrayProblem(Mesh &&m, const params_t &pp, const params_t &cp, MY_SIZE bs)
      : Problem<SOA>(std::move(m), pp, cp, bs) {}
};

template <bool SOA>
ArrayProblem<SOA> *make_problem(int loop, uint32_t n_cells,
                                const uint32_t *n_points,
                                const uint32_t *const *maps,
                                void *const *point_data,
                                void *const *cell_data, uint32_t block_size) {
  LoopBinding b;
  if (!binding(loop, b)) return nullptr;
  std::vector<MY_SIZE> np(n_points, n_points + b.mesh_dim.size());
  std::vector<const MY_SIZE *> mp(maps, maps + b.mesh_dim.size());
  auto *p = new ArrayProblem<SOA>(ArrayMesh(np, n_cells, b.mesh_dim, mp),
                                  b.point, b.cell, block_size);
  for (size_t k = 0; k < b.point.size(); ++k)
    std::memcpy(p->point_weights[k].begin(), point_data[k],
                (size_t)np[k] * b.point[k].first * b.point[k].second);
  for (size_t j = 0; j < b.cell.size(); ++j)
    std::memcpy(p->cell_weights[j].begin(), cell_data[j],
                (size_t)n_cells * b.cell[j].first * b.cell[j].second);
  return p;
}

template <bool SOA>
void copy_back(int loop, ArrayProblem<SOA> *p, uint32_t n_cells,
               void *const *point_data, void *const *cell_data) {
  LoopBinding b;
  binding(loop, b);
  std::memcpy(point_data[0], p->point_weights[0].begin(),
              (size_t)p->mesh.numPoints(0) * b.point[0].first * b.point[0].second);
  for (size_t j = 0; j < b.cell.size(); ++j)
    std::memcpy(cell_data[j], p->cell_weights[j].begin(),
                (size_t)n_cells * b.cell[j].first * b.cell[j].second);
}

template <bool SOA>
int run_serial(int loop, ArrayProblem<SOA> *p, uint32_t iters) {
  switch (loop) {
  case 0: p->template loopCPUCellCentred<res_calc::StepSeq>(iters); return 0;
  case 1: p->template loopCPUCellCentred<mini_aero::StepSeq>(iters); return 0;
  case 2: p->template loopCPUCellCentred<lulesh::StepSeq>(iters); return 0;
  case 3: p->template loopCPUCellCentred<volna::StepSeq>(iters); return 0;
  case 4: p->template loopCPUCellCentred<getacc::StepSeq>(iters); return 0;
  }
  return -1;
}

template <bool SOA>
int run_omp(int loop, ArrayProblem<SOA> *p, uint32_t iters) {
  switch (loop) {
  case 0: p->template loopCPUCellCentredOMP<res_calc::StepOMP>(iters); return 0;
  case 1: p->template loopCPUCellCentredOMP<mini_aero::StepOMP>(iters); return 0;
  case 2: p->template loopCPUCellCentredOMP<lulesh::StepOMP>(iters); return 0;
  case 3: p->template loopCPUCellCentredOMP<volna::StepOMP>(iters); return 0;
  case 4: p->template loopCPUCellCentredOMP<getacc::StepOMP>(iters); return 0;
  }
  return -1;
}

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

} // namespace

extern "C" {

/* Reference serial loop (problem.hpp:362-380) on caller arrays; point_data[0]
 * and the cell datasets are copied back.  seconds (optional) receives the
 * wall time of the loop call alone. */
int ref_loop_serial(int loop, int soa, uint32_t n_cells,
                    const uint32_t *n_points, const uint32_t *const *maps,
                    void *const *point_data, void *const *cell_data,
                    uint32_t iters, double *seconds) {
  int rc;
  double t0, t1;
  if (soa) {
    auto *p = make_problem<true>(loop, n_cells, n_points, maps, point_data, cell_data, 128);
    if (!p) return -1;
    t0 = now_s();
    rc = run_serial<true>(loop, p, iters);
    t1 = now_s();
    copy_back<true>(loop, p, n_cells, point_data, cell_data);
    delete p;
  } else {
    auto *p = make_problem<false>(loop, n_cells, n_points, maps, point_data, cell_data, 128);
    if (!p) return -1;
    t0 = now_s();
    rc = run_serial<false>(loop, p, iters);
    t1 = now_s();
    copy_back<false>(loop, p, n_cells, point_data, cell_data);
    delete p;
  }
  if (seconds) *seconds = t1 - t0;
  return rc;
}

/* Reference OpenMP loop (problem.hpp:405-437).  The loop driver colours the
 * mesh (mesh.hpp:117-162) on every call; that colouring is timed alone first
 * and reported in seconds_colouring, and seconds_loop is the whole call. */
int ref_loop_omp(int loop, int soa, uint32_t n_cells, const uint32_t *n_points,
                 const uint32_t *const *maps, void *const *point_data,
                 void *const *cell_data, uint32_t iters, double *seconds_loop,
                 double *seconds_colouring) {
  if (soa) return -2;
  auto *p = make_problem<false>(loop, n_cells, n_points, maps, point_data, cell_data, 128);
  if (!p) return -1;
  double t0 = now_s();
  auto colours = p->mesh.colourCells();
  double t1 = now_s();
  int rc = run_omp<false>(loop, p, iters);
  double t2 = now_s();
  copy_back<false>(loop, p, n_cells, point_data, cell_data);
  delete p;
  if (seconds_colouring) *seconds_colouring = t1 - t0;
  if (seconds_loop) *seconds_loop = t2 - t1;
  (void)colours;
  return rc;
}

/* The reference's host plan builder for the hierarchical executor
 * (colouring.hpp:44-147) on contiguous blocks of block_size cells: wall time,
 * block colours, blocks and the average number of thread colours. */
int ref_hier_plan(int loop, uint32_t n_cells, const uint32_t *n_points,
                  const uint32_t *const *maps, void *const *point_data,
                  void *const *cell_data, uint32_t block_size, double *seconds,
                  uint32_t *n_colours, uint32_t *n_blocks,
                  double *avg_thread_colours) {
  auto *p = make_problem<false>(loop, n_cells, n_points, maps, point_data, cell_data, block_size);
  if (!p) return -1;
  double t0 = now_s();
  HierarchicalColourMemory<false> memory(*p, p->partition_vector);
  double t1 = now_s();
  uint32_t nb = 0;
  double tc = 0;
  for (const auto &c : memory.colours) {
    nb += c.num_cell_colours.size();
    for (auto v : c.num_cell_colours) tc += v;
  }
  if (seconds) *seconds = t1 - t0;
  if (n_colours) *n_colours = memory.colours.size();
  if (n_blocks) *n_blocks = nb;
  if (avg_thread_colours) *avg_thread_colours = nb ? tc / nb : 0.0;
  delete p;
  return 0;
}

/* The reference's sector model (countCacheLinesForBlock, problem.hpp:654-672)
 * summed over blocks of cells_per_block consecutive cells of a mapping, as
 * loopGPUCellCentred applies it to a colour's cell list (problem.hpp:145-152):
 * `dim` and `type_size` describe point dataset 0. */
uint64_t ref_count_cache_lines(const uint32_t *map, uint32_t n_cells, uint32_t mesh_dim,
                               uint32_t cells_per_block, uint32_t dim, uint32_t type_size, int soa) {
  uint64_t total = 0;
  for (uint32_t c0 = 0; c0 < n_cells; c0 += cells_per_block) {
    const uint32_t c1 = std::min<uint32_t>(n_cells, c0 + cells_per_block);
    const uint32_t *b = map + (size_t)mesh_dim * c0, *e = map + (size_t)mesh_dim * c1;
    total += soa ? countCacheLinesForBlock<true>(b, e, dim, type_size)
                 : countCacheLinesForBlock<false>(b, e, dim, type_size);
  }
  return total;
}

} // extern "C"
