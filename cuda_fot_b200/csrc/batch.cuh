// Device views shared by the batched executors (batch.cu: hierarchical
// tiles; atomic_batch.cu: atomic tiles, compiled with multiply-add
// contraction like the other atomic units).
#pragma once

#include <cstdint>

#include "executors.cuh"

namespace fot {

struct BatchMesh {
  LoopData d;
  HierPlanDev P;
  int loop;
};

struct BatchDev {
  const BatchMesh *mesh;
  const uint32_t *tile_mesh;  // per tile of one iteration: mesh index
  const uint32_t *tile_block; // per tile: block of that mesh
  uint32_t tiles_per_iter;
  uint32_t total_tiles;
  uint32_t n_mesh;
  unsigned int *done; // per mesh
  Ctl *ctl;           // ticket / exited / error
};

constexpr uint32_t kAtomicTile = 1024;  // cells per tile of the atomic batch

// the atomic batch kernel for a set of loop kinds (atomic_batch.cu)
const void *batch_atomic_kernel_for(bool soa, bool agg, uint32_t loop_mask);

} // namespace fot
