// Batched atomic executor: tiles of kAtomicTile consecutive cells of every
// mesh and every iteration in one grid-stride launch (iterations need no
// ordering: the loops never read the dataset they increment).  Compiled with
// multiply-add contraction, like the single-mesh atomic units (see
// loop_atomic_impl.cuh); the functors are instantiated under res_calc_fma,
// ... to keep their symbols apart from the exact ones of batch.cu.
#define FOT_ADAPTER_ALL 1
#define FOT_NS_SUFFIX _fma
#include "batch.cuh"
#include "engine.hpp"
#include "loops.cuh"

namespace fot {

template <class... Ls> constexpr int max_reg_cap() {
  int m = 0;
  ((m = Ls::kRegCap > m ? Ls::kRegCap : m), ...);
  return m;
}

template <bool SOA, bool AGG, class... Ls>
__global__ void __launch_bounds__(256, (65536 / (256 * max_reg_cap<Ls...>())) > 0
                                           ? 65536 / (256 * max_reg_cap<Ls...>()) : 1)
    k_batch_atomic(BatchDev B) {
  const uint32_t warp = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < B.total_tiles; t += gridDim.x) {
    const uint32_t r = t % B.tiles_per_iter;
    const BatchMesh &m = B.mesh[B.tile_mesh[r]];
    const uint32_t start = B.tile_block[r];
#pragma unroll 1
    for (uint32_t k = 0; k < kAtomicTile / 256; ++k) {
      const uint32_t base = start + (k * 8u + warp) * 32u;
      ((m.loop == Ls::kLoop ? (atomic_warp<Ls, SOA, AGG>(m.d, base), 0) : 0), ...);
    }
  }
}

template <bool SOA, bool AGG> const void *batch_atomic_kernel(uint32_t loop_mask) {
  using RC = res_calc_fma::Loop;
  using MA = mini_aero_fma::Loop;
  using LU = lulesh_fma::Loop;
  using VO = volna_fma::Loop;
  using GA = getacc_fma::Loop;
  switch (loop_mask) {
  case 1u << FOT_LOOP_RES_CALC: return (const void *)&k_batch_atomic<SOA, AGG, RC>;
  case 1u << FOT_LOOP_MINI_AERO: return (const void *)&k_batch_atomic<SOA, AGG, MA>;
  case 1u << FOT_LOOP_LULESH: return (const void *)&k_batch_atomic<SOA, AGG, LU>;
  case 1u << FOT_LOOP_VOLNA: return (const void *)&k_batch_atomic<SOA, AGG, VO>;
  case 1u << FOT_LOOP_GETACC: return (const void *)&k_batch_atomic<SOA, AGG, GA>;
  case (1u << FOT_LOOP_RES_CALC) | (1u << FOT_LOOP_VOLNA):
    return (const void *)&k_batch_atomic<SOA, AGG, RC, VO>;
  }
  return nullptr;
}

const void *batch_atomic_kernel_for(bool soa, bool agg, uint32_t loop_mask) {
  if (soa) return agg ? batch_atomic_kernel<true, true>(loop_mask) : batch_atomic_kernel<true, false>(loop_mask);
  return agg ? batch_atomic_kernel<false, true>(loop_mask) : batch_atomic_kernel<false, false>(loop_mask);
}

} // namespace fot
