// Instantiates the atomic executor (a) for the loop selected by FOT_ADAPTER.
// Included once by each atomic_*.cu.  Those translation units are compiled
// WITH multiply-add contraction (the build compiles atomic_*.cu with
// -fmad=true, as the reference compiles its own device code): the atomic
// executor's results differ from the serial loop by summation order anyway
// (contract: normwise relative error <= 1e-12 FP64 / 1e-5 FP32), and the
// fused multiply-adds cut the instruction count of the heavy functors
// (mini_aero's Roe flux).  The coloured executors stay in the exact units
// (loop_*.cu, -fmad=false) where a run is bit-identical to its CPU replay.
#pragma once

#define FOT_NS_SUFFIX _fma
#include "engine.hpp"
#include "loops.cuh"

namespace fot {
namespace {

using LA = FOT_LNS(FOT_ADAPTER_NS)::Loop;

template <bool SOA, bool AGG>
int launch_atomic(const LoopData &d, uint32_t grid, cudaStream_t st) {
  k_atomic<LA, SOA, AGG><<<grid, 256, 0, st>>>(d);
  FOT_CUDA(cudaGetLastError());
  return FOT_OK;
}

template <bool SOA, bool AGG> const void *atomic_kernel() {
  return reinterpret_cast<const void *>(&k_atomic<LA, SOA, AGG>);
}

} // namespace

int FOT_CAT(atomic_run_, FOT_ADAPTER_NS)(const LoopData &d, bool soa, bool agg, uint32_t threads,
                                         uint32_t grid, cudaStream_t st) {
  if (threads != 256) return fail(FOT_ERR_ARG, "atomic executor runs 256 threads per CTA");
  if (soa) return agg ? launch_atomic<true, true>(d, grid, st) : launch_atomic<true, false>(d, grid, st);
  return agg ? launch_atomic<false, true>(d, grid, st) : launch_atomic<false, false>(d, grid, st);
}

int FOT_CAT(atomic_occupancy_, FOT_ADAPTER_NS)(bool soa, bool agg, int *per_sm) {
  const void *k = soa ? (agg ? atomic_kernel<true, true>() : atomic_kernel<true, false>())
                      : (agg ? atomic_kernel<false, true>() : atomic_kernel<false, false>());
  FOT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, 256, 0));
  return FOT_OK;
}

} // namespace fot
