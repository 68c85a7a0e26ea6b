// Instantiates the hierarchical-colour executors for the loop selected by
// FOT_ADAPTER and exposes them, with the atomic executor of the loop's
// atomic_*.cu unit, through a LoopOps table.  Included once by each
// loop_*.cu (compiled without multiply-add contraction: coloured runs are
// bit-identical to their CPU replay).
#pragma once

#include "engine.hpp"
#include "loops.cuh"

namespace fot {

// the atomic executor of this loop (atomic_*.cu, loop_atomic_impl.cuh)
int FOT_CAT(atomic_run_, FOT_ADAPTER_NS)(const LoopData &d, bool soa, bool agg, uint32_t threads,
                                         uint32_t grid, cudaStream_t st);
int FOT_CAT(atomic_occupancy_, FOT_ADAPTER_NS)(bool soa, bool agg, int *per_sm);

namespace FOT_ADAPTER_NS {

using L = Loop;

template <bool SOA, int T, bool STAGE> const void *hier_kernel(bool persistent) {
  return persistent ? reinterpret_cast<const void *>(&k_hier<L, SOA, T, STAGE>)
                    : reinterpret_cast<const void *>(&k_hier_colour<L, SOA, T, STAGE>);
}

template <bool SOA, bool STAGE> const void *hier_kernel_t(bool persistent, uint32_t threads) {
  switch (threads) {
  case 128: return hier_kernel<SOA, 128, STAGE>(persistent);
  case 256: return hier_kernel<SOA, 256, STAGE>(persistent);
  case 512: return hier_kernel<SOA, 512, STAGE>(persistent);
  case 1024: return hier_kernel<SOA, 1024, STAGE>(persistent);
  }
  return nullptr;
}

template <bool SOA, uint32_t SLOTS> const void *pipe_kernel(uint32_t threads) {
  switch (threads) {
  case 128: return reinterpret_cast<const void *>(&k_hier_pipe<L, SOA, 128, SLOTS>);
  case 256: return reinterpret_cast<const void *>(&k_hier_pipe<L, SOA, 256, SLOTS>);
  case 512: return reinterpret_cast<const void *>(&k_hier_pipe<L, SOA, 512, SLOTS>);
  }
  return nullptr;
}

template <bool SOA, uint32_t SLOTS> const void *split_kernel(uint32_t threads) {
  switch (threads) {
  case 128: return reinterpret_cast<const void *>(&k_hier_split<L, SOA, 128, SLOTS>);
  case 256: return reinterpret_cast<const void *>(&k_hier_split<L, SOA, 256, SLOTS>);
  case 512: return reinterpret_cast<const void *>(&k_hier_split<L, SOA, 512, SLOTS>);
  }
  return nullptr;
}

template <bool SOA> const void *dsplit_kernel(uint32_t threads) {
  switch (threads) {
  case 128: return reinterpret_cast<const void *>(&k_hier_dsplit<L, SOA, 128>);
  case 256: return reinterpret_cast<const void *>(&k_hier_dsplit<L, SOA, 256>);
  case 512: return reinterpret_cast<const void *>(&k_hier_dsplit<L, SOA, 512>);
  }
  return nullptr;
}

// variant: kVariantStage (staged reads), kVariantPipe (pipelined kernel),
// kVariantSplit (split write-back kernels: staged with kVariantPipe, else
// direct)
const void *kernel_for(int exec, bool soa, uint32_t threads, uint32_t variant) {
  if (exec == FOT_EXEC_ATOMIC) return nullptr;
  if (exec == FOT_EXEC_HIER && (variant & kVariantSplit) && !(variant & kVariantPipe))
    return soa ? dsplit_kernel<true>(threads) : dsplit_kernel<false>(threads);
  if (exec == FOT_EXEC_HIER && (variant & kVariantSplit)) {
    if (variant & kVariantSlots3) return soa ? split_kernel<true, 3>(threads) : split_kernel<false, 3>(threads);
    return soa ? split_kernel<true, 2>(threads) : split_kernel<false, 2>(threads);
  }
  if (exec == FOT_EXEC_HIER && (variant & kVariantPipe)) {
    if (variant & kVariantSlots3) return soa ? pipe_kernel<true, 3>(threads) : pipe_kernel<false, 3>(threads);
    return soa ? pipe_kernel<true, 2>(threads) : pipe_kernel<false, 2>(threads);
  }
  const bool persistent = exec == FOT_EXEC_HIER;
  const bool stage = variant & 1u;
  if (soa) return stage ? hier_kernel_t<true, true>(persistent, threads)
                        : hier_kernel_t<true, false>(persistent, threads);
  return stage ? hier_kernel_t<false, true>(persistent, threads)
               : hier_kernel_t<false, false>(persistent, threads);
}

int prepare(const void *k, size_t smem) {
  FOT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return FOT_OK;
}

int run_hier(const LoopData &d, const HierPlanDev &P, bool soa, uint32_t threads,
             uint32_t variant, uint32_t grid, size_t smem, cudaStream_t st) {
  const void *k = kernel_for(FOT_EXEC_HIER, soa, threads, variant);
  if (!k) return fail(FOT_ERR_ARG, "no hierarchical kernel for %u threads", threads);
  FOT_TRY(prepare(k, smem));
  void *args[] = {const_cast<LoopData *>(&d), const_cast<HierPlanDev *>(&P)};
  const uint32_t block = (variant & kVariantPipe) ? threads + 64 : threads;
  if (variant & kVariantSplit) {
    // One launch per iteration.  Launch `it` fills partial buffer it & 1 and
    // combines buffer (it - 1) & 1 (direct form: in comb_ctas extra CTAs;
    // staged form: in every CTA after its wait); a last, combine-only launch
    // of the direct kernel flushes the final iteration's buffer.  From the
    // second launch on, programmatic dependent launch lets the next grid
    // gather and compute while this one drains (the kernels wait before
    // they write); the first launch of a call is fully stream-ordered:
    // whatever precedes it may write the datasets it reads.
    const uint32_t iters = P.n_blocks ? P.total_tiles / P.n_blocks : 0;
    const bool direct = !(variant & kVariantPipe);
    const uint32_t comb_ctas = P.n_shared ? (P.n_shared + 4 * threads - 1) / (4 * threads) : 0;
    const void *flush = soa ? dsplit_kernel<true>(threads) : dsplit_kernel<false>(threads);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.stream = st;
    HierPlanDev Q = P;
    void *qargs[] = {const_cast<LoopData *>(&d), &Q};
    for (uint32_t it = 0; it <= iters; ++it) {
      const bool last = it == iters;
      if (last && P.n_shared == 0) break;
      Q.tiles_on = last ? 0u : 1u;
      Q.put_buf = it & 1u;
      Q.comb_on = it > 0 && P.n_shared > 0;
      Q.comb_ctas = (direct || last) && Q.comb_on ? comb_ctas : 0u;
      cfg.gridDim = dim3(last ? Q.comb_ctas : grid + (direct ? Q.comb_ctas : 0u));
      cfg.blockDim = dim3(last ? threads : block);
      cfg.dynamicSmemBytes = last ? 0 : smem;
      cfg.attrs = it > 0 ? attr : nullptr;
      cfg.numAttrs = it > 0 ? 1 : 0;
      FOT_CUDA(cudaLaunchKernelExC(&cfg, last ? flush : k, qargs));
    }
    return FOT_OK;
  }
  FOT_CUDA(cudaLaunchKernel(k, dim3(grid), dim3(block), args, smem, st));
  return FOT_OK;
}

int run_hier_colour(const LoopData &d, const HierPlanDev &P, bool soa, uint32_t threads,
                    uint32_t variant, uint32_t first, uint32_t count, size_t smem,
                    cudaStream_t st) {
  const void *k = kernel_for(FOT_EXEC_HIER_LAUNCH, soa, threads, variant);
  if (!k) return fail(FOT_ERR_ARG, "no hierarchical kernel for %u threads", threads);
  FOT_TRY(prepare(k, smem));
  void *args[] = {const_cast<LoopData *>(&d), const_cast<HierPlanDev *>(&P), &first};
  FOT_CUDA(cudaLaunchKernel(k, dim3(count), dim3(threads), args, smem, st));
  return FOT_OK;
}

int occupancy(int exec, bool soa, uint32_t threads, uint32_t variant, size_t smem, int *per_sm) {
  // atomic plans: `variant` bit 0 set = warp aggregation
  if (exec == FOT_EXEC_ATOMIC)
    return FOT_CAT(atomic_occupancy_, FOT_ADAPTER_NS)(soa, variant & 1u, per_sm);
  const void *k = kernel_for(exec, soa, threads, variant);
  if (!k) return fail(FOT_ERR_ARG, "no kernel for %u threads", threads);
  FOT_TRY(prepare(k, smem));
  int block = (int)threads;
  if (exec == FOT_EXEC_HIER && (variant & kVariantPipe)) block += 64;
  FOT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, block, smem));
  return FOT_OK;
}

void smem_layout(uint32_t cap0, uint32_t cap1, uint32_t variant, uint32_t rec_cap,
                 uint32_t threads, SmemLayout *out) {
  using out_t = typename L::out_t;
  using read_t = typename L::read_t;
  const bool stage = variant & kVariantStage;
  auto a16 = [](size_t v) { return (v + 15) & ~size_t(15); };
  SmemLayout s;
  size_t off = 0;
  if ((variant & kVariantSplit) && !(variant & kVariantPipe)) {
    // direct split write-back: the block's sums only
    s.acc_off = 0;
    s.total = a16((size_t)cap0 * L::kOut * sizeof(out_t));
    *out = s;
    return;
  }
  if (variant & kVariantPipe) {
    // 2 or 3 tile-record slots, 2 read-row slots, the per-slot increments, 2
    // prefetched-output-row slots (AOS output rows of a multiple of 16 bytes;
    // not in the split write-back kernel)
    auto a128 = [](size_t v) { return (v + 127) & ~size_t(127); };
    s.rec_slot = (uint32_t)a128(rec_cap);
    off = ((variant & kVariantSlots3) ? 3 : 2) * (size_t)s.rec_slot;
    s.rows_off = (uint32_t)off;
    size_t rows = 0;
    for (int r = 0; r < L::kNumRead; ++r) {
      s.read_off[r] = (uint32_t)rows;
      const uint32_t cap = L::read_class(r) == 0 ? cap0 : cap1;
      rows = a16(rows + (size_t)cap * L::read_dim(r) * sizeof(read_t));
    }
    s.rows_bytes = (uint32_t)a128(rows);
    off += 2 * (size_t)s.rows_bytes;
    s.inc_off = (uint32_t)off;
    off = a128(off + (size_t)L::kOut * L::kDim * threads * sizeof(out_t));
    s.outbuf_off = (uint32_t)off;
    if (!(variant & kVariantSplit) && (L::kOut * sizeof(out_t)) % 16 == 0) {
      s.outbuf_bytes = (uint32_t)a128((size_t)cap0 * L::kOut * sizeof(out_t));
      off += 2 * (size_t)s.outbuf_bytes;
    }
    s.total = off;
    *out = s;
    return;
  }
  if (stage) {
    for (int r = 0; r < L::kNumRead; ++r) {
      s.read_off[r] = (uint32_t)off;
      const uint32_t cap = L::read_class(r) == 0 ? cap0 : cap1;
      off = a16(off + (size_t)cap * L::read_dim(r) * sizeof(read_t));
    }
  }
  s.acc_off = (uint32_t)off;
  off = a16(off + (size_t)cap0 * L::kOut * sizeof(out_t));
  s.pts_off = (uint32_t)off;
  off += (size_t)(cap0 + (stage && L::kHasClass1 ? cap1 : 0)) * sizeof(uint32_t);
  s.total = a16(off);
  *out = s;
}

} // namespace FOT_ADAPTER_NS

extern const LoopOps FOT_OPS_NAME;
const LoopOps FOT_OPS_NAME = {FOT_CAT(atomic_run_, FOT_ADAPTER_NS), FOT_ADAPTER_NS::run_hier,
                              FOT_ADAPTER_NS::run_hier_colour, FOT_ADAPTER_NS::occupancy,
                              FOT_ADAPTER_NS::smem_layout};
} // namespace fot
