// Loop adapters: bind each application's per-cell user function to its data,
// the role of the reference's per-app StepSeq / StepGPUGlobal /
// StepGPUHierarchical wrappers (kernels/res_calc.hpp:29-89,
// mini_aero.hpp:43-111, lulesh.hpp:23-58, volna.hpp:30-75,
// getacc_scatter.hpp:29-75).
//
// An adapter describes
//   kDim          slots per cell (mesh_dim of mapping 0, the written mapping)
//   out_t, kOut   element type and dimension of point dataset 0 (incremented)
//   read sets     point datasets read through a mapping: point set index,
//                 mapping class (0: mapping 0; 1: a second, distinct mapping
//                 such as res_calc's edge->node), dimension, element type
//   direct sets   cell datasets (SOA), element type, and which are written
//                 (kWritesCell: the cell function writes a cell dataset)
// and a device function cell() that, given row pointers of the read sets for
// each slot (in global memory or staged in shared memory) and the cell's
// direct data, produces the signed per-slot increments inc[slot][k] such that
// point dataset 0 receives out[p_slot][k] += inc[slot][k].
//
// The user functions come from *_func.hpp files in the reference's drop-in
// format, included with USER_FUNCTION_SIGNATURE / RESTRICT defined; the
// directory is FOT_FUNCTOR_DIR (default: the engine's own files).
#pragma once

#include <cassert>
#include <cmath>
#include <cstdint>
#include <iostream>

#include "common.cuh"

// Each translation unit instantiates one loop: it defines FOT_ADAPTER to the
// loop id before including this header, so a user's drop-in *_func.hpp (and
// helpers with external linkage) is compiled exactly once.
#if !defined(FOT_ADAPTER) && !defined(FOT_ADAPTER_ALL)
#error "define FOT_ADAPTER to a FOT_LOOP_* id (or FOT_ADAPTER_ALL) before including loops.cuh"
#endif
#ifndef FOT_ADAPTER
#define FOT_ADAPTER (-1)
#endif

#ifndef FOT_FUNCTOR_DIR
#define FOT_FUNCTOR_DIR kernels
#endif
// Namespace of a loop's adapter and functor: the loop's name, plus
// FOT_NS_SUFFIX when a translation unit defines it (the atomic executor's
// units, compiled with multiply-add contraction, instantiate the same
// functors under res_calc_fma, ... so that their symbols stay apart from the
// exact instantiations of the coloured executors).
#ifndef FOT_NS_SUFFIX
#define FOT_NS_SUFFIX
#endif
#define FOT_CAT2(a, b) a##b
#define FOT_CAT(a, b) FOT_CAT2(a, b)
#define FOT_LNS(name) FOT_CAT(name, FOT_NS_SUFFIX)
// Resident CTAs per SM of the atomic executor, per loop (its register cap is
// 65536 / (256 * this)); measured choices, overridable at build time.
#ifndef FOT_ATOMIC_MINB_RES_CALC
#define FOT_ATOMIC_MINB_RES_CALC 4
#endif
#ifndef FOT_ATOMIC_MINB_MINI_AERO
#define FOT_ATOMIC_MINB_MINI_AERO 2
#endif
#ifndef FOT_ATOMIC_MINB_LULESH
#define FOT_ATOMIC_MINB_LULESH 2
#endif
#ifndef FOT_ATOMIC_MINB_VOLNA
#define FOT_ATOMIC_MINB_VOLNA 8
#endif
#ifndef FOT_ATOMIC_MINB_GETACC
#define FOT_ATOMIC_MINB_GETACC 2
#endif
// Whether the atomic executor (SOA form) prefetches the next chunk's mapping
// rows and direct data into L2 while it computes the current one (per loop;
// measured choices, overridable at build time: on for mini_aero's 96-byte
// face records, 2% faster after RCM; 2-11% slower for the other loops).
#ifndef FOT_ATOMIC_PREFETCH_RES_CALC
#define FOT_ATOMIC_PREFETCH_RES_CALC 0
#endif
#ifndef FOT_ATOMIC_PREFETCH_MINI_AERO
#define FOT_ATOMIC_PREFETCH_MINI_AERO 1
#endif
#ifndef FOT_ATOMIC_PREFETCH_LULESH
#define FOT_ATOMIC_PREFETCH_LULESH 0
#endif
#ifndef FOT_ATOMIC_PREFETCH_VOLNA
#define FOT_ATOMIC_PREFETCH_VOLNA 0
#endif
#ifndef FOT_ATOMIC_PREFETCH_GETACC
#define FOT_ATOMIC_PREFETCH_GETACC 0
#endif
#define FOT_STR2(x) #x
#define FOT_STR(x) FOT_STR2(x)
#define FOT_FUNCTOR(file) FOT_STR(FOT_FUNCTOR_DIR/file)

namespace fot {

// --------------------------------------------------------------------------
// res_calc: edge -> 2 cells; reads x through the edge->node mapping and q,
// adt through the edge->cell mapping (res_calc.hpp:29-89).
// --------------------------------------------------------------------------
#if FOT_ADAPTER == FOT_LOOP_RES_CALC || defined(FOT_ADAPTER_ALL)
namespace FOT_LNS(res_calc) {
#define USER_FUNCTION_SIGNATURE __device__ __forceinline__ void user_func_gpu
#define RESTRICT __restrict__
#include FOT_FUNCTOR(res_calc_func.hpp)

struct Loop {
  static constexpr int kLoop = FOT_LOOP_RES_CALC;
  static constexpr int kDim = 2;
  using out_t = double;
  static constexpr int kOut = 4;
  using read_t = double;
  static constexpr int kNumRead = 3;
  static constexpr bool kHasClass1 = true;
  static constexpr int kRegCap = 64; // registers per thread the tile kernels are held to
  // registers per thread of the direct split write-back kernel
  static constexpr int kDirectRegCap = 48;
  // resident 256-thread CTAs per SM the atomic executor is compiled for
  static constexpr int kAtomicMinBlocks = FOT_ATOMIC_MINB_RES_CALC;
  // the atomic executor prefetches the next chunk into L2
  static constexpr bool kAtomicPrefetch = FOT_ATOMIC_PREFETCH_RES_CALC;
  // read set r: x (set 1, class 1, dim 2), q (set 2, class 0, dim 4), adt (set 3, class 0, dim 1)
  __host__ __device__ static constexpr int read_set(int r) { return r + 1; }
  __host__ __device__ static constexpr int read_class(int r) { return r == 0 ? 1 : 0; }
  __host__ __device__ static constexpr int read_dim(int r) { return r == 0 ? 2 : (r == 1 ? 4 : 1); }
  static constexpr int kNumDirect = 0;
  static constexpr bool kWritesCell = false; // no cell dataset is written

  template <class Rows, class Direct>
  __device__ __forceinline__ static void cell(const Rows &rows, const Direct &,
                                              out_t (&inc)[kDim][kOut]) {
    user_func_gpu(rows.template ptr<0>(0), rows.template ptr<0>(1),
                  rows.template ptr<1>(0), rows.template ptr<1>(1),
                  rows.template ptr<2>(0), rows.template ptr<2>(1), inc[0],
                  inc[1], rows.template stride<0>(), rows.template stride<1>());
  }
};
} // namespace res_calc
#endif

// --------------------------------------------------------------------------
// mini_aero: face -> 2 cells; reads the 28-double cell record; the face
// record is direct data; left -= flux, right += flux (mini_aero.hpp:43-111).
// --------------------------------------------------------------------------
#if FOT_ADAPTER == FOT_LOOP_MINI_AERO || defined(FOT_ADAPTER_ALL)
namespace FOT_LNS(mini_aero) {
#define USER_FUNCTION_SIGNATURE __device__ __forceinline__ void user_func_gpu
#define RESTRICT __restrict__
#include FOT_FUNCTOR(mini_aero_func.hpp)

struct Loop {
  static constexpr int kLoop = FOT_LOOP_MINI_AERO;
  static constexpr int kDim = 2;
  using out_t = double;
  static constexpr int kOut = 5;
  using read_t = double;
  static constexpr int kNumRead = 1;
  static constexpr bool kHasClass1 = false;
  static constexpr int kRegCap = 128; // registers per thread the tile kernels are held to
  // registers per thread of the direct split write-back kernel
  static constexpr int kDirectRegCap = kRegCap;
  // resident 256-thread CTAs per SM the atomic executor is compiled for
  static constexpr int kAtomicMinBlocks = FOT_ATOMIC_MINB_MINI_AERO;
  // the atomic executor prefetches the next chunk into L2
  static constexpr bool kAtomicPrefetch = FOT_ATOMIC_PREFETCH_MINI_AERO;
  __host__ __device__ static constexpr int read_set(int) { return 1; }
  __host__ __device__ static constexpr int read_class(int) { return 0; }
  __host__ __device__ static constexpr int read_dim(int) { return 28; }
  static constexpr int kNumDirect = 1;
  static constexpr bool kWritesCell = false;

  template <class Rows, class Direct>
  __device__ __forceinline__ static void cell(const Rows &rows, const Direct &dir,
                                              out_t (&inc)[kDim][kOut]) {
    const double *L = rows.template ptr<0>(0);
    const double *R = rows.template ptr<0>(1);
    const unsigned s = rows.template stride<0>();
    const double *f = dir.template ptr<double>(0);
    const unsigned fs = dir.stride;
    double flux[5];
    user_func_gpu(flux, L, R, L + 5 * s, R + 5 * s, L + 8 * s, R + 8 * s,
                  L + 23 * s, R + 23 * s, f, f + 3 * fs, f + 6 * fs, f + 9 * fs,
                  s, fs);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      inc[0][k] = -flux[k];
      inc[1][k] = flux[k];
    }
  }
};
} // namespace mini_aero
#endif

// --------------------------------------------------------------------------
// lulesh: hex element -> 8 nodes; reads xyz, writes the element volume into
// the direct dataset determ (lulesh.hpp:23-58).
// --------------------------------------------------------------------------
#if FOT_ADAPTER == FOT_LOOP_LULESH || defined(FOT_ADAPTER_ALL)
namespace FOT_LNS(lulesh) {
static constexpr unsigned MESH_DIM = 8;
#define USER_FUNCTION_SIGNATURE __device__ __forceinline__ void user_func_gpu
#define RESTRICT __restrict__
#include FOT_FUNCTOR(lulesh_func.hpp)

struct Loop {
  static constexpr int kLoop = FOT_LOOP_LULESH;
  static constexpr int kDim = 8;
  using out_t = double;
  static constexpr int kOut = 3;
  using read_t = double;
  static constexpr int kNumRead = 1;
  static constexpr bool kHasClass1 = false;
  static constexpr int kRegCap = 96; // registers per thread the tile kernels are held to
  // registers per thread of the direct split write-back kernel
  static constexpr int kDirectRegCap = kRegCap;
  // resident 256-thread CTAs per SM the atomic executor is compiled for
  static constexpr int kAtomicMinBlocks = FOT_ATOMIC_MINB_LULESH;
  // the atomic executor prefetches the next chunk into L2
  static constexpr bool kAtomicPrefetch = FOT_ATOMIC_PREFETCH_LULESH;
  __host__ __device__ static constexpr int read_set(int) { return 1; }
  __host__ __device__ static constexpr int read_class(int) { return 0; }
  __host__ __device__ static constexpr int read_dim(int) { return 3; }
  static constexpr int kNumDirect = 2;
  static constexpr bool kWritesCell = true; // determ (cell dataset 1)

  template <class Rows, class Direct>
  __device__ __forceinline__ static void cell(const Rows &rows, const Direct &dir,
                                              out_t (&inc)[kDim][kOut]) {
    const double *xyz[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) xyz[j] = rows.template ptr<0>(j);
    double f[24];
    double determ;
    user_func_gpu(f, xyz, dir.template ptr<double>(0), determ,
                  rows.template stride<0>(), dir.stride);
    *dir.template wptr<double>(1) = determ;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) inc[j][i] = f[i * 8 + j];
  }
};
} // namespace lulesh
#endif

// --------------------------------------------------------------------------
// volna: edge -> 2 cells, FP32; reads the cell volumes; per-edge fluxes,
// bathymetry source, normals and the boundary flag are direct data
// (volna.hpp:30-75).
// --------------------------------------------------------------------------
#if FOT_ADAPTER == FOT_LOOP_VOLNA || defined(FOT_ADAPTER_ALL)
namespace FOT_LNS(volna) {
#define USER_FUNCTION_SIGNATURE __device__ __forceinline__ void user_func_gpu
#define RESTRICT __restrict__
#include FOT_FUNCTOR(volna_func.hpp)

struct Loop {
  static constexpr int kLoop = FOT_LOOP_VOLNA;
  static constexpr int kDim = 2;
  using out_t = float;
  static constexpr int kOut = 4;
  using read_t = float;
  static constexpr int kNumRead = 1;
  static constexpr bool kHasClass1 = false;
  static constexpr int kRegCap = 64; // registers per thread the tile kernels are held to
  // registers per thread of the direct split write-back kernel
  static constexpr int kDirectRegCap = kRegCap;
  // resident 256-thread CTAs per SM the atomic executor is compiled for
  static constexpr int kAtomicMinBlocks = FOT_ATOMIC_MINB_VOLNA;
  // the atomic executor prefetches the next chunk into L2
  static constexpr bool kAtomicPrefetch = FOT_ATOMIC_PREFETCH_VOLNA;
  __host__ __device__ static constexpr int read_set(int) { return 1; }
  __host__ __device__ static constexpr int read_class(int) { return 0; }
  __host__ __device__ static constexpr int read_dim(int) { return 1; }
  static constexpr int kNumDirect = 4;
  static constexpr bool kWritesCell = false;

  template <class Rows, class Direct>
  __device__ __forceinline__ static void cell(const Rows &rows, const Direct &dir,
                                              out_t (&inc)[kDim][kOut]) {
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int k = 0; k < 4; ++k) inc[s][k] = 0.0f;
    user_func_gpu(rows.template ptr<0>(0), rows.template ptr<0>(1), inc[0],
                  inc[1], dir.template ptr<float>(0), dir.template ptr<float>(1),
                  dir.template ptr<float>(2), dir.template ptr<int>(3), dir.stride);
  }
};
} // namespace volna
#endif

// --------------------------------------------------------------------------
// getacc: quad element -> 4 nodes; direct data only
// (getacc_scatter.hpp:29-75).
// --------------------------------------------------------------------------
#if FOT_ADAPTER == FOT_LOOP_GETACC || defined(FOT_ADAPTER_ALL)
namespace FOT_LNS(getacc) {
#define USER_FUNCTION_SIGNATURE __device__ __forceinline__ void user_func_gpu
#define RESTRICT __restrict__
#include FOT_FUNCTOR(getacc_scatter_func.hpp)

struct Loop {
  static constexpr int kLoop = FOT_LOOP_GETACC;
  static constexpr int kDim = 4;
  using out_t = double;
  static constexpr int kOut = 4;
  using read_t = double;
  static constexpr int kNumRead = 0;
  static constexpr bool kHasClass1 = false;
  static constexpr int kRegCap = 96; // registers per thread the tile kernels are held to
  // registers per thread of the direct split write-back kernel
  static constexpr int kDirectRegCap = kRegCap;
  // resident 256-thread CTAs per SM the atomic executor is compiled for
  static constexpr int kAtomicMinBlocks = FOT_ATOMIC_MINB_GETACC;
  // the atomic executor prefetches the next chunk into L2
  static constexpr bool kAtomicPrefetch = FOT_ATOMIC_PREFETCH_GETACC;
  __host__ __device__ static constexpr int read_set(int) { return 0; }
  __host__ __device__ static constexpr int read_class(int) { return 0; }
  __host__ __device__ static constexpr int read_dim(int) { return 1; }
  static constexpr int kNumDirect = 5;
  static constexpr bool kWritesCell = false;

  template <class Rows, class Direct>
  __device__ __forceinline__ static void cell(const Rows &, const Direct &dir,
                                              out_t (&inc)[kDim][kOut]) {
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int k = 0; k < 4; ++k) inc[s][k] = 0.0;
    user_func_gpu(dir.template ptr<double>(0), dir.template ptr<double>(1),
                  dir.template ptr<double>(2), dir.template ptr<double>(3),
                  dir.template ptr<double>(4), inc[0], inc[1], inc[2], inc[3],
                  dir.stride);
  }
};
} // namespace getacc
#endif

} // namespace fot
