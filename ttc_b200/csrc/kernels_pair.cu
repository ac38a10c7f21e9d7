// Instantiations of the plain kernels for one A/B type pair. This file is compiled once per pair
// with -DTTCB_PAIR=<0..7> (s, d, c, z, sd, ds, cz, zc) so the eight pairs build in parallel.
#include <cstring>
#include "batch_kernels.cuh"
#include "kernels.cuh"
#include "launch.h"

#ifndef TTCB_PAIR
#error "TTCB_PAIR must be defined"
#endif

namespace ttcb {

#if TTCB_PAIR == 0
using TA = float;
using TB = float;
#define PAIR_FN pick_kernel_ss
#define PAIR_BATCH_FN pick_batch_ss
#elif TTCB_PAIR == 1
using TA = double;
using TB = double;
#define PAIR_FN pick_kernel_dd
#define PAIR_BATCH_FN pick_batch_dd
#elif TTCB_PAIR == 2
using TA = float2;
using TB = float2;
#define PAIR_FN pick_kernel_cc
#define PAIR_BATCH_FN pick_batch_cc
#elif TTCB_PAIR == 3
using TA = double2;
using TB = double2;
#define PAIR_FN pick_kernel_zz
#define PAIR_BATCH_FN pick_batch_zz
#elif TTCB_PAIR == 4
using TA = float;
using TB = double;
#define PAIR_FN pick_kernel_sd
#define PAIR_BATCH_FN pick_batch_sd
#elif TTCB_PAIR == 5
using TA = double;
using TB = float;
#define PAIR_FN pick_kernel_ds
#define PAIR_BATCH_FN pick_batch_ds
#elif TTCB_PAIR == 6
using TA = float2;
using TB = double2;
#define PAIR_FN pick_kernel_cz
#define PAIR_BATCH_FN pick_batch_cz
#else
using TA = double2;
using TB = float2;
#define PAIR_FN pick_kernel_zc
#define PAIR_BATCH_FN pick_batch_zc
#endif

template <int VA, int VB, bool BETA, bool STREAM>
static cudaError_t launch_tile(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                               cudaStream_t stream, int blocks) {
  TA al;
  std::memcpy(&al, alpha, sizeof(TA));
  TB be;
  std::memset(&be, 0, sizeof(TB));
  if (BETA) std::memcpy(&be, beta, sizeof(TB));
  tile_kernel<TA, TB, VA, VB, BETA, STREAM><<<blocks, kThreads, p->smem_bytes, stream>>>(
      reinterpret_cast<const TileDesc*>(p->dev_desc), static_cast<const TA*>(A), static_cast<TB*>(B), al, be);
  return cudaGetLastError();
}

template <int V, bool BETA, bool STREAM>
static cudaError_t launch_row(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                              cudaStream_t stream, int blocks) {
  TA al;
  std::memcpy(&al, alpha, sizeof(TA));
  TB be;
  std::memset(&be, 0, sizeof(TB));
  if (BETA) std::memcpy(&be, beta, sizeof(TB));
  row_kernel<TA, TB, V, BETA, STREAM><<<blocks, kThreads, 0, stream>>>(
      reinterpret_cast<const RowDesc*>(p->dev_desc), static_cast<const TA*>(A), static_cast<TB*>(B), al, be);
  return cudaGetLastError();
}

template <int VA, int VB>
static KernelRef tile_ref(int variant) {
  KernelRef r;
  if (variant == 2) {
    r.fn = &launch_tile<VA, VB, true, false>;
    r.func = reinterpret_cast<const void*>(&tile_kernel<TA, TB, VA, VB, true, false>);
  } else if (variant == 1) {
    r.fn = &launch_tile<VA, VB, false, true>;
    r.func = reinterpret_cast<const void*>(&tile_kernel<TA, TB, VA, VB, false, true>);
  } else {
    r.fn = &launch_tile<VA, VB, false, false>;
    r.func = reinterpret_cast<const void*>(&tile_kernel<TA, TB, VA, VB, false, false>);
  }
  return r;
}

template <int V>
static KernelRef row_ref(int variant) {
  KernelRef r;
  if (variant == 2) {
    r.fn = &launch_row<V, true, false>;
    r.func = reinterpret_cast<const void*>(&row_kernel<TA, TB, V, true, false>);
  } else if (variant == 1) {
    r.fn = &launch_row<V, false, true>;
    r.func = reinterpret_cast<const void*>(&row_kernel<TA, TB, V, false, true>);
  } else {
    r.fn = &launch_row<V, false, false>;
    r.func = reinterpret_cast<const void*>(&row_kernel<TA, TB, V, false, false>);
  }
  return r;
}

KernelRef PAIR_FN(int kernel, int va, int vb, int variant) {
  constexpr int MA = 16 / sizeof(TA);
  constexpr int MB = 16 / sizeof(TB);
  constexpr int MR = MA < MB ? MA : MB;
  if (kernel == TTCB_KERNEL_ROW) {
    if (va > 1 && vb > 1) return row_ref<MR>(variant);
    return row_ref<1>(variant);
  }
  const bool a = va > 1, b = vb > 1;
  if (a && b) return tile_ref<MA, MB>(variant);
  if (a) return tile_ref<MA, 1>(variant);
  if (b) return tile_ref<1, MB>(variant);
  return tile_ref<1, 1>(variant);
}

template <bool BETA, bool STREAM>
static cudaError_t launch_batch(const void* probs, const int64_t* prefix, int count, unsigned long long total,
                                unsigned long long* counter, int* status, const void* alpha, const void* beta,
                                int blocks, int smem, cudaStream_t stream) {
  TA al;
  std::memcpy(&al, alpha, sizeof(TA));
  TB be;
  std::memset(&be, 0, sizeof(TB));
  if (BETA) std::memcpy(&be, beta, sizeof(TB));
  batch_kernel<TA, TB, BETA, STREAM><<<blocks, kThreads, smem, stream>>>(
      static_cast<const BatchProblem*>(probs), prefix, count, total, counter, status, al, be);
  return cudaGetLastError();
}

BatchKernelRef PAIR_BATCH_FN(int variant) {
  BatchKernelRef r;
  if (variant == 2) {
    r.fn = &launch_batch<true, false>;
    r.func = reinterpret_cast<const void*>(&batch_kernel<TA, TB, true, false>);
  } else if (variant == 1) {
    r.fn = &launch_batch<false, true>;
    r.func = reinterpret_cast<const void*>(&batch_kernel<TA, TB, false, true>);
  } else {
    r.fn = &launch_batch<false, false>;
    r.func = reinterpret_cast<const void*>(&batch_kernel<TA, TB, false, false>);
  }
  return r;
}

}  // namespace ttcb
