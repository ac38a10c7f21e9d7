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

template <int VA, int VB, bool BETA, bool STREAM, bool REG, bool DYN, bool BULK>
static cudaError_t launch_async(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                                cudaStream_t stream, int blocks) {
  TA al;
  std::memcpy(&al, alpha, sizeof(TA));
  TB be;
  std::memset(&be, 0, sizeof(TB));
  if (BETA) std::memcpy(&be, beta, sizeof(TB));
  unsigned int* sched = nullptr;
  if (DYN) {
    sched = plan_claim_slot(p);
    if (!sched) return cudaErrorInvalidValue;
  }
  // programmatic stream serialization: the kernel may start while the previous one in the stream
  // drains; it waits (griddepcontrol.wait) before it touches A or B
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = p->smem_async;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // shifted A runs: A's pointer lies a0 elements past a 16-byte boundary
  const int a0 = (int)(((uintptr_t)A / sizeof(TA)) & (uintptr_t)(VA - 1));
  return cudaLaunchKernelEx(&cfg, tile_async_kernel<TA, TB, VA, VB, BETA, STREAM, REG, DYN, BULK>,
                            reinterpret_cast<const TileDesc*>(p->dev_desc), static_cast<const TA*>(A),
                            static_cast<TB*>(B), al, be, sched, a0, BULK ? p->wait_status : nullptr,
                            (unsigned int)(p->claim_group > 0 ? p->claim_group : 1));
}

template <int VA, int VB, bool REG, bool DYN, bool BULK>
static KernelRef async_ref(int variant) {
  KernelRef r;
  if (variant == 2) {
    r.fn = &launch_async<VA, VB, true, false, REG, DYN, BULK>;
    r.func = reinterpret_cast<const void*>(&tile_async_kernel<TA, TB, VA, VB, true, false, REG, DYN, BULK>);
  } else if (variant == 1) {
    r.fn = &launch_async<VA, VB, false, true, REG, DYN, BULK>;
    r.func = reinterpret_cast<const void*>(&tile_async_kernel<TA, TB, VA, VB, false, true, REG, DYN, BULK>);
  } else {
    r.fn = &launch_async<VA, VB, false, false, REG, DYN, BULK>;
    r.func = reinterpret_cast<const void*>(&tile_async_kernel<TA, TB, VA, VB, false, false, REG, DYN, BULK>);
  }
  return r;
}

template <int VA, bool REG, bool DYN, bool BULK>
static KernelRef async_ref_b(int vb, int variant) {
  constexpr int MB = 16 / sizeof(TB);
  if (vb >= 4 && MB >= 4) return async_ref<VA, (MB >= 4 ? 4 : 1), REG, DYN, BULK>(variant);
  if (vb >= 2 && MB >= 2) return async_ref<VA, (MB >= 2 ? 2 : 1), REG, DYN, BULK>(variant);
  return async_ref<VA, 1, REG, DYN, BULK>(variant);
}

// The bulk-copy form exists for the full 16-byte A vector only (the launch asks for it only then).
template <bool REG, bool DYN, bool BULK>
static KernelRef async_ref_ab(int va, int vb, int variant) {
  constexpr int MA = 16 / sizeof(TA);
  if constexpr (BULK) {
    if (va != MA) return KernelRef{};
    return async_ref_b<MA, REG, DYN, true>(vb, variant);
  } else {
    if (va >= 4 && MA >= 4) return async_ref_b<(MA >= 4 ? 4 : 1), REG, DYN, false>(vb, variant);
    if (va >= 2 && MA >= 2) return async_ref_b<(MA >= 2 ? 2 : 1), REG, DYN, false>(vb, variant);
    return async_ref_b<1, REG, DYN, false>(vb, variant);
  }
}

template <int VA, int VB, bool BETA, bool STREAM, bool FAST>
static cudaError_t launch_tile(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                               cudaStream_t stream, int blocks) {
  TA al;
  std::memcpy(&al, alpha, sizeof(TA));
  TB be;
  std::memset(&be, 0, sizeof(TB));
  if (BETA) std::memcpy(&be, beta, sizeof(TB));
  const TileDesc* d = reinterpret_cast<const TileDesc*>(p->dev_desc);
  if (FAST)
    tile_fast_kernel<TA, TB, VA, VB, BETA, STREAM><<<blocks, kThreads, p->smem_fast, stream>>>(
        d, static_cast<const TA*>(A), static_cast<TB*>(B), al, be);
  else
    tile_kernel<TA, TB, VA, VB, BETA, STREAM><<<blocks, kThreads, p->smem_bytes, stream>>>(
        d, static_cast<const TA*>(A), static_cast<TB*>(B), al, be);
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

template <int VA, int VB, bool FAST>
static KernelRef tile_ref(int variant) {
  KernelRef r;
  if (variant == 2) {
    r.fn = &launch_tile<VA, VB, true, false, FAST>;
    r.func = FAST ? reinterpret_cast<const void*>(&tile_fast_kernel<TA, TB, VA, VB, true, false>)
                  : reinterpret_cast<const void*>(&tile_kernel<TA, TB, VA, VB, true, false>);
  } else if (variant == 1) {
    r.fn = &launch_tile<VA, VB, false, true, FAST>;
    r.func = FAST ? reinterpret_cast<const void*>(&tile_fast_kernel<TA, TB, VA, VB, false, true>)
                  : reinterpret_cast<const void*>(&tile_kernel<TA, TB, VA, VB, false, true>);
  } else {
    r.fn = &launch_tile<VA, VB, false, false, FAST>;
    r.func = FAST ? reinterpret_cast<const void*>(&tile_fast_kernel<TA, TB, VA, VB, false, false>)
                  : reinterpret_cast<const void*>(&tile_kernel<TA, TB, VA, VB, false, false>);
  }
  return r;
}

template <int VA, bool FAST>
static KernelRef tile_ref_b(int vb, int variant) {
  constexpr int MB = 16 / sizeof(TB);
  if (vb >= 4 && MB >= 4) return tile_ref<VA, (MB >= 4 ? 4 : 1), FAST>(variant);
  if (vb >= 2 && MB >= 2) return tile_ref<VA, (MB >= 2 ? 2 : 1), FAST>(variant);
  return tile_ref<VA, 1, FAST>(variant);
}

template <bool FAST>
static KernelRef tile_ref_ab(int va, int vb, int variant) {
  constexpr int MA = 16 / sizeof(TA);
  if (va >= 4 && MA >= 4) return tile_ref_b<(MA >= 4 ? 4 : 1), FAST>(vb, variant);
  if (va >= 2 && MA >= 2) return tile_ref_b<(MA >= 2 ? 2 : 1), FAST>(vb, variant);
  return tile_ref_b<1, FAST>(vb, variant);
}

template <bool BETA, bool STREAM>
static cudaError_t launch_ragged(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                                 cudaStream_t stream, int blocks) {
  TA al;
  std::memcpy(&al, alpha, sizeof(TA));
  TB be;
  std::memset(&be, 0, sizeof(TB));
  if (BETA) std::memcpy(&be, beta, sizeof(TB));
  tile_ragged_kernel<TA, TB, BETA, STREAM><<<blocks, kThreads, p->smem_ragged, stream>>>(
      reinterpret_cast<const TileDesc*>(p->dev_desc), static_cast<const TA*>(A), static_cast<TB*>(B), al, be);
  return cudaGetLastError();
}

static KernelRef ragged_ref(int variant) {
  KernelRef r;
  if (variant == 2) {
    r.fn = &launch_ragged<true, false>;
    r.func = reinterpret_cast<const void*>(&tile_ragged_kernel<TA, TB, true, false>);
  } else if (variant == 1) {
    r.fn = &launch_ragged<false, true>;
    r.func = reinterpret_cast<const void*>(&tile_ragged_kernel<TA, TB, false, true>);
  } else {
    r.fn = &launch_ragged<false, false>;
    r.func = reinterpret_cast<const void*>(&tile_ragged_kernel<TA, TB, false, false>);
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
    const int v = va < vb ? va : vb;
    if (v >= 4 && MR >= 4) return row_ref<(MR >= 4 ? 4 : 1)>(variant);
    if (v >= 2 && MR >= 2) return row_ref<(MR >= 2 ? 2 : 1)>(variant);
    return row_ref<1>(variant);
  }
  if (kernel == TTCB_KERNEL_TILE_FAST) return tile_ref_ab<true>(va, vb, variant);
  if (kernel == TTCB_KERNEL_TILE_ASYNC) return async_ref_ab<false, false, false>(va, vb, variant);
  if (kernel == TTCB_KERNEL_TILE_ASYNC_REG) return async_ref_ab<true, false, false>(va, vb, variant);
  if (kernel == TTCB_KERNEL_TILE_ASYNC_DYN) return async_ref_ab<false, true, false>(va, vb, variant);
  if (kernel == TTCB_KERNEL_TILE_ASYNC_REG_DYN) return async_ref_ab<true, true, false>(va, vb, variant);
  if (kernel == (TTCB_KERNEL_TILE_ASYNC | TTCB_KERNEL_BULK_FLAG)) return async_ref_ab<false, false, true>(va, vb, variant);
  if (kernel == (TTCB_KERNEL_TILE_ASYNC_REG | TTCB_KERNEL_BULK_FLAG)) return async_ref_ab<true, false, true>(va, vb, variant);
  if (kernel == (TTCB_KERNEL_TILE_ASYNC_DYN | TTCB_KERNEL_BULK_FLAG)) return async_ref_ab<false, true, true>(va, vb, variant);
  if (kernel == (TTCB_KERNEL_TILE_ASYNC_REG_DYN | TTCB_KERNEL_BULK_FLAG))
    return async_ref_ab<true, true, true>(va, vb, variant);
  if (kernel == TTCB_KERNEL_TILE_RAGGED) return ragged_ref(variant);
  return tile_ref_ab<false>(va, vb, variant);
}

template <bool BETA, bool STREAM>
static cudaError_t launch_batch(const void* probs, const int64_t* prefix, int count, unsigned long long total,
                                unsigned long long* counter, int* status, const void* alpha, const void* beta,
                                int blocks, int smem, int slots_bytes, int chunk, cudaStream_t stream) {
  TA al;
  std::memcpy(&al, alpha, sizeof(TA));
  TB be;
  std::memset(&be, 0, sizeof(TB));
  if (BETA) std::memcpy(&be, beta, sizeof(TB));
  batch_kernel<TA, TB, BETA, STREAM><<<blocks, kThreads, smem, stream>>>(
      static_cast<const BatchProblem*>(probs), prefix, count, total, counter, status, al, be, slots_bytes, chunk);
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
