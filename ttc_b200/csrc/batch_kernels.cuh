// Batched mode: thousands of independent transpositions in one persistent launch.
//
// Every problem keeps the schedule of its own plan (tile shape, access widths, loop order). Work
// items are numbered globally: problem i owns items [prefix[i], prefix[i+1]) - one tile for a tile
// plan, one group of 8 row units (one per warp) for a row plan. CTAs claim items from one atomic
// counter, so long and short problems balance across the GPU. Nothing waits on another CTA.
#pragma once
#include "kernels.cuh"

namespace ttcb {

struct BatchProblem {
  const void* A;
  void* B;
  const unsigned char* desc;  // TileDesc or RowDesc, followed by its tables (device memory)
  int32_t kind;               // TTCB_KERNEL_TILE / TTCB_KERNEL_ROW
  int32_t va, vb;             // access widths for this problem (1 = scalar)
  int32_t pad_;
};

// Batch status codes written by the device (0 = ok).
enum { kBatchBadItem = 1 };

template <typename TA, typename TB, bool BETA, bool STREAM>
__device__ __forceinline__ void batch_tile(const BatchProblem& bp, uint32_t t, TA alpha, TB beta, TA* tile) {
  const TileDesc& d = *reinterpret_cast<const TileDesc*>(bp.desc);
  const TileTables tt{reinterpret_cast<const int64_t*>(bp.desc + d.off_segA),
                      reinterpret_cast<const int64_t*>(bp.desc + d.off_segB),
                      reinterpret_cast<const uint16_t*>(bp.desc + d.off_perm)};
  const TA* A = static_cast<const TA*>(bp.A);
  TB* B = static_cast<TB*>(bp.B);
  constexpr int MA = 16 / sizeof(TA);
  constexpr int MB = 16 / sizeof(TB);
  // the widest access each side allows (16 bytes) or scalar; narrower plans run scalar here
  if (bp.va == MA && bp.vb == MB)
    tile_body<TA, TB, MA, MB, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
  else if (bp.va == MA)
    tile_body<TA, TB, MA, 1, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
  else if (bp.vb == MB)
    tile_body<TA, TB, 1, MB, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
  else
    tile_body<TA, TB, 1, 1, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
}

template <typename TA, typename TB, bool BETA, bool STREAM>
__device__ __forceinline__ void batch_row(const BatchProblem& bp, uint32_t item, TA alpha, TB beta) {
  const RowDesc& d = *reinterpret_cast<const RowDesc*>(bp.desc);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t u = item * (kThreads / 32) + warp;
  if (u >= (uint32_t)d.nunits) return;
  constexpr int MA = 16 / sizeof(TA);
  constexpr int MB = 16 / sizeof(TB);
  constexpr int MR = MA < MB ? MA : MB;
  const TA* A = static_cast<const TA*>(bp.A);
  TB* B = static_cast<TB*>(bp.B);
  if (bp.va == MR && bp.vb == MR)
    row_unit<TA, TB, MR, BETA, STREAM>(d, u, A, B, alpha, beta, lane);
  else
    row_unit<TA, TB, 1, BETA, STREAM>(d, u, A, B, alpha, beta, lane);
}

// counter[0]: next work item (zeroed before every launch); status[0]: first error code.
template <typename TA, typename TB, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 3) batch_kernel(const BatchProblem* __restrict__ probs,
                                                         const int64_t* __restrict__ prefix, int count,
                                                         unsigned long long total, unsigned long long* counter,
                                                         int* status, TA alpha, TB beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TA* tile = reinterpret_cast<TA*>(smem_raw);
  __shared__ unsigned long long s_item;
  __shared__ int s_prob;
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned long long it = atomicAdd(counter, 1ull);
      int pr = -1;
      unsigned long long local = 0;
      if (it < total) {
        // largest pr with prefix[pr] <= it (problems with no items have equal prefixes)
        int lo = 0, hi = count - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if ((unsigned long long)prefix[mid] <= it)
            lo = mid;
          else
            hi = mid - 1;
        }
        pr = lo;
        local = it - (unsigned long long)prefix[pr];
        if (local >= (unsigned long long)(prefix[pr + 1] - prefix[pr])) {
          atomicCAS(status, 0, (int)kBatchBadItem);
          pr = -1;
        }
      }
      s_item = local;
      s_prob = pr;
    }
    __syncthreads();
    const int pr = s_prob;
    const uint32_t item = (uint32_t)s_item;
    __syncthreads();
    if (pr < 0) break;
    const BatchProblem& bp = probs[pr];
    if (bp.kind == TTCB_KERNEL_TILE)
      batch_tile<TA, TB, BETA, STREAM>(bp, item, alpha, beta, tile);
    else
      batch_row<TA, TB, BETA, STREAM>(bp, item, alpha, beta);
  }
}

}  // namespace ttcb
