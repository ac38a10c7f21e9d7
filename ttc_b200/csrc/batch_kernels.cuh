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

// One access-width variant of the table-driven tile body as a call of its own: the batch kernel
// holds four of them and a row path, and separate register allocations keep them from spilling.
template <typename TA, typename TB, int VA, int VB, bool BETA, bool STREAM>
__device__ __noinline__ void batch_tile_body(const TileDesc& d, const TileTables& tt, uint32_t t,
                                             const TA* __restrict__ A, TB* __restrict__ B, TA alpha, TB beta,
                                             TA* tile) {
  tile_body<TA, TB, VA, VB, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
}

// One tile of a tile problem whose descriptor header (d) and tables (tt) are in shared memory.
template <typename TA, typename TB, bool BETA, bool STREAM>
__device__ __forceinline__ void batch_tile(const BatchProblem& bp, const TileDesc& d, const TileTables& tt, uint32_t t,
                                           TA alpha, TB beta, TA* tile) {
  const TA* A = static_cast<const TA*>(bp.A);
  TB* B = static_cast<TB*>(bp.B);
  constexpr int MA = 16 / sizeof(TA);
  constexpr int MB = 16 / sizeof(TB);
  // the widest access each side allows (16 bytes) or scalar; narrower plans run scalar here
  if (bp.va == MA && bp.vb == MB)
    batch_tile_body<TA, TB, MA, MB, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
  else if (bp.va == MA)
    batch_tile_body<TA, TB, MA, 1, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
  else if (bp.vb == MB)
    batch_tile_body<TA, TB, 1, MB, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
  else
    batch_tile_body<TA, TB, 1, 1, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
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
// A CTA claims `chunk` consecutive items per atomic and walks them in order; the problem index
// advances along the prefix array. A tile problem's descriptor header and run tables are copied
// into shared memory (after the `slots_bytes` tile buffer) when the CTA moves to it.
template <typename TA, typename TB, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 3) batch_kernel(const BatchProblem* __restrict__ probs,
                                                         const int64_t* __restrict__ prefix, int count,
                                                         unsigned long long total, unsigned long long* counter,
                                                         int* status, TA alpha, TB beta, int slots_bytes, int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TA* tile = reinterpret_cast<TA*>(smem_raw);
  __shared__ TileDesc d;
  __shared__ unsigned long long s_item;
  __shared__ int s_prob;
  int64_t* segA = reinterpret_cast<int64_t*>(smem_raw + slots_bytes);
  int cur = -1;  // problem whose header and tables are in shared memory
  TileTables tt{nullptr, nullptr, nullptr};
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned long long it = atomicAdd(counter, (unsigned long long)chunk);
      int pr = -1;
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
      }
      s_item = it;
      s_prob = pr;
    }
    __syncthreads();
    int pr = s_prob;
    const unsigned long long it0 = s_item;
    __syncthreads();
    if (pr < 0) break;
    const unsigned long long end = it0 + (unsigned long long)chunk < total ? it0 + (unsigned long long)chunk : total;
    for (unsigned long long it = it0; it < end; ++it) {
      while (pr < count - 1 && (unsigned long long)prefix[pr + 1] <= it) ++pr;
      const uint32_t local = (uint32_t)(it - (unsigned long long)prefix[pr]);
      if (local >= (uint32_t)(prefix[pr + 1] - prefix[pr])) {
        if (threadIdx.x == 0) atomicCAS(status, 0, (int)kBatchBadItem);
        continue;
      }
      const BatchProblem& bp = probs[pr];
      if (bp.kind == TTCB_KERNEL_TILE) {
        if (pr != cur) {
          // the previous tile ended with a barrier, so the old header and tables are free
          const TileDesc* gd = reinterpret_cast<const TileDesc*>(bp.desc);
          for (int i = threadIdx.x; i < (int)(sizeof(TileDesc) / 4); i += kThreads)
            reinterpret_cast<uint32_t*>(&d)[i] = reinterpret_cast<const uint32_t*>(gd)[i];
          __syncthreads();
          int64_t* sB = segA + d.nsegA;
          uint16_t* pt = reinterpret_cast<uint16_t*>(sB + d.nsegB);
          const int64_t* gA = reinterpret_cast<const int64_t*>(bp.desc + d.off_segA);
          const int64_t* gB = reinterpret_cast<const int64_t*>(bp.desc + d.off_segB);
          const uint32_t* gP = reinterpret_cast<const uint32_t*>(bp.desc + d.off_perm);
          for (int i = threadIdx.x; i < d.nsegA; i += kThreads) segA[i] = gA[i];
          for (int i = threadIdx.x; i < d.nsegB; i += kThreads) sB[i] = gB[i];
          for (int i = threadIdx.x; i < (d.P + 1) / 2; i += kThreads) reinterpret_cast<uint32_t*>(pt)[i] = gP[i];
          __syncthreads();
          tt = TileTables{segA, sB, pt};
          cur = pr;
        }
        batch_tile<TA, TB, BETA, STREAM>(bp, d, tt, local, alpha, beta, tile);
      } else {
        batch_row<TA, TB, BETA, STREAM>(bp, local, alpha, beta);
      }
    }
  }
}

}  // namespace ttcb
