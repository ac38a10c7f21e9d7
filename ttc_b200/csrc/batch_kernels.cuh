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
  int32_t full_only;          // tile problem: items are its complete tiles only (edge plans, problems
                              // of their own, move its ragged tiles)
};

// Stage buffers of the batched kernel's tile pipeline (tiles in flight ahead of the one written out:
// kBatchStages - 1).
#ifndef TTCB_BATCH_STAGES
#define TTCB_BATCH_STAGES 2
#endif
constexpr int kBatchStages = TTCB_BATCH_STAGES;
static_assert(kBatchStages == 2 || kBatchStages == 3, "the pending-tile queue holds at most two tiles");

// Batch status codes written by the device (0 = ok).
enum { kBatchBadItem = 1 };

// Complete tiles of a batched tile problem go through a two-buffer asynchronous-copy pipeline: the
// A tile is copied into shared memory in A order (element p at p + (p / sigmaA) * padA, the plan's
// staged layout) while the previous tile is written out in B order through the gather table. Each
// access-width variant is a call of its own, so their register allocations stay separate.
template <typename TA, int VA>
__device__ __noinline__ void batch_stage_issue(const TileDesc& d, const int64_t* segA, const TA* __restrict__ At,
                                               uint32_t stage) {
  const int P = d.P, LA = d.LA, padA = d.padA;
  for (int i = threadIdx.x; i < P / VA; i += kThreads) {
    const int p = i * VA;
    const int s = (int)fdiv((uint32_t)p, d.divLA);
    const int sp = (int)fdiv((uint32_t)p, d.divSigmaA);
    cp_async<VA * sizeof(TA)>(stage + (uint32_t)((p + sp * padA) * sizeof(TA)), At + (segA[s] + (p - s * LA)));
  }
}

template <typename TA, typename TB, int VB, bool BETA, bool STREAM>
__device__ __noinline__ void batch_stage_store(const TileDesc& d, const int64_t* segB, const uint16_t* gtab,
                                               TB* __restrict__ Bt, TA alpha, TB beta, const TA* st) {
  const int P = d.P, LB = d.LB;
  constexpr int U = 2;  // B vectors per thread in flight
  for (int i0 = threadIdx.x; i0 < P / VB; i0 += kThreads * U) {
    TB* dst[U];
    Vec<TB, VB> bv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * kThreads;
      dst[u] = nullptr;
      if (i < P / VB) {
        const int q = i * VB;
        const int s = (int)fdiv((uint32_t)q, d.divLB);
        dst[u] = Bt + (segB[s] + (q - s * LB));
        if (BETA) bv[u] = ld_stream<TB, VB>(dst[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!dst[u]) continue;
      const int q = (i0 + u * kThreads) * VB;
      uint16_t pos[VB];
      ld_u16s<TA, VB>(gtab + q, pos);
      Vec<TB, VB> out;
#pragma unroll
      for (int j = 0; j < VB; ++j) {
        const TA tj = scale_a(alpha, st[pos[j]]);
        if (BETA)
          out.v[j] = combine<TA, TB>(tj, bv[u].v[j], beta);
        else
          out.v[j] = finish<TA, TB>(tj);
      }
      st_vec<TB, VB>(dst[u], out, STREAM);
    }
  }
}

// A ragged tile (last block of a blocked dimension), element-wise, as a call of its own.
template <typename TA, typename TB, bool BETA, bool STREAM>
__device__ __noinline__ void batch_ragged(const TileDesc& d, TileTables tt, int lim0, int lim1,
                                          const TA* __restrict__ At, TB* __restrict__ Bt, TA alpha, TB beta,
                                          TA* tile) {
  const int lim[2] = {lim0, lim1};
  tile_ragged<TA, TB, BETA, STREAM>(d, tt, lim, At, Bt, alpha, beta, tile);
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
// advances along the prefix array. When it moves to a tile problem it copies that problem's
// descriptor header and run and gather tables into shared memory (after kBatchStages stage buffers
// of `slots_bytes` each) and pipelines the problem's consecutive complete tiles.
template <typename TA, typename TB, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 3) batch_kernel(const BatchProblem* __restrict__ probs,
                                                         const int64_t* __restrict__ prefix, int count,
                                                         unsigned long long total, unsigned long long* counter,
                                                         int* status, TA alpha, TB beta, int slots_bytes, int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ TileDesc d;
  __shared__ unsigned long long s_item;
  __shared__ int s_prob;
  constexpr int MA = 16 / sizeof(TA);
  constexpr int MB = 16 / sizeof(TB);
  const uint32_t stage0 = smem_u32(smem_raw);
  int64_t* segA = reinterpret_cast<int64_t*>(smem_raw + kBatchStages * slots_bytes);
  int64_t* segB = segA;
  uint16_t* gtab = nullptr;
  int cur = -1;  // problem whose header and tables are in shared memory
  const BatchProblem* bp = nullptr;
  // complete tiles whose copies are in flight, oldest first (at most kBatchStages - 1): B base and
  // stage buffer of each
  int npend = 0, next_buf = 0;
  int64_t pend_bB[2] = {0, 0};
  int pend_buf[2] = {0, 0};

  // writes out the oldest pending tile once its copies (and no newer ones: `newer` stay in flight)
  // have landed
  auto store_oldest = [&](int newer) {
    if (newer >= 2)
      cp_async_wait<2>();
    else if (newer == 1)
      cp_async_wait<1>();
    else
      cp_async_wait<0>();
    __syncthreads();
    TB* Bt = static_cast<TB*>(bp->B) + pend_bB[0];
    const TA* st = reinterpret_cast<const TA*>(smem_raw + pend_buf[0] * slots_bytes);
    if (bp->vb == MB)
      batch_stage_store<TA, TB, MB, BETA, STREAM>(d, segB, gtab, Bt, alpha, beta, st);
    else
      batch_stage_store<TA, TB, 1, BETA, STREAM>(d, segB, gtab, Bt, alpha, beta, st);
    __syncthreads();
    pend_bB[0] = pend_bB[1];
    pend_buf[0] = pend_buf[1];
    --npend;
  };
  auto flush = [&]() {
    while (npend > 0) store_oldest(npend - 1);
  };

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
      if (probs[pr].kind != TTCB_KERNEL_TILE) {
        flush();
        batch_row<TA, TB, BETA, STREAM>(probs[pr], local, alpha, beta);
        continue;
      }
      if (pr != cur) {
        flush();  // the pending tile belongs to the previous problem and its tables
        bp = &probs[pr];
        const TileDesc* gd = reinterpret_cast<const TileDesc*>(bp->desc);
        for (int i = threadIdx.x; i < (int)(sizeof(TileDesc) / 4); i += kThreads)
          reinterpret_cast<uint32_t*>(&d)[i] = reinterpret_cast<const uint32_t*>(gd)[i];
        __syncthreads();
        segB = segA + d.nsegA;
        gtab = reinterpret_cast<uint16_t*>(segB + d.nsegB);
        const int64_t* gA = reinterpret_cast<const int64_t*>(bp->desc + d.off_segA);
        const int64_t* gB = reinterpret_cast<const int64_t*>(bp->desc + d.off_segB);
        const uint32_t* gG = reinterpret_cast<const uint32_t*>(bp->desc + d.off_gtab);
        for (int i = threadIdx.x; i < d.nsegA; i += kThreads) segA[i] = gA[i];
        for (int i = threadIdx.x; i < d.nsegB; i += kThreads) segB[i] = gB[i];
        for (int i = threadIdx.x; i < (d.P + 1) / 2; i += kThreads) reinterpret_cast<uint32_t*>(gtab)[i] = gG[i];
        __syncthreads();
        cur = pr;
      }
      int64_t bA, bB;
      int lim[2];
      bool full = true;
      if (bp->full_only)
        decode_full_tile(d, local, bA, bB);
      else
        full = decode_tile(d, local, bA, bB, lim);
      const TA* A = static_cast<const TA*>(bp->A);
      if (full) {
        // the buffer after the newest pending one is free: its previous tile was written out
        // (followed by a barrier) before the pipeline last held kBatchStages - 1 tiles
        const int b = next_buf;
        next_buf = next_buf + 1 == kBatchStages ? 0 : next_buf + 1;
        if (bp->va == MA)
          batch_stage_issue<TA, MA>(d, segA, A + bA, stage0 + b * slots_bytes);
        else
          batch_stage_issue<TA, 1>(d, segA, A + bA, stage0 + b * slots_bytes);
        cp_async_commit();
        if (npend == kBatchStages - 1) store_oldest(kBatchStages - 1);
        if (npend == 0) {  // constant indices keep the queue in registers
          pend_bB[0] = bB;
          pend_buf[0] = b;
        } else {
          pend_bB[1] = bB;
          pend_buf[1] = b;
        }
        ++npend;
      } else {
        flush();
        const TileTables tt{segA, segB, reinterpret_cast<const uint16_t*>(bp->desc + d.off_perm)};
        batch_ragged<TA, TB, BETA, STREAM>(d, tt, lim[0], lim[1], A + bA, static_cast<TB*>(bp->B) + bB, alpha, beta,
                                           reinterpret_cast<TA*>(smem_raw));
      }
    }
    flush();
  }
}

}  // namespace ttcb
