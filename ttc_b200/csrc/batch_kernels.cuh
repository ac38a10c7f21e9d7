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

// Stage buffers of the batched kernel's tile ring: kBatchStages - 2 tiles of copies in flight ahead of
// the one written out, one CTA barrier per tile (the staged kernel's pipeline).
#ifndef TTCB_BATCH_STAGES
#define TTCB_BATCH_STAGES 3
#endif
constexpr int kBatchStages = TTCB_BATCH_STAGES;
static_assert(kBatchStages == 3 || kBatchStages == 4, "one or two tiles of copies in flight");
constexpr int kBatchAhead = kBatchStages - 2;

// Batch status codes written by the device (0 = ok).
enum { kBatchBadItem = 1 };

// A ragged tile (last block of a blocked dimension), element-wise, as a call of its own so that its
// registers stay apart from the ring's.
template <typename TA, typename TB, bool BETA, bool STREAM>
__device__ __noinline__ void batch_ragged(const TileDesc& d, TileTables tt, int lim0, int lim1,
                                          const TA* __restrict__ At, TB* __restrict__ Bt, TA alpha, TB beta,
                                          TA* tile) {
  const int lim[2] = {lim0, lim1};
  tile_ragged<TA, TB, BETA, STREAM>(d, tt, lim, At, Bt, alpha, beta, tile);
}

// The tiles [t0, t1) of one batched tile problem, whose descriptor header `d` and run and gather
// tables are in shared memory. Complete tiles go through the ring: the A tile is copied into a stage
// in A order (element p at p + (p / sigmaA) * padA, the plan's staged layout) while an earlier tile
// is written out in B order through the gather table. Each thread computes its tile-relative
// offsets once per call when they fit registers (beta = 0, P / VA and P / VB at most kRegVec *
// kThreads, the plan's staged bytes within 16 bits: the staged kernel's register path), else per
// vector from the run tables. A ragged tile empties the ring and goes element-wise. Every access-width pair is a
// function of its own, so that register allocations stay separate.
template <typename TA, typename TB, int VA, int VB, bool BETA, bool STREAM>
__device__ __noinline__ void batch_tiles(const TileDesc& d, const int64_t* segA, const int64_t* segB,
                                         const uint16_t* gtab, const uint16_t* gperm, const TA* __restrict__ A,
                                         TB* __restrict__ B, uint32_t t0, uint32_t t1, bool full_only, TA alpha,
                                         TB beta, unsigned char* smem_raw, int slots_bytes) {
  const int tid = threadIdx.x;
  const int P = d.P, LA = d.LA, LB = d.LB, padA = d.padA;
  const int nvA = P / VA, nvB = P / VB;
  // (with beta != 0 the register path's extra B stream spills the 128-register budget: table path)
  const bool reg = !BETA && d.reg_ok && nvA <= kRegVec * kThreads && nvB <= kRegVec * kThreads;
  const uint32_t stage0 = smem_u32(smem_raw);
  // register path: A source offsets, staged byte offsets (two per register), B offsets, gather byte
  // offsets (two per register) of the thread's vectors u = tid + k * kThreads
  int32_t rA[kRegVec], rB[kRegVec];
  uint32_t dA[kRegVec / 2];
  constexpr int kGp = (kRegVec * VB + 1) / 2;
  uint32_t gp[kGp];
#pragma unroll
  for (int e = 0; e < kGp; ++e) gp[e] = 0;
#pragma unroll
  for (int u = 0; u < kRegVec; ++u) {
    rA[u] = rB[u] = 0;
    if (!(u & 1)) dA[u >> 1] = 0;
  }
  if (reg) {
#pragma unroll
    for (int u = 0; u < kRegVec; ++u) {
      const int i = tid + u * kThreads;
      if (i < nvA) {
        const int p = i * VA;
        const int sg = (int)fdiv((uint32_t)p, d.divLA);
        const int sp = (int)fdiv((uint32_t)p, d.divSigmaA);
        rA[u] = (int32_t)(segA[sg] + (p - sg * LA));
        dA[u >> 1] |= ((uint32_t)(p + sp * padA) * (uint32_t)sizeof(TA)) << ((u & 1) * 16);
      }
      if (i < nvB) {
        const int q = i * VB;
        const int sg = (int)fdiv((uint32_t)q, d.divLB);
        rB[u] = (int32_t)(segB[sg] + (q - sg * LB));
#pragma unroll
        for (int j = 0; j < VB; ++j) {
          const int e = u * VB + j;
          const uint32_t v = (uint32_t)gtab[q + j] * (uint32_t)sizeof(TA);
          gp[e >> 1] |= (e & 1) ? (v << 16) : v;
        }
      }
    }
  }

  auto issue = [&](int64_t bA, int stage) {
    const TA* At = A + bA;
    const uint32_t sb = stage0 + (uint32_t)(stage * slots_bytes);
    if (reg) {
#pragma unroll
      for (int u = 0; u < kRegVec; ++u)
        if (tid + u * kThreads < nvA)
          cp_async<VA * sizeof(TA)>(sb + ((dA[u >> 1] >> ((u & 1) * 16)) & 0xffffu), At + rA[u]);
    } else {
      for (int i = tid; i < nvA; i += kThreads) {
        const int p = i * VA;
        const int sg = (int)fdiv((uint32_t)p, d.divLA);
        const int sp = (int)fdiv((uint32_t)p, d.divSigmaA);
        cp_async<VA * sizeof(TA)>(sb + (uint32_t)((p + sp * padA) * sizeof(TA)), At + (segA[sg] + (p - sg * LA)));
      }
    }
  };
  // one B vector: gather VB staged elements (byte offsets from the stage base), scale, combine, store
  auto out_vec = [&](const unsigned char* st, const uint32_t* off, TB* dst, const Vec<TB, VB>& bv) {
    Vec<TB, VB> out;
#pragma unroll
    for (int j = 0; j < VB; ++j) {
      const TA tj = scale_a(alpha, *reinterpret_cast<const TA*>(st + off[j]));
      if (BETA)
        out.v[j] = combine<TA, TB>(tj, bv.v[j], beta);
      else
        out.v[j] = finish<TA, TB>(tj);
    }
    st_vec<TB, VB>(dst, out, STREAM);
  };
  auto store = [&](int64_t bB, int stage) {
    TB* Bt = B + bB;
    const unsigned char* st = smem_raw + stage * slots_bytes;
    if (reg) {
      // two B vectors at a time: their B reads (beta) in flight together
#pragma unroll
      for (int u0 = 0; u0 < kRegVec; u0 += 2) {
        Vec<TB, VB> bv[2];
        if (BETA) {
#pragma unroll
          for (int k = 0; k < 2; ++k)
            if (tid + (u0 + k) * kThreads < nvB) bv[k] = ld_stream<TB, VB>(Bt + rB[u0 + k]);
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int u = u0 + k;
          if (tid + u * kThreads < nvB) {
            uint32_t off[VB];
#pragma unroll
            for (int j = 0; j < VB; ++j) {
              const int e = u * VB + j;
              off[j] = (e & 1) ? (gp[e >> 1] >> 16) : (gp[e >> 1] & 0xffffu);
            }
            out_vec(st, off, Bt + rB[u], bv[k]);
          }
        }
      }
    } else {
      constexpr int U = 2;  // B vectors per thread in flight
      for (int i0 = tid; i0 < nvB; i0 += kThreads * U) {
        TB* dst[U];
        Vec<TB, VB> bv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int i = i0 + u * kThreads;
          dst[u] = nullptr;
          if (i < nvB) {
            const int q = i * VB;
            const int sg = (int)fdiv((uint32_t)q, d.divLB);
            dst[u] = Bt + (segB[sg] + (q - sg * LB));
            if (BETA) bv[u] = ld_stream<TB, VB>(dst[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (!dst[u]) continue;
          const int q = (i0 + u * kThreads) * VB;
          uint16_t pos[VB];
          ld_u16s<TA, VB>(gtab + q, pos);
          uint32_t off[VB];
#pragma unroll
          for (int j = 0; j < VB; ++j) off[j] = (uint32_t)pos[j] * (uint32_t)sizeof(TA);
          out_vec(st, off, dst[u], bv[u]);
        }
      }
    }
  };

  // tiles issued and not yet written out, oldest first (at most kBatchAhead + 1 while a tile is
  // being pushed): B base and stage of each
  int npend = 0, next_stage = 0;
  int64_t pend_bB[kBatchAhead + 1];
  int pend_st[kBatchAhead + 1];
#pragma unroll
  for (int k = 0; k <= kBatchAhead; ++k) {
    pend_bB[k] = 0;
    pend_st[k] = 0;
  }
  // writes out the oldest pending tile once its copies have landed (`newer` copies stay in flight);
  // the barrier also tells every thread that the tile written out before it is done with its stage
  auto store_oldest = [&](int newer) {
    if (newer >= 2)
      cp_async_wait<2>();
    else if (newer == 1)
      cp_async_wait<1>();
    else
      cp_async_wait<0>();
    __syncthreads();
    store(pend_bB[0], pend_st[0]);
#pragma unroll
    for (int k = 0; k < kBatchAhead; ++k) {
      pend_bB[k] = pend_bB[k + 1];
      pend_st[k] = pend_st[k + 1];
    }
    --npend;
  };
  for (uint32_t t = t0; t < t1; ++t) {
    int64_t bA, bB;
    int lim[2];
    bool full = true;
    if (full_only)
      decode_full_tile(d, t, bA, bB);
    else
      full = decode_tile(d, t, bA, bB, lim);
    if (!full) {
      while (npend > 0) store_oldest(npend - 1);
      __syncthreads();  // the element-wise path reuses the stage buffers
      const TileTables tt{segA, segB, gperm};
      batch_ragged<TA, TB, BETA, STREAM>(d, tt, lim[0], lim[1], A + bA, B + bB, alpha, beta,
                                         reinterpret_cast<TA*>(smem_raw));
      next_stage = 0;
      continue;
    }
    // stage next_stage last held the tile written out kBatchAhead + 1 tiles ago, before the barrier
    // of the following one
    issue(bA, next_stage);
    cp_async_commit();
#pragma unroll
    for (int k = 0; k <= kBatchAhead; ++k)
      if (k == npend) {
        pend_bB[k] = bB;
        pend_st[k] = next_stage;
      }
    ++npend;
    next_stage = next_stage + 1 == kBatchStages ? 0 : next_stage + 1;
    if (npend > kBatchAhead) store_oldest(kBatchAhead);
  }
  while (npend > 0) store_oldest(npend - 1);
  __syncthreads();  // the caller may reuse the tables and the stages
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
// A CTA claims `chunk` consecutive items per atomic and walks them in order, a problem at a time; the
// problem index advances along the prefix array. When it moves to a tile problem it copies that
// problem's descriptor header and run and gather tables into shared memory (after kBatchStages
// stage buffers of `slots_bytes` each) and runs the problem's claimed tiles through batch_tiles.
template <typename TA, typename TB, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 2) batch_kernel(const BatchProblem* __restrict__ probs,
                                                         const int64_t* __restrict__ prefix, int count,
                                                         unsigned long long total, unsigned long long* counter,
                                                         int* status, TA alpha, TB beta, int slots_bytes, int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ TileDesc d;
  __shared__ unsigned long long s_item;
  __shared__ int s_prob;
  constexpr int MA = 16 / sizeof(TA);
  constexpr int MB = 16 / sizeof(TB);
  constexpr int HA = MA >= 2 ? MA / 2 : 1;  // the half-width vectors (8 bytes) where they differ
  constexpr int HB = MB >= 2 ? MB / 2 : 1;
  int64_t* segA = reinterpret_cast<int64_t*>(smem_raw + kBatchStages * slots_bytes);
  int64_t* segB = segA;
  uint16_t* gtab = nullptr;
  int cur = -1;  // problem whose header and tables are in shared memory

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
    for (unsigned long long it = it0; it < end;) {
      while (pr < count - 1 && (unsigned long long)prefix[pr + 1] <= it) ++pr;
      const unsigned long long pend = (unsigned long long)prefix[pr + 1];
      if (it < (unsigned long long)prefix[pr] || it >= pend) {
        if (threadIdx.x == 0) atomicCAS(status, 0, (int)kBatchBadItem);
        ++it;
        continue;
      }
      const unsigned long long seg_end = end < pend ? end : pend;
      const uint32_t l0 = (uint32_t)(it - (unsigned long long)prefix[pr]);
      const uint32_t l1 = (uint32_t)(seg_end - (unsigned long long)prefix[pr]);
      it = seg_end;
      const BatchProblem& bp = probs[pr];
      if (bp.kind != TTCB_KERNEL_TILE) {
        for (uint32_t local = l0; local < l1; ++local) batch_row<TA, TB, BETA, STREAM>(bp, local, alpha, beta);
        continue;
      }
      if (pr != cur) {
        const TileDesc* gd = reinterpret_cast<const TileDesc*>(bp.desc);
        for (int i = threadIdx.x; i < (int)(sizeof(TileDesc) / 4); i += kThreads)
          reinterpret_cast<uint32_t*>(&d)[i] = reinterpret_cast<const uint32_t*>(gd)[i];
        __syncthreads();
        segB = segA + d.nsegA;
        gtab = reinterpret_cast<uint16_t*>(segB + d.nsegB);
        const int64_t* gA = reinterpret_cast<const int64_t*>(bp.desc + d.off_segA);
        const int64_t* gB = reinterpret_cast<const int64_t*>(bp.desc + d.off_segB);
        const uint32_t* gG = reinterpret_cast<const uint32_t*>(bp.desc + d.off_gtab);
        for (int i = threadIdx.x; i < d.nsegA; i += kThreads) segA[i] = gA[i];
        for (int i = threadIdx.x; i < d.nsegB; i += kThreads) segB[i] = gB[i];
        for (int i = threadIdx.x; i < (d.P + 1) / 2; i += kThreads) reinterpret_cast<uint32_t*>(gtab)[i] = gG[i];
        __syncthreads();
        cur = pr;
      }
      const TA* A = static_cast<const TA*>(bp.A);
      TB* B = static_cast<TB*>(bp.B);
      const uint16_t* gperm = reinterpret_cast<const uint16_t*>(bp.desc + d.off_perm);
      const bool fo = bp.full_only != 0;
      const int va = bp.va >= MA ? MA : (bp.va >= HA ? HA : 1);
      const int vb = bp.vb >= MB ? MB : (bp.vb >= HB ? HB : 1);
#define TTCB_BATCH_TILES(VA_, VB_) \
  batch_tiles<TA, TB, VA_, VB_, BETA, STREAM>(d, segA, segB, gtab, gperm, A, B, l0, l1, fo, alpha, beta, smem_raw, slots_bytes)
      if (va == MA) {
        if (vb == MB) TTCB_BATCH_TILES(MA, MB);
        else if (vb == HB) TTCB_BATCH_TILES(MA, HB);
        else TTCB_BATCH_TILES(MA, 1);
      } else if (va == HA) {
        if (vb == MB) TTCB_BATCH_TILES(HA, MB);
        else if (vb == HB) TTCB_BATCH_TILES(HA, HB);
        else TTCB_BATCH_TILES(HA, 1);
      } else {
        if (vb == MB) TTCB_BATCH_TILES(1, MB);
        else if (vb == HB) TTCB_BATCH_TILES(1, HB);
        else TTCB_BATCH_TILES(1, 1);
      }
#undef TTCB_BATCH_TILES
    }
  }
}

}  // namespace ttcb
