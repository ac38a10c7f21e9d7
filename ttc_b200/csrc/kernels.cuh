// Device kernels of the transposition. Templated on the A/B element types, the access widths
// (VA elements per A load, VB per B store; 16 bytes when aligned) and the beta / streaming-store
// variants; the host picks an instantiation per plan and per call (pointer alignment).
//
// tile_body() processes one tile (see desc.h). It is shared by the plain persistent kernel, which
// stages the tile tables in shared memory once per CTA, and by the batched kernel, which reads the
// tables of whichever problem a work item belongs to through the read-only data path.
#pragma once
#include "common.cuh"
#include "desc.h"

namespace ttcb {

constexpr int kThreads = 256;  // threads per CTA (TTC's default threadsPerBlock, GPUtransposeGenerator.py:110)
constexpr int kUnroll = 4;     // independent global accesses in flight per thread and phase

// v[k] for a run-time k in [0, V): a select chain, so the vector stays in registers.
template <typename T, int V> __device__ __forceinline__ T vsel(const Vec<T, V>& v, int k) {
  T x = v.v[0];
#pragma unroll
  for (int i = 1; i < V; ++i)
    if (k == i) x = v.v[i];
  return x;
}

// Shared-memory slot of B-order position q (padding breaks power-of-two bank strides).
__device__ __forceinline__ int slot_of(int q, int pshift, int pad) { return q + ((q >> pshift) & -pad); }

// Decodes tile index t into A/B base offsets and the valid extents of blocked dimensions.
// Returns true when the tile is complete (no ragged edge).
__device__ __forceinline__ bool decode_tile(const TileDesc& d, uint32_t t, int64_t& bA, int64_t& bB, int* lim) {
  bA = 0;
  bB = 0;
  bool full = true;
  lim[0] = lim[1] = 0x7fffffff;
  const int ng = d.ngrid;
#pragma unroll 1  // a rolled loop keeps the callers' register budget
  for (int g = 0; g < ng; ++g) {
    const GridDimDesc& gd = d.g[g];
    const uint32_t q = fdiv(t, gd.div);
    const uint32_t blk = t - q * gd.div.d;
    t = q;
    bA += (int64_t)blk * gd.strideA;
    bB += (int64_t)blk * gd.strideB;
    if (gd.blocked >= 0) {
      const int64_t left = gd.n - (int64_t)blk * gd.e;
      const int l = left < gd.e ? (int)left : gd.e;
      if (gd.blocked == 0)  // constant indices keep lim[] in registers
        lim[0] = l;
      else
        lim[1] = l;
      if (l < gd.e) full = false;
    }
  }
  return full;
}

// Decodes complete-tile index t (numbered over the divf counts, which leave out the ragged last
// blocks) into A/B base offsets.
__device__ __forceinline__ void decode_full_tile(const TileDesc& d, uint32_t t, int64_t& bA, int64_t& bB) {
  bA = 0;
  bB = 0;
  const int ng = d.ngrid;
#pragma unroll 1  // a rolled loop keeps the callers' register budget
  for (int g = 0; g < ng; ++g) {
    const GridDimDesc& gd = d.g[g];
    const uint32_t q = fdiv(t, gd.divf);
    const uint32_t blk = t - q * gd.divf.d;
    t = q;
    bA += (int64_t)blk * gd.strideA;
    bB += (int64_t)blk * gd.strideB;
  }
}

struct TileTables {
  const int64_t* segA;
  const int64_t* segB;
  const uint16_t* ptab;
};

// out[j] = v[(j + r) mod V] for a run-time r in [0, V): two select stages, registers only.
template <typename T, int V> __device__ __forceinline__ Vec<T, V> rot_left(const Vec<T, V>& v, int r) {
  Vec<T, V> a = v;
  if constexpr (V >= 2) {
    Vec<T, V> b;
#pragma unroll
    for (int j = 0; j < V; ++j) b.v[j] = (r & 1) ? a.v[(j + 1) % V] : a.v[j];
    a = b;
  }
  if constexpr (V >= 4) {
    Vec<T, V> b;
#pragma unroll
    for (int j = 0; j < V; ++j) b.v[j] = (r & 2) ? a.v[(j + 2) % V] : a.v[j];
    a = b;
  }
  return a;
}

// Ragged tile (a blocked dimension's last block): element-wise, validity from the blocked
// dimensions' tile coordinates. Ends with a barrier.
template <typename TA, typename TB, bool BETA, bool STREAM>
__device__ __forceinline__ void tile_ragged(const TileDesc& d, const TileTables& tt, const int* lim, const TA* __restrict__ At,
                                         TB* __restrict__ Bt, TA alpha, TB beta, TA* tile) {
  const int tid = threadIdx.x;
  const int P = d.P, LA = d.LA, LB = d.LB;
  const int pshift = d.pshift, pad = d.pad;
  const int nb = d.nblocked;
  for (int p0 = tid; p0 < P; p0 += kThreads * kUnroll) {
    TA v[kUnroll];
    int slot[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int p = p0 + u * kThreads;
      slot[u] = -1;
      if (p < P) {
        bool ok = true;
        for (int b = 0; b < nb; ++b) {
          const uint32_t c = fdiv((uint32_t)p, d.bd[b].tsA);
          const uint32_t cc = c - fdiv(c, d.bd[b].ext) * d.bd[b].ext.d;
          ok = ok && ((int)cc < (b == 0 ? lim[0] : lim[1]));
        }
        if (ok) {
          const int s = (int)fdiv((uint32_t)p, d.divLA);
          v[u] = ld_scalar<TA>(At + (tt.segA[s] + (p - s * LA)));
          slot[u] = tt.ptab[p];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
      if (slot[u] >= 0) tile[slot[u]] = scale_a(alpha, v[u]);
  }
  __syncthreads();
  for (int q0 = tid; q0 < P; q0 += kThreads * kUnroll) {
    TB* dst[kUnroll];
    TB bv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int q = q0 + u * kThreads;
      dst[u] = nullptr;
      if (q < P) {
        bool ok = true;
        for (int b = 0; b < nb; ++b) {
          const uint32_t c = fdiv((uint32_t)q, d.bd[b].tsB);
          const uint32_t cc = c - fdiv(c, d.bd[b].ext) * d.bd[b].ext.d;
          ok = ok && ((int)cc < (b == 0 ? lim[0] : lim[1]));
        }
        if (ok) {
          const int s = (int)fdiv((uint32_t)q, d.divLB);
          dst[u] = Bt + (tt.segB[s] + (q - s * LB));
          if (BETA) bv[u] = ld_scalar<TB>(dst[u]);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (dst[u]) {
        const int q = q0 + u * kThreads;
        const TA tq = tile[slot_of(q, pshift, pad)];
        TB r;
        if (BETA)
          r = combine<TA, TB>(tq, bv[u], beta);
        else
          r = finish<TA, TB>(tq);
        st_scalar<TB>(dst[u], r, STREAM);
      }
    }
  }
  __syncthreads();
}

// One tile with the generic table-driven loops: load phase (A runs -> alpha*A -> shared slots in B
// order), barrier, store phase (shared slots -> B runs, with beta*B when BETA), barrier.
template <typename TA, typename TB, int VA, int VB, bool BETA, bool STREAM>
__device__ __forceinline__ void tile_body(const TileDesc& d, const TileTables& tt, uint32_t t, const TA* __restrict__ A,
                                          TB* __restrict__ B, TA alpha, TB beta, TA* tile) {
  const int tid = threadIdx.x;
  const int rot = (tid >> 3) & 3;  // lane-dependent access order (spreads shared-memory banks)
  const int P = d.P, LA = d.LA, LB = d.LB;
  const int pshift = d.pshift, pad = d.pad;
  int64_t bA, bB;
  int lim[2];
  const bool full = decode_tile(d, t, bA, bB, lim);
  const TA* At = A + bA;
  TB* Bt = B + bB;
  if (!full) {
    tile_ragged<TA, TB, BETA, STREAM>(d, tt, lim, At, Bt, alpha, beta, tile);
    return;
  }
  const int nvA = P / VA;
  for (int i0 = tid; i0 < nvA; i0 += kThreads * kUnroll) {
    Vec<TA, VA> v[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int i = i0 + u * kThreads;
      if (i < nvA) {
        const int p = i * VA;
        const int s = (int)fdiv((uint32_t)p, d.divLA);
        v[u] = ld_stream<TA, VA>(At + (tt.segA[s] + (p - s * LA)));
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int i = i0 + u * kThreads;
      if (i < nvA) {
        const int p = i * VA;
#pragma unroll
        for (int j = 0; j < VA; ++j) {
          const int jj = (j + rot) & (VA - 1);
          tile[tt.ptab[p + jj]] = scale_a(alpha, vsel<TA, VA>(v[u], jj));
        }
      }
    }
  }
  __syncthreads();
  const int nvB = P / VB;
  for (int i0 = tid; i0 < nvB; i0 += kThreads * kUnroll) {
    int64_t o[kUnroll];
    Vec<TB, VB> bv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int i = i0 + u * kThreads;
      if (i < nvB) {
        const int q = i * VB;
        const int s = (int)fdiv((uint32_t)q, d.divLB);
        o[u] = tt.segB[s] + (q - s * LB);
        if (BETA) bv[u] = ld_stream<TB, VB>(Bt + o[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int i = i0 + u * kThreads;
      if (i < nvB) {
        const int q = i * VB;
        Vec<TA, VB> tv;
#pragma unroll
        for (int j = 0; j < VB; ++j) {
          const int jj = (j + rot) & (VB - 1);
          tv.v[j] = tile[slot_of(q + jj, pshift, pad)];
        }
        Vec<TB, VB> out;
#pragma unroll
        for (int k = 0; k < VB; ++k) {
          const TA tk = vsel<TA, VB>(tv, (k - rot) & (VB - 1));
          if (BETA)
            out.v[k] = combine<TA, TB>(tk, bv[u].v[k], beta);
          else
            out.v[k] = finish<TA, TB>(tk);
        }
        st_vec<TB, VB>(Bt + o[u], out, STREAM);
      }
    }
  }
  __syncthreads();
}

// Shared-memory layout of the generic tile kernel: [tile slots][segA][segB][perm_tab].
__host__ __device__ inline size_t tile_slots_bytes(int phys_size, int elem_bytes) {
  return ((size_t)phys_size * elem_bytes + 15) & ~size_t(15);
}

template <typename TA, typename TB, int VA, int VB, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 4) tile_kernel(const TileDesc* __restrict__ desc, const TA* __restrict__ A,
                                                           TB* __restrict__ B, TA alpha, TB beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TileDesc& d = *desc;
  const int tid = threadIdx.x;
  TA* tile = reinterpret_cast<TA*>(smem_raw);
  int64_t* segA = reinterpret_cast<int64_t*>(smem_raw + tile_slots_bytes(d.phys_size, sizeof(TA)));
  int64_t* segB = segA + d.nsegA;
  uint16_t* ptab = reinterpret_cast<uint16_t*>(segB + d.nsegB);
  {
    const unsigned char* base = reinterpret_cast<const unsigned char*>(desc);
    const int64_t* gA = reinterpret_cast<const int64_t*>(base + d.off_segA);
    const int64_t* gB = reinterpret_cast<const int64_t*>(base + d.off_segB);
    const uint32_t* gP = reinterpret_cast<const uint32_t*>(base + d.off_perm);
    uint32_t* sP = reinterpret_cast<uint32_t*>(ptab);
    for (int i = tid; i < d.nsegA; i += kThreads) segA[i] = gA[i];
    for (int i = tid; i < d.nsegB; i += kThreads) segB[i] = gB[i];
    for (int i = tid; i < (d.P + 1) / 2; i += kThreads) sP[i] = gP[i];
  }
  __syncthreads();
  const TileTables tt{segA, segB, ptab};
  const uint32_t ntiles = (uint32_t)d.ntiles;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x)
    tile_body<TA, TB, VA, VB, BETA, STREAM>(d, tt, t, A, B, alpha, beta, tile);
}

// ------------------------------------------------------------------------------------------------
// Fast tile kernel. Each thread owns up to kMaxVec A-vectors and kMaxVec B-vectors of every tile;
// their tile-relative offsets and shared-memory slots do not depend on the tile, so they are
// computed once per CTA and kept in registers. The A loads of the next tile are issued before the
// store phase of the current one, so loads stay in flight across the barrier. Needs P/VA and P/VB
// <= kMaxVec * kThreads and 32-bit tile-relative offsets (TileDesc::fast).
constexpr int kMaxVec = 4;

template <typename TA, int VA>
__device__ __forceinline__ void fast_load(Vec<TA, VA>* va, const TA* __restrict__ At, const int32_t* relA) {
#pragma unroll
  for (int u = 0; u < kMaxVec; ++u)
    if (relA[u] >= 0) va[u] = ld_stream<TA, VA>(At + relA[u]);
}

template <typename TA, typename TB, int VA, int VB, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 3) tile_fast_kernel(const TileDesc* __restrict__ desc,
                                                                const TA* __restrict__ A, TB* __restrict__ B,
                                                                TA alpha, TB beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TA* tile = reinterpret_cast<TA*>(smem_raw);
  const TileDesc& d = *desc;
  const unsigned char* base = reinterpret_cast<const unsigned char*>(desc);
  const TileTables tt{reinterpret_cast<const int64_t*>(base + d.off_segA),
                      reinterpret_cast<const int64_t*>(base + d.off_segB),
                      reinterpret_cast<const uint16_t*>(base + d.off_perm)};
  const int tid = threadIdx.x;
  const int rotA = (tid >> 3) & (VA - 1);
  const int rotB = (tid >> 3) & (VB - 1);
  const int P = d.P, LA = d.LA, LB = d.LB;
  const int nvA = P / VA, nvB = P / VB;

  // tile-invariant per-thread offsets and slots (A-side slots in the thread's write order, two
  // 16-bit slots per register)
  constexpr int NSA = (VA + 1) / 2;
  int32_t relA[kMaxVec], relB[kMaxVec];
  uint32_t slA[kMaxVec][NSA];
#pragma unroll
  for (int u = 0; u < kMaxVec; ++u) {
    const int i = tid + u * kThreads;
    relA[u] = -1;
    if (i < nvA) {
      const int p = i * VA;
      const int s = p / LA;
      relA[u] = (int32_t)(tt.segA[s] + (p - s * LA));
#pragma unroll
      for (int j = 0; j < NSA; ++j) {
        const uint32_t lo = tt.ptab[p + ((2 * j + rotA) & (VA - 1))];
        const uint32_t hi = (2 * j + 1 < VA) ? tt.ptab[p + ((2 * j + 1 + rotA) & (VA - 1))] : 0u;
        slA[u][j] = lo | (hi << 16);
      }
    }
    relB[u] = -1;
    if (i < nvB) {
      const int q = i * VB;
      const int s = q / LB;
      relB[u] = (int32_t)(tt.segB[s] + (q - s * LB));
    }
  }
  const int pshift = d.pshift, pad = d.pad;

  const uint32_t ntiles = (uint32_t)d.ntiles;
  uint32_t t = blockIdx.x;
  int64_t bA = 0, bB = 0;
  int lim[2];
  Vec<TA, VA> va[kMaxVec];
  bool full = false;
  if (t < ntiles) {
    full = decode_tile(d, t, bA, bB, lim);
    if (full) fast_load<TA, VA>(va, A + bA, relA);
  }
  while (t < ntiles) {
    const uint32_t tn = t + gridDim.x;
    int64_t nA = 0, nB = 0;
    int nlim[2];
    bool nfull = false;
    if (full) {
#pragma unroll
      for (int u = 0; u < kMaxVec; ++u) {
        if (relA[u] >= 0) {
          const Vec<TA, VA> w = rot_left<TA, VA>(va[u], rotA);
#pragma unroll
          for (int j = 0; j < VA; ++j) {
            const uint32_t sl = (j & 1) ? (slA[u][j >> 1] >> 16) : (slA[u][j >> 1] & 0xffffu);
            tile[sl] = scale_a(alpha, w.v[j]);
          }
        }
      }
      __syncthreads();
      // next tile's A loads go out before this tile's stores
      if (tn < ntiles) {
        nfull = decode_tile(d, tn, nA, nB, nlim);
        if (nfull) fast_load<TA, VA>(va, A + nA, relA);
      }
      TB* Bt = B + bB;
      Vec<TB, VB> bv[kMaxVec];
      if (BETA) {
#pragma unroll
        for (int u = 0; u < kMaxVec; ++u)
          if (relB[u] >= 0) bv[u] = ld_stream<TB, VB>(Bt + relB[u]);
      }
#pragma unroll
      for (int u = 0; u < kMaxVec; ++u) {
        if (relB[u] >= 0) {
          const int slb = slot_of((tid + u * kThreads) * VB, pshift, pad);
          Vec<TA, VB> tv;
#pragma unroll
          for (int j = 0; j < VB; ++j) tv.v[j] = tile[slb + ((j + rotB) & (VB - 1))];
          tv = rot_left<TA, VB>(tv, (VB - rotB) & (VB - 1));
          Vec<TB, VB> out;
#pragma unroll
          for (int k = 0; k < VB; ++k) {
            if (BETA)
              out.v[k] = combine<TA, TB>(tv.v[k], bv[u].v[k], beta);
            else
              out.v[k] = finish<TA, TB>(tv.v[k]);
          }
          st_vec<TB, VB>(Bt + relB[u], out, STREAM);
        }
      }
      __syncthreads();
    } else {
      tile_ragged<TA, TB, BETA, STREAM>(d, tt, lim, A + bA, B + bB, alpha, beta, tile);
      if (tn < ntiles) {
        nfull = decode_tile(d, tn, nA, nB, nlim);
        if (nfull) fast_load<TA, VA>(va, A + nA, relA);
      }
    }
    t = tn;
    full = nfull;
    bA = nA;
    bB = nB;
    lim[0] = nlim[0];
    lim[1] = nlim[1];
  }
}

// ------------------------------------------------------------------------------------------------
// Staged tile kernel. A tiles are fetched with asynchronous global->shared copies (cp.async, no
// register cost) into an S-stage ring, so S-1 tiles of loads stay in flight per CTA while the
// current tile is written out. Shared memory holds A in A order (element p at
// p + (p/sigmaA)*padA, the pair chosen by the planner against bank conflicts of the gather); the
// store phase gathers B order through gtab[q] and applies alpha (and beta*B) on the way out. With
// beta != 0 the B tile is staged the same way, in B order.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Programmatic dependent launch: a kernel launched with programmatic stream serialization may start
// while the kernel before it in the stream drains. It lets its own successor start early as soon as
// every CTA has begun (launch_dependents), and it touches no tensor data before everything the
// previous kernel wrote is visible (wait). Both are no-ops in a launch without the attribute.
__device__ __forceinline__ void pdl_allow_next() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_previous() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

template <int BYTES> __device__ __forceinline__ void cp_async(uint32_t dst, const void* src) {
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
  else if constexpr (BYTES == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Bulk copies global -> shared (cp.async.bulk): one instruction moves a contiguous, 16-byte aligned
// range whose size is a multiple of 16 bytes, and signals the bytes it wrote to an mbarrier in
// shared memory (complete_tx). A phase of the barrier completes once its one expected arrival has
// come (arrive.expect_tx, which also adds the bytes to wait for) and every byte has landed.
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
// makes the initialised barriers visible to the bulk-copy unit before any copy signals them
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits for the barrier's phase of the given parity; false if it has not completed within limit_ns
// (the copies it counts never landed). try_wait itself suspends the thread for a while between
// checks, so the loop polls the clock only every 64 attempts.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t n = 1; n != 0; ++n) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((n & 63u) == 0 && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// A stage's bulk copies land within microseconds; a wait that lasts seconds means they never will.
constexpr uint64_t kBulkWaitLimitNs = 2000000000ull;
constexpr uint64_t kBulkDrainLimitNs = 200000000ull;  // the wait for the other stages, after that

// Shared-memory layout of the staged kernel: S stages of [A tile (staged A order)][B tile (B order,
// only when beta != 0)], then segA, segB, and gtab when the gather positions do not fit registers.
constexpr int kRegPos = 16;  // gather positions per thread kept in registers (P <= kRegPos * kThreads)
// Resident CTAs per SM that the staged kernel's register budget is sized for: with beta != 0 and
// wide accesses, 3 (80 registers: the extra B stream keeps more offsets live); otherwise 4 (64
// registers: narrow accesses need the extra warps to cover their larger instruction count).
constexpr int async_min_blocks(int bytes_a, int bytes_b, bool beta) {
  return (beta && bytes_a + bytes_b >= 24) ? 3 : 4;
}
constexpr int kRegVec = 4;   // vectors per thread and side whose offsets the register path keeps

// V consecutive 16-bit table entries (V-aligned) in one shared-memory access.
template <typename T, int V> __device__ __forceinline__ void ld_u16s(const uint16_t* p, uint16_t* out) {
  if constexpr (V == 4) {
    const uint2 w = *reinterpret_cast<const uint2*>(p);
    out[0] = (uint16_t)(w.x & 0xffffu);
    out[1] = (uint16_t)(w.x >> 16);
    out[2] = (uint16_t)(w.y & 0xffffu);
    out[3] = (uint16_t)(w.y >> 16);
  } else if constexpr (V == 2) {
    const uint32_t w = *reinterpret_cast<const uint32_t*>(p);
    out[0] = (uint16_t)(w & 0xffffu);
    out[1] = (uint16_t)(w >> 16);
  } else {
    out[0] = p[0];
  }
}

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }
__host__ __device__ inline size_t async_stage_bytes(int stage_elems, int P, int ea, int eb, bool beta) {
  return al16((size_t)stage_elems * ea) + (beta ? al16((size_t)P * eb) : 0);
}
__host__ __device__ inline size_t async_smem_bytes(int S, int stage_elems, int P, int nsegA, int nsegB, int ea, int eb,
                                                   bool beta) {
  return S * async_stage_bytes(stage_elems, P, ea, eb, beta) + 8 * (size_t)(nsegA + nsegB) +
         (P > kRegPos * kThreads ? al16((size_t)2 * P) : 0);
}

// Decoded tile, shared by the CTA. The first kDecodeBatch lanes of warp 0 decode tiles in batches:
// before the loop, tiles 0 .. 2 * kDecodeBatch - 1 of this CTA; after the barrier of iteration k (k a
// nonzero multiple of kDecodeBatch), tiles k + kDecodeBatch .. k + 2 * kDecodeBatch - 1, one per lane,
// into the ring entries (j % kInfoRing) of tiles k - kDecodeBatch .. k - 1, which every thread
// finished with before that barrier. Tile k + D, issued in iteration k, was decoded at the latest in
// iteration k - kDecodeBatch (D < kDecodeBatch), so one lane's decode costs warp 0 an eighth of a
// tile decode per iteration instead of a whole one.
struct TileInfo {
  int64_t bA, bB;
  int32_t state;  // 1: complete tile, 0: ragged tile, -1: past the last tile
  int32_t lim0, lim1, pad_;
};

// Static shared memory of the staged kernel (descriptor header + tile ring), on top of its dynamic
// shared memory.
constexpr int kDecodeBatch = 8;              // staged kernel: tiles decoded per batch
constexpr int kInfoRing = 2 * kDecodeBatch;  // decoded-tile ring entries (tile j in entry j % kInfoRing)
constexpr int kMaxStages = 7;                // S - 2 = D tiles in flight, D < kDecodeBatch
static_assert(kMaxStages - 2 < kDecodeBatch && kMaxStages - 2 <= 5,
              "tiles in flight must be decoded a batch ahead and covered by the copy-group wait");
constexpr size_t kAsyncStaticSmem = sizeof(TileDesc) + kInfoRing * sizeof(TileInfo) + kMaxStages * sizeof(uint64_t);

// REG: every tile-relative offset of this thread lives in registers (tiles of at most kRegVec
// vectors per thread and side whose offsets fit 32 bits and whose staged bytes fit 16 bits): A
// source offsets rA, staged byte offsets dA (two per register), B offsets rB, gather byte offsets
// gp (two per register; B vector u = tid + u * kThreads, element j). Otherwise offsets are computed
// per vector from the run tables in shared memory, with the gather positions in registers while
// P <= kRegPos * kThreads and in shared memory beyond. The number of stages (3 to kMaxStages) is the
// descriptor's.
// DYN: tiles are claimed in order from a counter in global memory (sched[0]) as the CTA goes, instead
// of the fixed round-robin blockIdx.x + k * gridDim.x. CTAs then stay on neighbouring tiles however
// their speeds differ, so the tiles in motion stay within a narrow span of A and B, and the last
// tiles go to whichever CTAs are free. Each claim takes claim_group consecutive tiles and is issued
// a group before its tiles are used; the last CTA to finish (sched[1] counts them) sets both words back to zero for the next
// launch that uses them, which runs after this grid completes (stream order, and griddepcontrol.wait
// before the first claim when the launch overlaps its predecessor).
// a0 (shifted A runs only): A's pointer is a0 elements past a 16-byte boundary.
// BULK (descriptor's bulkA; VA is the 16-byte vector): the lanes of warp 0 move each A run of a
// tile with one bulk copy, and the stage's mbarrier counts the bytes; every thread waits on it before
// the store phase, with a time limit. A wait that runs out adds 1 to *wait_status, waits (bounded
// again) for the copies of the other tiles in flight and ends the CTA's loop, so that the host
// learns of it and the context stays usable.
template <typename TA, typename TB, int VA, int VB, bool BETA, bool STREAM, bool REG, bool DYN, bool BULK>
__global__ void __launch_bounds__(kThreads, async_min_blocks(VA * sizeof(TA), VB * sizeof(TB), BETA))
    tile_async_kernel(
    const TileDesc* __restrict__ desc, const TA* __restrict__ A, TB* __restrict__ B, TA alpha, TB beta,
    unsigned int* __restrict__ sched, int a0, unsigned int* __restrict__ wait_status, unsigned int claim_group) {
  static_assert(!BULK || VA * sizeof(TA) == 16, "bulk copies move runs of whole 16-byte vectors");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ TileDesc d;  // the descriptor header, read once per CTA
  __shared__ TileInfo info[kInfoRing];  // kAsyncStaticSmem counts both, and the stage barriers
  __shared__ __align__(8) uint64_t abar[kMaxStages];  // BULK: one mbarrier per stage
  const int tid = threadIdx.x;
  pdl_allow_next();
  for (int i = tid; i < (int)(sizeof(TileDesc) / 4); i += kThreads)
    reinterpret_cast<uint32_t*>(&d)[i] = reinterpret_cast<const uint32_t*>(desc)[i];
  __syncthreads();
  const int P = d.P;
  const int S = d.nstages;
  const uint32_t a_bytes = (uint32_t)al16((size_t)d.stage_elems * sizeof(TA));
  const uint32_t sbytes = (uint32_t)async_stage_bytes(d.stage_elems, P, sizeof(TA), sizeof(TB), BETA);
  int64_t* segA = reinterpret_cast<int64_t*>(smem_raw + S * sbytes);
  int64_t* segB = segA + d.nsegA;
  uint16_t* gtab = reinterpret_cast<uint16_t*>(segB + d.nsegB);
  const bool reg_pos = REG || P <= kRegPos * kThreads;
  const unsigned char* base = reinterpret_cast<const unsigned char*>(desc);
  const uint16_t* ggtab = reinterpret_cast<const uint16_t*>(base + d.off_gtab);
  {
    const int64_t* gA = reinterpret_cast<const int64_t*>(base + d.off_segA);
    const int64_t* gB = reinterpret_cast<const int64_t*>(base + d.off_segB);
    if (!REG || BULK)
      for (int i = tid; i < d.nsegA; i += kThreads) segA[i] = gA[i];
    if (!REG) {
      for (int i = tid; i < d.nsegB; i += kThreads) segB[i] = gB[i];
      if (!reg_pos) {
        const uint32_t* gG = reinterpret_cast<const uint32_t*>(ggtab);
        uint32_t* sG = reinterpret_cast<uint32_t*>(gtab);
        for (int i = tid; i < (P + 1) / 2; i += kThreads) sG[i] = gG[i];
      }
    }
  }
  const bool shift = VA * sizeof(TA) == 16 && d.shiftA;
  // A copies per tile: VA-element vectors, or with shifted runs the chunk slots of every run
  const int nvA = shift ? d.nsegA * d.shiftCM : P / VA, nvB = P / VB;
  constexpr int kVecB = REG ? kRegVec : kRegPos / VB;  // B vectors per thread with positions in gp
  constexpr int kGp = (kVecB * VB + 1) / 2;
  // gather positions: byte offsets in the register path, element positions otherwise
  uint32_t gp[kGp];
  int32_t rA[REG ? kRegVec : 1], rB[REG ? kRegVec : 1];
  uint32_t dA[REG ? kRegVec / 2 : 1];
  // the tile shifts x for which each of the thread's A copies is made: x in [lo, hi), 4-bit fields
  // (lo + 1, hi) per copy; without shifted runs a copy is made at x = 0 when it exists
  uint32_t lohi = 0;
  // the register path's lane map (TileDesc::map_log2s): the B vector of thread slot i
  const bool lane_map = REG && d.map_log2s >= 0 && d.map_vb == VB;
  // (-1: the slot takes no vector)
  auto vec_of = [&](int i) -> int {
    if (!lane_map) return i < nvB ? i : -1;
    if (i >= d.map_nslots) return -1;
    const int w = i >> 5, l = i & 31, ls = d.map_log2s, nbx = d.map_nbx;
    const int y = (w / nbx) * (32 >> ls) + (l >> ls);
    if (y >= d.map_ny) return -1;
    const int run = d.off_runs ? (int)reinterpret_cast<const uint16_t*>(base + d.off_runs)[y] : y;
    return (w % nbx) * (1 << ls) + (l & ((1 << ls) - 1)) + d.map_nx * run;
  };
  uint32_t vmask = 0;  // register path: bit u set when the thread's slot u takes a B vector
  // BETA, register path: the B stage byte offset of each of the thread's B vectors (two per register)
  uint32_t qb[REG && BETA ? (kRegVec + 1) / 2 : 1];
#pragma unroll
  for (int e = 0; e < (int)(sizeof(qb) / sizeof(qb[0])); ++e) qb[e] = 0;
#pragma unroll
  for (int e = 0; e < kGp; ++e) gp[e] = 0;
  if (reg_pos) {
#pragma unroll
    for (int u = 0; u < kVecB; ++u) {
      const int vi = vec_of(tid + u * kThreads);
      if (vi >= 0) {
#pragma unroll
        for (int j = 0; j < VB; ++j) {
          const int e = u * VB + j;
          const uint32_t v = (uint32_t)ggtab[vi * VB + j] * (REG ? (uint32_t)sizeof(TA) : 1u);
          gp[e >> 1] |= (e & 1) ? (v << 16) : v;
        }
        if constexpr (REG && BETA) qb[u >> 1] |= ((uint32_t)(vi * VB * (int)sizeof(TB))) << ((u & 1) * 16);
      }
    }
  }
  if constexpr (REG) {
    const int64_t* gA = reinterpret_cast<const int64_t*>(base + d.off_segA);
    const int64_t* gB = reinterpret_cast<const int64_t*>(base + d.off_segB);
    const int LA = d.LA, LB = d.LB, padA = d.padA;
    const FastDiv divLA = d.divLA, divLB = d.divLB, divSig = d.divSigmaA;
#pragma unroll
    for (int u = 0; u < kRegVec; ++u) {
      const int i = tid + u * kThreads;
      rA[u] = rB[u] = 0;
      if (!(u & 1)) dA[u >> 1] = 0;
      if (BULK) {
        // the A runs are moved by warp 0's bulk copies
      } else if (i < nvA && shift) {
        // chunk c of run s: source V * (segA[s] / V + c) past the tile's aligned base, slot
        // s * shiftW + V * c; it covers run elements for lo <= x < hi
        const int s = (int)fdiv((uint32_t)i, d.divCM);
        const int c = i - s * d.shiftCM;
        const int y = (int)(gA[s] & (VA - 1));
        rA[u] = (int32_t)(gA[s] - y) + VA * c;
        dA[u >> 1] |= ((uint32_t)(s * d.shiftW + VA * c) * (uint32_t)sizeof(TA)) << ((u & 1) * 16);
        const int lo = max(c * VA - y - LA + 1, -1), hi = min((c + 1) * VA - y, VA + 1);
        lohi |= ((uint32_t)(lo + 1) | ((uint32_t)max(hi, 0) << 4)) << (8 * u);
      } else if (i < nvA) {
        const int p = i * VA;
        const int s = (int)fdiv((uint32_t)p, divLA);
        const int sp = (int)fdiv((uint32_t)p, divSig);
        rA[u] = (int32_t)(gA[s] + (p - s * LA));
        dA[u >> 1] |= ((uint32_t)(p + sp * padA) * (uint32_t)sizeof(TA)) << ((u & 1) * 16);
        lohi |= (1u | (1u << 4)) << (8 * u);  // x = 0 is in [0, 1)
      }
      const int vi = vec_of(i);
      if (vi >= 0) {
        const int q = vi * VB;
        const int s = (int)fdiv((uint32_t)q, divLB);
        rB[u] = (int32_t)(gB[s] + (q - s * LB));
        vmask |= 1u << u;
      }
    }
  }
  // B stage byte offset of the thread's u-th B vector (register path with beta)
  auto qb_of = [&](int u) -> uint32_t {
    if constexpr (REG && BETA) return (qb[u >> 1] >> ((u & 1) * 16)) & 0xffffu;
    return 0u;
  };

  const uint32_t ntiles = (uint32_t)d.nfull;  // the ragged tiles are the ragged-tile kernel's
  const uint32_t G = gridDim.x;
  const uint32_t stage0 = smem_u32(smem_raw);

  auto decode_into = [&](uint32_t t, TileInfo& ti) {
    if (t >= ntiles) {
      ti.state = -1;
      return;
    }
    decode_full_tile(d, t, ti.bA, ti.bB);
    ti.state = 1;
  };

  // the tile's shift: its first A element lies x elements past a 16-byte boundary (shifted runs)
  auto shift_of = [&](const TileInfo& ti) -> int { return shift ? (int)((a0 + ti.bA) & (VA - 1)) : 0; };

  auto issue = [&](const TileInfo& ti, int stage) {
    if (ti.state != 1) return;  // ragged tiles are moved by the ragged-tile kernel
    const int x = shift_of(ti);
    const TA* At = A + (ti.bA - x);  // 16-byte aligned with shifted runs
    const TB* Bt = B + ti.bB;
    const uint32_t sb = stage0 + (uint32_t)stage * sbytes;
    const uint32_t sbB = sb + a_bytes;
    if constexpr (BULK) {
      if (tid < 32) {
        const uint32_t bar = smem_u32(&abar[stage]);
        const int LA = d.LA, nsegA = d.nsegA;
        if (shift) {
          // run s, y = segA[s] mod V: its elements sit at x + y + j past the aligned chunk
          // segA[s] - y, so chunks (x + y) / V .. (x + y + LA - 1) / V hold it, every one of them
          // holding at least one run element
          uint32_t bytes = 0;
          for (int s = tid; s < nsegA; s += 32) {
            const int xy = x + (int)(segA[s] & (VA - 1));
            bytes += (uint32_t)((xy + LA - 1) / VA - xy / VA + 1) * 16u;
          }
          bytes = __reduce_add_sync(0xffffffffu, bytes);
          if (tid == 0) mbar_arrive_expect_tx(bar, bytes);
          __syncwarp();
          for (int s = tid; s < nsegA; s += 32) {
            const int y = (int)(segA[s] & (VA - 1));
            const int clo = (x + y) / VA, chi = (x + y + LA - 1) / VA;
            bulk_g2s(sb + (uint32_t)((s * d.shiftW + VA * clo) * (int)sizeof(TA)), At + (segA[s] - y + VA * clo),
                     (uint32_t)(chi - clo + 1) * 16u, bar);
          }
        } else {
          // piece j of run s (m = bulk_pieces pieces of LA / m elements, cut at the padding points)
          // at its staged position p + (p / sigmaA) * padA, p = s * LA + j * LA / m, contiguous
          if (tid == 0) mbar_arrive_expect_tx(bar, (uint32_t)(P * (int)sizeof(TA)));
          __syncwarp();
          const FastDiv divSig = d.divSigmaA, divM = d.divPieces;
          const int padA = d.padA, m = d.bulk_pieces, piece = LA / m;
          const uint32_t piece_bytes = (uint32_t)(piece * (int)sizeof(TA));
          for (int i = tid; i < nsegA * m; i += 32) {
            const int s = (int)fdiv((uint32_t)i, divM);
            const int j = i - s * m;
            const int p = s * LA + j * piece;
            const int sp = (int)fdiv((uint32_t)p, divSig);
            bulk_g2s(sb + (uint32_t)((p + sp * padA) * (int)sizeof(TA)), At + (segA[s] + j * piece), piece_bytes, bar);
          }
        }
      }
      if constexpr (BETA) {
        if constexpr (REG) {
#pragma unroll
          for (int u = 0; u < kRegVec; ++u)
            if ((vmask >> u) & 1u) cp_async<VB * sizeof(TB)>(sbB + qb_of(u), Bt + rB[u]);
        } else {
          const int LB = d.LB;
          const FastDiv divLB = d.divLB;
          for (int i = tid; i < nvB; i += kThreads) {
            const int q = i * VB;
            const int s = (int)fdiv((uint32_t)q, divLB);
            cp_async<VB * sizeof(TB)>(sbB + (uint32_t)(q * sizeof(TB)), Bt + (segB[s] + (q - s * LB)));
          }
        }
      }
      return;
    }
    if constexpr (REG) {
#pragma unroll
      for (int u = 0; u < kRegVec; ++u) {
        const uint32_t f = lohi >> (8 * u);
        if (x + 1 >= (int)(f & 15u) && x < (int)((f >> 4) & 15u))
          cp_async<VA * sizeof(TA)>(sb + ((dA[u >> 1] >> ((u & 1) * 16)) & 0xffffu), At + rA[u]);
        if (BETA && ((vmask >> u) & 1u)) cp_async<VB * sizeof(TB)>(sbB + qb_of(u), Bt + rB[u]);
      }
    } else {
      const int LA = d.LA, LB = d.LB, padA = d.padA;
      const FastDiv divLA = d.divLA, divLB = d.divLB, divSig = d.divSigmaA;
      if (shift) {
        for (int i = tid; i < nvA; i += kThreads) {
          const int s = (int)fdiv((uint32_t)i, d.divCM);
          const int c = i - s * d.shiftCM;
          const int y = (int)(segA[s] & (VA - 1));
          if (x >= c * VA - y - LA + 1 && x < (c + 1) * VA - y)
            cp_async<VA * sizeof(TA)>(sb + (uint32_t)((s * d.shiftW + VA * c) * sizeof(TA)),
                                      At + (segA[s] - y + VA * c));
        }
      } else {
        for (int i = tid; i < nvA; i += kThreads) {
          const int p = i * VA;
          const int s = (int)fdiv((uint32_t)p, divLA);
          const int sp = (int)fdiv((uint32_t)p, divSig);
          cp_async<VA * sizeof(TA)>(sb + (uint32_t)((p + sp * padA) * sizeof(TA)), At + (segA[s] + (p - s * LA)));
        }
      }
      if (BETA) {
        for (int i = tid; i < nvB; i += kThreads) {
          const int q = i * VB;
          const int s = (int)fdiv((uint32_t)q, divLB);
          cp_async<VB * sizeof(TB)>(sbB + (uint32_t)(q * sizeof(TB)), Bt + (segB[s] + (q - s * LB)));
        }
      }
    }
  };

  // one B vector: gather VB staged elements (byte offsets from the stage base), scale, combine, store
  auto out_vec = [&](const unsigned char* stage, const TB* sB, int q, const uint32_t* off, TB* dst) {
    Vec<TB, VB> out;
    Vec<TB, VB> bv;
    if (BETA) bv = *reinterpret_cast<const Vec<TB, VB>*>(sB + q);
#pragma unroll
    for (int j = 0; j < VB; ++j) {
      const TA tj = scale_a(alpha, *reinterpret_cast<const TA*>(stage + off[j]));
      if (BETA)
        out.v[j] = combine<TA, TB>(tj, bv.v[j], beta);
      else
        out.v[j] = finish<TA, TB>(tj);
    }
    st_vec<TB, VB>(dst, out, STREAM);
  };
  auto reg_pos_of = [&](int u, uint32_t* off) {
#pragma unroll
    for (int j = 0; j < VB; ++j) {
      const int e = u * VB + j;
      off[j] = (e & 1) ? (gp[e >> 1] >> 16) : (gp[e >> 1] & 0xffffu);
    }
  };

  // Pipeline: S stages, D = S - 2 tiles of copies in flight ahead of the tile being written, and one
  // CTA barrier per tile. Iteration k issues tile k + D into stage (k + D) % S, whose previous tile
  // (k - 2) every thread finished writing out before the barrier of iteration k - 1. Tiles are
  // decoded in batches (see TileInfo).
  const int D = S - 2;
  // DYN: thread 0 claims claim_group consecutive tiles per atomic, one group ahead: `pending` is the
  // first tile of the next group, `cbase` of the current one, `cleft` the current group's tiles left
  unsigned int pending = 0, cbase = 0, cleft = 0;
  uint32_t phase = 0;        // BULK: bit s = parity of the next phase of stage s's barrier
  if constexpr (BULK) {
    if (tid == 0) {
      for (int st = 0; st < S; ++st) mbar_init(smem_u32(&abar[st]), 1);
      mbar_fence_init();
    }
  }
  if constexpr (DYN) {
    // claims touch no tensor data, but the previous launch's reset of the counter must be visible
    pdl_wait_previous();
    if (tid < 32) {
      unsigned int base = 0;
      if (tid == 0) {
        base = atomicAdd(&sched[0], (unsigned int)(D + 2));
        pending = atomicAdd(&sched[0], claim_group);
      }
      base = __shfl_sync(0xffffffffu, base, 0);
      if (tid < D + 2) decode_into(base + tid, info[tid]);
    }
  } else {
    if (tid < kInfoRing) decode_into(blockIdx.x + tid * G, info[tid]);
  }
  __syncthreads();
  // everything above reads the plan's descriptor only; A and B are touched from here on
  pdl_wait_previous();
  for (int j = 0; j < D; ++j) {
    issue(info[j], j);
    cp_async_commit();
  }
  int cur = 0;   // stage of tile k
  int nxt = D;   // stage of tile k + D
  for (uint32_t k = 0;; ++k) {
    if constexpr (DYN) {
      if (info[k % kInfoRing].state < 0) break;  // claims grow, so every later one is past the end too
    } else {
      const uint32_t t = blockIdx.x + k * G;
      if (t >= ntiles) break;
    }
    issue(info[(k + D) % kInfoRing], nxt);
    if (!BULK || BETA) {
      cp_async_commit();
      // tile k's copies are complete once at most D groups (tiles k + 1 .. k + D) are pending
      switch (D) {
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        case 3: cp_async_wait<3>(); break;
        case 4: cp_async_wait<4>(); break;
        default: cp_async_wait<5>(); break;
      }
    }
    if constexpr (BULK) {
      bool late = false;
      if (info[k % kInfoRing].state == 1) {
        late = !mbar_wait_bounded(smem_u32(&abar[cur]), (phase >> cur) & 1u, kBulkWaitLimitNs);
        phase ^= 1u << cur;
      }
      if (__syncthreads_or(late)) {
        // tile k's copies never landed: record it, wait (bounded) for the copies of tiles k .. k + D
        // so that none writes shared memory after the CTA ends, and stop
        if (tid == 0 && wait_status) atomicAdd(wait_status, 1u);
        for (int j = 0, st = cur; j <= D; ++j, st = st + 1 == S ? 0 : st + 1) {
          if (info[(k + j) % kInfoRing].state != 1) continue;
          const uint32_t par = ((phase >> st) & 1u) ^ (j == 0 ? 1u : 0u);
          mbar_wait_bounded(smem_u32(&abar[st]), par, kBulkDrainLimitNs);
        }
        break;
      }
    } else {
      __syncthreads();
    }
    if constexpr (DYN) {
      // the tile of iteration k + D + 2 (read after the next barrier), and the next claim, whose
      // result thread 0 needs only an iteration later (decoding here, before thread 0's own stores,
      // timed 3% faster over the 200 MiB sweep than after them)
      if (tid == 0) {
        if (cleft == 0) {
          cbase = pending;
          cleft = claim_group;
          pending = atomicAdd(&sched[0], claim_group);
        }
        decode_into(cbase + (claim_group - cleft), info[(k + D + 2) % kInfoRing]);
        --cleft;
      }
    } else {
      const uint32_t t = blockIdx.x + k * G;
      if (tid < kDecodeBatch && k % kDecodeBatch == 0 && k != 0)
        decode_into(t + (kDecodeBatch + tid) * G, info[(k + kDecodeBatch + tid) % kInfoRing]);
    }
    const TileInfo& ti = info[k % kInfoRing];
    TB* Bt = B + ti.bB;
    const unsigned char* stage_base = smem_raw + cur * sbytes;
    const TB* sB = reinterpret_cast<const TB*>(stage_base + a_bytes);
    // gathers read the A data through the stage base moved by the tile's shift
    const unsigned char* stage = stage_base + shift_of(ti) * (int)sizeof(TA);
    if (ti.state == 1) {
      if constexpr (REG) {
#pragma unroll
        for (int u = 0; u < kRegVec; ++u) {
          if ((vmask >> u) & 1u) {
            uint32_t off[VB];
            reg_pos_of(u, off);
            out_vec(stage, reinterpret_cast<const TB*>(reinterpret_cast<const unsigned char*>(sB) + qb_of(u)), 0, off,
                    Bt + rB[u]);
          }
        }
      } else {
        const int LB = d.LB;
        const FastDiv divLB = d.divLB;
        if (reg_pos) {
#pragma unroll
          for (int u = 0; u < kVecB; ++u) {
            const int i = tid + u * kThreads;
            if (i < nvB) {
              const int q = i * VB;
              const int s = (int)fdiv((uint32_t)q, divLB);
              uint32_t off[VB];
              reg_pos_of(u, off);
#pragma unroll
              for (int j = 0; j < VB; ++j) off[j] *= (uint32_t)sizeof(TA);
              out_vec(stage, sB, q, off, Bt + (segB[s] + (q - s * LB)));
            }
          }
        } else {
          for (int i = tid; i < nvB; i += kThreads) {
            const int q = i * VB;
            const int s = (int)fdiv((uint32_t)q, divLB);
            uint16_t pos[VB];
            ld_u16s<TA, VB>(gtab + q, pos);
            uint32_t off[VB];
#pragma unroll
            for (int j = 0; j < VB; ++j) off[j] = (uint32_t)pos[j] * (uint32_t)sizeof(TA);
            out_vec(stage, sB, q, off, Bt + (segB[s] + (q - s * LB)));
          }
        }
      }
    }
    cur = cur + 1 == S ? 0 : cur + 1;
    nxt = nxt + 1 == S ? 0 : nxt + 1;
  }
  cp_async_wait<0>();
  if constexpr (DYN) {
    // every claim of this CTA is done; the last CTA to get here resets the counter words
    if (tid == 0) {
      __threadfence();
      if (atomicAdd(&sched[1], 1u) == gridDim.x - 1) {
        atomicExch(&sched[0], 0u);
        atomicExch(&sched[1], 0u);
        __threadfence();
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Ragged tiles of a plan whose complete tiles the staged kernel moved. Every CTA first tabulates,
// for each tile element, its tile-relative A and B offsets (32-bit) and its coordinates in the
// blocked dimensions (two 16-bit fields), which do not depend on the tile; a ragged tile then costs
// a compare per element. Each thread issues an element-wise asynchronous copy for every valid A
// element straight into its B-order shared-memory slot, so a whole tile of loads is in flight at
// once, and the next ragged tile is fetched into the second buffer while the current one is written
// out (alpha is applied on the way out, which rounds exactly as applying it on the way in).
struct RaggedTables {
  const int32_t* relA;  // A-order element p: offset from the tile's A base
  const uint32_t* crdA; // A-order element p: blocked coordinates (low 16 bits: dim 0, high: dim 1)
  const int32_t* relB;  // B-order element q: offset from the tile's B base
  const uint32_t* crdB; // B-order element q: blocked coordinates
  const uint16_t* ptab; // A-order element p: shared-memory slot
};

__device__ __forceinline__ bool ragged_valid(uint32_t crd, int lim0, int lim1) {
  return (int)(crd & 0xffffu) < lim0 && (int)(crd >> 16) < lim1;
}

template <typename TA>
__device__ __forceinline__ void ragged_issue(const TileDesc& d, const RaggedTables& rt, int lim0, int lim1,
                                             const TA* __restrict__ At, TA* tile) {
  const int P = d.P;
  for (int p = threadIdx.x; p < P; p += kThreads)
    if (ragged_valid(rt.crdA[p], lim0, lim1)) cp_async<sizeof(TA)>(smem_u32(tile + rt.ptab[p]), At + rt.relA[p]);
}

template <typename TA, typename TB, bool BETA, bool STREAM>
__device__ __forceinline__ void ragged_store(const TileDesc& d, const RaggedTables& rt, int lim0, int lim1,
                                             TB* __restrict__ Bt, TA alpha, TB beta, const TA* tile) {
  const int P = d.P, pshift = d.pshift, pad = d.pad;
  for (int q0 = threadIdx.x; q0 < P; q0 += kThreads * kUnroll) {
    TB* dst[kUnroll];
    TB bv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int q = q0 + u * kThreads;
      dst[u] = nullptr;
      if (q < P && ragged_valid(rt.crdB[q], lim0, lim1)) {
        dst[u] = Bt + rt.relB[q];
        if (BETA) bv[u] = ld_scalar<TB>(dst[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (dst[u]) {
        const int q = q0 + u * kThreads;
        const TA tq = scale_a(alpha, tile[slot_of(q, pshift, pad)]);
        TB r;
        if (BETA)
          r = combine<TA, TB>(tq, bv[u], beta);
        else
          r = finish<TA, TB>(tq);
        st_scalar<TB>(dst[u], r, STREAM);
      }
    }
  }
}

// Shared memory: two tile buffers of `slots` bytes each, then the per-element tables.
__host__ __device__ inline size_t ragged_smem_bytes(int phys_size, int elem_bytes, int P) {
  return 2 * tile_slots_bytes(phys_size, elem_bytes) + 16 * (size_t)P + al16((size_t)2 * P);
}

// Tile index of the r-th ragged tile (see TileDesc::rag_a): mixed radix over the grid dimensions
// with the ragged dimension pinned to its last block (and, in the second part, rag_a below its last).
__device__ __forceinline__ uint32_t ragged_tile_index(const TileDesc& d, uint32_t r) {
  int fixed = d.rag_a, excl = -1;
  if (r >= (uint32_t)d.nrag0) {
    r -= (uint32_t)d.nrag0;
    fixed = d.rag_b;
    excl = d.rag_a;
  }
  uint32_t t = 0, M = 1;
  for (int k = 0; k < d.ngrid; ++k) {
    const uint32_t cnt = d.g[k].div.d;
    uint32_t c;
    if (k == fixed) {
      c = cnt - 1;
    } else {
      const uint32_t radix = (k == excl) ? cnt - 1 : cnt;
      c = r % radix;
      r /= radix;
    }
    t += c * M;
    M *= cnt;
  }
  return t;
}

template <typename TA, typename TB, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 4) tile_ragged_kernel(const TileDesc* __restrict__ desc,
                                                                  const TA* __restrict__ A, TB* __restrict__ B,
                                                                  TA alpha, TB beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ TileDesc d;
  __shared__ TileInfo ri[2];
  const int tid = threadIdx.x;
  for (int i = tid; i < (int)(sizeof(TileDesc) / 4); i += kThreads)
    reinterpret_cast<uint32_t*>(&d)[i] = reinterpret_cast<const uint32_t*>(desc)[i];
  __syncthreads();
  const uint32_t R = (uint32_t)(d.nrag0 + d.nrag1);
  uint32_t r = blockIdx.x;
  if (r >= R) return;
  const int P = d.P;
  const size_t slots = tile_slots_bytes(d.phys_size, sizeof(TA));
  auto buf = [&](int i) { return reinterpret_cast<TA*>(smem_raw + (i & 1) * slots); };
  int32_t* relA = reinterpret_cast<int32_t*>(smem_raw + 2 * slots);
  uint32_t* crdA = reinterpret_cast<uint32_t*>(relA + P);
  int32_t* relB = reinterpret_cast<int32_t*>(crdA + P);
  uint32_t* crdB = reinterpret_cast<uint32_t*>(relB + P);
  uint16_t* ptab = reinterpret_cast<uint16_t*>(crdB + P);
  {
    const unsigned char* base = reinterpret_cast<const unsigned char*>(desc);
    const int64_t* gA = reinterpret_cast<const int64_t*>(base + d.off_segA);
    const int64_t* gB = reinterpret_cast<const int64_t*>(base + d.off_segB);
    const uint16_t* gP = reinterpret_cast<const uint16_t*>(base + d.off_perm);
    const int nb = d.nblocked;
    for (int p = tid; p < P; p += kThreads) {
      const int sa = (int)fdiv((uint32_t)p, d.divLA);
      relA[p] = (int32_t)(gA[sa] + (p - sa * d.LA));
      const int sb = (int)fdiv((uint32_t)p, d.divLB);
      relB[p] = (int32_t)(gB[sb] + (p - sb * d.LB));
      uint32_t ca = 0, cb = 0;
      for (int b = 0; b < nb; ++b) {
        const uint32_t x = fdiv((uint32_t)p, d.bd[b].tsA);
        const uint32_t y = fdiv((uint32_t)p, d.bd[b].tsB);
        ca |= (x - fdiv(x, d.bd[b].ext) * d.bd[b].ext.d) << (16 * b);
        cb |= (y - fdiv(y, d.bd[b].ext) * d.bd[b].ext.d) << (16 * b);
      }
      crdA[p] = ca;
      crdB[p] = cb;
      ptab[p] = gP[p];
    }
  }
  const RaggedTables rt{relA, crdA, relB, crdB, ptab};
  // thread 0 locates and decodes each ragged tile (the mixed-radix index uses integer division)
  // one iteration ahead; entry k & 1 holds the tile of iteration k
  auto locate = [&](uint32_t rr, TileInfo& ti) {
    int lim[2];
    decode_tile(d, ragged_tile_index(d, rr), ti.bA, ti.bB, lim);
    ti.lim0 = lim[0];
    ti.lim1 = lim[1];
  };
  if (tid == 0) locate(r, ri[0]);
  __syncthreads();
  ragged_issue<TA>(d, rt, ri[0].lim0, ri[0].lim1, A + ri[0].bA, buf(0));
  cp_async_commit();
  for (int k = 0;; ++k) {
    const uint32_t rn = r + gridDim.x;
    const bool more = rn < R;
    if (more && tid == 0) locate(rn, ri[(k + 1) & 1]);
    __syncthreads();
    if (more) {
      const TileInfo& nx = ri[(k + 1) & 1];
      ragged_issue<TA>(d, rt, nx.lim0, nx.lim1, A + nx.bA, buf(k + 1));
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const TileInfo& cu = ri[k & 1];
    ragged_store<TA, TB, BETA, STREAM>(d, rt, cu.lim0, cu.lim1, B + cu.bB, alpha, beta, buf(k));
    __syncthreads();
    if (!more) break;
    r = rn;
  }
}

// One row-copy work unit (row, chunk) processed by one warp.
template <typename TA, typename TB, int V, bool BETA, bool STREAM>
__device__ __forceinline__ void row_unit(const RowDesc& d, uint32_t u, const TA* __restrict__ A, TB* __restrict__ B,
                                         TA alpha, TB beta, int lane) {
  const uint32_t row = fdiv(u, d.divChunk);
  const uint32_t ck = u - row * (uint32_t)d.nchunk;
  int64_t oA = 0, oB = 0;
  uint32_t r = row;
  const int nd = d.nd;
  for (int k = 0; k < nd; ++k) {
    const uint32_t q = fdiv(r, d.div[k]);
    const uint32_t c = r - q * d.div[k].d;
    r = q;
    oA += (int64_t)c * d.sA[k];
    oB += (int64_t)c * d.sB[k];
  }
  const int64_t w = d.w;
  const int64_t e0 = (int64_t)ck * d.chunk;
  const int64_t e1 = (e0 + d.chunk < w) ? e0 + d.chunk : w;
  const TA* Ar = A + oA;
  TB* Br = B + oB;
  for (int64_t eb = e0 + (int64_t)lane * V; eb < e1; eb += 32 * V * kUnroll) {
    Vec<TA, V> av[kUnroll];
    Vec<TB, V> bv[kUnroll];
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const int64_t e = eb + (int64_t)k * 32 * V;
      if (e + V <= e1) {
        av[k] = ld_stream<TA, V>(Ar + e);
        if (BETA) bv[k] = ld_stream<TB, V>(Br + e);
      }
    }
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const int64_t e = eb + (int64_t)k * 32 * V;
      if (e + V <= e1) {
        Vec<TB, V> out;
#pragma unroll
        for (int j = 0; j < V; ++j) {
          const TA t = scale_a(alpha, av[k].v[j]);
          if (BETA)
            out.v[j] = combine<TA, TB>(t, bv[k].v[j], beta);
          else
            out.v[j] = finish<TA, TB>(t);
        }
        st_vec<TB, V>(Br + e, out, STREAM);
      } else if (e < e1) {
        for (int64_t x = e; x < e1; ++x) {
          const TA t = scale_a(alpha, ld_scalar<TA>(Ar + x));
          TB res;
          if (BETA)
            res = combine<TA, TB>(t, ld_scalar<TB>(Br + x), beta);
          else
            res = finish<TA, TB>(t);
          st_scalar<TB>(Br + x, res, STREAM);
        }
      }
    }
  }
}

// Direct row copy: A and B share their stride-1 dimension. One warp per (row, chunk) unit.
template <typename TA, typename TB, int V, bool BETA, bool STREAM>
__global__ void __launch_bounds__(kThreads, 4) row_kernel(const RowDesc* __restrict__ desc, const TA* __restrict__ A,
                                                       TB* __restrict__ B, TA alpha, TB beta) {
  const RowDesc& d = *desc;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kThreads) >> 5;
  for (int u = warp; u < d.nunits; u += nwarps) row_unit<TA, TB, V, BETA, STREAM>(d, (uint32_t)u, A, B, alpha, beta, lane);
}

}  // namespace ttcb
