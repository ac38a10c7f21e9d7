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
      lim[gd.blocked] = l;
      if (l < gd.e) full = false;
    }
  }
  return full;
}

struct TileTables {
  const int64_t* segA;
  const int64_t* segB;
  const uint16_t* ptab;
};

// One tile: load phase (A runs -> alpha*A -> shared slots in B order), barrier, store phase
// (shared slots -> B runs, with beta*B when BETA), barrier. All threads of the CTA take part.
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
  if (full) {
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
  } else {
    // ragged tile: element-wise, validity from the blocked dimensions' tile coordinates
    const int nb = d.nblocked;
    for (int p = tid; p < P; p += kThreads) {
      bool ok = true;
      for (int b = 0; b < nb; ++b) {
        const uint32_t c = fdiv((uint32_t)p, d.bd[b].tsA);
        const uint32_t cc = c - fdiv(c, d.bd[b].ext) * d.bd[b].ext.d;
        ok = ok && ((int)cc < lim[b]);
      }
      if (ok) {
        const int s = (int)fdiv((uint32_t)p, d.divLA);
        tile[tt.ptab[p]] = scale_a(alpha, ld_scalar<TA>(At + (tt.segA[s] + (p - s * LA))));
      }
    }
    __syncthreads();
    for (int q = tid; q < P; q += kThreads) {
      bool ok = true;
      for (int b = 0; b < nb; ++b) {
        const uint32_t c = fdiv((uint32_t)q, d.bd[b].tsB);
        const uint32_t cc = c - fdiv(c, d.bd[b].ext) * d.bd[b].ext.d;
        ok = ok && ((int)cc < lim[b]);
      }
      if (ok) {
        const int s = (int)fdiv((uint32_t)q, d.divLB);
        TB* dst = Bt + (tt.segB[s] + (q - s * LB));
        const TA tq = tile[slot_of(q, pshift, pad)];
        TB r;
        if (BETA)
          r = combine<TA, TB>(tq, ld_scalar<TB>(dst), beta);
        else
          r = finish<TA, TB>(tq);
        st_scalar<TB>(dst, r, STREAM);
      }
    }
  }
  __syncthreads();
}

// Shared-memory layout of the plain tile kernel: [tile slots][segA][segB][perm_tab].
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
