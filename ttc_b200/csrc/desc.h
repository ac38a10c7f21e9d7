// Device descriptors built once per plan by the host planner (plan.cpp) and read by the kernels.
//
// A plan is executed by one of two kernels:
//
//  * tile kernel: the index space is cut into tiles of P elements. A tile is a product set over a
//    subset T of the (fused) dimensions: the leading A dimensions (A's contiguous "run") and the
//    leading B dimensions (B's run), each either full or blocked. Inside a tile, elements are
//    numbered in A order (p) and in B order (q). The load phase walks p (contiguous runs of LA
//    elements in A, segment bases in segA[]), scales by alpha and scatters into shared memory at
//    slot perm_tab[p]; the store phase walks q (runs of LB elements in B, bases in segB[]) and
//    writes B. The remaining dimensions, and the block index of blocked dimensions, form the tile
//    grid, rasterised in the plan's loop order. This generalises TTC's 32x32 plane tiles
//    (CUDAtranspose.py:114-165, 289-388) to runs that span several dimensions.
//
//  * row kernel: when A's and B's stride-1 dimension is the same one and long (TTC's perm[0]==0
//    path, CUDAtranspose.py:179-243, and its identity copy, :781-799), rows are copied directly,
//    one warp per (row, chunk) unit, without staging.
#pragma once
#include <cstdint>
#include "common.cuh"

struct GridDimDesc {
  FastDiv div;      // number of grid steps along this dimension
  FastDiv divf;     // grid steps whose tile is complete (div, less the ragged last block if any)
  int64_t strideA;  // A element offset of one grid step (block extent * A stride)
  int64_t strideB;  // B element offset of one grid step
  int64_t n;        // full extent of the dimension
  int32_t e;        // tile extent (1 for dimensions outside the tile)
  int32_t blocked;  // index into TileDesc::bd for a blocked tile dimension, else -1
};

struct BlockedDesc {
  FastDiv tsA;  // stride of this dimension in the tile's A-order numbering p
  FastDiv tsB;  // stride in the tile's B-order numbering q
  FastDiv ext;  // tile extent e of the dimension
};

struct TileDesc {
  int32_t P;          // elements per tile
  int32_t LA, LB;     // contiguous run lengths (elements) in A and in B
  int32_t nsegA;      // P / LA
  int32_t nsegB;      // P / LB
  int32_t pshift;     // shared-memory slot of q: q + (q >> pshift) * pad
  int32_t pad;
  int32_t phys_size;  // shared-memory slots including padding
  int32_t ngrid;      // grid dimensions, fastest first
  int32_t nblocked;   // blocked tile dimensions (0..2)
  int32_t ntiles;
  int32_t off_segA;   // byte offsets of the tables, relative to the start of the descriptor
  int32_t off_segB;
  int32_t off_perm;
  int32_t smem_bytes; // dynamic shared memory the generic kernel needs (slots + tables)
  int32_t fast;       // 1: every tile-relative offset fits in 32 bits and the fast kernel applies
  // staged (asynchronous-copy) kernel: A tiles land in shared memory in A order, element p at
  // p + (p / LA) * padA; the store phase gathers B order through gtab[q]
  int32_t async_ok;   // 1: the staged kernel applies (32-bit offsets, <= 16 elements per thread)
  int32_t padA;       // padding after each A run in the staged layout (multiple of the A vector)
  int32_t stage_elems;// elements of one stage buffer (max of the staged layout and phys_size)
  int32_t nstages;    // staged kernel: stages (3..7; stages - 2 tiles of copies in flight)
  int32_t off_gtab;   // byte offset of gtab (uint16_t[P]) from the start of the descriptor
  int32_t sigmaA;     // staged layout: element p at p + (p / sigmaA) * padA
  int32_t reg_ok;     // 1: fast, and the staged tile's byte offsets fit 16 bits (register path)
  // ragged tiles (last block of a blocked dimension that does not divide its extent), which the
  // staged kernel leaves to the ragged-tile kernel: grid dimensions rag_a, rag_b (-1: none);
  // tiles with rag_a at its last block come first (nrag0), then those with rag_b at its last block
  // and rag_a not (nrag1)
  int32_t rag_a, rag_b, nrag0, nrag1;
  int32_t nfull;      // complete tiles (decoded over the divf counts of the grid dimensions)
  int32_t pad3_;
  FastDiv divLA, divLB;
  FastDiv divSigmaA;
  GridDimDesc g[TTCB_MAXR];
  BlockedDesc bd[2];
  // staged kernel, shifted A runs (A runs that 16-byte accesses cannot reach directly: odd lengths or
  // offsets): each run is copied as the 16-byte chunks that cover it. Run s keeps chunk slots
  // [s * shiftW, s * shiftW + shiftCM * V) (V = 16 / sizeof(TA)); a tile whose first A element lies
  // x elements past a 16-byte boundary (x = (a0 + tile base) mod V, a0 the misalignment of A's
  // pointer) puts element j of run s at s * shiftW + (segA[s] mod V) + x + j, which is gtab's position
  // plus x: the store phase reads through the stage base moved by x elements.
  int32_t shiftA;     // 1: A runs are copied as covering 16-byte chunks (the vector width is V)
  int32_t shiftW;     // staged stride of one A run (elements, a multiple of V)
  int32_t shiftCM;    // chunk slots per A run
  // 1: the staged kernel may move A with bulk copies (cp.async.bulk, completion counted on a
  // per-stage mbarrier) instead of per-thread 16-byte copies: one per shifted run, else one per
  // contiguous piece of a run in the staged layout - the whole run when sigmaA is a multiple of LA,
  // else bulk_pieces = LA / sigmaA pieces of sigmaA elements, each 16-byte aligned.
  int32_t bulkA;
  FastDiv divCM;      // divisor shiftCM
  int32_t bulk_pieces;  // bulk copies per A run (plain runs)
  // Lane map of the staged kernel's register path (when its B vector width is map_vb): a warp's
  // 32 lanes take map_s consecutive B vectors from each of 32 / map_s consecutive B runs instead of
  // 32 consecutive vectors, so that the gathers of one load fall into more banks (lanes in
  // different runs read different A positions). Warp w covers columns (w mod map_nbx) * map_s ..
  // + map_s - 1 of rows (w / map_nbx) * (32 / map_s) .. of the (B vectors per run) x (B runs) grid;
  // lane l takes column offset l mod map_s, row offset l / map_s. The last footprint row may reach
  // past the tile's B runs: those slots take no vector.
  int32_t map_log2s;  // log2 map_s, or -1: no map (lane i of the block takes vector i)
  int32_t map_nx;     // B vectors per B run (LB / map_vb)
  int32_t map_nbx;    // warp footprints across the B vectors of a run (map_nx / map_s)
  FastDiv divPieces;  // divisor bulk_pieces
  int32_t map_vb;     // the B vector width the map is planned for
  int32_t map_ny;     // B runs in the tile; thread slots whose row is past them take no vector
  int32_t map_nslots; // thread slots the map spans (map_nbx * ceil(map_ny / (32 / map_s)) * 32)
  // byte offset (from the descriptor start) of the map's run order, uint16_t[map_ny]: footprint
  // row y takes B run runs[y] (the runs sorted by the A position of their first element, so that
  // a warp's rows start at neighbouring A positions); 0: row y takes run y
  int32_t off_runs;
  // followed by: int64_t segA[nsegA]; int64_t segB[nsegB]; uint16_t perm_tab[P] (slots)
};

struct RowDesc {
  int64_t w;          // row length in elements (stride 1 in both A and B)
  int32_t chunk;      // elements per work unit
  int32_t nchunk;     // units per row
  int32_t nd;         // number of row dimensions
  int32_t nunits;     // rows * nchunk
  FastDiv divChunk;   // divisor nchunk
  FastDiv div[TTCB_MAXR];
  int64_t sA[TTCB_MAXR];
  int64_t sB[TTCB_MAXR];
};

enum { TTCB_KERNEL_TILE = 1, TTCB_KERNEL_ROW = 2 };
// Launch-time kernel choices for tile plans (never stored in a plan's kernel field): register-prefetch
// kernel, staged kernel with offsets computed from the run tables or held in registers, each staged
// form with the fixed round-robin tile order or with tiles claimed in order from a counter (_DYN).
enum { TTCB_KERNEL_TILE_FAST = 3, TTCB_KERNEL_TILE_ASYNC = 4, TTCB_KERNEL_TILE_ASYNC_REG = 5, TTCB_KERNEL_TILE_RAGGED = 6,
       TTCB_KERNEL_TILE_ASYNC_DYN = 7, TTCB_KERNEL_TILE_ASYNC_REG_DYN = 8 };
// Added to a staged-kernel id: the form that moves A runs with bulk copies (TileDesc::bulkA).
enum { TTCB_KERNEL_BULK_FLAG = 16 };
inline bool ttcb_is_staged_kernel(int k) {
  k &= ~TTCB_KERNEL_BULK_FLAG;
  return k == TTCB_KERNEL_TILE_ASYNC || k == TTCB_KERNEL_TILE_ASYNC_REG || k == TTCB_KERNEL_TILE_ASYNC_DYN ||
         k == TTCB_KERNEL_TILE_ASYNC_REG_DYN;
}
