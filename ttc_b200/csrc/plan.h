// Host-side plan: validation, index fusion, kernel choice and descriptor construction.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/ttcb200.h"
#include "desc.h"

struct FusedProblem {
  int rank = 0;
  int perm[TTCB_MAXR] = {0};     // B dim j <- A dim perm[j]
  int64_t n[TTCB_MAXR] = {0};    // extents (A order)
  int64_t sA[TTCB_MAXR] = {0};   // A stride of A-dim i
  int64_t sB[TTCB_MAXR] = {0};   // B stride of A-dim i
  int64_t oA = 0, oB = 0;        // offsets (elements) of A and B from a 16-byte boundary; only their
                                 // alignment matters (nonzero for the edge plans of another plan)
  int fused_of[TTCB_MAXR] = {0}; // the caller's dimension i belongs to fused dimension fused_of[i]
                                 // (-1: an extent-1 dimension, dropped)
};

// A box of a tile plan's ragged tiles (the last block of one ragged dimension; with two ragged
// dimensions, the second box leaves out the first's), as a transposition of its own in TTC's form:
// the parent's strides through lda/ldb, its first element at offA / offB.
struct EdgeBox {
  int rank = 0;
  int perm[TTCB_MAXR] = {0};
  int64_t size[TTCB_MAXR] = {0};
  int64_t lda[TTCB_MAXR] = {0};
  int64_t ldb[TTCB_MAXR] = {0};
  int64_t offA = 0, offB = 0;
};

struct ttcb_plan {
  // the problem as given
  int rank = 0;
  int perm[TTCB_MAXR] = {0};
  int64_t size[TTCB_MAXR] = {0};
  int64_t lda[TTCB_MAXR] = {0};
  int64_t ldb[TTCB_MAXR] = {0};
  ttcb_dtype ta = TTCB_S, tb = TTCB_S;
  int beta_nonzero = 0;
  ttcb_tuning tuning{};

  // after fusion
  FusedProblem f;
  int64_t N = 0;          // elements
  bool empty = false;

  // choice
  int kernel = 0;         // TTCB_KERNEL_TILE / TTCB_KERNEL_ROW
  int vecA = 1, vecB = 1; // elements per access assuming 16-byte aligned base pointers
  int blocks = 0;         // CTAs launched
  bool streaming = false;
  int loop_order = 0;
  int raster[TTCB_MAXR] = {0};  // grid dimensions (fused) from the fastest-varying to the slowest
  int nraster = 0;
  double est_cost = 0.0;  // planner's cost estimate (bytes-equivalent per element)

  // descriptor (host copy + device copy)
  std::vector<unsigned char> host_desc;
  void* dev_desc = nullptr;
  int smem_bytes = 0;     // generic tile kernel (slots + tables)
  int smem_fast = 0;      // fast tile kernel (slots only)
  int blocks_fast = 0;    // CTAs for the fast tile kernel
  int smem_async = 0;     // staged tile kernel (stages + tables)
  int blocks_async = 0;   // CTAs for the staged tile kernel
  int ctas_per_sm = 0;    // staged tile kernel: CTAs per SM the schedule asks for (0 = as many as fit)
  int blocks_ragged = 0;  // CTAs for the ragged-tile kernel that runs beside the staged kernel
  // the ragged-tile kernel runs on a side stream forked from (and joined back into) the caller's
  // stream; the mutex keeps one call's record/wait sequence whole when calls come from several threads
  void* side_stream = nullptr;  // cudaStream_t
  void* ev_fork = nullptr;      // cudaEvent_t
  void* ev_join = nullptr;      // cudaEvent_t
  void* fork_mutex = nullptr;   // std::mutex
  // staged kernel with claimed tiles: kClaimSlots pairs of counter words on the device (zeroed at
  // creation, reset by each launch's last CTA) and the host's running launch count
  unsigned int* claim_words = nullptr;
  int claim_group = 1;           // tiles per claim
  void* launch_count = nullptr;  // std::atomic<unsigned int>
  // staged kernel with bulk A copies: count of stage waits that ran out of time (device word, zeroed
  // at creation; read and cleared by ttcb_plan_wait_timeouts)
  unsigned int* wait_status = nullptr;
  int smem_ragged = 0;    // its dynamic shared memory (two tile buffers + tables)
  int device = 0;

  // ragged tiles: the fused dimensions whose last tile block is ragged and where that block starts
  int rag_dim[2] = {-1, -1};
  int64_t rag_start[2] = {0, 0};
  // edge plans: the boxes of the ragged tiles planned as transpositions of their own, which the
  // staged kernel moves on the side stream (instead of the element-wise ragged-tile kernel)
  int depth = 0;                     // 0 for a caller's plan, 1 for an edge plan
  int64_t base_offA = 0, base_offB = 0;  // an edge plan's offsets into its parent's A and B
  ttcb_plan* edge[2] = {nullptr, nullptr};
  int nedge = 0;

  // shape-only planning (candidate features for the learned selector): the tile choice without
  // descriptor tables
  bool shape_only = false;
  int64_t tile_P = 0, tile_LA = 0, tile_LB = 0, tile_ntiles = 0;
  int64_t tile_ext[TTCB_MAXR] = {0};  // tile extent per fused dimension (0 = not in the tile)
  int shape_stages = 0;                // the staged kernel's ring depth the schedule would use
  bool shape_shifted = false;          // the staged kernel would copy shifted A runs
  bool shape_bulk = false;             // the staged kernel would move A runs with bulk copies
};

// Fills everything except dev_desc / blocks (which need the CUDA device). Returns a status and a
// message in err on failure.
ttcb_status plan_build_host(ttcb_plan* p, std::string& err);

// Between these calls, plan_build_host on this thread enumerates the tile shapes of a problem once
// and reuses them for further tunings of the same problem (used to plan many candidates quickly).
void plan_tile_cache_begin();
void plan_tile_cache_end();

// Decodes an explicit loop order (ttcb_tuning::raster_lo/hi) into `order` (the caller's dimensions,
// fastest first); false unless it is a permutation of 0..rank-1.
bool unpack_raster(const ttcb_tuning& tu, int rank, int* order);

// Fusion of adjacent dimensions that stay adjacent in B (exposed for tests through the C ABI of
// the test helper in abi.cu).
void fuse_problem(int rank, const int* perm, const int64_t* n, const int64_t* sA, const int64_t* sB,
                  FusedProblem& out);

// The boxes of a tile plan's ragged tiles (0, 1 or 2); -1 when they cannot be written in TTC's form
// within the rank limit.
int plan_edge_boxes(const ttcb_plan* p, EdgeBox out[2]);

int dtype_bytes(ttcb_dtype t);
std::string plan_describe_json(const ttcb_plan* p);
