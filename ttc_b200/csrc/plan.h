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
  double est_cost = 0.0;  // planner's cost estimate (bytes-equivalent per element)

  // descriptor (host copy + device copy)
  std::vector<unsigned char> host_desc;
  void* dev_desc = nullptr;
  int smem_bytes = 0;     // generic tile kernel (slots + tables)
  int smem_fast = 0;      // fast tile kernel (slots only)
  int blocks_fast = 0;    // CTAs for the fast tile kernel
  int smem_async = 0;     // staged tile kernel (stages + tables)
  int blocks_async = 0;   // CTAs for the staged tile kernel
  int blocks_ragged = 0;  // CTAs for the ragged-tile kernel that runs beside the staged kernel
  // the ragged-tile kernel runs on a side stream forked from (and joined back into) the caller's
  // stream; the mutex keeps one call's record/wait sequence whole when calls come from several threads
  void* side_stream = nullptr;  // cudaStream_t
  void* ev_fork = nullptr;      // cudaEvent_t
  void* ev_join = nullptr;      // cudaEvent_t
  void* fork_mutex = nullptr;   // std::mutex
  int smem_ragged = 0;    // its dynamic shared memory (two tile buffers + tables)
  int device = 0;

  // shape-only planning (candidate features for the learned selector): the tile choice without
  // descriptor tables
  bool shape_only = false;
  int64_t tile_P = 0, tile_LA = 0, tile_LB = 0, tile_ntiles = 0;
  int64_t tile_ext[TTCB_MAXR] = {0};  // tile extent per fused dimension (0 = not in the tile)
};

// Fills everything except dev_desc / blocks (which need the CUDA device). Returns a status and a
// message in err on failure.
ttcb_status plan_build_host(ttcb_plan* p, std::string& err);

// Between these calls, plan_build_host on this thread enumerates the tile shapes of a problem once
// and reuses them for further tunings of the same problem (used to plan many candidates quickly).
void plan_tile_cache_begin();
void plan_tile_cache_end();

// Fusion of adjacent dimensions that stay adjacent in B (exposed for tests through the C ABI of
// the test helper in abi.cu).
void fuse_problem(int rank, const int* perm, const int64_t* n, const int64_t* sA, const int64_t* sB,
                  FusedProblem& out);

int dtype_bytes(ttcb_dtype t);
std::string plan_describe_json(const ttcb_plan* p);
