// C ABI of the plain transposition: plan creation (validation, fusion, descriptor upload),
// asynchronous execution, error reporting.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <sstream>
#include <vector>
#include <new>
#include <string>

#include "../../include/ttcb200.h"
#include "kernels.cuh"
#include "launch.h"
#include "plan.h"
#include "testing.h"

namespace ttcb {
KernelRef pick_kernel_ss(int, int, int, int);
KernelRef pick_kernel_dd(int, int, int, int);
KernelRef pick_kernel_cc(int, int, int, int);
KernelRef pick_kernel_zz(int, int, int, int);
KernelRef pick_kernel_sd(int, int, int, int);
KernelRef pick_kernel_ds(int, int, int, int);
KernelRef pick_kernel_cz(int, int, int, int);
KernelRef pick_kernel_zc(int, int, int, int);

KernelRef pick_kernel(ttcb_dtype ta, ttcb_dtype tb, int kernel, int va, int vb, int variant) {
  if (ta == TTCB_S && tb == TTCB_S) return pick_kernel_ss(kernel, va, vb, variant);
  if (ta == TTCB_D && tb == TTCB_D) return pick_kernel_dd(kernel, va, vb, variant);
  if (ta == TTCB_C && tb == TTCB_C) return pick_kernel_cc(kernel, va, vb, variant);
  if (ta == TTCB_Z && tb == TTCB_Z) return pick_kernel_zz(kernel, va, vb, variant);
  if (ta == TTCB_S && tb == TTCB_D) return pick_kernel_sd(kernel, va, vb, variant);
  if (ta == TTCB_D && tb == TTCB_S) return pick_kernel_ds(kernel, va, vb, variant);
  if (ta == TTCB_C && tb == TTCB_Z) return pick_kernel_cz(kernel, va, vb, variant);
  if (ta == TTCB_Z && tb == TTCB_C) return pick_kernel_zc(kernel, va, vb, variant);
  return KernelRef();
}
}  // namespace ttcb

static thread_local std::string g_last_error;

static ttcb_status fail(ttcb_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

static ttcb_status cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return fail(TTCB_ERR_CUDA, m);
}

static int variant_of(const ttcb_plan* p) { return p->beta_nonzero ? 2 : (p->streaming ? 1 : 0); }

namespace ttcb {
// Kernels whose shared memory (dynamic, plus the staged kernel's static descriptor header and tile
// ring) may exceed the 48 KB default get the opt-in once per device, always to the planner's
// ceiling (kMaxDynamicSmem), so that no caller ever lowers the limit another plan relies on.
bool needs_large_smem(int dynamic_smem) { return dynamic_smem + (int)kAsyncStaticSmem > 48 * 1024; }

void allow_large_smem(const void* func) {
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  for (const auto& x : done)
    if (x.first == func && x.second == dev) return;
  cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
  cudaGetLastError();
  done.emplace_back(func, dev);
}
}  // namespace ttcb

namespace ttcb {
unsigned int* plan_claim_slot(const ttcb_plan* p) {
  if (!p->claim_words || !p->launch_count) return nullptr;
  const unsigned int k = static_cast<std::atomic<unsigned int>*>(p->launch_count)->fetch_add(1);
  return p->claim_words + 2 * (k % kClaimSlots);
}
}  // namespace ttcb

using ttcb::allow_large_smem;
using ttcb::needs_large_smem;

// The staged kernel claims tiles from the plan's counters when the plan has them (the schedule asks
// for it with round_robin = -1, or the planner's rule below); otherwise it takes the round-robin
// order.
static bool uses_claims(const ttcb_plan* p) { return p->claim_words != nullptr; }
static constexpr int64_t kClaimMinTileBytes = 16 * 1024;
static constexpr int kClaimMinTilesPerCta = 16;
// The staged kernel moves A runs with bulk copies when the plan's layout allows it and A's pointer
// meets the layout's alignment (shifted runs take any pointer; plain runs need the 16-byte vector).
static bool uses_bulk(const ttcb_plan* p, const TileDesc* td, int va, int EA) {
  return td->bulkA && p->wait_status && (td->shiftA || va * EA == 16);
}
static int staged_kernel_id(const ttcb_plan* p, const TileDesc* td, bool reg, bool bulk) {
  const bool claims = uses_claims(p);
  const int k = reg ? (claims ? TTCB_KERNEL_TILE_ASYNC_REG_DYN : TTCB_KERNEL_TILE_ASYNC_REG)
                    : (claims ? TTCB_KERNEL_TILE_ASYNC_DYN : TTCB_KERNEL_TILE_ASYNC);
  return bulk ? (k | TTCB_KERNEL_BULK_FLAG) : k;
}

static ttcb_status plan_finish_device(ttcb_plan* p) {
  if (p->empty) return TTCB_OK;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaMalloc(&p->dev_desc, p->host_desc.size());
  if (e != cudaSuccess) {
    p->dev_desc = nullptr;
    cudaGetLastError();
    return fail(TTCB_ERR_ALLOC, std::string("cudaMalloc of the plan descriptor failed: ") + cudaGetErrorString(e));
  }
  e = cudaMemcpy(p->dev_desc, p->host_desc.data(), p->host_desc.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy of the plan descriptor");

  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
  int64_t work = 1;
  if (p->kernel == TTCB_KERNEL_TILE) {
    work = reinterpret_cast<const TileDesc*>(p->host_desc.data())->ntiles;
  } else {
    const RowDesc* rd = reinterpret_cast<const RowDesc*>(p->host_desc.data());
    work = (rd->nunits + (ttcb::kThreads / 32) - 1) / (ttcb::kThreads / 32);  // one warp per unit
  }
  auto grid_for = [&](int kernel_id, int smem, int* out, int64_t items = -1) -> ttcb_status {
    const int64_t work_k = items >= 0 ? std::max<int64_t>(items, 1) : work;
    ttcb::KernelRef k = ttcb::pick_kernel(p->ta, p->tb, kernel_id, p->vecA, p->vecB, variant_of(p));
    if (!k.func) return fail(TTCB_ERR_DTYPE, "no kernel for this type pair");
    if (needs_large_smem(smem)) allow_large_smem(k.func);
    int per_sm = 0;
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.func, ttcb::kThreads, smem);
    if (err != cudaSuccess) return cuda_fail(err, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return fail(TTCB_ERR_UNSUPPORTED, "tile does not fit in shared memory");
    // the staged kernel's schedule may ask for fewer CTAs per SM than fit (see the planner)
    if (ttcb_is_staged_kernel(kernel_id) && p->ctas_per_sm > 0)
      per_sm = std::min(per_sm, p->ctas_per_sm);
    int64_t resident = (int64_t)per_sm * sms;
    int64_t blocks;
    if (p->tuning.blocks > 0 && kernel_id != TTCB_KERNEL_TILE_RAGGED) {
      blocks = std::min<int64_t>(p->tuning.blocks, work_k);
    } else if (kernel_id == TTCB_KERNEL_ROW) {
      // one warp per row unit and the hardware's own block order: on a 200 MiB copy this ran at
      // 6335 GB/s against 5655 with the grid persistent over units (582 CTAs)
      blocks = std::min<int64_t>(work_k, 0x7fffffff);
    } else {
      int64_t per = (work_k + resident - 1) / resident;  // work items per CTA, balanced
      blocks = (work_k + per - 1) / per;
    }
    *out = (int)std::max<int64_t>(blocks, 1);
    return TTCB_OK;
  };
  ttcb_status s = grid_for(p->kernel, p->smem_bytes, &p->blocks);
  if (s != TTCB_OK) return s;
  if (p->kernel == TTCB_KERNEL_TILE) {
    const TileDesc* td = reinterpret_cast<const TileDesc*>(p->host_desc.data());
    if (td->fast) {
      s = grid_for(TTCB_KERNEL_TILE_FAST, p->smem_fast, &p->blocks_fast);
      if (s != TTCB_OK) return s;
    }
    if (td->async_ok) {
      // Tiles are claimed in order from counters when the schedule asks for it, or by default for
      // tiles of 16 KiB or more (A, B and B read back) when every CTA has at least 16 of them. Timed
      // over the 200 MiB sweep back to back, claims made such tiles 2-15% faster (CTAs stay on
      // neighbouring tiles, so the tiles in motion span a narrow stretch of A and B) and smaller
      // ones up to 19% slower (the claim's round trip is not hidden behind a short tile); a CTA
      // claims its first S tiles at once, which leaves CTAs idle when each has only a few (the 147 MB
      // 1000x768x16 transposition, 11 tiles per CTA: 10% slower).
      const int EA = dtype_bytes(p->ta);
      s = grid_for(staged_kernel_id(p, td, td->reg_ok, false), p->smem_async, &p->blocks_async, td->nfull);
      if (s != TTCB_OK) return s;
      const int64_t tile_bytes = (int64_t)td->P * (EA + dtype_bytes(p->tb) * (p->beta_nonzero ? 2 : 1));
      const bool claims_by_default = p->tuning.round_robin == 0 && tile_bytes >= kClaimMinTileBytes &&
                                     td->nfull >= (int64_t)kClaimMinTilesPerCta * p->blocks_async;
      // two tiles per claim: back to back over the sweep, 0.3% faster than one (three: 0.3% slower)
      p->claim_group = p->tuning.claim_group > 0 ? std::min(p->tuning.claim_group, 64) : 2;
      if (p->tuning.round_robin == -1 || claims_by_default) {
        e = cudaMalloc(&p->claim_words, sizeof(unsigned int) * 2 * ttcb::kClaimSlots);
        if (e != cudaSuccess) {
          p->claim_words = nullptr;
          cudaGetLastError();
          return fail(TTCB_ERR_ALLOC, std::string("cudaMalloc of the tile counters failed: ") + cudaGetErrorString(e));
        }
        if ((e = cudaMemset(p->claim_words, 0, sizeof(unsigned int) * 2 * ttcb::kClaimSlots)) != cudaSuccess)
          return cuda_fail(e, "cudaMemset of the tile counters");
        p->launch_count = new (std::nothrow) std::atomic<unsigned int>(0);
        if (!p->launch_count) return fail(TTCB_ERR_ALLOC, "host allocation of the launch counter failed");
      }
      if (td->bulkA) {
        e = cudaMalloc(&p->wait_status, sizeof(unsigned int));
        if (e != cudaSuccess) {
          p->wait_status = nullptr;
          cudaGetLastError();
          return fail(TTCB_ERR_ALLOC, std::string("cudaMalloc of the wait status failed: ") + cudaGetErrorString(e));
        }
        if ((e = cudaMemset(p->wait_status, 0, sizeof(unsigned int))) != cudaSuccess)
          return cuda_fail(e, "cudaMemset of the wait status");
      }
      s = grid_for(staged_kernel_id(p, td, td->reg_ok, uses_bulk(p, td, p->vecA, EA)), p->smem_async, &p->blocks_async,
                   td->nfull);
      if (s != TTCB_OK) return s;
      if (td->nrag0 + td->nrag1 > 0) {
        s = grid_for(TTCB_KERNEL_TILE_RAGGED, p->smem_ragged, &p->blocks_ragged, (int64_t)td->nrag0 + td->nrag1);
        if (s != TTCB_OK) return s;
        if (p->depth > 0) return TTCB_OK;  // an edge plan runs on its parent's side stream
        cudaStream_t side = nullptr;
        cudaEvent_t fork = nullptr, join = nullptr;
        if ((e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking)) != cudaSuccess)
          return cuda_fail(e, "cudaStreamCreateWithFlags");
        p->side_stream = side;
        if ((e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming)) != cudaSuccess)
          return cuda_fail(e, "cudaEventCreateWithFlags");
        p->ev_fork = fork;
        if ((e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming)) != cudaSuccess)
          return cuda_fail(e, "cudaEventCreateWithFlags");
        p->ev_join = join;
        p->fork_mutex = new (std::nothrow) std::mutex();
        if (!p->fork_mutex) return fail(TTCB_ERR_ALLOC, "host allocation of the plan's mutex failed");
      }
    }
  }
  return TTCB_OK;
}

// Launches a checked plan on stream st. The staged kernel moves complete tiles only; a plan with
// ragged tiles forks its side stream from st before the staged kernel and joins it back after, and
// the side stream moves the ragged tiles beside the staged kernel (they write disjoint parts of B):
// through the edge plans when there are some, else with the element-wise ragged-tile kernel. An
// edge plan with ragged tiles of its own runs its ragged-tile kernel after its staged kernel.
static ttcb_status launch_plan(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                               cudaStream_t st) {
  const int EA = dtype_bytes(p->ta), EB = dtype_bytes(p->tb);
  cudaError_t e;
  int va = p->vecA, vb = p->vecB;
  const bool shifted = p->kernel == TTCB_KERNEL_TILE &&
                       reinterpret_cast<const TileDesc*>(p->host_desc.data())->shiftA;
  // shifted A runs take any pointer (the kernel folds its misalignment into the tile shift)
  while (!shifted && va > 1 && (uintptr_t)A % (va * EA)) va /= 2;
  while (vb > 1 && (uintptr_t)B % (vb * EB)) vb /= 2;
  if (p->kernel == TTCB_KERNEL_ROW) va = vb = std::min(va, vb);
  int kernel = p->kernel, blocks = p->blocks, smem = p->smem_bytes;
  if (kernel == TTCB_KERNEL_TILE) {
    const TileDesc* td = reinterpret_cast<const TileDesc*>(p->host_desc.data());
    const int want = p->tuning.tile_variant;
    const bool fast_ok = td->fast && td->P / va <= 1024 && td->P / vb <= 1024;
    if (shifted && !((want == 0 || want == 3) && td->async_ok))
      return fail(TTCB_ERR_UNSUPPORTED, "a plan with shifted A runs runs only on the staged tile kernel");
    if ((want == 0 || want == 3) && td->async_ok) {
      kernel = staged_kernel_id(p, td, fast_ok && td->reg_ok, uses_bulk(p, td, va, EA));
      blocks = p->blocks_async;
      smem = p->smem_async;
    } else if ((want == 0 || want == 2) && fast_ok) {
      kernel = TTCB_KERNEL_TILE_FAST;
      blocks = p->blocks_fast;
      smem = p->smem_fast;
    }
  }
  ttcb::KernelRef k = ttcb::pick_kernel(p->ta, p->tb, kernel, va, vb, variant_of(p));
  if (!k.fn) return fail(TTCB_ERR_DTYPE, "no kernel for this type pair");
  if (needs_large_smem(smem)) allow_large_smem(k.func);
  const TileDesc* td = reinterpret_cast<const TileDesc*>(p->host_desc.data());
  const bool ragged = ttcb_is_staged_kernel(kernel) && td->nrag0 + td->nrag1 > 0;
  if (!ragged) {
    e = k.fn(p, A, B, alpha, beta, st, blocks);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return TTCB_OK;
  }
  ttcb::KernelRef kr{};
  if (p->nedge == 0) {
    kr = ttcb::pick_kernel(p->ta, p->tb, TTCB_KERNEL_TILE_RAGGED, 1, 1, variant_of(p));
    if (!kr.fn) return fail(TTCB_ERR_DTYPE, "no ragged-tile kernel for this type pair");
    if (needs_large_smem(p->smem_ragged)) allow_large_smem(kr.func);
  }
  if (p->depth > 0) {
    e = k.fn(p, A, B, alpha, beta, st, blocks);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    e = kr.fn(p, A, B, alpha, beta, st, p->blocks_ragged);
    if (e != cudaSuccess) return cuda_fail(e, "ragged-tile kernel launch");
    return TTCB_OK;
  }
  cudaStream_t side = static_cast<cudaStream_t>(p->side_stream);
  cudaEvent_t fork = static_cast<cudaEvent_t>(p->ev_fork), join = static_cast<cudaEvent_t>(p->ev_join);
  std::lock_guard<std::mutex> lk(*static_cast<std::mutex*>(p->fork_mutex));
  if ((e = cudaEventRecord(fork, st)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  if ((e = cudaStreamWaitEvent(side, fork, 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
  // once forked, the side stream is joined back even when a launch fails, so that the caller's
  // stream stays ordered after whatever was enqueued
  ttcb_status status = TTCB_OK;
  e = k.fn(p, A, B, alpha, beta, st, blocks);
  if (e != cudaSuccess) status = cuda_fail(e, "kernel launch");
  if (status == TTCB_OK && p->nedge > 0) {
    for (int j = 0; j < p->nedge && status == TTCB_OK; ++j) {
      const ttcb_plan* q = p->edge[j];
      status = launch_plan(q, static_cast<const char*>(A) + q->base_offA * EA,
                           static_cast<char*>(B) + q->base_offB * EB, alpha, beta, side);
    }
  } else if (status == TTCB_OK) {
    e = kr.fn(p, A, B, alpha, beta, side, p->blocks_ragged);
    if (e != cudaSuccess) status = cuda_fail(e, "ragged-tile kernel launch");
  }
  if ((e = cudaEventRecord(join, side)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  if ((e = cudaStreamWaitEvent(st, join, 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
  return status;
}

// Edge plans: the boxes of a staged-kernel plan's ragged tiles, each planned as a transposition of
// its own (default schedule, the caller's streaming choice) so that the staged kernel moves them
// too. A box that cannot be planned leaves all of them to the element-wise ragged-tile kernel.
static void plan_create_edges(ttcb_plan* p) {
  if (p->depth > 0 || p->empty || p->kernel != TTCB_KERNEL_TILE || p->tuning.ragged == 1) return;
  if (p->tuning.tile_variant == 1 || p->tuning.tile_variant == 2) return;  // kernels without ragged split
  const TileDesc* td = reinterpret_cast<const TileDesc*>(p->host_desc.data());
  if (!td->async_ok || td->nrag0 + td->nrag1 == 0) return;
  EdgeBox box[2];
  const int n = plan_edge_boxes(p, box);
  if (n <= 0) return;
  for (int k = 0; k < n; ++k) {
    ttcb_plan* q = new (std::nothrow) ttcb_plan();
    if (!q) break;
    q->rank = box[k].rank;
    for (int i = 0; i < q->rank; ++i) {
      q->perm[i] = box[k].perm[i];
      q->size[i] = box[k].size[i];
      q->lda[i] = box[k].lda[i];
      q->ldb[i] = box[k].ldb[i];
    }
    q->ta = p->ta;
    q->tb = p->tb;
    q->beta_nonzero = p->beta_nonzero;
    q->tuning.streaming = p->tuning.streaming;
    q->depth = 1;
    q->base_offA = box[k].offA;
    q->base_offB = box[k].offB;
    std::string err;
    if (plan_build_host(q, err) != TTCB_OK || plan_finish_device(q) != TTCB_OK) {
      ttcb_plan_destroy(q);
      break;
    }
    p->edge[p->nedge++] = q;
  }
  if (p->nedge != n) {
    for (int k = 0; k < p->nedge; ++k) ttcb_plan_destroy(p->edge[k]);
    p->edge[0] = p->edge[1] = nullptr;
    p->nedge = 0;
    g_last_error.clear();
  }
}

extern "C" {

ttcb_status ttcb_plan_create(ttcb_plan** plan, int rank, const int* perm, const int64_t* size, const int64_t* lda,
                             const int64_t* ldb, ttcb_dtype type_a, ttcb_dtype type_b, int beta_nonzero,
                             const ttcb_tuning* tuning) {
  if (!plan) return fail(TTCB_ERR_INVALID_ARG, "plan output pointer is NULL");
  *plan = nullptr;
  if (rank < 1 || rank > TTCB_MAX_RANK)
    return fail(TTCB_ERR_RANK, "rank must be in [1, " + std::to_string(TTCB_MAX_RANK) + "], got " + std::to_string(rank));
  if (!perm || !size) return fail(TTCB_ERR_INVALID_ARG, "perm and size must not be NULL");
  ttcb_plan* p = new (std::nothrow) ttcb_plan();
  if (!p) return fail(TTCB_ERR_ALLOC, "host allocation of the plan failed");
  p->rank = rank;
  for (int i = 0; i < rank; ++i) {
    p->perm[i] = perm[i];
    p->size[i] = size[i];
  }
  // perm must be checked before ldb's default uses it
  {
    bool seen[TTCB_MAX_RANK] = {false};
    for (int j = 0; j < rank; ++j) {
      if (perm[j] < 0 || perm[j] >= rank || seen[perm[j]]) {
        delete p;
        return fail(TTCB_ERR_BAD_PERM, "permutation is invalid");
      }
      seen[perm[j]] = true;
    }
  }
  for (int i = 0; i < rank; ++i) p->lda[i] = lda ? lda[i] : size[i];
  for (int j = 0; j < rank; ++j) p->ldb[j] = ldb ? ldb[j] : size[perm[j]];
  p->ta = type_a;
  p->tb = type_b;
  p->beta_nonzero = beta_nonzero ? 1 : 0;
  if (tuning) p->tuning = *tuning;
  std::string err;
  ttcb_status s = plan_build_host(p, err);
  if (s != TTCB_OK) {
    delete p;
    return fail(s, err);
  }
  s = plan_finish_device(p);
  if (s != TTCB_OK) {
    ttcb_plan_destroy(p);  // frees whatever the device set-up created
    return s;
  }
  plan_create_edges(p);
  *plan = p;
  return TTCB_OK;
}

void ttcb_plan_destroy(ttcb_plan* plan) {
  if (!plan) return;
  for (int k = 0; k < plan->nedge; ++k) ttcb_plan_destroy(plan->edge[k]);
  if (plan->dev_desc) cudaFree(plan->dev_desc);
  if (plan->claim_words) cudaFree(plan->claim_words);
  if (plan->wait_status) cudaFree(plan->wait_status);
  delete static_cast<std::atomic<unsigned int>*>(plan->launch_count);
  if (plan->side_stream) cudaStreamDestroy(static_cast<cudaStream_t>(plan->side_stream));
  if (plan->ev_fork) cudaEventDestroy(static_cast<cudaEvent_t>(plan->ev_fork));
  if (plan->ev_join) cudaEventDestroy(static_cast<cudaEvent_t>(plan->ev_join));
  delete static_cast<std::mutex*>(plan->fork_mutex);
  delete plan;
}

ttcb_status ttcb_transpose(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                           ttcb_stream_t stream) {
  if (!p) return fail(TTCB_ERR_INVALID_ARG, "plan is NULL");
  if (p->empty) return TTCB_OK;
  if (!A || !B || !alpha) return fail(TTCB_ERR_INVALID_ARG, "A, B and alpha must not be NULL");
  if (p->beta_nonzero && !beta) return fail(TTCB_ERR_BETA, "plan was created for beta != 0 but beta is NULL");
  const int EA = dtype_bytes(p->ta), EB = dtype_bytes(p->tb);
  const int natA = (p->ta == TTCB_C) ? 8 : EA, natB = (p->tb == TTCB_C) ? 8 : EB;
  if ((uintptr_t)A % natA || (uintptr_t)B % natB)
    return fail(TTCB_ERR_ALIGN, "A or B is not aligned to its element size");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != p->device)
    return fail(TTCB_ERR_INVALID_ARG, "plan was created on device " + std::to_string(p->device) +
                                          " but the current device is " + std::to_string(dev));
  return launch_plan(p, A, B, alpha, beta, reinterpret_cast<cudaStream_t>(stream));
}

size_t ttcb_plan_describe(const ttcb_plan* plan, char* buf, size_t len) {
  if (!plan) return 0;
  std::string s = plan_describe_json(plan);
  if (buf && len > 0) {
    size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size() + 1;
}

}  // extern "C"

namespace {
__global__ void bounded_wait_kernel(uint64_t limit_ns, int arrive, unsigned int* gave_up) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = ttcb::smem_u32(&bar);
  if (threadIdx.x == 0) {
    ttcb::mbar_init(b, 1);
    ttcb::mbar_fence_init();
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0) ttcb::mbar_arrive(b);
  const bool done = ttcb::mbar_wait_bounded(b, 0, limit_ns);
  if (__syncthreads_or(!done) && threadIdx.x == 0) atomicAdd(gave_up, 1u);
}
}  // namespace

extern "C" {
int ttcb_test_bounded_wait(uint64_t limit_ns, int arrive, unsigned int* gave_up) {
  unsigned int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(unsigned int));
  if (e != cudaSuccess) return (int)e;
  e = cudaMemset(d, 0, sizeof(unsigned int));
  if (e == cudaSuccess) {
    bounded_wait_kernel<<<1, 64>>>(limit_ns, arrive, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(gave_up, d, sizeof(unsigned int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

ttcb_status ttcb_plan_wait_timeouts(const ttcb_plan* p, unsigned int* count) {
  if (!p || !count) return fail(TTCB_ERR_INVALID_ARG, "plan and count must not be NULL");
  *count = 0;
  if (!p->wait_status) return TTCB_OK;
  cudaError_t e = cudaMemcpy(count, p->wait_status, sizeof(unsigned int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy of the wait status");
  if (*count && (e = cudaMemset(p->wait_status, 0, sizeof(unsigned int))) != cudaSuccess)
    return cuda_fail(e, "cudaMemset of the wait status");
  return TTCB_OK;
}

int64_t ttcb_plan_bytes(const ttcb_plan* p) {
  if (!p) return 0;
  return p->N * (dtype_bytes(p->ta) + (p->beta_nonzero ? 2 : 1) * dtype_bytes(p->tb));
}

const char* ttcb_last_error(void) { return g_last_error.c_str(); }

void ttcb_internal_set_error(const char* msg) { g_last_error = msg ? msg : ""; }

void ttcb_version(int* major, int* minor, int* patch) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  if (patch) *patch = 0;
}

// ---------------------------------------------------------------------------------------------
// Test hooks (declared in testing.h, not part of the public header).
int ttcb_test_fuse(int rank, const int* perm, const int64_t* n, const int64_t* sA, const int64_t* sB, int* out_rank,
                   int* out_perm, int64_t* out_n, int64_t* out_sA, int64_t* out_sB) {
  if (rank < 1 || rank > TTCB_MAX_RANK) return -1;
  FusedProblem f;
  fuse_problem(rank, perm, n, sA, sB, f);
  *out_rank = f.rank;
  for (int i = 0; i < f.rank; ++i) {
    out_perm[i] = f.perm[i];
    out_n[i] = f.n[i];
    out_sA[i] = f.sA[i];
    out_sB[i] = f.sB[i];
  }
  return 0;
}

// Builds the host part of a plan (no CUDA calls) and returns its JSON description.
size_t ttcb_test_plan_shapes(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                             int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tunings, int n, char* buf,
                             size_t len) {
  std::string js = "[";
  plan_tile_cache_begin();
  for (int k = 0; k < n; ++k) {
    ttcb_plan p;
    p.shape_only = true;
    bool ok = rank >= 1 && rank <= TTCB_MAX_RANK;
    for (int j = 0; ok && j < rank; ++j) ok = perm[j] >= 0 && perm[j] < rank;
    if (ok) {
      p.rank = rank;
      for (int i = 0; i < rank; ++i) {
        p.perm[i] = perm[i];
        p.size[i] = size[i];
        p.lda[i] = lda ? lda[i] : size[i];
      }
      for (int j = 0; j < rank; ++j) p.ldb[j] = ldb ? ldb[j] : size[perm[j]];
      p.ta = (ttcb_dtype)type_a;
      p.tb = (ttcb_dtype)type_b;
      p.beta_nonzero = beta_nonzero;
      if (tunings) p.tuning = tunings[k];
      std::string err;
      ok = plan_build_host(&p, err) == TTCB_OK;
    }
    js += (k ? "," : "");
    js += ok ? plan_describe_json(&p) : std::string("null");
  }
  plan_tile_cache_end();
  js += "]";
  if (buf && len) {
    size_t m = std::min(len - 1, js.size());
    std::memcpy(buf, js.data(), m);
    buf[m] = 0;
  }
  return js.size() + 1;
}

int ttcb_test_plan_host(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                        int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tuning, char* buf, size_t len) {
  ttcb_plan p;
  p.rank = rank;
  if (rank < 1 || rank > TTCB_MAX_RANK) return TTCB_ERR_RANK;
  for (int i = 0; i < rank; ++i) {
    p.perm[i] = perm[i];
    p.size[i] = size[i];
  }
  for (int j = 0; j < rank; ++j)
    if (perm[j] < 0 || perm[j] >= rank) return TTCB_ERR_BAD_PERM;
  for (int i = 0; i < rank; ++i) p.lda[i] = lda ? lda[i] : size[i];
  for (int j = 0; j < rank; ++j) p.ldb[j] = ldb ? ldb[j] : size[perm[j]];
  p.ta = (ttcb_dtype)type_a;
  p.tb = (ttcb_dtype)type_b;
  p.beta_nonzero = beta_nonzero;
  if (tuning) p.tuning = *tuning;
  std::string err;
  ttcb_status s = plan_build_host(&p, err);
  if (s != TTCB_OK) {
    g_last_error = err;
    return s;
  }
  std::string js = plan_describe_json(&p);
  if (buf && len) {
    size_t n = std::min(len - 1, js.size());
    std::memcpy(buf, js.data(), n);
    buf[n] = 0;
  }
  return 0;
}

// Host-side copy of a plan's descriptor tables (for CPU checks of the tile tables).
size_t ttcb_test_plan_desc(const ttcb_plan* p, void* buf, size_t len) {
  if (!p) return 0;
  if (buf && len >= p->host_desc.size()) std::memcpy(buf, p->host_desc.data(), p->host_desc.size());
  return p->host_desc.size();
}

// Host-only plan build that returns the descriptor bytes (tile or row tables) and the kernel kind.
size_t ttcb_test_plan_host_desc(int rank, const int* perm, const int64_t* size, const int64_t* lda,
                                const int64_t* ldb, int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tuning,
                                int* kernel, void* buf, size_t len) {
  ttcb_plan p;
  if (rank < 1 || rank > TTCB_MAX_RANK) return 0;
  p.rank = rank;
  for (int i = 0; i < rank; ++i) {
    p.perm[i] = perm[i];
    p.size[i] = size[i];
  }
  for (int j = 0; j < rank; ++j)
    if (perm[j] < 0 || perm[j] >= rank) return 0;
  for (int i = 0; i < rank; ++i) p.lda[i] = lda ? lda[i] : size[i];
  for (int j = 0; j < rank; ++j) p.ldb[j] = ldb ? ldb[j] : size[perm[j]];
  p.ta = (ttcb_dtype)type_a;
  p.tb = (ttcb_dtype)type_b;
  p.beta_nonzero = beta_nonzero;
  if (tuning) p.tuning = *tuning;
  std::string err;
  if (plan_build_host(&p, err) != TTCB_OK) {
    g_last_error = err;
    return 0;
  }
  if (kernel) *kernel = p.kernel;
  if (buf && len >= p.host_desc.size()) std::memcpy(buf, p.host_desc.data(), p.host_desc.size());
  return p.host_desc.size();
}

size_t ttcb_test_plan_edges(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                            int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tuning, char* buf, size_t len) {
  ttcb_plan p;
  if (rank < 1 || rank > TTCB_MAX_RANK) return 0;
  p.rank = rank;
  for (int i = 0; i < rank; ++i) {
    p.perm[i] = perm[i];
    p.size[i] = size[i];
  }
  for (int j = 0; j < rank; ++j)
    if (perm[j] < 0 || perm[j] >= rank) return 0;
  for (int i = 0; i < rank; ++i) p.lda[i] = lda ? lda[i] : size[i];
  for (int j = 0; j < rank; ++j) p.ldb[j] = ldb ? ldb[j] : size[perm[j]];
  p.ta = (ttcb_dtype)type_a;
  p.tb = (ttcb_dtype)type_b;
  p.beta_nonzero = beta_nonzero;
  if (tuning) p.tuning = *tuning;
  std::string err;
  if (plan_build_host(&p, err) != TTCB_OK) {
    g_last_error = err;
    return 0;
  }
  EdgeBox box[2];
  const int n = p.kernel == TTCB_KERNEL_TILE ? plan_edge_boxes(&p, box) : 0;
  std::ostringstream o;
  o << "[";
  for (int k = 0; k < n; ++k) {
    const EdgeBox& b = box[k];
    o << (k ? "," : "") << "{\"rank\":" << b.rank;
    const char* names[] = {"perm", "size", "lda", "ldb"};
    for (int a = 0; a < 4; ++a) {
      o << ",\"" << names[a] << "\":[";
      for (int i = 0; i < b.rank; ++i)
        o << (i ? "," : "") << (a == 0 ? (int64_t)b.perm[i] : a == 1 ? b.size[i] : a == 2 ? b.lda[i] : b.ldb[i]);
      o << "]";
    }
    o << ",\"offA\":" << b.offA << ",\"offB\":" << b.offB << "}";
  }
  o << "]";
  const std::string js = o.str();
  if (buf && len) {
    size_t m = std::min(len - 1, js.size());
    std::memcpy(buf, js.data(), m);
    buf[m] = 0;
  }
  return js.size() + 1;
}

// Layout of the descriptor structs, so host-side checkers can parse them.
void ttcb_test_desc_layout(int64_t* out) {
  out[0] = sizeof(TileDesc);
  out[1] = offsetof(TileDesc, divLA);
  out[2] = offsetof(TileDesc, g);
  out[3] = sizeof(GridDimDesc);
  out[4] = offsetof(TileDesc, bd);
  out[5] = sizeof(BlockedDesc);
  out[6] = sizeof(RowDesc);
  out[7] = offsetof(RowDesc, div);
  out[8] = offsetof(RowDesc, sA);
  out[9] = offsetof(RowDesc, sB);
  out[10] = sizeof(FastDiv);
  out[11] = offsetof(GridDimDesc, strideA);
  out[12] = offsetof(TileDesc, shiftA);
}

uint32_t ttcb_test_fastdiv(uint32_t n, uint32_t d) {
  FastDiv f = make_fastdiv(d);
  return fdiv(n, f);
}

}  // extern "C"
