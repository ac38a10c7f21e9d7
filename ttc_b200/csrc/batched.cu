// C ABI of batched mode: one persistent launch (optionally replayed from a captured CUDA graph)
// for many independent transpositions, each with the schedule of its own plan.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <memory>
#include <vector>

#include "../../include/ttcb200.h"
#include "batch_kernels.cuh"
#include "launch.h"
#include "plan.h"

namespace ttcb {
BatchKernelRef pick_batch_ss(int);
BatchKernelRef pick_batch_dd(int);
BatchKernelRef pick_batch_cc(int);
BatchKernelRef pick_batch_zz(int);
BatchKernelRef pick_batch_sd(int);
BatchKernelRef pick_batch_ds(int);
BatchKernelRef pick_batch_cz(int);
BatchKernelRef pick_batch_zc(int);

BatchKernelRef pick_batch_kernel(ttcb_dtype ta, ttcb_dtype tb, int variant) {
  if (ta == TTCB_S && tb == TTCB_S) return pick_batch_ss(variant);
  if (ta == TTCB_D && tb == TTCB_D) return pick_batch_dd(variant);
  if (ta == TTCB_C && tb == TTCB_C) return pick_batch_cc(variant);
  if (ta == TTCB_Z && tb == TTCB_Z) return pick_batch_zz(variant);
  if (ta == TTCB_S && tb == TTCB_D) return pick_batch_sd(variant);
  if (ta == TTCB_D && tb == TTCB_S) return pick_batch_ds(variant);
  if (ta == TTCB_C && tb == TTCB_Z) return pick_batch_cz(variant);
  if (ta == TTCB_Z && tb == TTCB_C) return pick_batch_zc(variant);
  return BatchKernelRef();
}
}  // namespace ttcb

struct ttcb_batch {
  int count = 0;
  ttcb_dtype ta = TTCB_S, tb = TTCB_S;
  int beta_nonzero = 0;
  bool streaming = false;
  int device = 0;
  unsigned char alpha[16] = {0};
  unsigned char beta[16] = {0};
  int64_t bytes = 0;
  unsigned long long total = 0;
  int blocks = 0;
  int smem = 0;         // the stage buffers + the largest problem's tables
  int slots_bytes = 0;  // one stage buffer (the largest staged tile)
  int chunk = 1;        // items claimed per atomic
  void* d_probs = nullptr;
  int64_t* d_prefix = nullptr;
  unsigned char* d_desc = nullptr;
  unsigned long long* d_counter = nullptr;  // [0] next item, [1] status word (as int)
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaStream_t capture_stream = nullptr;
};

// The thread-local last-error message lives in abi.cu.
extern "C" void ttcb_internal_set_error(const char* msg);
static ttcb_status bfail(ttcb_status s, const std::string& msg) {
  ttcb_internal_set_error(msg.c_str());
  return s;
}
static ttcb_status bcuda(cudaError_t e, const char* what) {
  return bfail(TTCB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

static void batch_free(ttcb_batch* b) {
  if (!b) return;
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  if (b->d_probs) cudaFree(b->d_probs);
  if (b->d_prefix) cudaFree(b->d_prefix);
  if (b->d_desc) cudaFree(b->d_desc);
  if (b->d_counter) cudaFree(b->d_counter);
  delete b;
}

static int batch_variant(const ttcb_batch* b) { return b->beta_nonzero ? 2 : (b->streaming ? 1 : 0); }

extern "C" {

ttcb_status ttcb_batch_create(ttcb_batch** out, int count, const ttcb_plan* const* plans, const void* const* A,
                              void* const* B, const void* alpha, const void* beta, int blocks) {
  if (!out) return bfail(TTCB_ERR_INVALID_ARG, "batch output pointer is NULL");
  *out = nullptr;
  if (count < 1 || !plans || !A || !B || !alpha) return bfail(TTCB_ERR_INVALID_ARG, "empty batch or NULL argument");
  const ttcb_plan* p0 = plans[0];
  if (!p0) return bfail(TTCB_ERR_INVALID_ARG, "plan 0 is NULL");
  if (p0->beta_nonzero && !beta) return bfail(TTCB_ERR_BETA, "plans were created for beta != 0 but beta is NULL");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bcuda(e, "cudaGetDevice");
  const int EA = dtype_bytes(p0->ta), EB = dtype_bytes(p0->tb);

  ttcb_batch* b = new (std::nothrow) ttcb_batch();
  if (!b) return bfail(TTCB_ERR_ALLOC, "host allocation of the batch failed");
  b->count = count;
  b->ta = p0->ta;
  b->tb = p0->tb;
  b->beta_nonzero = p0->beta_nonzero;
  b->streaming = p0->streaming;
  b->device = dev;
  std::memcpy(b->alpha, alpha, EA);
  if (p0->beta_nonzero) std::memcpy(b->beta, beta, EB);

  // Problems of the batch: every plan, and for a plan whose ragged tiles its edge plans move, those
  // edge plans as problems of their own (offset into the plan's A and B) while the plan keeps only
  // its complete tiles.
  struct Entry {
    const ttcb_plan* p;
    const void* A;
    void* B;
    int full_only;  // the plan's complete tiles only (its edge plans follow it)
    int user;       // index of the caller's plan
    int own;        // 1: the caller's plan itself (0: one of its edge plans)
  };
  std::vector<Entry> ent;
  ent.reserve(count);
  for (int i = 0; i < count; ++i) {
    const ttcb_plan* p = plans[i];
    if (!p) {
      batch_free(b);
      return bfail(TTCB_ERR_INVALID_ARG, "plan " + std::to_string(i) + " is NULL");
    }
    if (p->ta != b->ta || p->tb != b->tb || p->beta_nonzero != b->beta_nonzero) {
      batch_free(b);
      return bfail(TTCB_ERR_INVALID_ARG, "all plans of a batch need the same types and beta flag");
    }
    if (p->device != dev && !p->empty) {
      batch_free(b);
      return bfail(TTCB_ERR_INVALID_ARG, "plan " + std::to_string(i) + " belongs to another device");
    }
    if (!p->empty && (!A[i] || !B[i])) {
      batch_free(b);
      return bfail(TTCB_ERR_INVALID_ARG, "A or B of problem " + std::to_string(i) + " is NULL");
    }
    const bool edges = !p->empty && p->kernel == TTCB_KERNEL_TILE && p->nedge > 0;
    ent.push_back({p, A[i], B[i], edges ? 1 : 0, i, 1});
    for (int k = 0; edges && k < p->nedge; ++k) {
      const ttcb_plan* q = p->edge[k];
      ent.push_back({q, static_cast<const char*>(A[i]) + q->base_offA * EA,
                     static_cast<char*>(B[i]) + q->base_offB * EB, 0, i, 0});
    }
  }
  // The batched kernel stages A in the plain layout (element p at p + (p / sigmaA) * padA); a plan
  // with shifted A runs takes part through a host copy of itself planned without them.
  std::vector<std::unique_ptr<ttcb_plan>> unshifted;
  for (Entry& e : ent) {
    const ttcb_plan* p = e.p;
    if (p->empty || p->kernel != TTCB_KERNEL_TILE) continue;
    if (!reinterpret_cast<const TileDesc*>(p->host_desc.data())->shiftA) continue;
    std::unique_ptr<ttcb_plan> q(new (std::nothrow) ttcb_plan());
    if (!q) {
      batch_free(b);
      return bfail(TTCB_ERR_ALLOC, "host allocation of a batch problem failed");
    }
    q->rank = p->rank;
    for (int i = 0; i < p->rank; ++i) {
      q->perm[i] = p->perm[i];
      q->size[i] = p->size[i];
      q->lda[i] = p->lda[i];
      q->ldb[i] = p->ldb[i];
    }
    q->ta = p->ta;
    q->tb = p->tb;
    q->beta_nonzero = p->beta_nonzero;
    q->tuning = p->tuning;
    q->tuning.shifted_runs = -1;
    q->depth = p->depth;
    q->base_offA = p->base_offA;
    q->base_offB = p->base_offB;
    q->device = p->device;
    std::string err;
    if (plan_build_host(q.get(), err) != TTCB_OK || q->kernel != TTCB_KERNEL_TILE ||
        q->host_desc.size() < sizeof(TileDesc)) {
      batch_free(b);
      return bfail(TTCB_ERR_UNSUPPORTED, "a batch problem could not be planned for the batched kernel: " + err);
    }
    // the batch moves the complete tiles of the same grid: the tile must not change
    const TileDesc* a = reinterpret_cast<const TileDesc*>(p->host_desc.data());
    const TileDesc* c = reinterpret_cast<const TileDesc*>(q->host_desc.data());
    if (a->P != c->P || a->ntiles != c->ntiles || a->nfull != c->nfull) {
      batch_free(b);
      return bfail(TTCB_ERR_UNSUPPORTED, "a batch problem planned without shifted runs changed its tiles");
    }
    e.p = q.get();
    unshifted.push_back(std::move(q));
  }
  const int n = (int)ent.size();
  b->count = n;

  // descriptors back to back, 16-byte aligned
  std::vector<int64_t> desc_off(n, -1);
  int64_t desc_bytes = 0;
  for (int i = 0; i < n; ++i) {
    if (!ent[i].p->empty) {
      desc_off[i] = desc_bytes;
      desc_bytes += (ent[i].p->host_desc.size() + 15) & ~size_t(15);
    }
  }
  std::vector<unsigned char> hdesc(std::max<int64_t>(desc_bytes, 16), 0);
  std::vector<ttcb::BatchProblem> hp(n);
  std::vector<int64_t> prefix(n + 1, 0);
  int max_slots_bytes = 0, max_table_bytes = 0;
  for (int i = 0; i < n; ++i) {
    const ttcb_plan* p = ent[i].p;
    ttcb::BatchProblem& q = hp[i];
    std::memset(&q, 0, sizeof(q));
    int64_t items = 0;
    if (!p->empty) {
      std::memcpy(hdesc.data() + desc_off[i], p->host_desc.data(), p->host_desc.size());
      q.A = ent[i].A;
      q.B = ent[i].B;
      q.kind = p->kernel;
      q.va = p->vecA;
      q.vb = p->vecB;
      q.full_only = ent[i].full_only;
      while (q.va > 1 && (uintptr_t)q.A % (q.va * EA)) q.va /= 2;
      while (q.vb > 1 && (uintptr_t)q.B % (q.vb * EB)) q.vb /= 2;
      if (p->kernel == TTCB_KERNEL_ROW) {
        q.va = q.vb = std::min(q.va, q.vb);
        const RowDesc* rd = reinterpret_cast<const RowDesc*>(p->host_desc.data());
        items = (rd->nunits + 7) / 8;
      } else {
        const TileDesc* td = reinterpret_cast<const TileDesc*>(p->host_desc.data());
        items = ent[i].full_only ? td->nfull : td->ntiles;
        // one stage buffer: the staged layout (or, for a ragged tile, the slots), 16-byte aligned
        max_slots_bytes = std::max<int>(
            max_slots_bytes, (int)ttcb::al16((size_t)std::max(td->stage_elems, td->phys_size) * EA));
        max_table_bytes = std::max<int>(max_table_bytes, 8 * (td->nsegA + td->nsegB) + 4 * ((td->P + 1) / 2));
      }
      if (ent[i].own) b->bytes += ttcb_plan_bytes(p);  // an edge plan's bytes are its parent's
    }
    prefix[i + 1] = prefix[i] + items;
  }
  b->total = (unsigned long long)prefix[n];
  b->slots_bytes = (int)((max_slots_bytes + 15) & ~15);
  b->smem = ttcb::kBatchStages * b->slots_bytes + max_table_bytes;  // stage buffers, then the tables

  // device copies
  if ((e = cudaMalloc(&b->d_desc, hdesc.size())) != cudaSuccess ||
      (e = cudaMalloc(&b->d_probs, sizeof(ttcb::BatchProblem) * n)) != cudaSuccess ||
      (e = cudaMalloc(&b->d_prefix, sizeof(int64_t) * (n + 1))) != cudaSuccess ||
      (e = cudaMalloc(&b->d_counter, 2 * sizeof(unsigned long long))) != cudaSuccess) {
    cudaGetLastError();
    batch_free(b);
    return bfail(TTCB_ERR_ALLOC, std::string("cudaMalloc for the batch failed: ") + cudaGetErrorString(e));
  }
  for (int i = 0; i < n; ++i)
    if (desc_off[i] >= 0) hp[i].desc = b->d_desc + desc_off[i];
  if ((e = cudaMemcpy(b->d_desc, hdesc.data(), hdesc.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->d_probs, hp.data(), sizeof(ttcb::BatchProblem) * n, cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemcpy(b->d_prefix, prefix.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemset(b->d_counter, 0, 2 * sizeof(unsigned long long))) != cudaSuccess) {
    batch_free(b);
    return bcuda(e, "batch descriptor upload");
  }

  ttcb::BatchKernelRef k = ttcb::pick_batch_kernel(b->ta, b->tb, batch_variant(b));
  if (!k.func) {
    batch_free(b);
    return bfail(TTCB_ERR_DTYPE, "no batched kernel for this type pair");
  }
  if (b->smem + (int)sizeof(TileDesc) + 64 > 48 * 1024)  // + its static header copy, item and problem index
    ttcb::allow_large_smem(k.func);
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.func, ttcb::kThreads, b->smem);
  if (e != cudaSuccess || per_sm < 1) {
    batch_free(b);
    return e != cudaSuccess ? bcuda(e, "occupancy query") : bfail(TTCB_ERR_UNSUPPORTED, "batch tile too large");
  }
  int64_t resident = (int64_t)per_sm * sms;
  int64_t nb = blocks > 0 ? blocks : resident;
  nb = std::min<int64_t>(nb, std::max<unsigned long long>(b->total, 1ull));
  b->blocks = (int)std::max<int64_t>(nb, 1);
  // about sixteen claims per CTA keep the tail balanced while amortising the claim and its search
  b->chunk = (int)std::max<unsigned long long>(1ull, std::min<unsigned long long>(
                                                         32ull, b->total / (16ull * (unsigned long long)b->blocks)));
  *out = b;
  return TTCB_OK;
}

static ttcb_status batch_enqueue(ttcb_batch* b, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return bcuda(e, "counter reset");
  if (b->total == 0) return TTCB_OK;
  ttcb::BatchKernelRef k = ttcb::pick_batch_kernel(b->ta, b->tb, batch_variant(b));
  e = k.fn(b->d_probs, b->d_prefix, b->count, b->total, b->d_counter,
           reinterpret_cast<int*>(b->d_counter + 1), b->alpha, b->beta, b->blocks, b->smem, b->slots_bytes,
           b->chunk, s);
  if (e != cudaSuccess) return bcuda(e, "batched kernel launch");
  return TTCB_OK;
}

ttcb_status ttcb_batch_launch(ttcb_batch* b, ttcb_stream_t stream) {
  if (!b) return bfail(TTCB_ERR_INVALID_ARG, "batch is NULL");
  return batch_enqueue(b, reinterpret_cast<cudaStream_t>(stream));
}

ttcb_status ttcb_batch_graph_launch(ttcb_batch* b, ttcb_stream_t stream) {
  if (!b) return bfail(TTCB_ERR_INVALID_ARG, "batch is NULL");
  cudaError_t e;
  if (!b->graph_exec) {
    // capture once on a private stream (the legacy default stream cannot be captured)
    if ((e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
      return bcuda(e, "cudaStreamCreate");
    if ((e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return bcuda(e, "cudaStreamBeginCapture");
    ttcb_status st = batch_enqueue(b, b->capture_stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->capture_stream, &g);
    if (st != TTCB_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return bcuda(e, "cudaStreamEndCapture");
    b->graph = g;
    if ((e = cudaGraphInstantiate(&b->graph_exec, g, 0)) != cudaSuccess) {
      b->graph_exec = nullptr;
      return bcuda(e, "cudaGraphInstantiate");
    }
  }
  if ((e = cudaGraphLaunch(b->graph_exec, reinterpret_cast<cudaStream_t>(stream))) != cudaSuccess)
    return bcuda(e, "cudaGraphLaunch");
  return TTCB_OK;
}

ttcb_status ttcb_batch_status(ttcb_batch* b, ttcb_stream_t stream) {
  if (!b) return bfail(TTCB_ERR_INVALID_ARG, "batch is NULL");
  int st = 0;
  cudaError_t e = cudaMemcpyAsync(&st, b->d_counter + 1, sizeof(int), cudaMemcpyDeviceToHost,
                                  reinterpret_cast<cudaStream_t>(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return bcuda(e, "batch status read");
  if (st != 0) return bfail(TTCB_ERR_INVALID_ARG, "batched kernel reported status " + std::to_string(st));
  return TTCB_OK;
}

int64_t ttcb_batch_bytes(const ttcb_batch* b) { return b ? b->bytes : 0; }

void ttcb_batch_destroy(ttcb_batch* b) { batch_free(b); }

}  // extern "C"
