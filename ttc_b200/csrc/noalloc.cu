// Allocation-free entry point: ttcb_transpose_noalloc().
//
// Who needs it: code that may not allocate device memory at the point where it transposes - for
// example a caller whose device memory is owned by an external pool that hands out only the
// tensors themselves, or a caller in a section where cudaMalloc is forbidden (it can synchronize the
// device or fail). ttcb_plan_create() allocates a small device descriptor with cudaMalloc; this
// entry point instead writes the descriptor into one fixed scratch array that is part of the
// library image, so no device allocation happens at all.
//
// The scratch array is a file-scope __device__ array of kNoAllocScratchBytes. Every GPU that loads
// the library keeps it until the process exits. Each call rewrites all scratch bytes that its kernel
// reads (nothing must start at zero), so back-to-back calls on one stream are safe; calls that
// overlap on the GPU (different streams, or several host threads) race on the array.
//
// On the first call on each device this entry point looks up the device address of the array with
// cudaGetSymbolAddress (the symbol's name is only a host-side stand-in, not a device address). That
// first call on a device should therefore come before any stream capture.
//
// The descriptor reaches the scratch array through a cudaMemcpyAsync from host memory that exists
// only while the call runs. A call made while its stream is being captured would record a copy node
// that reads that host memory again at every replay, long after it was freed, so such a call is
// refused with TTCB_ERR_UNSUPPORTED before anything is enqueued.
//
// The kernels' dynamic shared memory limit is raised through the same once-per-device opt-in as
// the plan entry points use (ttcb::allow_large_smem), which never lowers a limit that a plan made
// earlier relies on.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/ttcb200.h"
#include "kernels.cuh"
#include "launch.h"
#include "plan.h"

static constexpr size_t kNoAllocScratchBytes = 64 * 1024;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Largest descriptor the entry point accepts: the scratch size, or less when a CPU test lowers it
// (ttcb_test_noalloc_limit) to reach the rejection path with an ordinary problem.
static size_t g_noalloc_limit = kNoAllocScratchBytes;

extern "C" void ttcb_internal_set_error(const char* msg);

static ttcb_status na_fail(ttcb_status s, const std::string& m) {
  ttcb_internal_set_error(m.c_str());
  return s;
}

static ttcb_status na_cuda(cudaError_t e, const char* what) {
  return na_fail(TTCB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

// Device address of the scratch array for the current device, looked up once per device.
static ttcb_status scratch_address(int dev, void** out) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  if (dev < 0 || dev >= 64) return na_fail(TTCB_ERR_UNSUPPORTED, "device index beyond 63");
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return na_cuda(e, "cudaGetSymbolAddress of the no-allocation scratch");
    addr[dev] = p;
  }
  *out = addr[dev];
  return TTCB_OK;
}

extern "C" ttcb_status ttcb_transpose_noalloc(int rank, const int* perm, const int64_t* size, const int64_t* lda,
                                              const int64_t* ldb, ttcb_dtype type_a, ttcb_dtype type_b,
                                              const void* A, void* B, const void* alpha, const void* beta,
                                              ttcb_stream_t stream) {
  if (rank < 1 || rank > TTCB_MAX_RANK)
    return na_fail(TTCB_ERR_RANK, "rank must be in [1, " + std::to_string(TTCB_MAX_RANK) + "]");
  if (!perm || !size || !A || !B || !alpha) return na_fail(TTCB_ERR_INVALID_ARG, "NULL argument");
  ttcb_plan p;
  p.rank = rank;
  for (int i = 0; i < rank; ++i) {
    p.perm[i] = perm[i];
    p.size[i] = size[i];
  }
  for (int j = 0; j < rank; ++j)
    if (perm[j] < 0 || perm[j] >= rank) return na_fail(TTCB_ERR_BAD_PERM, "permutation is invalid");
  for (int i = 0; i < rank; ++i) p.lda[i] = lda ? lda[i] : size[i];
  for (int j = 0; j < rank; ++j) p.ldb[j] = ldb ? ldb[j] : size[perm[j]];
  p.ta = type_a;
  p.tb = type_b;
  p.beta_nonzero = beta ? 1 : 0;
  p.tuning.kernel = TTCB_KERNEL_TILE;  // one kernel family: the staged tile transpose
  std::string err;
  ttcb_status s = plan_build_host(&p, err);
  if (s != TTCB_OK) return na_fail(s, err);
  if (p.empty) return TTCB_OK;
  const TileDesc* td = reinterpret_cast<const TileDesc*>(p.host_desc.data());
  if (!td->async_ok) return na_fail(TTCB_ERR_UNSUPPORTED, "problem needs offsets beyond 32 bits");
  if (p.host_desc.size() > g_noalloc_limit)
    return na_fail(TTCB_ERR_UNSUPPORTED, "descriptor needs " + std::to_string(p.host_desc.size()) +
                                             " bytes of scratch; the no-allocation entry point holds at most " +
                                             std::to_string(g_noalloc_limit));
  const int EA = dtype_bytes(p.ta), EB = dtype_bytes(p.tb);
  const int natA = (p.ta == TTCB_C) ? 8 : EA, natB = (p.tb == TTCB_C) ? 8 : EB;
  if ((uintptr_t)A % natA || (uintptr_t)B % natB)
    return na_fail(TTCB_ERR_ALIGN, "A or B is not aligned to its element size");

  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return na_cuda(e, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return na_fail(TTCB_ERR_UNSUPPORTED,
                   "ttcb_transpose_noalloc cannot be called while its stream is being captured: it uploads the "
                   "descriptor from host memory that exists only during the call");
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_cuda(e, "cudaGetDevice");
  void* scratch = nullptr;
  if ((s = scratch_address(dev, &scratch)) != TTCB_OK) return s;
  e = cudaMemcpyAsync(scratch, p.host_desc.data(), p.host_desc.size(), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return na_cuda(e, "descriptor upload to the scratch array");
  p.dev_desc = scratch;
  p.device = dev;

  int va = p.vecA, vb = p.vecB;
  while (!td->shiftA && va > 1 && (uintptr_t)A % (va * EA)) va /= 2;  // shifted runs take any pointer
  while (vb > 1 && (uintptr_t)B % (vb * EB)) vb /= 2;
  const bool reg = td->reg_ok && td->P / va <= 1024 && td->P / vb <= 1024;
  const int kernel = reg ? TTCB_KERNEL_TILE_ASYNC_REG : TTCB_KERNEL_TILE_ASYNC;
  const int variant = p.beta_nonzero ? 2 : (p.streaming ? 1 : 0);
  ttcb::KernelRef k = ttcb::pick_kernel(p.ta, p.tb, kernel, va, vb, variant);
  if (!k.fn) return na_fail(TTCB_ERR_DTYPE, "no kernel for this type pair");
  if (ttcb::needs_large_smem(p.smem_async)) ttcb::allow_large_smem(k.func);
  int sms = 0, per_sm = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return na_cuda(e, "cudaDeviceGetAttribute");
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.func, ttcb::kThreads, p.smem_async)) !=
      cudaSuccess)
    return na_cuda(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (per_sm < 1) return na_fail(TTCB_ERR_UNSUPPORTED, "tile does not fit in shared memory");
  const int64_t work = td->nfull, resident = (int64_t)per_sm * sms;
  const int64_t per = (work + resident - 1) / resident;
  p.blocks_async = (int)std::max<int64_t>((work + per - 1) / per, 1);
  e = k.fn(&p, A, B, alpha, beta, st, p.blocks_async);
  if (e == cudaSuccess && td->nrag0 + td->nrag1 > 0) {
    // the staged kernel moves complete tiles only; the ragged ones follow on the same stream
    ttcb::KernelRef kr = ttcb::pick_kernel(p.ta, p.tb, TTCB_KERNEL_TILE_RAGGED, 1, 1, variant);
    if (!kr.fn) {
      p.dev_desc = nullptr;
      return na_fail(TTCB_ERR_DTYPE, "no ragged-tile kernel for this type pair");
    }
    if (ttcb::needs_large_smem(p.smem_ragged)) ttcb::allow_large_smem(kr.func);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kr.func, ttcb::kThreads, p.smem_ragged)) ==
        cudaSuccess) {
      const int64_t rw = (int64_t)td->nrag0 + td->nrag1, rres = (int64_t)std::max(per_sm, 1) * sms;
      const int64_t rper = (rw + rres - 1) / rres;
      e = kr.fn(&p, A, B, alpha, beta, st, (int)std::max<int64_t>((rw + rper - 1) / rper, 1));
    }
  }
  p.dev_desc = nullptr;  // the scratch belongs to the library, not to this stack plan
  if (e != cudaSuccess) return na_cuda(e, "kernel launch");
  return TTCB_OK;
}

// Test hook (testing.h): lowers the largest descriptor the entry point accepts (0 restores the
// scratch size), so that a CPU test reaches the rejection with an ordinary problem. No CUDA call.
extern "C" size_t ttcb_test_noalloc_limit(size_t bytes) {
  g_noalloc_limit = (bytes == 0 || bytes > kNoAllocScratchBytes) ? kNoAllocScratchBytes : bytes;
  return kNoAllocScratchBytes;
}
