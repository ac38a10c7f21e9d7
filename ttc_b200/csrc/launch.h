// Launch dispatch shared by the plain and batched entry points.
#pragma once
#include <cuda_runtime.h>
#include "plan.h"

namespace ttcb {

// Launches one plan. va/vb are the access widths actually used (the plan's widths, or 1 when a
// pointer is not 16-byte aligned). variant: 0 = beta==0, 1 = beta==0 with streaming stores,
// 2 = beta != 0.
using LaunchFn = cudaError_t (*)(const ttcb_plan* p, const void* A, void* B, const void* alpha, const void* beta,
                                 cudaStream_t stream, int blocks);

struct KernelRef {
  LaunchFn fn = nullptr;
  const void* func = nullptr;  // the __global__ function (for occupancy queries and attributes)
};

// One definition per A/B type pair lives in kernels_<pair>.cu.
KernelRef pick_kernel(ttcb_dtype ta, ttcb_dtype tb, int kernel, int va, int vb, int variant);

// The counter words (claim, finished CTAs) of the next launch of a plan's staged kernel with claimed
// tiles: one of the plan's kClaimSlots slot pairs, taken in turn, so launches of one plan on
// different streams use different words (up to kClaimSlots of them in flight). Null when the plan
// has no counters.
constexpr int kClaimSlots = 64;
unsigned int* plan_claim_slot(const ttcb_plan* p);

// Dynamic shared memory ceiling of every plan (the planner never exceeds it).
constexpr int kMaxDynamicSmem = 200 * 1024;
// True when a launch with this much dynamic shared memory needs the opt-in above 48 KB.
bool needs_large_smem(int dynamic_smem);
// Raises func's dynamic shared memory limit to kMaxDynamicSmem on the current device, once; it
// never lowers it. Every entry point that launches a kernel goes through this (defined in abi.cu).
void allow_large_smem(const void* func);

using BatchLaunchFn = cudaError_t (*)(const void* probs, const int64_t* prefix, int count, unsigned long long total,
                                      unsigned long long* counter, int* status, const void* alpha, const void* beta,
                                      int blocks, int smem, int slots_bytes, int chunk, cudaStream_t stream);
struct BatchKernelRef {
  BatchLaunchFn fn = nullptr;
  const void* func = nullptr;
};
BatchKernelRef pick_batch_kernel(ttcb_dtype ta, ttcb_dtype tb, int variant);

}  // namespace ttcb
