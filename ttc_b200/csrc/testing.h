// Test hooks exported by libttcb200.so for unit tests. They are not part of the public ABI
// (include/ttcb200.h); all but ttcb_test_bounded_wait make no CUDA calls.
#pragma once
#include <cstddef>
#include <cstdint>
#include "../../include/ttcb200.h"

extern "C" {
int ttcb_test_fuse(int rank, const int* perm, const int64_t* n, const int64_t* sA, const int64_t* sB, int* out_rank,
                   int* out_perm, int64_t* out_n, int64_t* out_sA, int64_t* out_sB);
int ttcb_test_plan_host(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                        int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tuning, char* buf, size_t len);
size_t ttcb_test_plan_desc(const ttcb_plan* p, void* buf, size_t len);
uint32_t ttcb_test_fastdiv(uint32_t n, uint32_t d);
size_t ttcb_test_plan_host_desc(int rank, const int* perm, const int64_t* size, const int64_t* lda,
                                const int64_t* ldb, int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tuning,
                                int* kernel, void* buf, size_t len);
// Sizes and offsets of the descriptor structs (13 entries), so host-side checkers can parse them.
void ttcb_test_desc_layout(int64_t* out);
// Shape-only plans of one problem under n tunings (the learned selector's candidate features):
// writes a JSON array (one plan description per tuning, null where planning failed) into buf and
// returns the length it needs including the terminator.
size_t ttcb_test_plan_shapes(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                             int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tunings, int n, char* buf,
                             size_t len);
// Lowers the largest descriptor ttcb_transpose_noalloc accepts to `bytes` (0 restores the full
// scratch size) and returns the scratch size. Makes no CUDA call.
size_t ttcb_test_noalloc_limit(size_t bytes);
// The boxes a plan's ragged tiles are moved as (edge plans), host-only: a JSON array of
// {"rank","perm","size","lda","ldb","offA","offB"}; returns the length needed, 0 on failure.
size_t ttcb_test_plan_edges(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                            int type_a, int type_b, int beta_nonzero, const ttcb_tuning* tuning, char* buf, size_t len);
// GPU hook (the one that launches a kernel): one CTA waits, with a limit of limit_ns, on an mbarrier
// phase - the bounded wait of the staged kernel's bulk-copy form. With arrive = 0 nothing completes
// the phase, so the wait must give up; with arrive = 1 the CTA arrives first, so it must not. Writes
// to *gave_up how many CTAs gave up (0 or 1); returns the CUDA error code.
int ttcb_test_bounded_wait(uint64_t limit_ns, int arrive, unsigned int* gave_up);
}
