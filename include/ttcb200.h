/*
 * ttcb200.h -- C ABI of the B200-native out-of-place tensor transposition
 *
 *     B_{pi(i0,i1,...,iN-1)} = alpha * A_{i0,i1,...,iN-1} + beta * B_{pi(i0,i1,...,iN-1)}
 *
 * Conventions (identical to TTC):
 *   - Column-major: dimension 0 of a tensor has stride 1.
 *   - perm[j] = the A-dimension that becomes B-dimension j; B-dimension j has extent size[perm[j]].
 *   - lda[i] / ldb[j] are "outer sizes": stride of A-dim i is prod_{k<i} lda[k]; stride of B-dim j is
 *     prod_{k<j} ldb[k]. Passing NULL means "dense" (lda = size, ldb[j] = size[perm[j]]).
 *   - A and B are DEVICE pointers owned by the caller. Plans own a small device descriptor that is
 *     created once; ttcb_transpose() itself never allocates.
 *   - All calls return a ttcb_status; they never exit() and never trap. ttcb_last_error() returns a
 *     thread-local message describing the last failure on the calling thread.
 *
 * Every entry point below names the TTC interface it replaces (file:line inside the TTC project).
 */
#ifndef TTCB200_H
#define TTCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A cudaStream_t, declared without including the CUDA headers. 0/NULL = the legacy default stream. */
typedef struct CUstream_st* ttcb_stream_t;

#define TTCB_MAX_RANK 10   /* TTC's tuning database stores up to 10 dimensions (ttc.py:226-240) */

/* Element types. TTC's --dataType letters map as s=float, d=double, c=float complex,
 * z=double complex; a mixed pair "xy" means A has type x and B has type y (ttc.py:1218-1244). */
typedef enum {
  TTCB_S = 0, /* float                        */
  TTCB_D = 1, /* double                       */
  TTCB_C = 2, /* float complex  (cuFloatComplex layout: re, im)  */
  TTCB_Z = 3  /* double complex (cuDoubleComplex layout: re, im) */
} ttcb_dtype;

typedef enum {
  TTCB_OK = 0,
  TTCB_ERR_INVALID_ARG = 1,   /* null plan / pointer where one is required, bad enum             */
  TTCB_ERR_RANK = 2,          /* rank < 1 or rank > TTCB_MAX_RANK                                */
  TTCB_ERR_BAD_PERM = 3,      /* perm is not a permutation of 0..rank-1 (ttc.py:754-758)          */
  TTCB_ERR_BAD_LD = 4,        /* lda[i] < size[i] or ldb[j] < size[perm[j]] (ttc.py:739-746)      */
  TTCB_ERR_DTYPE = 5,         /* unsupported A/B type pair (only s,d,c,z,sd,ds,cz,zc exist)       */
  TTCB_ERR_ALIGN = 6,         /* a pointer is not aligned to its element size                     */
  TTCB_ERR_CUDA = 7,          /* a CUDA runtime call failed; the message holds the CUDA error     */
  TTCB_ERR_ALLOC = 8,         /* host or device allocation failed                                 */
  TTCB_ERR_UNSUPPORTED = 9,   /* a size/extent beyond what the kernels index (see message)        */
  TTCB_ERR_TIMEOUT = 10,      /* a bounded device-side wait gave up (batched mode)                */
  TTCB_ERR_BETA = 11          /* beta given to a plan made for beta == 0, or missing when needed  */
} ttcb_status;

/* Kernel selection and schedule knobs. Every field 0 means "planner default".
 * These are the candidate dimensions the autotuner searches (tile shape x vector width x loop
 * order x block count), the B200 counterparts of TTC's blocking / loop order / threadsPerBlock
 * search space (GPUtransposeGenerator.py:165-230, 258-285). */
typedef struct {
  int32_t kernel;        /* 0 auto, 1 = staged tile transpose, 2 = direct row copy            */
  int32_t tile_elems;    /* target elements per shared-memory tile (tile kernel)              */
  int32_t run_bytes;     /* target contiguous run length on each side, in bytes               */
  int32_t vec;           /* 0 = widest legal 16-byte vectors, 1 = force scalar accesses        */
  int32_t blocks;        /* CTAs launched (persistent grid); 0 = all tiles / occupancy bound  */
  int32_t loop_order;    /* raster of the tile grid: 0 = planner's choice (B-major when B's runs
                            are under 256 bytes and B exceeds 64 MiB, else A-major), 1 = B-major,
                            2 = reverse A, 3 = A-major, 4 = the explicit order in raster_lo/hi  */
  int32_t streaming;     /* 0 = default (streaming stores when beta == 0), 1 = on, -1 = off     */
  int32_t tile_variant;  /* tile kernel: 0 auto, 1 table-driven, 2 register-resident prefetch,
                            3 staged asynchronous copies                                        */
  int32_t ragged;        /* staged tile kernel's ragged tiles (last blocks of dimensions that
                            the tile does not divide): 0 = planned as transpositions of their
                            own and moved by the staged kernel, 1 = element-wise kernel         */
  /* loop_order == 4: TTC's loop order (--loopPerm, GPUtransposeGenerator.py:203-230), the caller's
     dimensions from the fastest-varying tile index to the slowest, packed 4 bits per dimension as
     (dimension + 1): dimensions 0..7 of the order in raster_lo (first in the low bits), 8..9 in
     raster_hi. Dimensions that index fused groups are ordered by their first appearance; those the
     tile covers whole do not step the grid. Every dimension must appear exactly once. */
  int32_t raster_lo;
  int32_t raster_hi;
  int32_t stages;        /* staged tile kernel: shared-memory ring stages (3..7, stages - 2 tiles of
                            copies in flight); 0 = planner's choice                             */
  int32_t ctas_per_sm;   /* staged tile kernel: resident CTAs per SM (1..8, capped by what fits);
                            0 = planner's choice. `blocks`, when set, takes precedence          */
  int32_t round_robin;   /* staged tile kernel: 0 = planner's choice (claims for tiles of 16 KiB
                            or more when every CTA has 16 or more), 1 = fixed round-robin order
                            (tile blockIdx + k * CTAs), -1 = CTAs claim tiles in order from
                            counters the plan owns                                              */
  int32_t shifted_runs;  /* staged tile kernel: 1 = copy A runs that 16-byte accesses cannot
                            reach directly (odd lengths or offsets) as the 16-byte chunks that
                            cover them; 0 = planner's choice (plain copies), -1 = never         */
  int32_t bulk_copies;   /* staged tile kernel: 1 = move A with one bulk copy per run or run
                            piece (cp.async.bulk into the stage, completion counted on an
                            mbarrier) where the runs allow it (16-byte aligned runs, or shifted
                            runs); 0 or -1 = per-thread 16-byte copies                          */
  int32_t lane_map;      /* staged tile kernel, register path: 1 = a warp takes B vectors from
                            several B runs (in their order, or sorted by A position) when the
                            planner's model finds fewer bank conflicts in the gather that way;
                            0 or -1 = a warp takes 32 consecutive B vectors                     */
  int32_t claim_group;   /* staged tile kernel with claimed tiles: consecutive tiles per claim
                            (1..64); 0 = planner's choice (2)                                   */
} ttcb_tuning;

typedef struct ttcb_plan ttcb_plan;

/* Replaces the generated TTC wrapper's per-call set-up (CUDAtranspose.py:395-429: cudaMalloc +
 * cudaMemcpy of size/lda/ldb on every call) and the planning that ttc.py does before generating
 * code (index fusion ttc_util.py:214-276, validation ttc.py:733-768, path choice
 * CUDAtranspose.py:34-42). Extents are 64-bit (TTC used int, capping tensors at 2^31 elements).
 * size[i] == 0 is allowed and yields a plan whose transpose is a no-op. */
ttcb_status ttcb_plan_create(ttcb_plan** plan, int rank, const int* perm, const int64_t* size,
                             const int64_t* lda, const int64_t* ldb, ttcb_dtype type_a,
                             ttcb_dtype type_b, int beta_nonzero, const ttcb_tuning* tuning);

/* Replaces the generated entry point
 *   extern "C" void <p>CuTranspose_<perm>_<sizes>[_bz](const TA* A, TB* B, const Talpha alpha,
 *        [const Tbeta beta,] const int* size, const int* lda, const int* ldb)
 * (CUDAtranspose.py:438-451, named at :473-527). Stream-ordered and asynchronous; it never
 * allocates and never synchronizes. alpha points to one value of A's precision: float for s/sd,
 * double for d/ds, {float re, im} for c/cz, {double re, im} for z/zc (TTC takes a real alpha; a
 * complex one is an extension). beta likewise in B's precision; it is ignored (may be NULL) for a
 * plan created with beta_nonzero == 0. */
ttcb_status ttcb_transpose(const ttcb_plan* plan, const void* A, void* B, const void* alpha,
                           const void* beta, ttcb_stream_t stream);
/* Calls with one plan may overlap on the GPU (several streams). A plan whose staged kernel claims
 * tiles from counters ("claims" in its description) takes the counter words in turn from 64 slot
 * pairs, so up to 64 of its launches can be in flight at once; a launch captured in a CUDA graph
 * keeps its slot, and replays of that graph must not overlap each other. */

/* Allocation-free transposition, for callers that may not allocate device memory (their memory is
 * owned by an external pool, or cudaMalloc is forbidden where they run). It has no counterpart in
 * TTC, whose every call allocates. Plans on the host and writes the plan's descriptor into a 64 KiB
 * scratch array built into the library (held by every GPU that loads the library until exit);
 * never calls cudaMalloc/cudaFree. Uses the staged tile kernel; beta == NULL means beta = 0.
 * Problems whose descriptor exceeds the scratch size fail with TTCB_ERR_UNSUPPORTED (with the
 * planner's tile limits a descriptor stays under about 34 KiB). Calls that overlap on the GPU race
 * on the scratch array; calls in order on one stream do not. The first call on each device looks up
 * the scratch address and should come before any stream capture. The descriptor is uploaded from
 * host memory that lives only during the call, so a call on a stream that is being captured is
 * refused with TTCB_ERR_UNSUPPORTED before anything is enqueued. */
ttcb_status ttcb_transpose_noalloc(int rank, const int* perm, const int64_t* size, const int64_t* lda,
                                   const int64_t* ldb, ttcb_dtype type_a, ttcb_dtype type_b,
                                   const void* A, void* B, const void* alpha, const void* beta,
                                   ttcb_stream_t stream);

/* Frees the plan's device descriptor. Safe on NULL. */
void ttcb_plan_destroy(ttcb_plan* plan);

/* One-line JSON description of a plan (fused problem, chosen kernel, tile, vectors, grid).
 * Writes at most len bytes including the terminating NUL; returns the full length needed. */
size_t ttcb_plan_describe(const ttcb_plan* plan, char* buf, size_t len);

/* Algorithmic bytes of one call: N*(sizeof(TA) + sizeof(TB)*(1 + [beta != 0])), N = prod size,
 * the bandwidth convention of GPUtransposeGenerator.py:589-592 (padding excluded). */
int64_t ttcb_plan_bytes(const ttcb_plan* plan);

/* Stage waits of the plan's staged kernel that ran out of time since the plan was created or last
 * asked (a plan with bulk A copies waits on its stage barriers with a limit of 2 s; a wait that runs
 * out means copies never landed, and that launch left tiles of B unwritten). Writes the count and
 * clears it; 0 for plans without bulk copies. Copies from the device, so it waits for the device's
 * work that is ordered before it on the legacy default stream. No counterpart in TTC. */
ttcb_status ttcb_plan_wait_timeouts(const ttcb_plan* plan, unsigned int* count);

/* Message of the last failure on this thread ("" if none). Replaces ttc_util.py:135-141, which
 * printed the CUDA error and called exit(-1). */
const char* ttcb_last_error(void);

/* Library version {major, minor, patch}. */
void ttcb_version(int* major, int* minor, int* patch);

/* ---------------------------------------------------------------------------------------------
 * Batched mode: many independent transpositions in one persistent launch.
 * No counterpart in TTC, which can only call one generated wrapper per transposition (each with its
 * own cudaMalloc/cudaMemcpy/cudaDeviceSynchronize, CUDAtranspose.py:395-429). The batch owns a
 * device table of per-problem descriptors, a prefix sum of tile counts and a work counter.
 * ------------------------------------------------------------------------------------------- */
typedef struct ttcb_batch ttcb_batch;

/* Builds a batch from already-created plans (each keeps its own schedule; the batch copies what
 * it needs, so the plans may be destroyed afterwards). A[i]/B[i] are device pointers bound now. */
ttcb_status ttcb_batch_create(ttcb_batch** batch, int count, const ttcb_plan* const* plans,
                              const void* const* A, void* const* B, const void* alpha,
                              const void* beta, int blocks);

/* Runs every problem of the batch in one persistent kernel launch on stream. */
ttcb_status ttcb_batch_launch(ttcb_batch* batch, ttcb_stream_t stream);

/* Captures the batch launch (counter reset + kernel) into a CUDA graph once and replays it. */
ttcb_status ttcb_batch_graph_launch(ttcb_batch* batch, ttcb_stream_t stream);

/* Device status word of the last launch: 0 = ok, otherwise a TTCB_ERR_* code set on the device. */
ttcb_status ttcb_batch_status(ttcb_batch* batch, ttcb_stream_t stream);

int64_t ttcb_batch_bytes(const ttcb_batch* batch);
void ttcb_batch_destroy(ttcb_batch* batch);

#ifdef __cplusplus
}
#endif
#endif /* TTCB200_H */
