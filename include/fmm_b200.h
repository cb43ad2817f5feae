/*
 * fmm_b200 — B200-native (sm_100a) generated fast matrix multiplication, C ABI.
 *
 * Semantics match the reference's generated entry points: column-major FP64,
 * C += A * B (alpha = beta = 1, no transposes).  Unlike the reference, C needs no
 * padding or alignment: any ldc >= m works.
 *
 * Two families of entry points:
 *   1. Drop-in symbols with the reference's exact signatures (host pointers,
 *      synchronous).  They run the plan bound with fmm_bind_default_plan(); a job
 *      library written by the generator (fmm_gen_b200.control) binds its plan when
 *      it is loaded, so one job library per algorithm configuration, as in the
 *      reference.
 *   2. Stream-ordered device-pointer entry points with status codes (the form a
 *      PyTorch custom op or another GPU library binds).
 *
 * Every function that returns int returns FMM_OK (0) or a negative FMM_E* code;
 * fmm_error_string() names it.  The void drop-in symbols record their status in
 * fmm_last_error().
 */
#ifndef FMM_B200_H
#define FMM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FMM_OK 0
#define FMM_E_INVALID (-1)      /* bad dimension, leading dimension or pointer */
#define FMM_E_NOPLAN (-2)       /* no default plan bound */
#define FMM_E_CUDA (-3)         /* a CUDA runtime call failed */
#define FMM_E_NOMEM (-4)        /* device or host allocation failed */
#define FMM_E_PLAN (-5)         /* malformed plan tables */
#define FMM_E_UNSUPPORTED (-6)  /* pack type or option not supported */
#define FMM_E_TIMEOUT (-7)      /* a bounded device-side wait gave up */
#define FMM_E_TOO_LARGE (-8)    /* beyond the fixed limits of fmm_dgemm_dev_noalloc */

#define FMM_PACK_ABC 0    /* sums fused into operand staging, products scattered into C */
#define FMM_PACK_AB 1     /* each product to a workspace M_r, then M_Add (sums fused into staging,
                             or pre-summed in HBM for large sub-blocks) */
#define FMM_PACK_NAIVE 2  /* explicit S_r, T_r temporaries, plain GEMM into M_r, then scatter */

typedef struct fmm_plan fmm_plan;

/* ---- drop-in symbols (reference: common/include/bl_dgemm.h:60-70, 96-130) ---- */

/* Classical C += A*B (reference bl_dgemm, common/dgemm/my_dgemm.c:115-210). */
void bl_dgemm(int m, int n, int k, double *A, int lda, double *B, int ldb, double *C, int ldc);

/* Generated FMM entry points (reference bl_dgemm_strassen_abc/_ab/_naive, emitted by
 * meta/abc_gen_mix.py:448-472, meta/ab_gen_mix.py:430-456, meta/naive_gen_mix.py:412-429).
 * They run the default plan. */
void bl_dgemm_strassen_abc(int m, int n, int k, double *A, int lda, double *B, int ldb, double *C, int ldc);
void bl_dgemm_strassen_ab(int m, int n, int k, double *A, int lda, double *B, int ldb, double *C, int ldc);
void bl_dgemm_strassen_naive(int m, int n, int k, double *A, int lda, double *B, int ldb, double *C, int ldc);

/* Fringe GEMMs around the FMM core (reference bl_dynamic_peeling,
 * common/dgemm/bl_dgemm_util.c:316-353); host pointers. */
void bl_dynamic_peeling(int m, int n, int k, double *A, int lda, double *B, int ldb, double *C, int ldc,
                        int dim1, int dim2, int dim3);

/* Status of the last drop-in call on this host thread. */
int fmm_last_error(void);
const char *fmm_error_string(int code);

/* ---- plans ---- */

/* Create a plan from composed term lists (the generator's output).
 *   dims[3]       = (prod mt, prod kt, prod nt) over all levels
 *   rank          = number of products R
 *   nterms[3*R]   = per product r: #A terms, #B terms, #C terms
 *   rows, cols, coefs: the terms, product-major, A terms then B then C per product;
 *                   (row, col) is the global block position in the composed grid.
 * Replaces the reference's per-configuration generated code (meta/abc_gen_mix.py:407-472). */
int fmm_plan_create(const int dims[3], int rank, const int *nterms, const int *rows, const int *cols,
                    const double *coefs, fmm_plan **out);
int fmm_plan_destroy(fmm_plan *plan);
int fmm_plan_rank(const fmm_plan *plan);
/* The stored-products combine pass's tables of a plan (no counterpart in the reference):
 * C blocks in groups that share products, the merged entries (one per product of a
 * group's union) and their chunks of 8.  groups = 0: the tables did not pass their checks
 * and the per-block scatter runs instead.  Any output pointer may be NULL. */
int fmm_plan_combine_info(const fmm_plan *plan, int *groups, int *entries, int *chunks);
int fmm_bind_default_plan(fmm_plan *plan);
fmm_plan *fmm_default_plan(void);

/* ---- stream-ordered device entry points ---- */

/* FMM C += A*B on device pointers, enqueued on `stream` (a cudaStream_t; NULL = legacy
 * default stream).  Workspace for AB/NAIVE comes from the stream-ordered allocator. */
int fmm_dgemm_dev(const fmm_plan *plan, int pack_type, int m, int n, int k, const double *A, long lda,
                  const double *B, long ldb, double *C, long ldc, void *stream);

/* Classical C += A*B on device pointers (the comparator and fringe engine). */
int fmm_plain_dgemm_dev(int m, int n, int k, const double *A, long lda, const double *B, long ldb, double *C,
                        long ldc, void *stream);

/* Host-pointer FMM with an explicit plan: copies A, B, C to the device, runs, copies C
 * back, synchronises.  The drop-in symbols above call this with the default plan.  When C
 * has at least 2^22 elements and n >= 4096 the call runs as up to four column panels
 * C[:, J] += A * B[:, J] whose copies in and out overlap the compute (fastest with pinned
 * host buffers); each panel is partitioned like an m x |J| x k call. */
int fmm_dgemm_host(const fmm_plan *plan, int pack_type, int m, int n, int k, const double *A, int lda,
                   const double *B, int ldb, double *C, int ldc);

/* Device-side status of the current device: FMM_E_TIMEOUT if a bounded wait inside a
 * kernel gave up since the last clear (results of that call are then unreliable),
 * FMM_OK otherwise.  Covers every entry point, fmm_dgemm_dev_noalloc's status word
 * included.  Synchronises with the device; clear != 0 resets the words.  The
 * synchronous host entry points check it themselves. */
int fmm_device_status(int clear);

/* Workspace of the pre-summed operands (the ABC pack type's large products) -- the
 * reference's counterpart is its packing pool (common/dgemm/bl_dgemm_util.c:375-394),
 * sized by the first call and never bounded.  One call's workspace is capped at `bytes`
 * (default 8 GiB; bytes <= 0 restores it): a call whose sums would need more runs its
 * products in groups over two halves of a capped workspace, the next group's sums formed
 * while the current group runs; results are unchanged.  The groups' workspace is
 * 2 G (ms + ns) kk 8 bytes for groups of G >= 1 products (kk: the k extent per product
 * rounded up to 8), so a cap below two products' sums is exceeded by that much.  Returns
 * the previous cap.
 * fmm_last_workspace_bytes: pre-summed workspace bytes of the calling thread's last
 * fmm_dgemm_dev / host call (0 when it used none).  The stored products of a call whose C
 * traffic the library routes through one combine pass (8 R ms ns bytes) are not capped. */
long long fmm_set_workspace_limit(long long bytes);
long long fmm_last_workspace_bytes(void);

/* Test hooks -- no counterpart in the reference, whose code has no device-side waits.
 *   FMM_DEBUG_WAIT_LIMIT_NS: time limit of every bounded device-side wait on the current
 *     device, in ns (default 4e9; value <= 0 restores the default).
 *   FMM_DEBUG_TICKET_FILL: byte written into every ticket of a single-problem FMM launch
 *     before it runs (default 0).  0xFF starts every ticket at -1, which no launch ever
 *     releases, so the launch's first ticket waits run out: the kernel records
 *     FMM_E_TIMEOUT after the limit, stops waiting for tickets, and finishes (its result
 *     is then unreliable); fmm_device_status() reports it.  Lets a test check the
 *     timeout path without a fault.
 *   FMM_DEBUG_COMBINE_POSITIONS: form of the stored-products combine pass: 0 (default) the
 *     shared-memory-staged form where the operands allow it, 1 or 2 the register form with
 *     that many element positions per thread; results are unchanged, for sweeps.
 *   FMM_DEBUG_KSPLIT: k split S (1..8) of every launch the model would consider splitting
 *     (launches of few waves); 0 restores the model's choice.  For sweeps; results change
 *     within rounding.
 *   FMM_DEBUG_SPLIT_OPERANDS: how the split-BF16 path forms its operand planes: 0 (default)
 *     every product's sums from one staged read of each operand, 1 one product per CTA (the
 *     two give identical planes; for tests and sweeps).
 * Process-wide settings for tests; restore them before other work.  FMM_E_INVALID for an
 * unknown setting or a value outside its range. */
#define FMM_DEBUG_WAIT_LIMIT_NS 1
#define FMM_DEBUG_TICKET_FILL 2
#define FMM_DEBUG_COMBINE_POSITIONS 3
#define FMM_DEBUG_KSPLIT 4
#define FMM_DEBUG_SPLIT_OPERANDS 5
int fmm_debug_set(int what, long long value);

/* FMM C += A*B (pack type ABC) that allocates no memory -- no counterpart in the
 * reference.  For callers that cannot allocate device memory at call time: frameworks
 * that own all device memory through their own arena or caching allocator, and
 * latency-critical paths where an allocation is not acceptable.  Operand sums are
 * folded while staging (no workspace); the only scratch -- per-tile tickets, a work-unit
 * counter, a status word and the plan's tables -- lives in one statically allocated device array (about
 * 384 KB, held by every GPU that loads the library until the process exits).
 *   Limits: plan with <= 1024 products and <= 12288 terms; <= 16384 tiles of 128 x 128
 *   in a product (ms x ns); beyond them it returns FMM_E_TOO_LARGE without running.
 *   The first call on a device resolves the array's address (cudaGetSymbolAddress),
 *   configures the kernels and writes the fringe strips' constant tables and a zero
 *   status word with blocking copies; make that first call before any stream capture.
 *   Every call shares the array: calls that overlap on the GPU (other streams, other
 *   host threads) race; serialise them on one stream.
 *   sync != 0: synchronise the stream and report a device-side wait timeout
 *   (FMM_E_TIMEOUT, then the word is cleared); sync == 0: stream-ordered, launch errors
 *   only -- a timeout stays recorded in the status word until a sync != 0 call or
 *   fmm_device_status() reports it. */
int fmm_dgemm_dev_noalloc(const fmm_plan *plan, int m, int n, int k, const double *A, long lda, const double *B,
                          long ldb, double *C, long ldc, void *stream, int sync);

/* Split-BF16 FMM on the tensor cores -- no counterpart in the reference (FP64 only).
 * C += A*B with FP32 A (m x k), B (k x n) and FP64 C, column-major device pointers,
 * enqueued on `stream`.  Same partition, product order and fringe peeling as
 * fmm_dgemm_dev (plan == NULL: classical).  Each product's operand sums are formed in
 * FP64 and split into three bf16 planes; the product is six bf16 plane products
 * accumulated in FP32 over 256-deep k chunks and in FP64 across chunks; W[l,r] * M_r is
 * added to C in FP64.  Relative Frobenius error against the FP64 product of the same
 * FP32 inputs: about 1e-7 (classical) and a few 1e-7 for two Strassen levels.
 * Workspace from the stream-ordered allocator: 6 R (ms + ns) kpad bytes of bf16 planes
 * (kpad = ks rounded up to 64) and, for R > 1, 8 R ms ns bytes of product tiles that a
 * final pass adds into C. */
int fmm_split_gemm_dev(const fmm_plan *plan, int m, int n, int k, const float *A, long lda, const float *B,
                       long ldb, double *C, long ldc, void *stream);

/* ---- batches: many independent problems in one persistent launch ----
 * The reference runs one generated entry point per call (meta/abc_gen_mix.py:448-472);
 * a batch runs many problems C_i += A_i * B_i (FP64, column-major), each with its own
 * plan (NULL = classical), in one persistent launch of the FMM kernel whose work units
 * span every problem, longest units first.  Each problem is partitioned exactly as
 * fmm_dgemm_dev partitions it (FMM core plus fringe strips), so results are identical
 * to calling fmm_dgemm_dev per problem.  A second launch handles the k-fringe strips
 * (they update the same C region as their core), and a launch before them forms the
 * pre-summed operands of the large FMM problems.
 *
 * fmm_batch_create fixes the shapes and plans and allocates (cudaMalloc) the job tables,
 * tickets and workspaces; the plans must outlive the batch.  fmm_batch_dgemm takes this
 * call's device pointers and enqueues the work on `stream` without allocating; it may be
 * captured in a CUDA graph.  The job tables go to the device from host staging buffers
 * owned by the batch, so a graph replays with the operands of the batch's most recent
 * fmm_batch_dgemm call (the captured one, unless the batch was called again since).
 * Destroy a batch only after its work has completed. */
typedef struct fmm_batch fmm_batch;
int fmm_batch_create(int count, const fmm_plan *const *plans, const int *m, const int *n, const int *k,
                     fmm_batch **out);
/* The same with a tile height per problem: tile_m[i] = 128 (the default, also 0) or 64 rows per
 * work unit (problem i's FMM core and fringe strips).  64-row tiles halve a problem's unit
 * length and double its unit count (a finer split of the batch's work over the SMs); they run
 * in phases of the direct variant (pre-summed or classical jobs) and fall back to 128 rows
 * elsewhere.  Results of a 64-row problem equal a single call's up to rounding (two partial k
 * sums per tile), not bit for bit. */
int fmm_batch_create_tiled(int count, const fmm_plan *const *plans, const int *m, const int *n, const int *k,
                           const int *tile_m, fmm_batch **out);
int fmm_batch_dgemm(fmm_batch *batch, const double *const *A, const long *lda, const double *const *B,
                    const long *ldb, double *const *C, const long *ldc, void *stream);
/* A batch formed, run and released in one stream-ordered call, for request loops that
 * form a new batch at every step: no cudaMalloc or cudaFree (both synchronise the
 * device, which would stop requests already on the GPU from overlapping with the next
 * batch).  Device buffers come from the stream-ordered pool; the job tables are staged
 * through a ring of 8 pinned host buffers owned by the library, each reused only after
 * the copy out of it has completed (so at most 8 calls' copies are pending).  Same
 * results as fmm_batch_create + fmm_batch_dgemm; not meant for stream capture. */
int fmm_batch_submit(int count, const fmm_plan *const *plans, const int *m, const int *n, const int *k,
                     const double *const *A, const long *lda, const double *const *B, const long *ldb,
                     double *const *C, const long *ldc, void *stream);

/* Work units of the main launch (phase 0) or of the k-fringe launch (phase 1). */
int fmm_batch_units(const fmm_batch *batch, int phase);
int fmm_batch_destroy(fmm_batch *batch);

/* Number of kernels the library launched since load (all entry points, all streams). */
long long fmm_kernel_launch_count(void);

/* Per-kernel timing (no counterpart in the reference, which only times whole calls with
 * bl_clock, common/dgemm/bl_dgemm_util.c:106-182).  Between begin and end every launch
 * is bracketed by CUDA events on its stream; end() synchronises those events and
 * writes, per kernel kind (0 .. fmm_profile_num_kinds()-1), the summed milliseconds and
 * launch counts. */
int fmm_profile_begin(void);
int fmm_profile_end(double *ms_out, long long *count_out);
int fmm_profile_num_kinds(void);
const char *fmm_profile_kind_name(int kind);

#ifdef __cplusplus
}
#endif

#endif /* FMM_B200_H */
