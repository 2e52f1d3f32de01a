/*
 * bbk_ldlt.h -- C ABI of the B200-native blocked Bunch-Kaufman LDL^T library
 * (libbbk_b200.so).  Plain pointers, sizes and status codes only; every entry
 * point is `extern "C"` and safe to bind from ctypes, cgo, JNI or C.
 *
 * Storage convention shared by every entry point: a symmetric matrix of
 * order n is an n x lda row-major array whose upper triangle (i <= j) holds
 * the matrix, which is the dense equivalent of the reference's BlockMatrix
 * upper-block storage (include/block_matrix.h:24-72 in
 * wentianshu/BlockedBunchKaufmanLDLT).  The strict lower triangle is never
 * read; the factorization uses it as scratch only where stated.
 *
 * Compact factors: after factorization the upper triangle holds D on the
 * diagonal and, for a 2x2 pivot starting at k, D(k,k+1) at (k,k+1); every
 * other strictly-upper entry (k,i) holds U(k,i) = L(i,k).  perm[i] is the
 * original index at factored position i, so (P A P^T)(i,j) = A(perm[i],
 * perm[j]) = (L D L^T)(i,j); pivot_types[i] is 1, 2 (first of a 2x2) or -2
 * (second of a 2x2).  This is exactly the reference's compact layout
 * (src/block_ldlt_decomposition.cc:633-704, tests/block_ldlt_decomposition_
 * test.cc:421-450).
 *
 * Errors: every function returns a bbk_status; bbk_last_error() gives a
 * thread-local message.  The C++ surface (include/block_ldlt_decomposition.h)
 * maps these onto the reference's exception types.
 */
#ifndef BBK_LDLT_H_
#define BBK_LDLT_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BBK_ABI_VERSION 1

typedef enum bbk_status {
  BBK_OK = 0,
  BBK_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument */
  BBK_ERR_OUT_OF_RANGE = 2,     /* reference: std::out_of_range */
  BBK_ERR_LOGIC = 3,            /* reference: std::logic_error */
  BBK_ERR_ALLOC = 4,            /* reference: std::bad_alloc */
  BBK_ERR_CUDA = 5,             /* a CUDA runtime call failed */
  BBK_ERR_TIMEOUT = 6,          /* a device-side bounded wait ran out */
  BBK_ERR_NO_DEVICE = 7,        /* no usable sm_100 device */
  BBK_ERR_WORKSPACE = 8         /* caller workspace smaller than required */
} bbk_status;

/* Arithmetic of the factorization.  The panel (pivot search, interchanges,
 * scaling, in-panel row updates) is always FP64, with the 1x1/2x2 tests,
 * determinants and divisions in the reference's own operation order; its
 * in-panel dot products keep the reference's summation order only in
 * BBK_UPDATE_FP64_ORDERED (elsewhere they are reassociated FMA chains). */
typedef enum bbk_update_mode {
  BBK_UPDATE_FP64 = 0,         /* FP64 tensor cores (DMMA mma.sync f64) for the
                                  trailing update */
  BBK_UPDATE_FP64_ORDERED = 1, /* FP64, reference summation order: bitwise
                                  identical to the reference */
  BBK_UPDATE_FP32 = 2,         /* operands rounded to FP32, FP32 accumulate,
                                  result subtracted in FP64 */
  BBK_UPDATE_BF16 = 3,         /* operands scaled by per-64-block powers of two
                                  and rounded to BF16, FP32 accumulation on
                                  tensor cores, result subtracted in FP64 */
  BBK_UPDATE_BF16X3 = 4        /* as BF16, each operand split into three BF16
                                  terms (six products): about FP32 accuracy
                                  at BF16 tensor-core rates */
} bbk_update_mode;

/* ---- version / diagnostics ------------------------------------------- */
int bbk_abi_version(void);
const char* bbk_last_error(void);
const char* bbk_status_string(int status);
/* Number of kernels this library has launched in this process. */
unsigned long long bbk_kernel_launch_count(void);
/* Upper bound, in nanoseconds, on every device-side spin wait (grid-wide
 * pivot exchanges).  A wait that runs out aborts the factorization with
 * BBK_ERR_TIMEOUT instead of hanging.  Default 5 s. */
int bbk_set_wait_timeout_ns(unsigned long long timeout_ns);
/* Test hook for the bounded-wait machinery: launches one cooperative grid of
 * `ctas` (1..223) blocks whose exchange also waits for one participant that
 * does not exist, so the wait must run out.  Returns BBK_ERR_TIMEOUT when the bound
 * works (and leaves the context usable), BBK_OK never. */
int bbk_probe_bounded_wait(int ctas, unsigned long long timeout_ns, void* stream);
/* Diagnostics: runs `iters` back-to-back grid exchanges (the panel kernel's
 * barrier + all-gather) on `ctas` (1..224) co-resident blocks and reports the
 * mean device nanoseconds per exchange. */
int bbk_probe_exchange_ns(int ctas, int iters, double* ns_per_exchange, void* stream);

/* Per-kernel-class device timing for benchmarks: between begin and end,
 * every launch of this library is bracketed by CUDA events on its own
 * stream.  end() waits for the events and writes the summed milliseconds
 * per class into ms[0..4] = {init, panel, finalize, trailing update, solve}
 * and the launch counts into counts[0..4] (either may be NULL). */
int bbk_profile_begin(void);
int bbk_profile_end(double* ms, long long* counts);
/* Panel-kernel phase timing (diagnostics): enable != 0 zeroes and arms the
 * counters; enable == 0 disarms them and copies 10 counters to out: summed
 * nanoseconds of CTA 0 in {row update, first exchange, candidate column,
 * second exchange, interchange + scaling}, pivots, candidate evaluations,
 * (unused), and over all exchanges the summed nanoseconds between CTA 0's
 * publish and the last CTA's publish, and between the last publish and
 * CTA 0 seeing every record. */
int bbk_panel_stats(int enable, unsigned long long* out);
/* The raw diagnostic counter array behind bbk_panel_stats (first `words`
 * words): [0..15] the counters above, then per panel-CTA how often it
 * published last in an exchange, then per CTA its own 5 phase totals. */
int bbk_panel_stats_raw(unsigned long long* out, size_t words);

/* ---- factorization ------------------------------------------------------
 * Replaces BlockLdltDecomposition(const BlockMatrix&, mode) + Factorize()
 * (reference include/block_ldlt_decomposition.h:18-23,
 * src/block_ldlt_decomposition.cc:30-59).  `block_size` is the reference's
 * BlockMatrix block size: it sets the panel width, the panel boundaries
 * (and so the same pivot sequence and boundary shifts as the reference).
 *
 * Device variant: a, perm, pivot_types, panel_end are device pointers;
 * panel_end (ceil(n/block_size) ints, may be NULL) receives the first row
 * after each panel, from which the reference's block geometry (boundary
 * shifts, src/block_ldlt_decomposition.cc:589-631) follows.  `workspace`
 * may be NULL (the library allocates with cudaMallocAsync on `stream`),
 * else it must hold bbk_factor_workspace_size(n, block_size) bytes.  The call
 * enqueues on `stream` and then waits for it, returning the device status. */
size_t bbk_factor_workspace_size(int n, int block_size);
int bbk_factor_device(int n, int block_size, double* a, long long lda,
                      int* perm, int* pivot_types, int* panel_end,
                      int update_mode, void* workspace,
                      size_t workspace_bytes, void* stream);
/* Same, without the final wait: the device status (a bbk_status) is
 * written to *status_device when the stream reaches it.  Capturable in a
 * CUDA graph when `workspace` is given. */
int bbk_factor_device_async(int n, int block_size, double* a, long long lda,
                            int* perm, int* pivot_types, int* panel_end,
                            int update_mode, void* workspace,
                            size_t workspace_bytes, int* status_device,
                            void* stream);
/* Optional outputs of bbk_factor_device_ex (no reference entry point: the
 * reference keeps both inside its object).  Any pointer may be NULL.
 *
 * pivot_log (device, 4 * n doubles): what every Bunch-Kaufman decision
 *   compared, so a decision that another summation order could flip (a
 *   near-tie) can be recognised.  At the factored position p where each
 *   pivot step's pivot starts: |W(p,p)| (tested against alpha * omega,
 *   src/block_ldlt_decomposition.cc:90-92), omega = max_{j>p} |W(p,j)|
 *   (FindCurrentRowMax, :164-182), sigma = max_{i>=p, i!=r} |W(i,r)| and
 *   |W(r,r)| (FindCandidateColumnMax and SelectPivot, :354-390; NaN when the
 *   first test kept the 1x1 pivot).  Every other entry is NaN (the second
 *   row of a 2x2 pivot).
 * workspace_rows (device, n x workspace_ld row-major): each panel's
 *   workspace rows W = D U (the unscaled updated pivot rows) at the columns
 *   the trailing update reads, i.e. W(p, j) for the panel's rows p and
 *   j >= the panel's end, in the column order at the panel's end -- the
 *   contents of the reference's Workspace() outside its diagonal blocks
 *   (written by FactorPanel, :80-120, and read by UpdateTrailingBlocks,
 *   :706-744).  Nothing else of the array is written. */
typedef struct bbk_factor_extras {
  double* pivot_log;
  double* workspace_rows;
  long long workspace_ld;
} bbk_factor_extras;
/* bbk_factor_device_async with the optional outputs above. */
int bbk_factor_device_ex(int n, int block_size, double* a, long long lda,
                         int* perm, int* pivot_types, int* panel_end,
                         int update_mode, const bbk_factor_extras* extras,
                         void* workspace, size_t workspace_bytes,
                         int* status_device, void* stream);
/* Host variant: a (n x lda, in/out), perm, pivot_types, panel_end are host
 * memory.  Copies in, factors on the current device, copies out. */
int bbk_factor_host(int n, int block_size, double* a, long long lda,
                    int* perm, int* pivot_types, int* panel_end,
                    int update_mode);

/* ---- solve with compact factors (no reference counterpart: the reference
 * exposes no solve; semantics follow its compact-storage reading rules,
 * tests/block_ldlt_large_stress_test.cc:160-194) --------------------------
 * Solves A X = B for nrhs right-hand sides stored column after column
 * (b[c*ldb + i]); X overwrites B.  A zero 1x1 pivot yields a zero component
 * (the reference zeroes that column of L); a singular 2x2 pivot divides by
 * zero.  The triangular sweeps are latency-bound (one dependent step per 64
 * rows): up to 32 right-hand sides go through them 8 per launch, each CTA
 * gathering every solved block into its next own block; more go through a
 * single launch that reads the factor once for all of them. */
size_t bbk_solve_workspace_size(int n, int nrhs);
int bbk_solve_device(int n, const double* factors, long long ldf,
                     const int* perm, const int* pivot_types, int nrhs,
                     double* b, long long ldb, void* workspace,
                     size_t workspace_bytes, void* stream);
int bbk_solve_host(int n, const double* factors, long long ldf,
                   const int* perm, const int* pivot_types, int nrhs,
                   double* b, long long ldb);

/* No counterpart in the reference (which has no solve).  The same solve as
 * bbk_solve_device, for callers that cannot allocate device memory: a
 * framework whose caching allocator owns the device's memory, a fixed pool
 * set up once, or a latency-critical loop that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree.  It allocates nothing: its
 * 2 * n * nrhs doubles of scratch come from one fixed 8 MiB array inside the
 * library that every GPU loading the library holds until the process exits,
 * so n * nrhs may be at most BBK_SOLVE_NOALLOC_MAX_ELEMENTS (larger sizes are
 * rejected with BBK_ERR_INVALID_ARGUMENT).  The first call on each device
 * may load the library's device code to find that array's address; make
 * that first call before any stream capture.  All calls on a device share
 * the array and it keeps the last call's contents (nothing in it needs
 * clearing: every element is written before it is read), so calls whose
 * work overlaps on the GPU -- different streams, or different host threads
 * -- race and corrupt each other.  Enqueues on `stream` and returns without
 * waiting; device pointers.  Because it returns before the solve runs, it
 * cannot report a solve whose device-side bounded wait ran out (the
 * synchronous bbk_solve_device returns BBK_ERR_TIMEOUT for that); the
 * sweeps' waits only run out if the GPU cannot keep their blocks resident
 * together, and the right-hand sides are then left partly solved. */
#define BBK_SOLVE_NOALLOC_MAX_ELEMENTS 524288
int bbk_solve_device_noalloc(int n, const double* factors, long long ldf,
                             const int* perm, const int* pivot_types,
                             int nrhs, double* b, long long ldb,
                             void* stream);

/* ---- FP64 iterative refinement (no reference counterpart) -------------
 * Solves A X = B with factors that may come from a low-precision update
 * (BBK_UPDATE_FP32 / BBK_UPDATE_BF16), refining in FP64 against the original
 * matrix `a` (upper triangle, lda) until every right-hand side's backward
 * error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol or
 * max_iter outer steps.  method BBK_REFINE_CLASSICAL: x += (LDL^T)^{-1} r;
 * BBK_REFINE_GMRES: restarted FGMRES(restart) on the correction equation,
 * right-preconditioned by the factors (for factor error x condition number
 * too large for classical refinement).  Device pointers; b and x are
 * column-major (b[c*ldb + i]).  `workspace` may be NULL (allocated with
 * cudaMallocAsync), else bbk_solve_refined_workspace_size bytes. */
typedef struct bbk_refine_info {
  int iterations;                /* outer refinement steps */
  int inner_iterations;          /* preconditioner applications */
  int converged;                 /* 1 when backward_error <= tol */
  int reserved;
  double initial_backward_error; /* of the unrefined solution */
  double backward_error;         /* final, max over right-hand sides */
} bbk_refine_info;

#define BBK_REFINE_CLASSICAL 0
#define BBK_REFINE_GMRES 1

size_t bbk_solve_refined_workspace_size(int n, int nrhs, int restart);
int bbk_solve_refined_device(int n, const double* a, long long lda,
                             const double* factors, long long ldf,
                             const int* perm, const int* pivot_types, int nrhs,
                             const double* b, long long ldb, double* x,
                             long long ldx, double tol, int max_iter,
                             int method, int restart, bbk_refine_info* info,
                             void* workspace, size_t workspace_bytes,
                             void* stream);

/* ---- factor + solve in one call, host buffers (the end-to-end path) ----
 * a (in: matrix, out: compact factors), b (in: right-hand sides, out:
 * solutions). */
int bbk_factor_solve_host(int n, int block_size, double* a, long long lda,
                          int* perm, int* pivot_types, int* panel_end,
                          int nrhs, double* b, long long ldb, int update_mode);

/* ---- reconstruction (reference ReconstructOriginal,
 * src/block_ldlt_decomposition.cc:61-78) --------------------------------
 * out (n x ldo row-major, full) = P^T L D L^T P from compact factors.
 * M = L D and L^T are formed on the device and the upper triangle of their
 * product runs on the FP64 tensor cores (the trailing-update tile kernels);
 * the result is mirrored and permuted.  Temporary device memory: 3 x ld^2
 * doubles, ld = n rounded up to 128.  Device pointers. */
int bbk_reconstruct_device(int n, const double* factors, long long ldf,
                           const int* perm, const int* pivot_types,
                           double* out, long long ldo, void* stream);
/* ExtractRegularFactorsFromCompact (src/block_ldlt_decomposition.cc:746-763)
 * on the device: dense L (n x ldl row-major, unit lower: L(i,k) = F(k,i)
 * for i > k, except the coupling entry of a 2x2 pivot) and D (n x ldd,
 * block diagonal: F(k,k), and F(k,k+1) at (k,k+1) and (k+1,k) of a 2x2),
 * the kFull mode's LFactor() / DFactor().  Either output may be NULL.
 * Device pointers; waits for `stream`. */
int bbk_extract_ld_device(int n, const double* factors, long long ldf,
                          const int* pivot_types, double* l, long long ldl,
                          double* d, long long ldd, void* stream);

/* ---- sampled residual (the reference's large-matrix check,
 * tests/block_ldlt_large_stress_test.cc:160-244) -------------------------
 * For `count` sampled entries (rows[k], cols[k]) of the original matrix `a`
 * (upper triangle read, lda), the same entry of P^T L D L^T P computed
 * straight from the compact factors, without forming L D L^T; *residual
 * (host) = sqrt(sum (reconstructed - original)^2) / max(sqrt(sum original^2),
 * 1).  Every sample is summed over the pivots in the reference's order with
 * each product and sum rounded separately, and the sums run in sample
 * order, so equal factors give the reference's value bit for bit.  rows and
 * cols are device int arrays; a, factors, perm, pivot_types device memory.
 * A sample outside [0, n) or a perm that is not a permutation makes the
 * result NaN.  Waits for `stream`. */
int bbk_sampled_residual_device(int n, const double* a, long long lda,
                                const double* factors, long long ldf,
                                const int* perm, const int* pivot_types,
                                int count, const int* rows, const int* cols,
                                double* residual, void* stream);

/* ---- the reference's kernel boundary (include/kernels.h:6-23,
 * src/kernels.cc:11-91), device pointers, element strides -------------- */
/* kernels::ScaleOneByOnePivot: dst[i*ds] = src[i*ss] / pivot, or 0 when
 * pivot == 0. */
int bbk_scale_one_by_one(int count, double pivot, const double* source,
                         int source_stride, double* destination,
                         int destination_stride, void* stream);
/* kernels::ScaleTwoByTwoPivot: [d1; d2] = inv([[a, b], [b, c]]) [s1; s2],
 * or zeros when the determinant is 0. */
int bbk_scale_two_by_two(int count, double a, double b, double c,
                         const double* first_source, int first_source_stride,
                         const double* second_source, int second_source_stride,
                         double* first_destination,
                         int first_destination_stride,
                         double* second_destination,
                         int second_destination_stride, void* stream);
/* kernels::UpdateTrailingBlock: target[rows x cols] -= left^T ws, with left
 * inner x rows and ws inner x cols, all row-major with the given strides. */
int bbk_update_trailing_block(int rows, int cols, int inner_dim,
                              const double* left_panel, int left_panel_stride,
                              const double* workspace_panel,
                              int workspace_panel_stride, double* target,
                              int target_stride, int update_mode,
                              void* stream);

/* ---------------------------------------------------------------------------
 * Batched factor + solve: many independent small symmetric matrices, each
 * factored with the reference's blocked Bunch-Kaufman algorithm
 * (BlockLdltDecomposition::Factorize, src/block_ldlt_decomposition.cc:
 * 28-78) and solved for one right-hand side, all in one persistent launch
 * (one CTA per matrix at a time, largest matrices first).  No reference
 * counterpart as a batch: the reference factors one matrix per object.
 *
 * Buffers are device memory.  Item k's matrix is n x lda row-major at
 * a + items[k].a (upper triangle read; compact factors written in place),
 * its right-hand side at x + items[k].rhs (overwritten by the solution), and
 * its perm / pivot_types at perm + items[k].piv / pivot_types +
 * items[k].piv.  Block sizes are chosen per size bucket (n <= 32, 64, 128,
 * 256, 512, 1024); the library clamps each to what shared memory holds.
 * ------------------------------------------------------------------------- */
#define BBK_BATCH_MAX_N 1024
#define BBK_BATCH_BUCKETS 6
typedef struct bbk_batch_item {
  int n;          /* order, 1..BBK_BATCH_MAX_N */
  int lda;        /* leading dimension, >= n */
  long long a;    /* element offset of the matrix in the a buffer */
  long long rhs;  /* element offset of the right-hand side in the x buffer */
  long long piv;  /* element offset of perm / pivot_types entries */
} bbk_batch_item;

typedef struct bbk_batch_info {
  int iterations;        /* refinement steps taken (0 without refinement) */
  int converged;         /* 1: backward error <= tol (always 1 without refinement) */
  double backward_error; /* max|b - A x| / (||A||_inf ||x||_inf + ||b||_inf) (refined modes) */
} bbk_batch_info;

/* Bytes of workspace for `count` items whose largest order is max_n. */
size_t bbk_batched_workspace_size(int count, int max_n);
/* Set-up (host, synchronous on `stream`): sorts the items largest first,
 * picks each item's block size from block_sizes[bucket] (NULL or 0 entries:
 * built-in defaults; BBK_BATCH_BUCKETS entries), writes the block size used
 * for item k to chosen_blocks[k] when that array is non-NULL, and stores the
 * schedule in the workspace. */
int bbk_batched_plan(int count, const bbk_batch_item* items_host,
                     const int* block_sizes, int* chosen_blocks,
                     void* workspace, size_t workspace_bytes, void* stream);
/* Factor and solve every planned item (asynchronous, allocates nothing; the
 * launch sequence can be captured in a CUDA graph).  update_mode:
 * BBK_UPDATE_FP64_ORDERED (the reference's arithmetic bit for bit),
 * BBK_UPDATE_FP64, or BBK_UPDATE_FP32 (FP32 trailing updates; with a_orig
 * non-NULL and max_iter > 0 the solution is refined in FP64 against the
 * original matrices at a_orig + items[k].a until the backward error is <=
 * tol).  info (device, optional) receives one record per item, in the
 * caller's item order. */
int bbk_batched_factor_solve(int count, double* a, const double* a_orig,
                             double* x, int* perm, int* pivot_types,
                             int update_mode, double tol, int max_iter,
                             bbk_batch_info* info, void* workspace,
                             size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BBK_LDLT_H_ */
