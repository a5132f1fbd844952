/*
 * b2blas.h -- C ABI of libb2blas.so, the B200 (sm_100a) dense BLAS-3 library.
 *
 * Two layers:
 *   1. Drop-in Fortran-BLAS symbols with the exact signatures of the reference
 *      (column-major, every argument by pointer, int32 dimensions, no hidden
 *      string-length arguments).  Host or device pointers are accepted; host
 *      buffers are staged through device memory and the call is synchronous.
 *      These return void like the reference; argument errors and CUDA errors
 *      never abort -- they leave C untouched and are reported by
 *      b2_last_error() / b2_last_info() on the calling thread.
 *   2. Extended b2_* entry points on DEVICE pointers, ordered on a caller
 *      stream (cudaStream_t passed as void*; NULL = the library's per-thread
 *      stream), returning a b2_status.
 *
 * Conventions shared with the reference (src/gemm_driver.c:18-19,131-132):
 *   - trans char 'N'/'n' = no transpose, any other char = transpose;
 *   - beta != 1 multiplies C by beta, so beta == 0 keeps a NaN already in C;
 *   - alpha == 0 skips the product (C is only scaled by beta).
 */
#ifndef B2BLAS_H
#define B2BLAS_H

#if defined(B2_BUILD) && defined(__GNUC__)
#define B2_API __attribute__((visibility("default")))
#else
#define B2_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status                                                                    */
/* ------------------------------------------------------------------------ */
enum b2_status {
  B2_OK = 0,
  B2_ERR_ARG = 1,          /* invalid argument; b2_last_info() = its 1-based position */
  B2_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  B2_ERR_NOMEM = 3,        /* device or pinned allocation failed */
  B2_ERR_TIMEOUT = 4,      /* a bounded device-side wait gave up; results invalid */
  B2_ERR_UNSUPPORTED = 5,  /* method/shape combination not available */
  B2_ERR_NO_DEVICE = 6     /* no sm_100 device visible */
};

/* Method selectors. */
enum b2_method {
  B2_METHOD_DEFAULT = 0,   /* library default for the routine */
  B2_METHOD_FP64 = 1,      /* plain FP64 (DMMA tensor-core path) */
  B2_METHOD_OZAKI = 2,     /* INT8 Ozaki emulation of FP64 (tcgen05 kind::i8) */
  B2_METHOD_AUTO = 3,      /* selector picks method, tile config and slice count */
  B2_METHOD_FP32 = 10,     /* SGEMM: native FP32 on the CUDA cores */
  B2_METHOD_TF32 = 11,     /* SGEMM: 1xTF32 on tcgen05 kind::tf32, FP32 accumulate */
  B2_METHOD_TF32X3 = 12,   /* SGEMM: split 3xTF32, FP32 accumulate */
  B2_METHOD_BF16X3 = 13    /* SGEMM: split 3xBF16 on tcgen05 kind::f16, FP32 accumulate */
};

B2_API int b2_last_error(void);                 /* status of the last call on this thread */
B2_API int b2_last_info(void);                  /* xerbla-style argument position, 0 if none */
B2_API const char *b2_status_string(int status);
B2_API int b2_device_count(void);               /* visible sm_100 devices */
B2_API int b2_version(void);                    /* MAJOR*10000 + MINOR*100 + PATCH */

/* Default method of the drop-in dgemm_ (B2_METHOD_FP64 / _OZAKI / _AUTO) and the
 * Ozaki slice (modulus) count, 0 = chosen per call from K and the requested
 * accuracy.  Also settable by env B2_METHOD=fp64|ozaki|auto, B2_SLICES=n. */
B2_API int b2_set_dgemm_method(int method, int slices);
/* Default method of the drop-in sgemm_ (FP32 / TF32 / TF32X3 / BF16X3);
 * env B2_SGEMM_METHOD=fp32|tf32|tf32x3|bf16x3. */
B2_API int b2_set_sgemm_method(int method);

/* Argument checking of the real drop-in GEMMs (dgemm_, sgemm_, SGEMM_), process-wide:
 *   B2_ARGS_BLAS (default): BLAS argument positions (xerbla numbering) reported
 *     through b2_last_error()/b2_last_info(), C untouched;
 *   B2_ARGS_OPENBLAS: the checks of the reference's OpenBLAS-like dgemm_
 *     (OpenBLAS-like_implementation/dgemm.c:488-498): M < 1 or N < 1 returns
 *     silently; LDA / LDB below the rows of A / B print the reference's
 *     "ERROR: ... Please check input parameters." line on stdout and return.
 *     LDC < M is still refused (B2_ERR_ARG, info 13): C is staged row by row.
 * Also settable by env B2_ARG_MODE=blas|openblas.  Returns the previous mode, or
 * -1 (nothing changed) for an unknown mode. */
#define B2_ARGS_BLAS 0
#define B2_ARGS_OPENBLAS 1
B2_API int b2_set_arg_mode(int mode);

/* ------------------------------------------------------------------------ */
/* Drop-in Fortran-BLAS symbols                                              */
/* ------------------------------------------------------------------------ */

/* Replaces GEMM_DRIVER built as dgemm_ (src/gemm_driver.c:116, -DDOUBLE per
 * Makefile:11-12) and the OpenBLAS-like dgemm_ (OpenBLAS-like_implementation/
 * dgemm.c:484).  C <- alpha*op(A)*op(B) + beta*C. */
B2_API void dgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
            const double *alpha, const double *a, const int *lda, const double *b,
            const int *ldb, const double *beta, double *c, const int *ldc);

/* Replaces GEMM_DRIVER built as sgemm_ (src/gemm_driver.c:116, Makefile:14-15). */
B2_API void sgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
            const float *alpha, const float *a, const int *lda, const float *b, const int *ldb,
            const float *beta, float *c, const int *ldc);

/* Replaces the upper-case serial harness symbol SGEMM_ of
 * OpenBLAS-like_implementation/sgemm.c:579 (same contract as sgemm_). */
B2_API void SGEMM_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
            const float *alpha, const float *a, const int *lda, const float *b, const int *ldb,
            const float *beta, float *c, const int *ldc);

/* Fortran-BLAS dtrsm_.  The reference ships the solve kernels
 * dtrsm_solve_{ln,lt,rn,rt}_m*n* (OpenBLAS-like_implementation/dtrsm_16x4/
 * dtrsm_kernel_16x4_skylakex.S:1863-2536, semantics in
 * dtrsm_kernel_16x4_tester.c:66-199) that an OpenBLAS trsm driver calls; this
 * symbol is that driver and its kernels.  side 'L': op(A) X = alpha B,
 * side 'R': X op(A) = alpha B; B is overwritten by X. */
B2_API void dtrsm_(const char *side, const char *uplo, const char *transa, const char *diag,
            const int *m, const int *n, const double *alpha, const double *a, const int *lda,
            double *b, const int *ldb);

/* 3M complex GEMM (interleaved re/im; alpha, beta and matrices complex;
 * ld in complex elements; trans 'N','T','C' conjugate-transpose,'R' conjugate).
 * Replaces the OpenBLAS gemm3m driver + kernels
 * zgemm3m_kernel_2x8_skylakex.c:336-351 (and the 8x4 variant :309-334) and
 * cgemm3m_kernel_16x4_skylakex.c:415-440.  zgemm3m products below 2^35
 * multiply-adds (2048^3 included) and cgemm3m products below 2^24 run all
 * three real products and the pre/post additions in one fused launch;
 * larger ones run the three real products as FP64 DMMA GEMMs (zgemm3m) or
 * 3xTF32 tensor-core GEMMs (cgemm3m, FP32-class accuracy) between a pre-add
 * pass and a combine pass. */
B2_API void zgemm3m_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
              const double *alpha, const double *a, const int *lda, const double *b,
              const int *ldb, const double *beta, double *c, const int *ldc);
B2_API void cgemm3m_(const char *transa, const char *transb, const int *m, const int *n, const int *k,
              const float *alpha, const float *a, const int *lda, const float *b,
              const int *ldb, const float *beta, float *c, const int *ldc);

/* ------------------------------------------------------------------------ */
/* Extended API (device pointers, stream-ordered, returns b2_status)         */
/* ------------------------------------------------------------------------ */

/* Same contract as dgemm_ (src/gemm_driver.c:116) on device memory.
 * method: B2_METHOD_FP64 / _OZAKI / _AUTO / _DEFAULT; slices: Ozaki modulus
 * count (0 = automatic).  Host pointers are rejected with B2_ERR_ARG. */
B2_API int b2_dgemm(char transa, char transb, int m, int n, int k, double alpha, const double *A,
             int lda, const double *B, int ldb, double beta, double *C, int ldc, int method,
             int slices, void *stream);

/* dgemm_ (src/gemm_driver.c:116, where the reference splits N over OpenMP
 * threads at :136-149) split over several GPUs of one node: C's columns are
 * cut into ndev contiguous blocks (sizes differ by at most one column) and
 * block j is computed on GPU devices[j] through the drop-in host path (copy
 * pipeline, method and modulus count as given; B2_METHOD_DEFAULT = the calling
 * thread's method).  No data crosses between GPUs: each receives A and its
 * columns of B and C.  Host memory only (device or managed pointers return
 * B2_ERR_ARG, info 7/9/12); a device index may repeat (several shards on one
 * GPU).  Synchronous; one persistent host thread per (device, occurrence)
 * keeps its streams and workspaces between calls; sharded calls from several
 * host threads are serialised.  Argument errors use dgemm_'s positions;
 * ndev outside 1..64, an unknown or pre-sm_100 device, a bad method or slice
 * count give B2_ERR_ARG with info 0.  dgemm_ itself shards a product of at
 * least 2^32 flops on host operands this way when the environment variable
 * B2_DEVICES lists two or more devices ("0,1,2,3"). */
B2_API int b2_dgemm_multi(int ndev, const int *devices, char transa, char transb, int m, int n,
                          int k, double alpha, const double *A, int lda, const double *B,
                          int ldb, double beta, double *C, int ldc, int method, int slices);

/* Plan of the last Ozaki DGEMM on this thread: out[0] = modulus (slice)
 * count, out[1] = number of K chunks (K is cut at 32768 per exact INT32 pass).
 * With slices = 0 the count (15, or 16 for heavy-tailed rows) is chosen on the
 * device; this call waits for that choice to be copied back. */
B2_API int b2_ozaki_last_plan(int *out, int n);

/* Allocation-free INT8 Ozaki DGEMM.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory at call time -- a real-time
 * loop that must stay out of the allocator, or a process whose device memory
 * another framework reserved up front, where a cudaMalloc during the call
 * would fail or stall.  Same contract and result as b2_dgemm(...,
 * B2_METHOD_OZAKI, slices, stream) on device pointers (slices 0 means 15
 * moduli here: the heavy-tail switch to 16 of the allocating path is not
 * made), but all scratch lives in one static device array of
 * B2_NOALLOC_SCRATCH_BYTES per device, and the call never allocates or frees.
 * The array sits in its own device module: under lazy module loading (the
 * CUDA default) it is reserved on a device at the first call there and held
 * until the process exits; processes that never call this entry point do not
 * pay for it.  Limit: problems whose scratch exceeds the array -- square ones
 * above n = 1200 at 15 moduli (1161 at 16), or K > 32768 -- return
 * B2_ERR_ARG without touching C.  Every call on a device shares the array and
 * it keeps the last call's contents, so calls that overlap on the GPU race
 * and must be serialised by the caller.  The first call on a device resolves
 * the array's device address and uploads constant tables (synchronising its
 * stream); make it before any stream capture.  The status comes back only as
 * the return value (b2_last_error() is not updated); a bounded device wait
 * that gave up is read with b2_dgemm_ozaki_noalloc_error.  stream NULL = the
 * legacy default stream. */
#define B2_NOALLOC_SCRATCH_BYTES (64ull << 20)
B2_API int b2_dgemm_ozaki_noalloc(char transa, char transb, int m, int n, int k, double alpha,
                                  const double *A, int lda, const double *B, int ldb,
                                  double beta, double *C, int ldc, int slices, void *stream);
/* Error word of the last b2_dgemm_ozaki_noalloc on the current device (kept
 * in its static array; allocation-free): B2_ERR_TIMEOUT when a bounded device
 * wait of that call gave up, else 0.  Synchronises `stream`; clear resets the
 * word.  No counterpart in the reference. */
B2_API int b2_dgemm_ozaki_noalloc_error(int clear, void *stream);

/* Same contract as sgemm_ (src/gemm_driver.c:116) on device memory. */
B2_API int b2_sgemm(char transa, char transb, int m, int n, int k, float alpha, const float *A,
             int lda, const float *B, int ldb, float beta, float *C, int ldc, int method,
             void *stream);

/* Double-double GEMM (the accuracy yardstick): Chi + Clo ~= alpha*op(A)*op(B)
 * + beta*C0 to ~2^-104 relative, beta semantics as dgemm_.  C0 may be NULL
 * (treated as zero); Clo may be NULL.  Outputs are m x n with leading
 * dimension ldo.  No counterpart in the reference: it is the oracle every
 * result's error is stated against. */
B2_API int b2_dgemm_dd(char transa, char transb, int m, int n, int k, double alpha, const double *A,
                int lda, const double *B, int ldb, double beta, const double *C0, int ldc,
                double *Chi, double *Clo, int ldo, void *stream);

/* Same contract as dtrsm_ on device memory.  update_method selects the GEMM
 * that performs the trailing updates (B2_METHOD_FP64 or B2_METHOD_OZAKI);
 * block = diagonal block order (0 = 128). */
B2_API int b2_dtrsm(char side, char uplo, char transa, char diag, int m, int n, double alpha,
             const double *A, int lda, double *B, int ldb, int update_method, int block,
             void *stream);

/* Same contracts as zgemm3m_ / cgemm3m_ on device memory. */
B2_API int b2_zgemm3m(char transa, char transb, int m, int n, int k, const double *alpha,
               const double *A, int lda, const double *B, int ldb, const double *beta, double *C,
               int ldc, void *stream);
B2_API int b2_cgemm3m(char transa, char transb, int m, int n, int k, const float *alpha,
               const float *A, int lda, const float *B, int ldb, const float *beta, float *C,
               int ldc, void *stream);

/* ------------------------------------------------------------------------ */
/* OpenBLAS kernel-level ABI on device pointers: what an OpenBLAS-style       */
/* level-3 driver calls on its packed blocks.  Packed layout (the reference's */
/* copy routines, OpenBLAS-like_implementation/dgemm.c:304-403): an operand   */
/* of R rows (rows of A, columns of B) and depth k is cut into full panels of */
/* `unroll` rows, then panels of unroll/2, unroll/4, ..., 1; a panel of width */
/* w starting at row r0 sits at offset r0*k and holds (r, kk) at              */
/* r0*k + kk*w + (r - r0).  Unrolls are powers of two <= 64.  All pointers    */
/* are device memory; the calls are asynchronous on `stream` (NULL = the      */
/* library stream) and return a b2_status.                                   */
/* ------------------------------------------------------------------------ */

/* C (m x n, ldc) += alpha * A * B on packed A (unroll_m) and B (unroll_n):
 * the CNAME kernels of dgemm.c:247-263 (16x2), dgemm_kernel_4x8_skylakex_2.c:
 * 661-668 (4x8), kernel_avx512_opt8x8.c / kernel_avx512_standard8x8.c (8x8). */
B2_API int b2_dgemm_kernel(int unroll_m, int unroll_n, long m, long n, long k, double alpha,
                           const double *sa, const double *sb, double *C, long ldc, void *stream);
/* FP32 version: the CNAME kernel of sgemm.c:397-412 (16x4). */
B2_API int b2_sgemm_kernel(int unroll_m, int unroll_n, long m, long n, long k, float alpha,
                           const float *sa, const float *sb, float *C, long ldc, void *stream);
/* 3M step: C_cplx (m x n, ldc in complex elements, interleaved re/im) +=
 * (alphar + i alphai) * A * B with real packed A and B: the CNAME kernels of
 * zgemm3m_kernel_2x8_skylakex.c:336-351 and cgemm3m_kernel_16x4_skylakex.c:
 * 415-440. */
B2_API int b2_zgemm3m_kernel(int unroll_m, int unroll_n, long m, long n, long k, double alphar,
                             double alphai, const double *sa, const double *sb, double *C,
                             long ldc, void *stream);
B2_API int b2_cgemm3m_kernel(int unroll_m, int unroll_n, long m, long n, long k, float alphar,
                             float alphai, const float *sa, const float *sb, float *C, long ldc,
                             void *stream);
/* DTRSM solve kernels dtrsm_solve_{ln,lt,rn,rt}_m*n* (dtrsm_kernel_16x4_skylakex.S:
 * 1863-2536), contract of dtrsm_kernel_16x4_tester.c:66-199, for any m, n:
 * side 'L'/'R' and trans 'N'/'T' select ln, lt, rn, rt.  The packed triangle
 * carries its inverted diagonal; the incoming update is added to C, the
 * solution is written to C and back into the packed right-hand side (sb for
 * the left kernels, sa for the right ones). */
B2_API int b2_dtrsm_kernel(char side, char trans, long m, long n, double *sa, double *sb,
                           double *C, long ldb, long ldc, void *stream);

/* ------------------------------------------------------------------------ */
/* Grouped GEMM: many independent problems in one persistent launch.  No     */
/* counterpart API in the reference, whose parallel drivers split one GEMM   */
/* (src/gemm_driver.c:136-149; OpenBLAS-like_implementation/dgemm.c:449-483   */
/* task queue); here the queue spans a whole batch.  Pointers are device     */
/* pointers; each problem follows the dgemm_/sgemm_ contract, or for the     */
/* complex dtypes the zgemm3m_/cgemm3m_ contract: the 3M method's three real */
/* products (zgemm3m_kernel_2x8_skylakex.c:336-351, cgemm3m_kernel_16x4_     */
/* skylakex.c:415-440) and their pre/post additions run inside the same      */
/* launch, one tile of C per queue entry.                                    */
/* ------------------------------------------------------------------------ */
typedef struct b2_gemm_problem {
  int dtype;            /* 0 = FP64 (double), 1 = FP32 (float), 2 = complex128
                           (zgemm3m_), 3 = complex64 (cgemm3m_) */
  char transa, transb;  /* real: 'N'/'n' = no transpose, anything else =
                           transpose; complex: 'N', 'T', 'C' (conjugate
                           transpose) or 'R' (conjugate, no transpose) */
  int m, n, k;
  double alpha, beta;   /* real parts for the complex dtypes; rounded to
                           float for dtypes 1 and 3 */
  const void *A;        /* complex dtypes: interleaved (re, im) pairs, */
  int lda;              /* leading dimensions in complex elements */
  const void *B;
  int ldb;
  void *C;
  int ldc;
  double alpha_i, beta_i; /* imaginary parts of alpha and beta (dtypes 2, 3) */
} b2_gemm_problem;

/* One-shot: build and upload the descriptors (through pinned staging, on
 * `stream`) and launch; returns once the launch is enqueued, so the caller's
 * `problems` array may be reused at once.  Consecutive calls alternate two
 * descriptor slots: a call waits only for the launch two calls back.
 * On an invalid problem returns B2_ERR_ARG with b2_last_info() = its 1-based index. */
B2_API int b2_gemm_grouped(int count, const b2_gemm_problem *problems, void *stream);
/* Plan: descriptors uploaded once and "reset queue + launch" captured in a CUDA
 * graph; b2_grouped_plan_launch replays it (one graph launch) on `stream`. */
B2_API int b2_grouped_plan_create(int count, const b2_gemm_problem *problems, void **plan);
B2_API int b2_grouped_plan_launch(void *plan, void *stream);
B2_API int b2_grouped_plan_destroy(void *plan);

/* Error statistics of C against a double-double reference computed on the
 * device from the same inputs: normwise ||C - Cdd||_F / ||Cdd||_F and
 * max_ij |C - Cdd| / max_ij |Cdd|.  Synchronous.  Allocates scratch. */
B2_API int b2_dgemm_error(char transa, char transb, int m, int n, int k, double alpha,
                   const double *A, int lda, const double *B, int ldb, double beta,
                   const double *C0, const double *C, int ldc, double *normwise,
                   double *maxelem, void *stream);

/* Device-side error word of this thread's context: B2_ERR_TIMEOUT after a
 * bounded wait inside one of its kernels gave up (the reference's own waits
 * spin forever, src/gemm_driver.c:21-31).  The synchronous drop-in symbols
 * read and clear it themselves after their final synchronisation and report
 * B2_ERR_TIMEOUT through b2_last_error(); the asynchronous b2_* calls cannot
 * know at return, so after synchronising their stream call this.  Reading it
 * synchronizes the library stream; clear resets it. */
B2_API int b2_device_error(int clear);

/* Test hook of the failure detection: every later tensor-core launch (the
 * tcgen05 engines of the Ozaki, split-SGEMM and 3M paths) gives up a wait
 * after wait_ns nanoseconds instead of 2 s (wait_ns <= 0 restores 2 s; the
 * value is clamped to [0.1 ms, 10 s]), and the next withhold_launches
 * launches post their first K-block's byte count without issuing its copy,
 * so that the wait for it runs out: the kernel records B2_ERR_TIMEOUT, drains
 * and returns, and the call reports the timeout.  Nothing faults or hangs;
 * results of a withheld launch are invalid.  Process-wide. */
B2_API int b2_test_bounded_wait(long long wait_ns, int withhold_launches);


/* ------------------------------------------------------------------------ */
/* Tuning hooks (replace the compile-time block sizes of dgemm_tune.h:6-15,  */
/* sgemm_tune.h:6-15 and src/gemm_set_parameters.h:10-82)                    */
/* ------------------------------------------------------------------------ */

/* Per-thread override of the plain-FP64 kernel configuration used by every
 * later FP64 GEMM on this thread: tile 0 = 128x128, 1 = 128x64, 2 = 64x64;
 * mmak = DMMA K shape 4, 8 or 16; split_k >= 1.  tile < 0 clears the
 * override (the selector decides again). */
B2_API int b2_set_fp64_config(int tile, int mmak, int split_k);

/* DGEMM configuration space of the autotuner: b2_tune_config_count() (= 48)
 * configurations; 0..35 plain FP64 DMMA (tile {128x128,128x64,64x64} x DMMA K
 * {4,8,16} x split-K {1,2,4,8}), 36..47 INT8 Ozaki (moduli {13..16} x INT8
 * engine shape {128x256/4 stages, 128x128/6, 128x128/4}). */
B2_API int b2_tune_config_count(void);
/* Run one DGEMM (device pointers) with a given configuration. */
B2_API int b2_dgemm_config(char transa, char transb, int m, int n, int k, double alpha,
                           const double *A, int lda, const double *B, int ldb, double beta,
                           double *C, int ldc, int config, void *stream);
/* Exhaustive autotuner: shapes[6*i..] = {m, n, k, transA, transB, beta_is_zero};
 * out_ms[48*i + c] = per-call time of configuration c, the fastest of `reps`
 * CUDA-event timings of a batch of back-to-back calls (batch sized to ~100 us,
 * at most 32 calls) on resident random inputs.  Synchronous; allocates its own
 * buffers. */
B2_API int b2_tune_sweep(int nshapes, const int *shapes, int reps, float *out_ms);

/* SGEMM configuration space of the tensor-core methods (the selector's dtype
 * 1): config c = method c / 16 (0 = TF32, 1 = TF32X3, 2 = BF16X3) and, for
 * c % 16 < 12, engine (c % 16) / 4 (0 = single CTA 128x256 / 4 stages,
 * 1 = single CTA 128x128 / 6 stages, 2 = CTA pair 256x256 / 6 stages) x
 * split-K 1 << (c % 4); c % 16 >= 12 is unused (B2_ERR_ARG).  Replaces the
 * compile-time SGEMM block sizes of sgemm_tune.h:6-15. */
B2_API int b2_sgemm_config(char transa, char transb, int m, int n, int k, float alpha,
                           const float *A, int lda, const float *B, int ldb, float beta,
                           float *C, int ldc, int config, void *stream);
/* Exhaustive SGEMM sweep over those 48 slots (unused slots NaN); same shape
 * layout and timing rule as b2_tune_sweep, FP32 inputs. */
B2_API int b2_tune_sweep_sgemm(int nshapes, const int *shapes, int reps, float *out_ms);
/* Configuration the tensor-core SGEMM method `method` runs for this shape
 * (the selector's pick when weights are installed and every dimension is at
 * most 2048, else the library default); -1 for a non-tensor method. */
B2_API int b2_sgemm_selector_choose(int method, char transa, char transb, int m, int n, int k,
                                    int beta_zero);

/* Learned selector: a 7-64-64-48 ReLU MLP predicting log2(ms) per
 * configuration from (log2 M, log2 N, log2 K centred at 7 and scaled by 1/3,
 * transA, transB, dtype (0 = FP64: the 48 DGEMM configurations, 1 = FP32:
 * the 48 SGEMM slots above), beta == 0).  b2_mlp_param_count() floats, layout
 * W1[7][64] b1 W2[64][64] b2 W3[64][48] b3.  Training, gradients and batched
 * inference run in this library's own CUDA kernels. */
B2_API int b2_mlp_param_count(void);
B2_API int b2_mlp_train(int n, const float *X, const float *T, int epochs, int batch, float lr,
                        int seed, const float *weights_in, float *weights_out,
                        float *final_loss);
B2_API int b2_mlp_forward(const float *weights, int n, const float *X, float *Y);
B2_API int b2_mlp_gradient(const float *weights, int n, const float *X, const float *T,
                           float *loss, float *grad);
/* Install (or clear with NULL) the selector weights used by B2_METHOD_AUTO;
 * b2_selector_choose returns the configuration AUTO would run (Ozaki
 * configurations only with >= min_slices moduli), b2_selector_predict the 48
 * predictions. */
B2_API int b2_selector_set(const float *weights);
B2_API int b2_selector_choose(char transa, char transb, int m, int n, int k, int beta_zero,
                              int min_slices);
B2_API int b2_selector_predict(char transa, char transb, int m, int n, int k, int beta_zero,
                               float *pred);

/* ------------------------------------------------------------------------ */
/* Tracing (no counterpart in the reference, whose only instrumentation is   */
/* the tester's clock_gettime loops, dtrsm_kernel_16x4_tester.c:267-287)     */
/* ------------------------------------------------------------------------ */

/* Kernel launches this library has issued in this process (all threads). */
B2_API long long b2_launch_count(void);
/* Per-thread kernel timing: when on, every launch is bracketed by CUDA events
 * on its own stream.  b2_profile_report synchronizes those events, writes one
 * line "name launches total_ms" per kernel into buf (NUL-terminated, at most
 * len bytes) and clears the records; returns the number of kernels listed. */
B2_API int b2_profile_enable(int on);
B2_API int b2_profile_report(char *buf, int len);
/* The same records as a timeline: one line "name start_ms end_ms" per launch
 * in issue order, times relative to the earliest start among the records
 * (launches on different streams may overlap, and a later-issued launch may
 * start first); lines that do not fit in buf are dropped
 * whole.  Clears the records and returns how many launches were listed. */
B2_API int b2_profile_timeline(char *buf, int len);

#ifdef __cplusplus
}
#endif
#endif /* B2BLAS_H */
