// b2_methods.cuh -- method-level entry points shared by the API layer.
#pragma once

#include "b2_internal.cuh"

#define B2_MAX_MODULI 20

namespace b2 {

bool is_device_ptr(const void *p);
int stage_in(Ctx *c, int slot, const void *host, int rows, int cols, int ld, size_t elem,
             void **dev, int *dld, cudaStream_t s);
int stage_out(void *host, int ld, const void *dev, int dld, int rows, int cols, size_t elem,
              cudaStream_t s);
int check_gemm(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc, const void *a,
               const void *b, const void *c, int *info);

// DGEMM dispatch on device pointers (method may be DEFAULT/AUTO).
int dgemm_device(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                 const double *B, int ldb, double beta, double *C, int ldc, int method,
                 int slices, cudaStream_t s);
int sgemm_device(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                 const float *B, int ldb, float beta, float *C, int ldc, int method,
                 cudaStream_t s);

// Method selection for B2_METHOD_AUTO (tuner.cu): configuration chosen by the
// learned selector when installed, else by the measured heuristic.
int select_dgemm_method(Ctx *c, char ta, char tb, int m, int n, int k, int *slices);
int dgemm_auto(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
               const double *B, int ldb, double beta, double *C, int ldc, int slices,
               cudaStream_t s);

// INT8 Ozaki emulation of DGEMM (ozaki.cu).  slices = modulus count, 0 = auto.
int dgemm_ozaki(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                const double *B, int ldb, double beta, double *C, int ldc, int slices,
                cudaStream_t s);
int ozaki_auto_moduli(int k);
// The allocation-free Ozaki DGEMM on a caller-provided scratch area (base,
// cap bytes, 256-byte aligned; word 0 is the kernels' error word): scratch
// bytes one call needs, and the call itself (B2_ERR_ARG when it does not fit).
size_t ozaki_noalloc_bytes(int m, int n, int k, int s);
int ozaki_noalloc_run(unsigned char *base, size_t cap, int dev, int sm_count, char transa,
                      char transb, int m, int n, int k, double alpha, const double *A, int lda,
                      const double *B, int ldb, double beta, double *C, int ldc, int slices,
                      cudaStream_t st);
void ozaki_set_variant(int v);  // INT8 engine shape of the allocating path (0..4; -1 = default)
// Host-operand pipeline state of this thread: the next Ozaki DGEMM computes
// rows [r0, r0 + m) of op(A) for column block j, op(A) being m_full rows whose
// row 0 is at a_full (device).  A's exponents and residue slices are kept for
// all m_full rows and reused by later blocks.  j < 0 ends the pipeline and
// drops what was kept.
void ozaki_pipeline_rows(int j, const double *a_full, int m_full, int r0);

// SGEMM methods (sgemm.cu).
int sgemm_dispatch(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                   const float *B, int ldb, float beta, float *C, int ldc, int method,
                   cudaStream_t s);
int sgemm_tensor(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                 const float *B, int ldb, float beta, float *C, int ldc, int method,
                 cudaStream_t s);
// Engine configuration of a tensor-core SGEMM (sgemm_tc.cu): engine 0 =
// single CTA 128 x 256 / 4 stages, 1 = single CTA 128 x 128 / 6 stages, 2 =
// CTA pair 256 x 256 / 6 stages; split = K ranges (0 = automatic).
struct SgCfg {
  int engine = 0;
  int split = 0;
};
SgCfg sgemm_default_cfg(int m, int n, int k, int method);
// The selector's pick for a tensor-core SGEMM (tuner.cu; default without weights).
SgCfg sgemm_pick_cfg(char ta, char tb, int m, int n, int k, int beta0, int method);
int sgemm_tensor_cfg(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                     const float *B, int ldb, float beta, float *C, int ldc, int method,
                     const SgCfg &cfg, cudaStream_t s);
int sgemm_simt(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
               const float *B, int ldb, float beta, float *C, int ldc, cudaStream_t s);
// 3xTF32 operand split (sgemm_tc.cu): the R x K view X (element (r, k) at
// X[r*sr + k*sk]) as R rows of [big | small] TF32 segments of kp floats each
// (row pitch 2 kp floats), the layout the tensor-core engine reads.
int sgemm_split_tf32x3(const float *X, long long sr, long long sk, int R, int K, int kp,
                       float *out, cudaStream_t s);
// C(m, n) = alpha * sum_ks W[ks * plane + n * ldw + m] + beta C (beta != 1
// multiplies), the S partials summed in FP64 in K order and rounded once.
int sgemm_splitk_reduce(const float *W, long long plane, int ldw, int S, int m, int n,
                        float alpha, float beta, float *C, int ldc, cudaStream_t s);

// Blocked triangular solve (trsm.cu).
int dtrsm_device(char side, char uplo, char transa, char diag, int m, int n, double alpha,
                 const double *A, int lda, double *B, int ldb, int method, int block,
                 cudaStream_t s);

// Grouped GEMM (grouped.cu).
int grouped_device(int count, const b2_gemm_problem *problems, cudaStream_t s, int *info);
int grouped_plan_create(int count, const b2_gemm_problem *problems, void **plan, int *info);
int grouped_plan_launch(void *plan, cudaStream_t s);
int grouped_plan_destroy(void *plan);

// 3M complex GEMM, one fused launch (gemm3m.cu); alpha/beta are (re, im) pairs.
template <typename T>
int gemm3m_device(char ta, char tb, int m, int n, int k, const T *alpha, const T *A, int lda,
                  const T *B, int ldb, const T *beta, T *C, int ldc, cudaStream_t s);

}  // namespace b2
