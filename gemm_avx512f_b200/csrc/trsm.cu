// trsm.cu -- blocked triangular solve on the GPU (dtrsm_).
//
// The reference ships DTRSM solve kernels for packed panels
// (OpenBLAS-like_implementation/dtrsm_16x4/dtrsm_kernel_16x4_skylakex.S:1863-2536,
// semantics in dtrsm_kernel_16x4_tester.c:66-199: add the incoming GEMM update,
// solve against the triangle whose diagonal is stored inverted, write X back),
// driven by an OpenBLAS trsm driver.  Here the driver is a recursive split of
// the triangle: solve the leading part, update the trailing right-hand sides
// with one large GEMM (plain FP64 DMMA or the INT8 Ozaki emulation), solve the
// trailing part.  Leaves have order <= 128: all diagonal blocks op(A_kk) are
// inverted up front in one batched launch (trtri_batched_kernel, substitution
// against the identity with the diagonal inverted first, the reference
// kernels' convention), and each leaf solve is then a small FP64 DMMA GEMM
// X_k = inv(op(A_kk)) Z_k (side 'L') or Z_k inv(op(A_kk)) (side 'R').
// Trailing updates use the INT8 Ozaki GEMM when requested and the product is
// large enough to amortise its slicing passes, plain FP64 otherwise.
#include "b2_methods.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace {

constexpr int TB = 128;        // leaf order
constexpr int TB_LD = TB + 1;  // shared row stride

// Invert every diagonal block T_b = op(A)[kb:kb+bs, kb:kb+bs] (lower or upper,
// unit or not); block b goes to Tinv + b*TB*TB (column-major, ld TB, zero
// outside the triangle and beyond bs).  T(i,j) = A[(kb+i) + (kb+j)*lda] when
// !a_swap, A[(kb+j) + (kb+i)*lda] when a_swap.  Thread j computes column j of
// inv(T) by substitution against e_j, multiplying by the inverted diagonal;
// the column lives in the output buffer (thread-private, L1 resident).
__global__ void __launch_bounds__(TB)
    trtri_batched_kernel(const double *__restrict__ A, int lda, int n, int lower, int a_swap,
                         int unit, double *__restrict__ Tinv) {
  extern __shared__ double tsm[];
  double *T = tsm;               // T[j*TB_LD + i] = T(i, j)
  double *inv = tsm + TB * TB_LD;
  const int kb = blockIdx.x * TB;
  const int bs = min(TB, n - kb);
  for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
    const int i = idx % bs, j = idx / bs;
    const long long r = a_swap ? (long long)(kb + j) + (long long)(kb + i) * lda
                               : (long long)(kb + i) + (long long)(kb + j) * lda;
    T[j * TB_LD + i] = A[r];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bs; i += blockDim.x) inv[i] = unit ? 1.0 : 1.0 / T[i * TB_LD + i];
  __syncthreads();
  const int j = threadIdx.x;
  double *x = Tinv + (long long)blockIdx.x * TB * TB + (long long)j * TB;  // column j
  for (int i = 0; i < TB; ++i) x[i] = 0.0;
  if (j >= bs) return;
  if (lower) {
    for (int i = j; i < bs; ++i) {
      double acc = (i == j) ? 1.0 : 0.0;
      for (int k = j; k < i; ++k) acc = fma(-T[k * TB_LD + i], x[k], acc);
      x[i] = acc * inv[i];
    }
  } else {
    for (int i = j; i >= 0; --i) {
      double acc = (i == j) ? 1.0 : 0.0;
      for (int k = i + 1; k <= j; ++k) acc = fma(-T[k * TB_LD + i], x[k], acc);
      x[i] = acc * inv[i];
    }
  }
}

__global__ void fill_zero_kernel(int M, int N, double *__restrict__ B, int ldb) {
  const long long total = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x)
    B[(idx / M) * ldb + idx % M] = 0.0;
}

struct TrsmPlan {
  bool left, upper, trans, unit;
  int m, n;
  const double *A;
  int lda;
  double *B;
  int ldb;
  int method;
  int leaf;
  cudaStream_t s;
  int sm_count;
  double *tinv;  // inverted diagonal blocks, TB x TB each
  double *tmp;   // leaf product scratch (max(m,n) x TB)
};

// Trailing-update GEMM: the INT8 emulation only where its slicing passes are
// amortised (measured: below ~2^33 multiply-adds or K < 1024 plain FP64 wins).
int update_gemm(const TrsmPlan &p, char ta, char tb, int m, int n, int k, const double *A,
                int lda, const double *B, int ldb, double *C, int ldc) {
  int meth = p.method;
  if (meth != B2_METHOD_FP64 && ((double)m * n * k < 8.6e9 || k < 1024)) meth = B2_METHOD_FP64;
  return dgemm_device(ta, tb, m, n, k, -1.0, A, lda, B, ldb, 1.0, C, ldc, meth, 0, p.s);
}

int diag_solve(const TrsmPlan &p, int kk, int bs) {
  const double *Ti = p.tinv + (long long)(kk / TB) * TB * TB;
  int rc;
  if (p.left) {  // X_k = inv(T) Z_k, Z_k = B[kk:kk+bs, :]
    B2_CUDA_TRY(cudaMemsetAsync(p.tmp, 0, (size_t)bs * p.n * sizeof(double), p.s));
    rc = dgemm_device('N', 'N', bs, p.n, bs, 1.0, Ti, TB, p.B + kk, p.ldb, 0.0, p.tmp, bs,
                      B2_METHOD_FP64, 0, p.s);
    if (rc != B2_OK) return rc;
    B2_CUDA_TRY(cudaMemcpy2DAsync(p.B + kk, (size_t)p.ldb * sizeof(double), p.tmp,
                                  (size_t)bs * sizeof(double), (size_t)bs * sizeof(double), p.n,
                                  cudaMemcpyDeviceToDevice, p.s));
    return B2_OK;
  }
  // X_k = Z_k inv(T), Z_k = B[:, kk:kk+bs]
  B2_CUDA_TRY(cudaMemsetAsync(p.tmp, 0, (size_t)p.m * bs * sizeof(double), p.s));
  rc = dgemm_device('N', 'N', p.m, bs, bs, 1.0, p.B + (long long)kk * p.ldb, p.ldb, Ti, TB, 0.0,
                    p.tmp, p.m, B2_METHOD_FP64, 0, p.s);
  if (rc != B2_OK) return rc;
  B2_CUDA_TRY(cudaMemcpy2DAsync(p.B + (long long)kk * p.ldb, (size_t)p.ldb * sizeof(double), p.tmp,
                                (size_t)p.m * sizeof(double), (size_t)p.m * sizeof(double), bs,
                                cudaMemcpyDeviceToDevice, p.s));
  return B2_OK;
}

// Solve the order-nr diagonal part starting at k0 (rows of B for side 'L',
// columns for side 'R').
int solve_range(const TrsmPlan &p, int k0, int nr) {
  if (nr <= p.leaf) return diag_solve(p, k0, nr);
  int n1 = (nr / 2 + p.leaf - 1) / p.leaf * p.leaf;
  if (n1 >= nr) n1 = nr - p.leaf;
  const int n2 = nr - n1;
  const int k1 = k0 + n1;
  const bool opA_lower = (!p.upper && !p.trans) || (p.upper && p.trans);
  const char tA = p.trans ? 'T' : 'N';
  // op(A)[r, c] block pointer for a GEMM operand: op(A)(i,j) = A[i,j] (N) or A[j,i] (T)
  auto opA_block = [&](int r0, int c0) -> const double * {
    return p.trans ? p.A + c0 + (long long)r0 * p.lda : p.A + r0 + (long long)c0 * p.lda;
  };
  int rc;
  if (p.left) {
    if (opA_lower) {  // forward: solve top, B2 -= op(A)21 X1, solve bottom
      rc = solve_range(p, k0, n1);
      if (rc != B2_OK) return rc;
      rc = update_gemm(p, tA, 'N', n2, p.n, n1, opA_block(k1, k0), p.lda, p.B + k0, p.ldb,
                       p.B + k1, p.ldb);
      if (rc != B2_OK) return rc;
      return solve_range(p, k1, n2);
    }
    // backward: solve bottom, B1 -= op(A)12 X2, solve top
    rc = solve_range(p, k1, n2);
    if (rc != B2_OK) return rc;
    rc = update_gemm(p, tA, 'N', n1, p.n, n2, opA_block(k0, k1), p.lda, p.B + k1, p.ldb,
                     p.B + k0, p.ldb);
    if (rc != B2_OK) return rc;
    return solve_range(p, k0, n1);
  }
  // side 'R': X op(A) = B over column blocks
  if (!opA_lower) {  // op(A) upper: forward over columns
    rc = solve_range(p, k0, n1);
    if (rc != B2_OK) return rc;
    rc = update_gemm(p, 'N', tA, p.m, n2, n1, p.B + (long long)k0 * p.ldb, p.ldb,
                     opA_block(k0, k1), p.lda, p.B + (long long)k1 * p.ldb, p.ldb);
    if (rc != B2_OK) return rc;
    return solve_range(p, k1, n2);
  }
  rc = solve_range(p, k1, n2);  // op(A) lower: backward over columns
  if (rc != B2_OK) return rc;
  rc = update_gemm(p, 'N', tA, p.m, n1, n2, p.B + (long long)k1 * p.ldb, p.ldb,
                   opA_block(k1, k0), p.lda, p.B + (long long)k0 * p.ldb, p.ldb);
  if (rc != B2_OK) return rc;
  return solve_range(p, k0, n1);
}

}  // namespace

int dtrsm_device(char side, char uplo, char transa, char diag, int m, int n, double alpha,
                 const double *A, int lda, double *B, int ldb, int method, int block,
                 cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  if (alpha == 0.0) {  // BLAS: B := 0
    const long long total = (long long)m * n;
    const int blocks = (int)((total + 255) / 256 > 4096 ? 4096 : (total + 255) / 256);
    B2_PROF("trsm_zero", s);
    fill_zero_kernel<<<blocks, 256, 0, s>>>(m, n, B, ldb);
    B2_CUDA_TRY(cudaGetLastError());
    return B2_OK;
  }
  if (alpha != 1.0) {
    const int rc = scale_matrix_d(m, n, alpha, B, ldb, s);
    if (rc != B2_OK) return rc;
  }
  TrsmPlan p;
  p.left = (side == 'L' || side == 'l');
  p.upper = (uplo == 'U' || uplo == 'u');
  p.trans = !(transa == 'N' || transa == 'n');
  p.unit = (diag == 'U' || diag == 'u');
  p.m = m;
  p.n = n;
  p.A = A;
  p.lda = lda;
  p.B = B;
  p.ldb = ldb;
  p.method = method == B2_METHOD_DEFAULT ? B2_METHOD_FP64 : method;
  (void)block;  // leaves are the TB-order inverted diagonal blocks
  p.leaf = TB;
  p.s = s;
  p.sm_count = cx->sm_count;
  const int na = p.left ? m : n;
  const int nblk = (na + TB - 1) / TB;
  const int nvec = p.left ? n : m;
  p.tinv = (double *)workspace(cx, WS_TRSM_INV, (size_t)nblk * TB * TB * sizeof(double));
  p.tmp = (double *)workspace(cx, WS_TRSM_TMP, (size_t)nvec * TB * sizeof(double));
  if (!p.tinv || !p.tmp) return B2_ERR_NOMEM;
  {
    const bool opA_lower = (!p.upper && !p.trans) || (p.upper && p.trans);
    const int smem = (TB * TB_LD + TB) * (int)sizeof(double);
    B2_CUDA_TRY(cudaFuncSetAttribute(trtri_batched_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    B2_PROF("trsm_trtri", s);
    trtri_batched_kernel<<<nblk, TB, smem, s>>>(A, lda, na, opA_lower ? 1 : 0, p.trans ? 1 : 0,
                                                p.unit ? 1 : 0, p.tinv);
    B2_CUDA_TRY(cudaGetLastError());
  }
  return solve_range(p, 0, na);
}

}  // namespace b2
