// sgemm.cu -- SGEMM methods.
//
// Native FP32 replaces the reference's AVX-512 SGEMM (src/gemm_driver.c:116
// built without -DDOUBLE driving the 48x8 tile of src/kernel/gemm_kernel.S,
// and the m16 x n24 tiles of OpenBLAS-like_implementation/sgemm.c:366-412):
// a CUDA-core FFMA kernel with a 128x128 CTA tile, 8x8 outputs per thread in
// registers, double-buffered shared-memory K panels.  The tensor-core forms
// (TF32, 3xTF32, 3xBF16) run on the tcgen05 engine in umma_gemm.cu.
#include "b2_methods.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace {

constexpr int SB_M = 128, SB_N = 128, SB_K = 8, SB_PAD = 4;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256, 2)
    sgemm_simt_kernel(int M, int N, int K, float alpha, const float *__restrict__ A, int lda,
                      const float *__restrict__ B, int ldb, float beta, float *__restrict__ C,
                      int ldc) {
  __shared__ __align__(16) float As[2][SB_K][SB_M + SB_PAD];
  __shared__ __align__(16) float Bs[2][SB_K][SB_N + SB_PAD];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int m0 = blockIdx.x * SB_M, n0 = blockIdx.y * SB_N;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  float ra[4], rb[4];
  auto gload = [&](int k0) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = tid + 256 * e;
      int kk, mm;
      if (TA) { kk = idx % SB_K; mm = idx / SB_K; } else { kk = idx / SB_M; mm = idx % SB_M; }
      const int gm = m0 + mm, gk = k0 + kk;
      ra[e] = (gm < M && gk < K) ? (TA ? A[(size_t)gm * lda + gk] : A[(size_t)gk * lda + gm]) : 0.f;
      int nn;
      if (!TB) { kk = idx % SB_K; nn = idx / SB_K; } else { kk = idx / SB_N; nn = idx % SB_N; }
      const int gn = n0 + nn, gk2 = k0 + kk;
      rb[e] = (gn < N && gk2 < K) ? (TB ? B[(size_t)gk2 * ldb + gn] : B[(size_t)gn * ldb + gk2]) : 0.f;
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = tid + 256 * e;
      int kk, mm;
      if (TA) { kk = idx % SB_K; mm = idx / SB_K; } else { kk = idx / SB_M; mm = idx % SB_M; }
      As[buf][kk][mm] = ra[e];
      int nn;
      if (!TB) { kk = idx % SB_K; nn = idx / SB_K; } else { kk = idx / SB_N; nn = idx % SB_N; }
      Bs[buf][kk][nn] = rb[e];
    }
  };

  const int KT = (K + SB_K - 1) / SB_K;
  gload(0);
  sstore(0);
  __syncthreads();
  for (int kt = 0; kt < KT; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < KT) gload((kt + 1) * SB_K);
#pragma unroll
    for (int kk = 0; kk < SB_K; ++kk) {
      float a[8], b[8];
      const float4 a0 = *reinterpret_cast<const float4 *>(&As[buf][kk][tx * 4]);
      const float4 a1 = *reinterpret_cast<const float4 *>(&As[buf][kk][64 + tx * 4]);
      const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][ty * 4]);
      const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][64 + ty * 4]);
      a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
      a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
      b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
      b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (kt + 1 < KT) {
      sstore(buf ^ 1);
      __syncthreads();
    }
  }
  const bool beta_one = (beta == 1.f);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int n = n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
    if (n >= N) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int m = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
      if (m >= M) continue;
      float *p = C + (size_t)n * ldc + m;
      *p = beta_one ? fmaf(alpha, acc[i][j], *p) : fmaf(alpha, acc[i][j], beta * *p);
    }
  }
}

}  // namespace

int sgemm_simt(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
               const float *B, int ldb, float beta, float *C, int ldc, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  if (k <= 0 || alpha == 0.f) return beta == 1.f ? B2_OK : scale_matrix_s(m, n, beta, C, ldc, s);
  const bool TA = !(ta == 'N' || ta == 'n');
  const bool TB = !(tb == 'N' || tb == 'n');
  dim3 grid((m + SB_M - 1) / SB_M, (n + SB_N - 1) / SB_N);
  B2_PROF("sgemm_simt", s);
  if (TA && TB)
    sgemm_simt_kernel<true, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  else if (TA)
    sgemm_simt_kernel<true, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  else if (TB)
    sgemm_simt_kernel<false, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  else
    sgemm_simt_kernel<false, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int sgemm_dispatch(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                   const float *B, int ldb, float beta, float *C, int ldc, int method,
                   cudaStream_t s) {
  switch (method) {
    case B2_METHOD_FP32:
    case B2_METHOD_DEFAULT:
      return sgemm_simt(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    case B2_METHOD_TF32:
    case B2_METHOD_TF32X3:
    case B2_METHOD_BF16X3:
      return sgemm_tensor(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, method, s);
    default:
      return B2_ERR_UNSUPPORTED;
  }
}

}  // namespace b2
