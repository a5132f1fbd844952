// dd_gemm.cu -- double-double GEMM on the FP64 pipe: the accuracy yardstick
// every result's error is stated against.
//
// Each product a*b is split exactly into p + e with TwoProd via fma (Dekker
// 1971: e = fma(a, b, -p) is exact), and added into a (hi, lo) pair with
// TwoSum (Knuth, TAOCP vol. 2, sec. 4.2.2).  The low words collect the
// rounding errors of the running sum, so hi + lo carries ~2^-100 relative
// accuracy for the K used here.  The final alpha/beta step is done in the
// same arithmetic, with the reference's beta semantics (C scaled whenever
// beta != 1, src/gemm_driver.c:131).
#include "b2_internal.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace {

constexpr int DD_BM = 64, DD_BN = 64, DD_BK = 16;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) dd_gemm_kernel(int M, int N, int K, double alpha,
                                                      const double *__restrict__ A, int lda,
                                                      const double *__restrict__ B, int ldb,
                                                      double beta,
                                                      const double *__restrict__ C0, int ldc,
                                                      double *__restrict__ Chi,
                                                      double *__restrict__ Clo, int ldo) {
  __shared__ double As[DD_BK][DD_BM + 1];
  __shared__ double Bs[DD_BK][DD_BN + 1];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int m0 = blockIdx.x * DD_BM, n0 = blockIdx.y * DD_BN;
  double sh[4][4], sl[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) sh[i][j] = sl[i][j] = 0.0;

  if (alpha != 0.0) {
    for (int k0 = 0; k0 < K; k0 += DD_BK) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int idx = tid + 256 * e;
        int kk, mm;
        if (TA) { kk = idx % DD_BK; mm = idx / DD_BK; } else { kk = idx / DD_BM; mm = idx % DD_BM; }
        const int gm = m0 + mm, gk = k0 + kk;
        double v = 0.0;
        if (gm < M && gk < K) v = TA ? A[(size_t)gm * lda + gk] : A[(size_t)gk * lda + gm];
        As[kk][mm] = v;
        int nn;
        if (!TB) { kk = idx % DD_BK; nn = idx / DD_BK; } else { kk = idx / DD_BN; nn = idx % DD_BN; }
        const int gn = n0 + nn, gk2 = k0 + kk;
        double w = 0.0;
        if (gn < N && gk2 < K) w = TB ? B[(size_t)gk2 * ldb + gn] : B[(size_t)gn * ldb + gk2];
        Bs[kk][nn] = w;
      }
      __syncthreads();
#pragma unroll 4
      for (int kk = 0; kk < DD_BK; ++kk) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const double p = a[i] * b[j];
            const double pe = fma(a[i], b[j], -p);
            const double s = sh[i][j] + p;
            const double bb = s - sh[i][j];
            const double te = (sh[i][j] - (s - bb)) + (p - bb);
            sh[i][j] = s;
            sl[i][j] += te + pe;
          }
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {  // renormalise (FastTwoSum)
          const double s = sh[i][j] + sl[i][j];
          sl[i][j] = sl[i][j] - (s - sh[i][j]);
          sh[i][j] = s;
        }
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int m = m0 + tx + 16 * i, n = n0 + ty + 16 * j;
      if (m >= M || n >= N) continue;
      // (ph, pl) = alpha * (sh, sl)
      double ph = sh[i][j] * alpha;
      double pl = fma(sh[i][j], alpha, -ph) + sl[i][j] * alpha;
      const double c = C0 ? C0[(size_t)n * ldc + m] : 0.0;
      double qh, ql;
      if (beta != 1.0) { qh = beta * c; ql = fma(beta, c, -qh); } else { qh = c; ql = 0.0; }
      const double s = ph + qh;
      const double bb = s - ph;
      double te = (ph - (s - bb)) + (qh - bb);
      te += pl + ql;
      const double hi = s + te;
      const double lo = te - (hi - s);
      Chi[(size_t)n * ldo + m] = hi;
      if (Clo) Clo[(size_t)n * ldo + m] = lo;
    }
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  // non-negative doubles (and NaN) order like their bit patterns
  atomicMax((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

__global__ void error_stats_kernel(int M, int N, const double *__restrict__ C, int ldc,
                                   const double *__restrict__ R, int ldr, double *out) {
  double s_dd = 0.0, s_rr = 0.0, mx_d = 0.0, mx_r = 0.0;
  const size_t total = (size_t)M * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M), n = (int)(idx / M);
    const double r = R[(size_t)n * ldr + m];
    const double d = C[(size_t)n * ldc + m] - r;
    s_dd = fma(d, d, s_dd);
    s_rr = fma(r, r, s_rr);
    mx_d = fmax(mx_d, fabs(d));
    mx_r = fmax(mx_r, fabs(r));
    if (d != d) mx_d = d;  // keep NaN visible
  }
  for (int o = 16; o > 0; o >>= 1) {
    s_dd += __shfl_down_sync(0xffffffffu, s_dd, o);
    s_rr += __shfl_down_sync(0xffffffffu, s_rr, o);
    mx_d = fmax(mx_d, __shfl_down_sync(0xffffffffu, mx_d, o));
    mx_r = fmax(mx_r, __shfl_down_sync(0xffffffffu, mx_r, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out + 0, s_dd);
    atomicAdd(out + 1, s_rr);
    atomic_max_nonneg(out + 2, mx_d != mx_d ? mx_d : fabs(mx_d));
    atomic_max_nonneg(out + 3, mx_r);
  }
}

}  // namespace

int dgemm_dd(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
             const double *B, int ldb, double beta, const double *C0, int ldc, double *Chi,
             double *Clo, int ldo, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  const bool TA = !(ta == 'N' || ta == 'n');
  const bool TB = !(tb == 'N' || tb == 'n');
  if (k <= 0) alpha = 0.0;
  dim3 grid((m + DD_BM - 1) / DD_BM, (n + DD_BN - 1) / DD_BN);
  B2_PROF("dgemm_dd", s);
  if (TA && TB)
    dd_gemm_kernel<true, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C0, ldc, Chi, Clo, ldo);
  else if (TA)
    dd_gemm_kernel<true, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C0, ldc, Chi, Clo, ldo);
  else if (TB)
    dd_gemm_kernel<false, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C0, ldc, Chi, Clo, ldo);
  else
    dd_gemm_kernel<false, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C0, ldc, Chi, Clo, ldo);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int error_stats(int m, int n, const double *C, int ldc, const double *Ref, int ldr, double *out,
                cudaStream_t s) {
  B2_CUDA_TRY(cudaMemsetAsync(out, 0, 4 * sizeof(double), s));
  if (m <= 0 || n <= 0) return B2_OK;
  const size_t total = (size_t)m * n;
  const int blocks = (int)((total + 255) / 256 > 2048 ? 2048 : (total + 255) / 256);
  B2_PROF("error_stats", s);
  error_stats_kernel<<<blocks, 256, 0, s>>>(m, n, C, ldc, Ref, ldr, out);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

}  // namespace b2
