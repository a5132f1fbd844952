// kernel_abi.cu -- the OpenBLAS kernel-level ABI of the reference, on device
// pointers: packed-panel GEMM kernels (real and 3M complex) and the DTRSM
// solve kernels, so an OpenBLAS-style level-3 driver can hand its packed
// blocks to the GPU.
//
// Packed layout (the reference's copy routines, dgemm.c:304-403): an operand
// of R rows (rows of A, or columns of B) and depth K is cut into full panels
// of `unroll` rows followed by panels of unroll/2, unroll/4, ..., 1 for the
// remainder; a panel of width w starting at row r0 sits at offset r0*K and
// holds element (r, k) at r0*K + k*w + (r - r0).
//
// The GEMM kernels unpack both operands into K-contiguous rows (one HBM pass)
// and run the library's own GEMMs (DMMA FP64, FFMA FP32); the reference's
// kernels accumulate, C += alpha * A B, and so do these.  The solve kernels
// restate dtrsm_kernel_16x4_tester.c:66-199 (the contract of
// dtrsm_kernel_16x4_skylakex.S:1863-2536) for any M, N: columns (left side)
// or rows (right side) are independent, one thread each.
#include "b2_methods.cuh"

namespace b2 {
namespace {

bool pow2_unroll(int u) { return u >= 1 && u <= 64 && (u & (u - 1)) == 0; }

// Row r of a packed operand: panel start r0 and width w.
__device__ __forceinline__ void panel_of(long long r, long long rows, int unroll, long long *r0,
                                         long long *w) {
  const long long full = rows / unroll * unroll;
  if (r < full) {
    *r0 = r / unroll * unroll;
    *w = unroll;
    return;
  }
  const long long rem = rows - full;
  long long base = full;
  for (long long ww = unroll >> 1; ww >= 1; ww >>= 1) {
    if (rem & ww) {
      if (r < base + ww) {
        *r0 = base;
        *w = ww;
        return;
      }
      base += ww;
    }
  }
  *r0 = r;  // unreachable for r < rows
  *w = 1;
}

// dst[r*K + k] = packed(r, k): threads over k (x), rows over y (strided).
template <typename T>
__global__ void unpack_panels_kernel(const T *__restrict__ src, long long rows, long long K,
                                     int unroll, T *__restrict__ dst) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= K) return;
  for (long long r = blockIdx.y; r < rows; r += gridDim.y) {
    long long r0, w;
    panel_of(r, rows, unroll, &r0, &w);
    dst[r * K + k] = src[r0 * K + k * w + (r - r0)];
  }
}

template <typename T>
int unpack(const T *src, long long rows, long long K, int unroll, T *dst, cudaStream_t s) {
  dim3 grid((unsigned)((K + 127) / 128), (unsigned)(rows < 4096 ? rows : 4096));
  unpack_panels_kernel<T><<<grid, 128, 0, s>>>(src, rows, K, unroll, dst);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

// C_cplx(i, j) += (ar + i ai) * D(i, j); C interleaved, ldc in complex elements.
template <typename T>
__global__ void add_3m_kernel(const T *__restrict__ D, long long m, long long n, T ar, T ai,
                              T *__restrict__ C, long long ldc) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m) return;
  for (long long j = blockIdx.y; j < n; j += gridDim.y) {
    const T d = D[i + j * m];
    T *c = C + 2 * (i + j * ldc);
    c[0] = fma(ar, d, c[0]);
    c[1] = fma(ai, d, c[1]);
  }
}

template <typename T>
int gemm_kernel_packed(int um, int un, long long m, long long n, long long k, T ar, T ai,
                       const T *sa, const T *sb, T *C, long long ldc, bool cplx, void *stream) {
  if (!pow2_unroll(um) || !pow2_unroll(un) || m < 0 || n < 0 || k < 0) return B2_ERR_ARG;
  if (m > 0x7fffffffll || n > 0x7fffffffll || k > 0x7fffffffll) return B2_ERR_ARG;
  if (ldc < (m > 1 ? m : 1)) return B2_ERR_ARG;
  if (m == 0 || n == 0 || k == 0 || (ar == (T)0 && ai == (T)0)) return B2_OK;
  if (!is_device_ptr(sa) || !is_device_ptr(sb) || !is_device_ptr(C)) return B2_ERR_ARG;
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  cudaStream_t s = pick_stream(c, stream);
  T *A = (T *)workspace(c, WS_KABI_A, (size_t)m * k * sizeof(T));
  T *B = (T *)workspace(c, WS_KABI_B, (size_t)n * k * sizeof(T));
  T *D = cplx ? (T *)workspace(c, WS_KABI_D, (size_t)m * n * sizeof(T)) : nullptr;
  if (!A || !B || (cplx && !D)) return B2_ERR_NOMEM;
  int st = unpack(sa, m, k, um, A, s);
  if (st == B2_OK) st = unpack(sb, n, k, un, B, s);
  if (st != B2_OK) return st;
  // The 3M product goes to scratch with beta = 0, and beta = 0 multiplies
  // (a NaN left in the scratch would survive): start it at zero.
  if (cplx) B2_CUDA_TRY(cudaMemsetAsync(D, 0, (size_t)m * n * sizeof(T), s));
  // A as k x m column-major (op 'T'), B as k x n column-major (op 'N')
  T *out = cplx ? D : C;
  const long long ldo = cplx ? m : ldc;
  const T al = cplx ? (T)1 : ar, be = cplx ? (T)0 : (T)1;
  if constexpr (sizeof(T) == 8)
    st = dgemm_fp64('T', 'N', (int)m, (int)n, (int)k, al, A, (int)k, B, (int)k, be, out, (int)ldo,
                    s, nullptr);
  else
    st = sgemm_dispatch('T', 'N', (int)m, (int)n, (int)k, al, A, (int)k, B, (int)k, be, out,
                        (int)ldo, B2_METHOD_FP32, s);
  if (st != B2_OK || !cplx) return st;
  dim3 grid((unsigned)((m + 127) / 128), (unsigned)(n < 4096 ? n : 4096));
  add_3m_kernel<T><<<grid, 128, 0, s>>>(D, m, n, ar, ai, C, ldc);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

// Left side (tester.c:145-199): per group of up to 4 columns, C += the packed
// update in sb (element (m, j) at sb[j + m*n_group]), then substitution with
// the inverted diagonal of the packed triangle sa (element (r, c) at
// sa[c*M + r]); X goes to C and back into sb.  One thread per column.
__global__ void trsm_left_kernel(bool forward, long long M, long long N, const double *sa,
                                 double *sb, double *C, long long LDB, long long LDC) {
  const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (col >= N) return;
  const long long g = col / 4, j = col % 4;
  const long long gw = N - 4 * g < 4 ? N - 4 * g : 4;
  double *sbg = sb + g * 4 * LDB;
  double *c = C + (g * 4 + j) * LDC;
  for (long long m = 0; m < M; ++m) c[m] += sbg[j + m * gw];
  for (long long t = 0; t < M; ++t) {
    const long long mk = forward ? t : M - 1 - t;
    const double b0 = c[mk] * sa[mk * M + mk];
    c[mk] = b0;
    sbg[mk * gw + j] = b0;
    if (forward)
      for (long long ml = mk + 1; ml < M; ++ml) c[ml] = fma(-b0, sa[mk * M + ml], c[ml]);
    else
      for (long long mu = 0; mu < mk; ++mu) c[mu] = fma(-b0, sa[mk * M + mu], c[mu]);
  }
}

// Right side (tester.c:91-143): C += the packed update in sa (element (m, j)
// at sa[m + j*M]), then substitution along the columns with the packed
// triangle sb (4-column panels of pitch 4*LDB, get_b of tester.c:91-95); X
// goes to C and back into sa.  One thread per row.
__global__ void trsm_right_kernel(bool forward, long long M, long long N, double *sa,
                                  const double *sb, double *C, long long LDB, long long LDC) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= M) return;
  const long long un = N > 4 ? 4 : N;
  auto gb = [&](long long kk, long long nn) {
    return sb[(nn >> 2) * (LDB << 2) + kk * un + (nn & 3)];
  };
  for (long long j = 0; j < N; ++j) C[m + j * LDC] += sa[m + j * M];
  for (long long t = 0; t < N; ++t) {
    const long long nk = forward ? t : N - 1 - t;
    const double x = C[m + nk * LDC] * gb(nk, nk);
    C[m + nk * LDC] = x;
    sa[m + nk * M] = x;
    if (forward)
      for (long long nr = nk + 1; nr < N; ++nr)
        C[m + nr * LDC] = fma(-x, gb(nk, nr), C[m + nr * LDC]);
    else
      for (long long nl = 0; nl < nk; ++nl)
        C[m + nl * LDC] = fma(-x, gb(nk, nl), C[m + nl * LDC]);
  }
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" {

int b2_dgemm_kernel(int unroll_m, int unroll_n, long m, long n, long k, double alpha,
                    const double *sa, const double *sb, double *C, long ldc, void *stream) {
  return gemm_kernel_packed<double>(unroll_m, unroll_n, m, n, k, alpha, 0.0, sa, sb, C, ldc,
                                    false, stream);
}

int b2_sgemm_kernel(int unroll_m, int unroll_n, long m, long n, long k, float alpha,
                    const float *sa, const float *sb, float *C, long ldc, void *stream) {
  return gemm_kernel_packed<float>(unroll_m, unroll_n, m, n, k, alpha, 0.0f, sa, sb, C, ldc,
                                   false, stream);
}

int b2_zgemm3m_kernel(int unroll_m, int unroll_n, long m, long n, long k, double alphar,
                      double alphai, const double *sa, const double *sb, double *C, long ldc,
                      void *stream) {
  return gemm_kernel_packed<double>(unroll_m, unroll_n, m, n, k, alphar, alphai, sa, sb, C, ldc,
                                    true, stream);
}

int b2_cgemm3m_kernel(int unroll_m, int unroll_n, long m, long n, long k, float alphar,
                      float alphai, const float *sa, const float *sb, float *C, long ldc,
                      void *stream) {
  return gemm_kernel_packed<float>(unroll_m, unroll_n, m, n, k, alphar, alphai, sa, sb, C, ldc,
                                   true, stream);
}

int b2_dtrsm_kernel(char side, char trans, long m, long n, double *sa, double *sb, double *C,
                    long ldb, long ldc, void *stream) {
  const bool left = side == 'L' || side == 'l';
  const bool tr = !(trans == 'N' || trans == 'n');
  if (m < 0 || n < 0 || ldc < (m > 1 ? m : 1) || ldb < 0) return B2_ERR_ARG;
  if (m == 0 || n == 0) return B2_OK;
  if (!is_device_ptr(sa) || !is_device_ptr(sb) || !is_device_ptr(C)) return B2_ERR_ARG;
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  cudaStream_t s = pick_stream(c, stream);
  // lt / rn solve forward, ln / rt backward (tester.c:97-199)
  const bool forward = left ? tr : !tr;
  if (left) {
    trsm_left_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(forward, m, n, sa, sb, C, ldb,
                                                                  ldc);
  } else {
    trsm_right_kernel<<<(unsigned)((m + 127) / 128), 128, 0, s>>>(forward, m, n, sa, sb, C, ldb,
                                                                   ldc);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

}  // extern "C"
