// sgemm.cu -- SGEMM methods.
//
// Native FP32 replaces the reference's AVX-512 SGEMM (src/gemm_driver.c:116
// built without -DDOUBLE driving the 48x8 tile of src/kernel/gemm_kernel.S,
// and the m16 x n24 tiles of OpenBLAS-like_implementation/sgemm.c:366-412):
// a CUDA-core kernel of paired FP32 FMAs (fma.rn.f32x2) with a 128x128 CTA
// tile, 8x8 outputs per thread in registers, double-buffered shared-memory K
// panels.  The tensor-core forms (TF32, 3xTF32, 3xBF16) run on the tcgen05
// engine (sgemm_tc.cu).
#include "b2_methods.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace {

// ----------------------------------------------------------------------
// Paired-FMA FP32 kernel (sm_100 fma.rn.f32x2: two FP32 FMAs per issued
// instruction, so the FFMA pipe, not instruction issue, is the limit).
// CTA tile 128 x 128, K blocks of 16, 256 threads of 8 x 8 outputs, K panels
// staged through registers (16-byte global loads when the layout allows)
// into double-buffered shared memory.  Thread (tx, ty) owns rows
// 4 tx + {0..3} + 64 h' and columns 4 ty + {0..3} + 64 h (h', h = 0, 1): per
// K step it reads two 16-byte A vectors and two 16-byte B vectors (64 bytes
// for 64 FMAs -- the shared-memory rate of 128 bytes per clock per SM then
// matches the 128 FMAs per clock) and forms the broadcast pairs (a, a) in
// registers.  Storing A duplicated in shared memory instead (one 16-byte load
// giving two pairs) cost 96 bytes per 64 FMAs and made the kernel
// shared-memory bound (ncu at 4096^3: L1 84 % busy, FMA pipe 55 %).  Two CTAs
// per SM (128 registers, a few bytes spilled) beat one CTA with 150 registers:
// 54.4 against 51.3 TFLOPS at 8192^3, 52.6 against 49.0 at 4096^3.
constexpr int S2_M = 128, S2_N = 128, S2_K = 16, S2_APAD = 4, S2_BPAD = 4;
constexpr int S2_ALD = S2_M + S2_APAD;  // floats per k row of the A panel
constexpr int S2_BLD = S2_N + S2_BPAD;
constexpr int S2_SMEM = (2 * S2_K * S2_ALD + 2 * S2_K * S2_BLD) * 4;

__device__ __forceinline__ unsigned long long dup2(float a) {
  unsigned long long d;
  asm("mov.b64 %0, {%1, %1};" : "=l"(d) : "f"(a));
  return d;
}

__device__ __forceinline__ void ffma2(unsigned long long &c, unsigned long long a,
                                      unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(c) : "l"(a), "l"(b));
}

// Four consecutive floats starting at p (16-byte aligned when VEC), or fewer
// at the matrix edge (lim = elements available from p), zero beyond.
template <bool VEC>
__device__ __forceinline__ float4 load4(const float *p, int lim) {
  if (VEC && lim >= 4) return __ldg(reinterpret_cast<const float4 *>(p));
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  if (lim > 0) v.x = p[0];
  if (lim > 1) v.y = p[1];
  if (lim > 2) v.z = p[2];
  if (lim > 3) v.w = p[3];
  return v;
}

template <bool TA, bool TB, bool VEC, bool SPLIT>
__global__ void __launch_bounds__(256, 2)
    sgemm_ffma2_kernel(int M, int N, int K, float alpha, const float *__restrict__ A, int lda,
                       const float *__restrict__ B, int ldb, float beta, float *__restrict__ C,
                       int ldc, int kchunk, float *__restrict__ P, long long plane, int ldp) {
  // Slice blockIdx.z of a split-K launch reads its own K range: either the
  // operand bases shift to it and K shortens (SHIFT), or K stays and kbeg /
  // kend bound the range.  The form per transpose pair is the one ptxas
  // compiles with the fewest spilled registers (NN shifts by 64-bit offsets).
  constexpr bool SHIFT = SPLIT && (TA || !TB);
  if (SHIFT) {
    if (TA) {
      const int kb = blockIdx.z * kchunk;
      A += (size_t)kb;
      B += TB ? (size_t)kb * ldb : (size_t)kb;
      K = min(kchunk, K - kb);
    } else {
      const long long kb = (long long)blockIdx.z * kchunk;
      A += kb * lda;
      B += kb;
      K = min(kchunk, K - (int)kb);
    }
  }
  extern __shared__ __align__(16) float s2mem[];
  float *As = s2mem;                        // [2][S2_K][S2_ALD]
  float *Bs = s2mem + 2 * S2_K * S2_ALD;    // [2][S2_K][S2_BLD]
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * S2_M, n0 = blockIdx.y * S2_N;
  // K range of this CTA (kchunk a multiple of S2_K); a split-K slice writes
  // its raw sums to P + z * plane.
  const int kbeg = (SPLIT && !SHIFT) ? blockIdx.z * kchunk : 0;
  const int kend = (SPLIT && !SHIFT) ? min(K, kbeg + kchunk) : K;

  unsigned long long acc[8][4];  // row r: 4tx + (r&3) + 64(r>>2); column pair c
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0ull;

  // Register staging of one K block: 8 A values and 8 B values per thread.
  // A: element (m, k) at A[k*lda + m] ('N') or A[m*lda + k] ('T');
  // B: element (k, n) at B[n*ldb + k] ('N') or B[k*ldb + n] ('T').
  float4 ra[2], rb[2];
  auto gload = [&](int k0) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = tid + 256 * h;
      if (!TA) {  // 4 consecutive m of one k
        const int kk = c >> 5, mm = (c & 31) * 4, gm = m0 + mm, gk = k0 + kk;
        ra[h] = gk < kend ? load4<VEC>(A + (size_t)gk * lda + gm, M - gm) : make_float4(0.f, 0.f, 0.f, 0.f);
      } else {    // 4 consecutive k of one m
        const int mm = c >> 2, kk = (c & 3) * 4, gm = m0 + mm, gk = k0 + kk;
        ra[h] = gm < M ? load4<VEC>(A + (size_t)gm * lda + gk, kend - gk) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (TB) {   // 4 consecutive n of one k
        const int kk = c >> 5, nn = (c & 31) * 4, gn = n0 + nn, gk = k0 + kk;
        rb[h] = gk < kend ? load4<VEC>(B + (size_t)gk * ldb + gn, N - gn) : make_float4(0.f, 0.f, 0.f, 0.f);
      } else {    // 4 consecutive k of one n
        const int nn = c >> 2, kk = (c & 3) * 4, gn = n0 + nn, gk = k0 + kk;
        rb[h] = gn < N ? load4<VEC>(B + (size_t)gn * ldb + gk, kend - gk) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  };
  auto sstore = [&](int buf) {
    float *as = As + buf * S2_K * S2_ALD;
    float *bs = Bs + buf * S2_K * S2_BLD;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = tid + 256 * h;
      if (!TA) {
        const int kk = c >> 5, mm = (c & 31) * 4;
        *reinterpret_cast<float4 *>(as + kk * S2_ALD + mm) = ra[h];
      } else {
        const int mm = c >> 2, kk = (c & 3) * 4;
        const float av[4] = {ra[h].x, ra[h].y, ra[h].z, ra[h].w};
#pragma unroll
        for (int e = 0; e < 4; ++e) as[(kk + e) * S2_ALD + mm] = av[e];
      }
      if (TB) {
        const int kk = c >> 5, nn = (c & 31) * 4;
        *reinterpret_cast<float4 *>(bs + kk * S2_BLD + nn) = rb[h];
      } else {
        const int nn = c >> 2, kk = (c & 3) * 4;
        const float bv[4] = {rb[h].x, rb[h].y, rb[h].z, rb[h].w};
#pragma unroll
        for (int e = 0; e < 4; ++e) bs[(kk + e) * S2_BLD + nn] = bv[e];
      }
    }
  };

  const int KT = (kend - kbeg + S2_K - 1) / S2_K;
  gload(kbeg);
  sstore(0);
  __syncthreads();
  for (int kt = 0; kt < KT; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < KT) gload(kbeg + (kt + 1) * S2_K);
    const float *as = As + buf * S2_K * S2_ALD;
    const float *bs = Bs + buf * S2_K * S2_BLD;
#pragma unroll
    for (int kk = 0; kk < S2_K; ++kk) {
      float av[8];  // rows 4tx + i + 64h'
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const float4 v = *reinterpret_cast<const float4 *>(as + kk * S2_ALD + 64 * hh + 4 * tx);
        av[4 * hh] = v.x;
        av[4 * hh + 1] = v.y;
        av[4 * hh + 2] = v.z;
        av[4 * hh + 3] = v.w;
      }
      ulonglong2 b2[2];  // columns 64h + 4ty .. 64h + 4ty + 3
#pragma unroll
      for (int h = 0; h < 2; ++h)
        b2[h] = *reinterpret_cast<const ulonglong2 *>(bs + kk * S2_BLD + 64 * h + 4 * ty);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const unsigned long long a = dup2(av[r]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          ffma2(acc[r][2 * h], a, b2[h].x);
          ffma2(acc[r][2 * h + 1], a, b2[h].y);
        }
      }
    }
    if (kt + 1 < KT) {
      // the other buffer was last read in the previous iteration, which every
      // thread finished before that iteration's closing barrier
      sstore(buf ^ 1);
      __syncthreads();
    }
  }
  const bool beta_one = (beta == 1.f);
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int m = m0 + 4 * tx + (r & 3) + 64 * (r >> 2);
    if (m >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float2 v = *reinterpret_cast<const float2 *>(&acc[r][c]);
      const int nb = n0 + 64 * (c >> 1) + 4 * ty + 2 * (c & 1);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int n = nb + e;
        if (n >= N) continue;
        const float x = e ? v.y : v.x;
        if (SPLIT) {
          P[blockIdx.z * plane + (long long)n * ldp + m] = x;
          continue;
        }
        float *p = C + (size_t)n * ldc + m;
        *p = beta_one ? fmaf(alpha, x, *p) : fmaf(alpha, x, beta * *p);
      }
    }
  }
}

// K slices for a grid of `tiles` CTAs at two per SM: 1 when the tiles fill
// the slots, else the count (at most 8, each slice >= 32 K blocks of 16)
// whose work units best fill whole waves of 2 * sms.  8192 x 256 x 8192 has
// 128 tiles for the 296 slots of 148 SMs; 2 slices fill them 86 %.
int ffma2_ksplit(long long tiles, int kblocks, int sms) {
  const long long slots = 2ll * sms;
  if (tiles >= slots) return 1;
  int best = 1;
  double best_eff = (double)tiles / slots;
  for (int S = 2; S <= 8 && S * 32 <= kblocks; ++S) {
    const long long units = tiles * S, waves = (units + slots - 1) / slots;
    const double eff = (double)units / (double)(waves * slots);
    if (eff > best_eff + 0.02) {
      best = S;
      best_eff = eff;
    }
  }
  return best;
}

template <bool TA, bool TB, bool VEC>
int launch_ffma2(int m, int n, int k, float alpha, const float *A, int lda, const float *B,
                 int ldb, float beta, float *C, int ldc, cudaStream_t s) {
  auto kern = sgemm_ffma2_kernel<TA, TB, VEC, false>;
  auto kern_split = sgemm_ffma2_kernel<TA, TB, VEC, true>;
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  const int gx = (m + S2_M - 1) / S2_M, gy = (n + S2_N - 1) / S2_N;
  const int kblocks = (k + S2_K - 1) / S2_K;
  const int S = ffma2_ksplit((long long)gx * gy, kblocks, cx->sm_count);
  if (S == 1) {
    B2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S2_SMEM));
    B2_PROF("sgemm_simt", s);
    kern<<<dim3(gx, gy), 256, S2_SMEM, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, k,
                                             nullptr, 0, 0);
    B2_CUDA_TRY(cudaGetLastError());
    return B2_OK;
  }
  // Split-K: S raw partial products of K ranges (multiples of S2_K), then one
  // reduction adding them in K order (FP64 sums, rounded once) into C.
  const int kchunk = (kblocks + S - 1) / S * S2_K;
  const int S_used = (k + kchunk - 1) / kchunk;
  const long long plane = (long long)n * m;
  float *P = (float *)workspace(cx, WS_MISC, (size_t)plane * S_used * sizeof(float));
  if (!P) return B2_ERR_NOMEM;
  {
    B2_CUDA_TRY(
        cudaFuncSetAttribute(kern_split, cudaFuncAttributeMaxDynamicSharedMemorySize, S2_SMEM));
    B2_PROF("sgemm_simt", s);
    kern_split<<<dim3(gx, gy, S_used), 256, S2_SMEM, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C,
                                                           ldc, kchunk, P, plane, m);
    B2_CUDA_TRY(cudaGetLastError());
  }
  return sgemm_splitk_reduce(P, plane, m, S_used, m, n, alpha, beta, C, ldc, s);
}

}  // namespace

int sgemm_simt(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
               const float *B, int ldb, float beta, float *C, int ldc, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  if (k <= 0 || alpha == 0.f) return beta == 1.f ? B2_OK : scale_matrix_s(m, n, beta, C, ldc, s);
  const bool TA = !(ta == 'N' || ta == 'n');
  const bool TB = !(tb == 'N' || tb == 'n');
  // 16-byte loads need 16-byte aligned bases and leading dimensions of 4k floats
  const bool vec = (lda % 4 == 0) && (ldb % 4 == 0) && (((uintptr_t)A & 15) == 0) &&
                   (((uintptr_t)B & 15) == 0);
  if (vec) {
    if (TA && TB) return launch_ffma2<true, true, true>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    if (TA) return launch_ffma2<true, false, true>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    if (TB) return launch_ffma2<false, true, true>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    return launch_ffma2<false, false, true>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
  }
  if (TA && TB) return launch_ffma2<true, true, false>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
  if (TA) return launch_ffma2<true, false, false>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
  if (TB) return launch_ffma2<false, true, false>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
  return launch_ffma2<false, false, false>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
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
