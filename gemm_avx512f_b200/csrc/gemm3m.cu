// gemm3m.cu -- complex GEMM by the 3M method.
//
// zgemm3m runs in ONE fused launch (zgemm3m_dmma_kernel, FP64 DMMA) below 2^35
// multiply-adds and as three FP64 DMMA GEMMs between a pre-add pass and a
// combine pass above; cgemm3m runs in one fused FFMA launch below 2^24
// multiply-adds and otherwise as three 3xTF32 tensor-core GEMMs
// (gemm3m_three_gemms, at the end).
//
// Replaces the OpenBLAS gemm3m driver + the reference's 3M kernels
// (zgemm3m_kernel_2x8_skylakex.c:336-351, zgemm3m_kernel_8x4_skylakex.c:309-334,
// cgemm3m_kernel_16x4_skylakex.c:415-440).  The reference kernels compute
// C_cplx += (alpha_r + i alpha_i) (A_real_packed . B_real_packed) and are called
// three times by the driver on pre-added panels.  Here every CTA owns one tile
// of C and forms all three real products from the same staged tiles:
//     P1 = Ar Br,  P2 = Ai Bi,  P3 = (Ar + Ai)(Br + Bi)
//     Re(AB) = P1 - P2,  Im(AB) = P3 - P1 - P2
// The pre-additions (and conjugation for 'C'/'R') happen while the complex
// tiles are de-interleaved into shared memory; the post-additions and the
// complex alpha/beta happen in the epilogue.  beta follows the reference
// drivers (C scaled whenever beta != 1, src/gemm_driver.c:131).
//   zgemm3m: FP64 DMMA (mma.sync.m16n8k4.f64), 64x64 tile, 8 warps of 32x16.
//   cgemm3m: FP32 FFMA, 64x64 tile, 256 threads of 4x4 outputs.
#include <stdlib.h>

#include "b2_methods.cuh"
#include "b2_profile.cuh"
#include "umma.cuh"

namespace b2 {
namespace {

constexpr int G_BM = 64, G_BN = 64, G_BK = 16, G_PAD = 4;
constexpr int G_LD = G_BM + G_PAD;  // [k][m] / [k][n] row stride (68 = 4 mod 16 doubles)

__device__ __forceinline__ bool tr_is_t(char c) {
  return !(c == 'N' || c == 'n' || c == 'R' || c == 'r');
}
__device__ __forceinline__ bool tr_is_conj(char c) {
  return c == 'C' || c == 'c' || c == 'R' || c == 'r';
}

// Stage one BK-deep complex K panel of op(A) (G_BM rows) and op(B) (G_BN
// columns) into registers.  Element (m,k) of op(A) is A[m*lda+k] when
// transposed, else A[k*lda+m] (complex units); element (k,n) of op(B) is
// B[k*ldb+n] when transposed, else B[n*ldb+k].
template <typename T, int NT>
struct Stage3M {
  static constexpr int PER = G_BM * G_BK / NT;  // complex elements per thread per operand
  T ar[PER], ai[PER], br[PER], bi[PER];
  __device__ __forceinline__ void load(const T *A, int lda, const T *B, int ldb, int M, int N,
                                       int K, int m0, int n0, int k0, bool tA, bool tB,
                                       T sa, T sb, int tid) {
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      const int idx = tid + NT * e;
      int mm, kk;
      if (tA) { kk = idx % G_BK; mm = idx / G_BK; } else { mm = idx % G_BM; kk = idx / G_BM; }
      const int gm = m0 + mm, gk = k0 + kk;
      T re = 0, im = 0;
      if (gm < M && gk < K) {
        const T *p = A + 2 * (tA ? ((long long)gm * lda + gk) : ((long long)gk * lda + gm));
        re = p[0];
        im = sa * p[1];
      }
      ar[e] = re;
      ai[e] = im;
      int nn;
      if (tB) { nn = idx % G_BN; kk = idx / G_BN; } else { kk = idx % G_BK; nn = idx / G_BK; }
      const int gn = n0 + nn, gk2 = k0 + kk;
      re = 0;
      im = 0;
      if (gn < N && gk2 < K) {
        const T *p = B + 2 * (tB ? ((long long)gk2 * ldb + gn) : ((long long)gn * ldb + gk2));
        re = p[0];
        im = sb * p[1];
      }
      br[e] = re;
      bi[e] = im;
    }
  }
  // shared layout: [3][BK][G_LD] for A (r, i, r+i) and the same for B
  __device__ __forceinline__ void store(T *sA, T *sB, bool tA, bool tB, int tid) const {
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      const int idx = tid + NT * e;
      int mm, kk;
      if (tA) { kk = idx % G_BK; mm = idx / G_BK; } else { mm = idx % G_BM; kk = idx / G_BM; }
      sA[(0 * G_BK + kk) * G_LD + mm] = ar[e];
      sA[(1 * G_BK + kk) * G_LD + mm] = ai[e];
      sA[(2 * G_BK + kk) * G_LD + mm] = ar[e] + ai[e];
      int nn;
      if (tB) { nn = idx % G_BN; kk = idx / G_BN; } else { kk = idx % G_BK; nn = idx / G_BK; }
      sB[(0 * G_BK + kk) * G_LD + nn] = br[e];
      sB[(1 * G_BK + kk) * G_LD + nn] = bi[e];
      sB[(2 * G_BK + kk) * G_LD + nn] = br[e] + bi[e];
    }
  }
};

template <typename T>
__device__ __forceinline__ void epilogue3m(T *C, int ldc, int m, int n, T p1, T p2, T p3,
                                           T ar, T ai, T br, T bi) {
  const T re = p1 - p2, im = p3 - p1 - p2;
  T *c = C + 2 * ((long long)n * ldc + m);
  T cr = c[0], ci = c[1];
  if (!(br == (T)1 && bi == (T)0)) {
    const T tr = br * cr - bi * ci, ti = br * ci + bi * cr;
    cr = tr;
    ci = ti;
  }
  c[0] = cr + (ar * re - ai * im);
  c[1] = ci + (ar * im + ai * re);
}

// ---------------------------------------------------- zgemm3m: FP64 DMMA --
__global__ void __launch_bounds__(256)
    zgemm3m_kernel(int M, int N, int K, const double *__restrict__ A, int lda,
                   const double *__restrict__ B, int ldb, double *__restrict__ C, int ldc,
                   double ar, double ai, double br, double bi, char transa, char transb) {
  extern __shared__ __align__(16) double zsm[];  // [2][3*BK*LD] A, then [2][3*BK*LD] B
  double *sA[2] = {zsm, zsm + 3 * G_BK * G_LD};
  double *sB[2] = {zsm + 6 * G_BK * G_LD, zsm + 9 * G_BK * G_LD};
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp >> 2) * 32, wn0 = (warp & 3) * 16;
  const int m0 = blockIdx.x * G_BM, n0 = blockIdx.y * G_BN;
  const bool tA = tr_is_t(transa), tB = tr_is_t(transb);
  const double sa = tr_is_conj(transa) ? -1.0 : 1.0, sb = tr_is_conj(transb) ? -1.0 : 1.0;
  double acc[3][2][2][4];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[p][i][j][v] = 0.0;

  Stage3M<double, 256> st;
  const int KT = (K + G_BK - 1) / G_BK;
  st.load(A, lda, B, ldb, M, N, K, m0, n0, 0, tA, tB, sa, sb, tid);
  st.store(sA[0], sB[0], tA, tB, tid);
  __syncthreads();
  for (int kt = 0; kt < KT; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < KT) st.load(A, lda, B, ldb, M, N, K, m0, n0, (kt + 1) * G_BK, tA, tB, sa, sb, tid);
    const double *As = sA[buf], *Bs = sB[buf];
#pragma unroll
    for (int kk = 0; kk < G_BK; kk += 4) {
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        double af[2][2], bf[2];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int v = 0; v < 2; ++v)
            af[i][v] = As[(p * G_BK + kk + t) * G_LD + wm0 + i * 16 + g + 8 * v];
#pragma unroll
        for (int j = 0; j < 2; ++j) bf[j] = Bs[(p * G_BK + kk + t) * G_LD + wn0 + j * 8 + g];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j)
            asm volatile(
                "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, "
                "{%6}, {%0,%1,%2,%3};\n"
                : "+d"(acc[p][i][j][0]), "+d"(acc[p][i][j][1]), "+d"(acc[p][i][j][2]),
                  "+d"(acc[p][i][j][3])
                : "d"(af[i][0]), "d"(af[i][1]), "d"(bf[j]));
      }
    }
    if (kt + 1 < KT) {
      st.store(sA[buf ^ 1], sB[buf ^ 1], tA, tB, tid);
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int m = m0 + wm0 + i * 16 + g + 8 * (v >> 1);
        const int n = n0 + wn0 + j * 8 + 2 * t + (v & 1);
        if (m < M && n < N)
          epilogue3m<double>(C, ldc, m, n, acc[0][i][j][v], acc[1][i][j][v], acc[2][i][j][v],
                             ar, ai, br, bi);
      }
}

// ---------------------------------------------------- cgemm3m: FP32 FFMA --
__global__ void __launch_bounds__(256)
    cgemm3m_kernel(int M, int N, int K, const float *__restrict__ A, int lda,
                   const float *__restrict__ B, int ldb, float *__restrict__ C, int ldc,
                   float ar, float ai, float br, float bi, char transa, char transb) {
  extern __shared__ __align__(16) float csm[];
  float *sA[2] = {csm, csm + 3 * G_BK * G_LD};
  float *sB[2] = {csm + 6 * G_BK * G_LD, csm + 9 * G_BK * G_LD};
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * G_BM, n0 = blockIdx.y * G_BN;
  const bool tA = tr_is_t(transa), tB = tr_is_t(transb);
  const float sa = tr_is_conj(transa) ? -1.f : 1.f, sb = tr_is_conj(transb) ? -1.f : 1.f;
  float acc[3][4][4];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[p][i][j] = 0.f;
  Stage3M<float, 256> st;
  const int KT = (K + G_BK - 1) / G_BK;
  st.load(A, lda, B, ldb, M, N, K, m0, n0, 0, tA, tB, sa, sb, tid);
  st.store(sA[0], sB[0], tA, tB, tid);
  __syncthreads();
  for (int kt = 0; kt < KT; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < KT) st.load(A, lda, B, ldb, M, N, K, m0, n0, (kt + 1) * G_BK, tA, tB, sa, sb, tid);
    const float *As = sA[buf], *Bs = sB[buf];
#pragma unroll
    for (int kk = 0; kk < G_BK; ++kk) {
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const float4 a = *reinterpret_cast<const float4 *>(&As[(p * G_BK + kk) * G_LD + tx * 4]);
        const float4 b = *reinterpret_cast<const float4 *>(&Bs[(p * G_BK + kk) * G_LD + ty * 4]);
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[p][i][j] = fmaf(av[i], bv[j], acc[p][i][j]);
      }
    }
    if (kt + 1 < KT) {
      st.store(sA[buf ^ 1], sB[buf ^ 1], tA, tB, tid);
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int m = m0 + tx * 4 + i, n = n0 + ty * 4 + j;
      if (m < M && n < N)
        epilogue3m<float>(C, ldc, m, n, acc[0][i][j], acc[1][i][j], acc[2][i][j], ar, ai, br, bi);
    }
}

// --------------------------------------- zgemm3m: one-launch FP64 DMMA --
// The fused 3M product for complex128 at any size, on the FP64 tensor path
// (mma.sync.m16n8k8.f64; tcgen05 has no f64 kind).  CTA tile 64 x 64 complex
// outputs, 16 warps of 16 x 16, K in blocks of 16 complex elements streamed
// global -> shared by cp.async (one 16-byte complex element per copy, zero
// filled outside the matrix) through a 4-deep ring.  The smem tile keeps the
// interleaved (re, im) pairs, so one 16-byte shared load gives a fragment
// element's real and imaginary part; per K step every warp issues
//     P1 += Ar Br,   P2 += Ai Bi,   P3 += (Ar + sa Ai)(Br + sb Bi)
// with the pre-additions made on the fragments in registers (sa, sb = -1 for
// conjugated operands), and the epilogue forms
//     Re = P1 - sa sb P2,   Im = P3 - P1 - sa sb P2
// and applies the complex alpha and beta (beta != 1 scales C, as the
// reference drivers do: src/gemm_driver.c:131).  Padding: +4 complex per row
// when K is contiguous, +2 otherwise, so both orientations' 16-byte fragment
// loads are conflict free.
constexpr int Z_BM = 64, Z_BN = 64, Z_BK = 16, Z_WM = 4, Z_WN = 4, Z_STAGES = 4;
constexpr int Z_NT = Z_WM * Z_WN * 32;

template <bool KC>
__host__ __device__ constexpr int z_stage_elems(int outer) {
  return KC ? outer * (Z_BK + 4) : Z_BK * (outer + 2);
}

// One OUTER x BK complex tile; element (o, k) at g[o*ld + k] when KC (K
// contiguous) else g[k*ld + o] (complex units).  Shared: KC -> [o][BK+4],
// else [k][OUTER+2].
template <int OUTER, bool KC>
__device__ __forceinline__ void z_load_tile(uint32_t sbase, const double2 *__restrict__ g, int ld,
                                            int o0, int k0, int olim, int klim, int tid) {
  constexpr int TOTAL = OUTER * Z_BK;
  static_assert(TOTAL % Z_NT == 0, "tile/thread mismatch");
#pragma unroll
  for (int i = 0; i < TOTAL / Z_NT; ++i) {
    const int c = tid + i * Z_NT;
    int o, k;
    if (KC) { o = c / Z_BK; k = c % Z_BK; } else { k = c / OUTER; o = c % OUTER; }
    const int go = o0 + o, gk = k0 + k;
    const bool ok = go < olim && gk < klim;
    const double2 *src = ok ? g + (KC ? (size_t)go * ld + gk : (size_t)gk * ld + go) : g;
    const uint32_t dst = sbase + (uint32_t)(KC ? o * (Z_BK + 4) + k : k * (OUTER + 2) + o) * 16u;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                 "r"(ok ? 16 : 0));
  }
}

template <bool A_KC, bool B_KC>
__global__ void __launch_bounds__(Z_NT, 1)
    zgemm3m_dmma_kernel(int M, int N, int K, const double2 *__restrict__ A, int lda,
                        const double2 *__restrict__ B, int ldb, double2 *__restrict__ C, int ldc,
                        double ar, double ai, double br, double bi, double sa, double sb) {
  constexpr int A_ST = z_stage_elems<A_KC>(Z_BM), B_ST = z_stage_elems<B_KC>(Z_BN);
  extern __shared__ __align__(16) double2 zsh[];
  double2 *sA = zsh;
  double2 *sB = zsh + Z_STAGES * A_ST;
  const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA);
  const uint32_t sB_u = (uint32_t)__cvta_generic_to_shared(sB);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp / Z_WN) * 16, wn0 = (warp % Z_WN) * 16;
  const int m0 = blockIdx.x * Z_BM, n0 = blockIdx.y * Z_BN;
  const int KT = (K + Z_BK - 1) / Z_BK;

  double acc[3][2][4];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[p][j][v] = 0.0;

  auto load_stage = [&](int st, int kt) {
    const int k0 = kt * Z_BK;
    z_load_tile<Z_BM, A_KC>(sA_u + st * A_ST * 16, A, lda, m0, k0, M, K, tid);
    z_load_tile<Z_BN, B_KC>(sB_u + st * B_ST * 16, B, ldb, n0, k0, N, K, tid);
  };
#pragma unroll
  for (int st = 0; st < Z_STAGES - 1; ++st) {
    if (st < KT) load_stage(st, st);
    asm volatile("cp.async.commit_group;\n" ::);
  }
  for (int kt = 0; kt < KT; ++kt) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(Z_STAGES - 2));
    __syncthreads();
    {
      const int kn = kt + Z_STAGES - 1;
      if (kn < KT) load_stage(kn % Z_STAGES, kn);
      asm volatile("cp.async.commit_group;\n" ::);
    }
    const double2 *As = sA + (kt % Z_STAGES) * A_ST;
    const double2 *Bs = sB + (kt % Z_STAGES) * B_ST;
#pragma unroll
    for (int kk = 0; kk < Z_BK; kk += 8) {
      double are[4], aim[4], bre[2][2], bim[2][2];
#pragma unroll
      for (int v1 = 0; v1 < 2; ++v1)
#pragma unroll
        for (int v0 = 0; v0 < 2; ++v0) {
          const int m = wm0 + g + 8 * v0, k = kk + t + 4 * v1;
          const double2 x = A_KC ? As[m * (Z_BK + 4) + k] : As[k * (Z_BM + 2) + m];
          are[v0 + 2 * v1] = x.x;
          aim[v0 + 2 * v1] = x.y;
        }
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const int n = wn0 + j * 8 + g, k = kk + t + 4 * v;
          const double2 x = B_KC ? Bs[n * (Z_BK + 4) + k] : Bs[k * (Z_BN + 2) + n];
          bre[j][v] = x.x;
          bim[j][v] = x.y;
        }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+d"(acc[0][j][0]), "+d"(acc[0][j][1]), "+d"(acc[0][j][2]), "+d"(acc[0][j][3])
            : "d"(are[0]), "d"(are[1]), "d"(are[2]), "d"(are[3]), "d"(bre[j][0]), "d"(bre[j][1]));
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+d"(acc[1][j][0]), "+d"(acc[1][j][1]), "+d"(acc[1][j][2]), "+d"(acc[1][j][3])
            : "d"(aim[0]), "d"(aim[1]), "d"(aim[2]), "d"(aim[3]), "d"(bim[j][0]), "d"(bim[j][1]));
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) are[v] = fma(sa, aim[v], are[v]);
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int v = 0; v < 2; ++v) bre[j][v] = fma(sb, bim[j][v], bre[j][v]);
#pragma unroll
      for (int j = 0; j < 2; ++j)
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+d"(acc[2][j][0]), "+d"(acc[2][j][1]), "+d"(acc[2][j][2]), "+d"(acc[2][j][3])
            : "d"(are[0]), "d"(are[1]), "d"(are[2]), "d"(are[3]), "d"(bre[j][0]), "d"(bre[j][1]));
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::);

  // Fragment (j, v): row g + 8 (v >> 1), column 2t + (v & 1) of the warp tile.
  const double s2 = sa * sb;
  const bool beta_one = br == 1.0 && bi == 0.0;
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int m = m0 + wm0 + g + 8 * (v >> 1);
      const int n = n0 + wn0 + j * 8 + 2 * t + (v & 1);
      if (m < M && n < N) {
        const double p1 = acc[0][j][v], p2 = s2 * acc[1][j][v], p3 = acc[2][j][v];
        const double re = p1 - p2, im = p3 - p1 - p2;
        double2 *c = C + (size_t)n * ldc + m;
        double2 cv = *c;
        if (!beta_one) cv = make_double2(br * cv.x - bi * cv.y, br * cv.y + bi * cv.x);
        *c = make_double2(cv.x + (ar * re - ai * im), cv.y + (ar * im + ai * re));
      }
    }
}

template <bool AK, bool BKc>
int launch_zgemm3m_dmma(int m, int n, int k, const double *A, int lda, const double *B, int ldb,
                        double *C, int ldc, double ar, double ai, double br, double bi, double sa,
                        double sb, cudaStream_t s) {
  constexpr size_t SMEM =
      (size_t)Z_STAGES * (z_stage_elems<AK>(Z_BM) + z_stage_elems<BKc>(Z_BN)) * 16;
  auto kern = zgemm3m_dmma_kernel<AK, BKc>;
  B2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM));
  dim3 grid((unsigned)((m + Z_BM - 1) / Z_BM), (unsigned)((n + Z_BN - 1) / Z_BN));
  B2_PROF("zgemm3m_dmma", s);
  kern<<<grid, Z_NT, SMEM, s>>>(m, n, k, reinterpret_cast<const double2 *>(A), lda,
                                reinterpret_cast<const double2 *>(B), ldb,
                                reinterpret_cast<double2 *>(C), ldc, ar, ai, br, bi, sa, sb);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

template <typename T>
__global__ void cscale_kernel(int M, int N, T br, T bi, T *__restrict__ C, int ldc) {
  const long long total = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M), n = (int)(idx / M);
    T *c = C + 2 * ((long long)n * ldc + m);
    const T cr = c[0], ci = c[1];
    c[0] = br * cr - bi * ci;
    c[1] = br * ci + bi * cr;
  }
}

}  // namespace

// ------------------------------------------ large products: 3 real GEMMs --
// Real and imaginary parts of op(X) (R x Cc, element (r, c) at
// X[2*(r*ld + c)] when transposed, else X[2*(c*ld + r)]; imaginary part times
// sgn for conjugation) and their sum, column-major with leading dimension R.
template <typename T>
__global__ void prep3m_kernel(const T *__restrict__ X, int ld, bool trans, T sgn, int R, int Cc,
                              T *__restrict__ outr, T *__restrict__ outi, T *__restrict__ outs) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= R) return;
  for (long long c = blockIdx.y; c < Cc; c += gridDim.y) {
    const T *p = X + 2 * (trans ? r * ld + c : c * ld + r);
    const T re = p[0], im = sgn * p[1];
    const long long o = r + c * (long long)R;
    outr[o] = re;
    outi[o] = im;
    outs[o] = re + im;
  }
}

// C = alpha (P1 - P2 + i (P3 - P1 - P2)) + beta C, beta applied when != 1.
template <typename T>
__global__ void combine3m_kernel(const T *__restrict__ P, long long plane, int M, int N, T ar,
                                 T ai, T br, T bi, T *__restrict__ C, int ldc) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= M) return;
  for (long long n = blockIdx.y; n < N; n += gridDim.y) {
    const long long o = m + n * M;
    const T p1 = P[o], p2 = P[plane + o], p3 = P[2 * plane + o];
    epilogue3m(C, ldc, (int)m, (int)n, p1, p2, p3, ar, ai, br, bi);
  }
}

// Products of at least 2^24 multiply-adds: the three real products run as
// the library's own GEMMs (FP64 DMMA for zgemm3m; 3xTF32 tensor-core SGEMM,
// FP32-class accuracy, for cgemm3m) between one pre-add pass and one
// post-combination pass -- both HBM-bound -- instead of the fused tile kernel,
// whose in-register pre-adds cap it below the plain GEMMs' rate.
template <typename T>
int gemm3m_three_gemms(char ta, char tb, int m, int n, int k, T ar, T ai, T br, T bi,
                       const T *A, int lda, const T *B, int ldb, T *C, int ldc, cudaStream_t s) {
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  const bool tA = !(ta == 'N' || ta == 'n' || ta == 'R' || ta == 'r');
  const bool tB = !(tb == 'N' || tb == 'n' || tb == 'R' || tb == 'r');
  const T sA = (ta == 'C' || ta == 'c' || ta == 'R' || ta == 'r') ? (T)-1 : (T)1;
  const T sB = (tb == 'C' || tb == 'c' || tb == 'R' || tb == 'r') ? (T)-1 : (T)1;
  const long long pa = (long long)m * k, pb = (long long)k * n, pc = (long long)m * n;
  T *W = (T *)workspace(cx, WS_3M, (size_t)(3 * pa + 3 * pb + 3 * pc) * sizeof(T));
  if (!W) return B2_ERR_NOMEM;
  T *Ar = W, *Ai = Ar + pa, *As = Ai + pa;
  T *Br = As + pa, *Bi = Br + pb, *Bs = Bi + pb;
  T *P = Bs + pb;
  {
    B2_PROF("gemm3m_prep", s);
    dim3 ga((unsigned)((m + 255) / 256), (unsigned)(k < 4096 ? k : 4096));
    prep3m_kernel<T><<<ga, 256, 0, s>>>(A, lda, tA, sA, m, k, Ar, Ai, As);
    dim3 gb((unsigned)((k + 255) / 256), (unsigned)(n < 4096 ? n : 4096));
    prep3m_kernel<T><<<gb, 256, 0, s>>>(B, ldb, tB, sB, k, n, Br, Bi, Bs);
    B2_CUDA_TRY(cudaGetLastError());
  }
  // beta = 0 still multiplies the output (reference semantics): start at zero
  B2_CUDA_TRY(cudaMemsetAsync(P, 0, (size_t)(3 * pc) * sizeof(T), s));
  const T *X[3] = {Ar, Ai, As}, *Y[3] = {Br, Bi, Bs};
  for (int t = 0; t < 3; ++t) {
    int st;
    if constexpr (sizeof(T) == 8)
      st = dgemm_fp64('N', 'N', m, n, k, 1.0, X[t], m, Y[t], k, 0.0, P + t * pc, m, s, nullptr);
    else
      st = sgemm_dispatch('N', 'N', m, n, k, 1.0f, X[t], m, Y[t], k, 0.0f, P + t * pc, m,
                          B2_METHOD_TF32X3, s);
    if (st != B2_OK) return st;
  }
  B2_PROF("gemm3m_combine", s);
  dim3 gc((unsigned)((m + 255) / 256), (unsigned)(n < 4096 ? n : 4096));
  combine3m_kernel<T><<<gc, 256, 0, s>>>(P, pc, m, n, ar, ai, br, bi, C, ldc);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

// cgemm3m in ONE tensor-core GEMM launch: the three real products of the 3M
// method run as 3xTF32 on the single-CTA tcgen05 engine in its three-
// accumulator mode -- each work unit is a 128 x 128 tile of C that multiplies
// batch 0 (Br, Ar), 1 (Bi, Ai) and 2 (Br + Bi, Ar + Ai) of the split operands
// into three TMEM accumulators of 128 columns, and the epilogue forms
// Re = P1 - P2, Im = P3 - P1 - P2 and C = alpha (Re + i Im) + beta C from
// them, so P1/P2/P3 never leave the SM.  The pre-adds (and conjugation /
// transposition) and the TF32 big/small splits stay passes in front.
constexpr int C3M_BN = 128, C3M_STAGES = 6;  // 128 x 128 tiles, one accumulator set

struct C3MEpi {
  float *C;
  int ldc;
  int M, N;  // C is M x N; the engine's P runs over N, Q over M
  float ar, ai, br, bi;
  __device__ __forceinline__ void operator()(int p, int q0, const uint32_t (&v0)[32],
                                             const uint32_t (&v1)[32],
                                             const uint32_t (&v2)[32]) const {
    if (p >= N || q0 >= M) return;
    const int nq = min(32, M - q0);
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (j < nq)
        epilogue3m<float>(C, ldc, q0 + j, p, __uint_as_float(v0[j]), __uint_as_float(v1[j]),
                          __uint_as_float(v2[j]), ar, ai, br, bi);
  }
};

int cgemm3m_fused_tc(char ta, char tb, int m, int n, int k, float ar, float ai, float br,
                     float bi, const float *A, int lda, const float *B, int ldb, float *C,
                     int ldc, cudaStream_t s) {
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  const bool tA = !(ta == 'N' || ta == 'n' || ta == 'R' || ta == 'r');
  const bool tB = !(tb == 'N' || tb == 'n' || tb == 'R' || tb == 'r');
  const float sA = (ta == 'C' || ta == 'c' || ta == 'R' || ta == 'r') ? -1.f : 1.f;
  const float sB = (tb == 'C' || tb == 'c' || tb == 'R' || tb == 'r') ? -1.f : 1.f;
  const long long pa = (long long)m * k, pb = (long long)k * n;
  float *W = (float *)workspace(cx, WS_3M, (size_t)(3 * pa + 3 * pb) * sizeof(float));
  if (!W) return B2_ERR_NOMEM;
  float *Ar = W, *Ai = Ar + pa, *As = Ai + pa;
  float *Br = As + pa, *Bi = Br + pb, *Bs = Bi + pb;
  {
    B2_PROF("gemm3m_prep", s);
    dim3 ga((unsigned)((m + 255) / 256), (unsigned)(k < 4096 ? k : 4096));
    prep3m_kernel<float><<<ga, 256, 0, s>>>(A, lda, tA, sA, m, k, Ar, Ai, As);
    dim3 gb((unsigned)((k + 255) / 256), (unsigned)(n < 4096 ? n : 4096));
    prep3m_kernel<float><<<gb, 256, 0, s>>>(B, ldb, tB, sB, k, n, Br, Bi, Bs);
    B2_CUDA_TRY(cudaGetLastError());
  }
  // split planes: Y[t] = rows of op(A) parts (m x [big|small]), X[t] = columns
  // of op(B) parts (n x [big|small]), t = 0, 1, 2 the three products
  const int kp = (int)((k + 31) / 32 * 32);
  const long long ks = 2LL * kp;
  float *Yp = (float *)workspace(cx, WS_SPLIT_Y, (size_t)(3 * m * ks) * sizeof(float));
  float *Xp = (float *)workspace(cx, WS_SPLIT_X, (size_t)(3 * n * ks) * sizeof(float));
  if (!Yp || !Xp) return B2_ERR_NOMEM;
  const float *Ya[3] = {Ar, Ai, As}, *Xb[3] = {Br, Bi, Bs};
  for (int t = 0; t < 3; ++t) {
    int rc = sgemm_split_tf32x3(Ya[t], 1, m, m, k, kp, Yp + t * m * ks, s);
    if (rc == B2_OK) rc = sgemm_split_tf32x3(Xb[t], k, 1, n, k, kp, Xp + t * n * ks, s);
    if (rc != B2_OK) return rc;
  }
  CUtensorMap tmX, tmY;
  int rc = umma::make_kmajor_map(&tmX, umma::KIND_TF32, Xp, ks, n, 3, ks * 4, (long long)n * ks * 4,
                                 umma::BM);
  if (rc == B2_OK)
    rc = umma::make_kmajor_map(&tmY, umma::KIND_TF32, Yp, ks, m, 3, ks * 4, (long long)m * ks * 4,
                               C3M_BN);
  if (rc != B2_OK) return rc;
  // three-term interleave as in the 3xTF32 SGEMM: terms (Bb, Ab), (Bs, Ab), (Bb, As)
  const int seg_kb = kp * 4 / umma::KBLOCK_BYTES;
  C3MEpi epi{C, ldc, m, n, ar, ai, br, bi};
  return umma::launch<umma::KIND_TF32, C3M_BN, C3M_STAGES, C3MEpi, 3>(tmX, tmY, n, m, 3LL * kp, 3, epi,
                                                         cx->sm_count, cx->derr, s,
                                                         "cgemm3m_umma", 0, nullptr, 1, seg_kb,
                                                         0x2u, 0x4u);
}

template <typename T>
int gemm3m_device(char ta, char tb, int m, int n, int k, const T *alpha, const T *A, int lda,
                  const T *B, int ldb, const T *beta, T *C, int ldc, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  const T ar = alpha[0], ai = alpha[1], br = beta[0], bi = beta[1];
  if (k <= 0 || (ar == (T)0 && ai == (T)0)) {
    if (br == (T)1 && bi == (T)0) return B2_OK;
    const long long total = (long long)m * n;
    const int blocks = (int)((total + 255) / 256 > 4096 ? 4096 : (total + 255) / 256);
    B2_PROF("gemm3m_scale", s);
    cscale_kernel<T><<<blocks, 256, 0, s>>>(m, n, br, bi, C, ldc);
    B2_CUDA_TRY(cudaGetLastError());
    return B2_OK;
  }
  if constexpr (sizeof(T) == 8) {
    // complex128: the one-launch DMMA kernel (16-byte aligned operands, the
    // normal case; an odd-aligned pointer takes the other paths) below 2^35
    // multiply-adds, 2048^3 included: the pre-adds, the three products and
    // the combination never leave the SM, and no intermediate planes are
    // allocated (the three-GEMM form needs 3 (m k + k n + m n) doubles of
    // workspace, 302 MB at 2048^3).  It runs 4 % below the three DMMA GEMMs
    // there (36.4 against 38.0 TFLOPS effective; tensor pipe 75 % against 84 %
    // active: the 512-thread fused CTA holds one CTA per SM).  The three
    // GEMMs take over from 2^35: at 4096^3 they run at 41.8 TFLOPS effective
    // against 36.9 for the one launch.  B2_Z3M_FUSED_MAX (multiply-adds)
    // moves the limit.
    static const double fused_max = [] {
      const char *e = getenv("B2_Z3M_FUSED_MAX");
      return e ? atof(e) : 34359738368.0;
    }();
    const bool al16 = (((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) & 15) == 0;
    if (al16 && (double)m * n * k < fused_max) {
      const bool tA = !(ta == 'N' || ta == 'n' || ta == 'R' || ta == 'r');
      const bool tB = !(tb == 'N' || tb == 'n' || tb == 'R' || tb == 'r');
      const double sA = (ta == 'C' || ta == 'c' || ta == 'R' || ta == 'r') ? -1.0 : 1.0;
      const double sB = (tb == 'C' || tb == 'c' || tb == 'R' || tb == 'r') ? -1.0 : 1.0;
      const bool ak = tA, bk = !tB;  // K contiguous in memory
      if (ak && bk)
        return launch_zgemm3m_dmma<true, true>(m, n, k, A, lda, B, ldb, C, ldc, ar, ai, br, bi, sA, sB, s);
      if (ak)
        return launch_zgemm3m_dmma<true, false>(m, n, k, A, lda, B, ldb, C, ldc, ar, ai, br, bi, sA, sB, s);
      if (bk)
        return launch_zgemm3m_dmma<false, true>(m, n, k, A, lda, B, ldb, C, ldc, ar, ai, br, bi, sA, sB, s);
      return launch_zgemm3m_dmma<false, false>(m, n, k, A, lda, B, ldb, C, ldc, ar, ai, br, bi, sA, sB, s);
    }
  }
  if ((double)m * n * k >= 16777216.0) {
    if constexpr (sizeof(T) == 4) {
      // One tensor-core launch (cgemm3m_fused_tc) when B2_C3M_FUSED=1 and its
      // 128 x 128 tiles fill the SMs.  Off by default: at 2048^3 it measured
      // 0.597 ms against 0.541 ms for the three GEMMs (which split K over the
      // SMs and use the CTA pair; 4096^3: 3.15 against 2.07 ms), and its
      // full-K FP32 accumulation gives 2.1e-5 relative error against 2.4e-6.
      static const bool fused_on = [] {
        const char *e = getenv("B2_C3M_FUSED");
        return e && e[0] == '1';
      }();
      Ctx *cx = ctx();
      const long long tiles = (long long)((n + 127) / 128) * ((m + C3M_BN - 1) / C3M_BN);
      if (fused_on && cx && tiles >= cx->sm_count)
        return cgemm3m_fused_tc(ta, tb, m, n, k, ar, ai, br, bi, A, lda, B, ldb, C, ldc, s);
    }
    return gemm3m_three_gemms<T>(ta, tb, m, n, k, ar, ai, br, bi, A, lda, B, ldb, C, ldc, s);
  }
  dim3 grid((m + G_BM - 1) / G_BM, (n + G_BN - 1) / G_BN);
  const int smem = (int)(12 * G_BK * G_LD * sizeof(T));
  if constexpr (sizeof(T) == 8) {
    B2_CUDA_TRY(cudaFuncSetAttribute(zgemm3m_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    B2_PROF("zgemm3m_fused", s);
    zgemm3m_kernel<<<grid, 256, smem, s>>>(m, n, k, A, lda, B, ldb, C, ldc, ar, ai, br, bi, ta, tb);
  } else {
    B2_CUDA_TRY(cudaFuncSetAttribute(cgemm3m_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    B2_PROF("cgemm3m_fused", s);
    cgemm3m_kernel<<<grid, 256, smem, s>>>(m, n, k, A, lda, B, ldb, C, ldc, ar, ai, br, bi, ta, tb);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

template int gemm3m_device<double>(char, char, int, int, int, const double *, const double *, int,
                                   const double *, int, const double *, double *, int,
                                   cudaStream_t);
template int gemm3m_device<float>(char, char, int, int, int, const float *, const float *, int,
                                  const float *, int, const float *, float *, int, cudaStream_t);

}  // namespace b2
