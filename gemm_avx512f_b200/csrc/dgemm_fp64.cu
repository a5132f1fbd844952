// dgemm_fp64.cu -- plain FP64 GEMM on the sm_100 FP64 tensor-core path.
//
// Replaces the reference's cache-blocked AVX-512 DGEMM (src/gemm_driver.c:116-195
// driving the 24x8 register tile of src/kernel/gemm_kernel.S:822-1213, and the
// OpenBLAS-like 16x2 / 4x8 / 8x8 kernels).  tcgen05 has no f64 kind, so the
// FP64 tensor path on sm_100 is the warp-level DMMA instruction
// mma.sync.aligned.m16n8k{4,8,16}.row.col.f64 with accumulators in registers.
//
// Design:
//  * CTA tile BM x BN (128x128 / 128x64 / 64x64), warp tile 64x32 or 32x32.
//  * op(A)/op(B) tiles streamed global->shared with cp.async (16 B when the
//    leading dimension and base allow it, else 8 B) through a STAGES-deep ring;
//    the reference's packing (src/gemm_copy.c) disappears: the smem tile keeps
//    the global orientation, padded so every DMMA fragment load is
//    bank-conflict free for both orientations (+4 doubles per row).
//  * alpha/beta are applied once in the epilogue (the reference folds alpha
//    into packed B, src/gemm_copy.c:64, and pre-scales C, :131).
//  * Optional split-K: each z-slice writes an FP64 partial into workspace and
//    a reduction kernel adds them in slice order (deterministic) and applies
//    alpha/beta.  Measured on B200 against an in-kernel fixup (the tile's last
//    slice to arrive adds the partials): the separate reduction is faster on
//    every shape tried, 14 us against 66 us at 128x128x1024 with 8 slices and
//    83 us against 118 us at 1024^3 with 4.
#include "b2_internal.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace {

template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void *src, int src_bytes) {
  if constexpr (BYTES == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                 "r"(src_bytes));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                 "r"(src_bytes));
  }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Load an OUTER x BK operand tile.  Element (o, k) of the operand lives at
// g[o*ld + k] when KCONT (k contiguous in memory) else g[k*ld + o].
// Shared layout: KCONT -> [o][BK+4], else [k][OUTER+4].
template <int OUTER, int BK, bool KCONT, int VEC, int NT>
__device__ __forceinline__ void load_tile(uint32_t sbase, const double *__restrict__ g, int ld,
                                          int o0, int k0, int olim, int klim, int tid) {
  if constexpr (KCONT) {
    constexpr int CPR = BK / VEC;
    constexpr int TOTAL = OUTER * CPR;
    static_assert(TOTAL % NT == 0, "tile/thread mismatch");
#pragma unroll
    for (int i = 0; i < TOTAL / NT; ++i) {
      const int c = tid + i * NT;
      const int o = c / CPR, kc = (c % CPR) * VEC;
      const int go = o0 + o, gk = k0 + kc;
      int valid = (go < olim) ? min(VEC, klim - gk) : 0;
      valid = valid < 0 ? 0 : valid;
      const double *src = valid ? g + (size_t)go * ld + gk : g;
      cp_async<VEC * 8>(sbase + (uint32_t)(o * (BK + 4) + kc) * 8u, src, valid * 8);
    }
  } else {
    constexpr int CPR = OUTER / VEC;
    constexpr int TOTAL = BK * CPR;
    static_assert(TOTAL % NT == 0, "tile/thread mismatch");
#pragma unroll
    for (int i = 0; i < TOTAL / NT; ++i) {
      const int c = tid + i * NT;
      const int kr = c / CPR, oc = (c % CPR) * VEC;
      const int go = o0 + oc, gk = k0 + kr;
      int valid = (gk < klim) ? min(VEC, olim - go) : 0;
      valid = valid < 0 ? 0 : valid;
      const double *src = valid ? g + (size_t)gk * ld + go : g;
      cp_async<VEC * 8>(sbase + (uint32_t)(kr * (OUTER + 4) + oc) * 8u, src, valid * 8);
    }
  }
}

template <int MMAK>
__device__ __forceinline__ void dmma(double (&c)[4], const double *a, const double *b) {
  if constexpr (MMAK == 4) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(b[0]));
  } else if constexpr (MMAK == 8) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
  } else {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
          "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
  }
}

// A_KCONT = transA (op(A)(m,k) = A[m*lda+k]); B_KCONT = !transB (op(B)(k,n) = B[n*ldb+k]).
// Output: when P != nullptr the raw product of this CTA's K range is written to
// P + z*ldp*N (split-K partial); otherwise C = alpha*acc + beta*C (beta==1: C += alpha*acc).
template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MMAK, bool A_KCONT,
          bool B_KCONT, int VEC>
__global__ void __launch_bounds__(WM *WN * 32, 1)
    dgemm_dmma_kernel(int M, int N, int K, int kchunk, double alpha,
                      const double *__restrict__ A, int lda, const double *__restrict__ B,
                      int ldb, double beta, double *__restrict__ C, int ldc,
                      double *__restrict__ P, int ldp) {
  constexpr int NT = WM * WN * 32;
  constexpr int TM = BM / WM, TN = BN / WN;  // warp tile
  constexpr int MT = TM / 16, NTL = TN / 8;
  constexpr int A_ST = A_KCONT ? BM * (BK + 4) : BK * (BM + 4);
  constexpr int B_ST = B_KCONT ? BN * (BK + 4) : BK * (BN + 4);
  static_assert(TM % 16 == 0 && TN % 8 == 0 && BK % MMAK == 0, "bad tile");

  extern __shared__ __align__(16) double smem[];
  double *sA = smem;
  double *sB = smem + STAGES * A_ST;
  const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA);
  const uint32_t sB_u = (uint32_t)__cvta_generic_to_shared(sB);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp / WN) * TM, wn0 = (warp % WN) * TN;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kbeg = blockIdx.z * kchunk;
  const int kend = min(K, kbeg + kchunk);
  const int KT = (kend - kbeg + BK - 1) / BK;

  double acc[MT][NTL][4];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NTL; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

  auto load_stage = [&](int st, int kt) {
    const int k0 = kbeg + kt * BK;
    load_tile<BM, BK, A_KCONT, VEC, NT>(sA_u + st * A_ST * 8, A, lda, m0, k0, M, kend, tid);
    load_tile<BN, BK, B_KCONT, VEC, NT>(sB_u + st * B_ST * 8, B, ldb, n0, k0, N, kend, tid);
  };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_stage(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int kn = kt + STAGES - 1;
      if (kn < KT) load_stage(kn % STAGES, kn);
      cp_async_commit();
    }
    const double *As = sA + (kt % STAGES) * A_ST;
    const double *Bs = sB + (kt % STAGES) * B_ST;
#pragma unroll
    for (int kk = 0; kk < BK; kk += MMAK) {
      double af[MT][MMAK / 2];
      double bf[NTL][MMAK / 4];
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int v1 = 0; v1 < MMAK / 4; ++v1)
#pragma unroll
          for (int v0 = 0; v0 < 2; ++v0) {
            const int m = wm0 + i * 16 + g + 8 * v0, k = kk + t + 4 * v1;
            af[i][v0 + 2 * v1] = A_KCONT ? As[m * (BK + 4) + k] : As[k * (BM + 4) + m];
          }
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int v = 0; v < MMAK / 4; ++v) {
          const int n = wn0 + j * 8 + g, k = kk + t + 4 * v;
          bf[j][v] = B_KCONT ? Bs[n * (BK + 4) + k] : Bs[k * (BN + 4) + n];
        }
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NTL; ++j) dmma<MMAK>(acc[i][j], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();

  // Epilogue.  Fragment (i, j, v): row g + 8*(v>>1), column 2t + (v&1).
  if (P != nullptr) {
    double *Pz = P + (size_t)blockIdx.z * ldp * N;
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int m = m0 + wm0 + i * 16 + g + 8 * (v >> 1);
          const int n = n0 + wn0 + j * 8 + 2 * t + (v & 1);
          if (m < M && n < N) Pz[(size_t)n * ldp + m] = acc[i][j][v];
        }
    return;
  }
  const bool beta_one = (beta == 1.0);
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NTL; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int m = m0 + wm0 + i * 16 + g + 8 * (v >> 1);
        const int n = n0 + wn0 + j * 8 + 2 * t + (v & 1);
        if (m < M && n < N) {
          double *p = C + (size_t)n * ldc + m;
          const double c_old = *p;
          *p = beta_one ? fma(alpha, acc[i][j][v], c_old) : fma(alpha, acc[i][j][v], beta * c_old);
        }
      }
}

__global__ void splitk_reduce_kernel(int M, int N, int splits, const double *__restrict__ P,
                                     int ldp, double alpha, double beta, double *__restrict__ C,
                                     int ldc) {
  const size_t total = (size_t)M * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M), n = (int)(idx / M);
    double s = 0.0;
    for (int z = 0; z < splits; ++z) s += P[(size_t)z * ldp * N + (size_t)n * ldp + m];
    double *p = C + (size_t)n * ldc + m;
    *p = (beta == 1.0) ? fma(alpha, s, *p) : fma(alpha, s, beta * *p);
  }
}

template <typename T>
__global__ void scale_kernel(int M, int N, T beta, T *__restrict__ C, int ldc) {
  const size_t total = (size_t)M * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M), n = (int)(idx / M);
    C[(size_t)n * ldc + m] *= beta;
  }
}

struct LaunchArgs {
  int M, N, K, kchunk;
  double alpha;
  const double *A;
  int lda;
  const double *B;
  int ldb;
  double beta;
  double *C;
  int ldc;
  double *P;
  int ldp;
  int splits;
};

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MMAK, bool AK, bool BKc,
          int VEC>
cudaError_t launch_one(const LaunchArgs &a, cudaStream_t s) {
  constexpr int A_ST = AK ? BM * (BK + 4) : BK * (BM + 4);
  constexpr int B_ST = BKc ? BN * (BK + 4) : BK * (BN + 4);
  constexpr size_t SMEM = (size_t)STAGES * (A_ST + B_ST) * sizeof(double);
  auto kern = dgemm_dmma_kernel<BM, BN, BK, WM, WN, STAGES, MMAK, AK, BKc, VEC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid((a.M + BM - 1) / BM, (a.N + BN - 1) / BN, a.splits);
  B2_PROF("dgemm_dmma", s);
  kern<<<grid, WM * WN * 32, SMEM, s>>>(a.M, a.N, a.K, a.kchunk, a.alpha, a.A, a.lda, a.B, a.ldb,
                                        a.beta, a.C, a.ldc, a.P, a.ldp);
  return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, int STAGES, int MMAK, int VEC>
cudaError_t launch_layout(bool ak, bool bk, const LaunchArgs &a, cudaStream_t s) {
  if (ak && bk) return launch_one<BM, BN, 16, WM, WN, STAGES, MMAK, true, true, VEC>(a, s);
  if (ak && !bk) return launch_one<BM, BN, 16, WM, WN, STAGES, MMAK, true, false, VEC>(a, s);
  if (!ak && bk) return launch_one<BM, BN, 16, WM, WN, STAGES, MMAK, false, true, VEC>(a, s);
  return launch_one<BM, BN, 16, WM, WN, STAGES, MMAK, false, false, VEC>(a, s);
}

template <int MMAK, int VEC>
cudaError_t launch_tile(int tile, bool ak, bool bk, const LaunchArgs &a, cudaStream_t s) {
  switch (tile) {
    case 0: return launch_layout<128, 128, 2, 4, 4, MMAK, VEC>(ak, bk, a, s);
    case 1: return launch_layout<128, 64, 2, 2, 4, MMAK, VEC>(ak, bk, a, s);
    default: return launch_layout<64, 64, 2, 2, 4, MMAK, VEC>(ak, bk, a, s);
  }
}

inline bool is_notrans(char c) { return c == 'N' || c == 'n'; }

}  // namespace

Fp64Cfg fp64_default_cfg(int m, int n, int k, int sm_count) {
  // Measured on B200: the 64x64 tile with two CTAs per SM is best from 1024^3
  // to 8192^3 (31.5 TF at 4096^3); in the exhaustive sweep over 22000 shapes
  // with M, N, K in [16, 1024] split-K 8 on that tile was the best single
  // choice, so grids below ~1024 tiles split K up to 8 ways as long as every
  // slice keeps >= 8 of K (2.6 % mean regret against the per-shape best of
  // all 36 FP64 configurations; 32 % when slices had to keep >= 32: small-K
  // products are latency-bound and gain from any split).  The split also
  // stops at 1024 work units (tiles x slices): 1024^3 runs in 83 us with 4
  // slices (25.9 TFLOPS) against 87 us unsplit and 90 us with 8; the
  // partials' extra reduction traffic outweighs the finer wave fit.
  (void)sm_count;
  Fp64Cfg c;
  c.tile = 2;
  c.mmak = 8;
  const long t64 = (long)((m + 63) / 64) * ((n + 63) / 64);
  int sk = 1;
  if (t64 < 1024)
    while (sk < 8 && k / (2 * sk) >= 8 && t64 * sk * 2 <= 1024) sk *= 2;
  c.split_k = sk;
  return c;
}

Fp64Cfg &fp64_override_cfg() {
  static thread_local Fp64Cfg cfg;
  return cfg;
}

int scale_matrix_d(int m, int n, double beta, double *C, int ldc, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  const size_t total = (size_t)m * n;
  const int blocks = (int)((total + 255) / 256 > 8192 ? 8192 : (total + 255) / 256);
  B2_PROF("scale_matrix", s);
  scale_kernel<double><<<blocks, 256, 0, s>>>(m, n, beta, C, ldc);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int scale_matrix_s(int m, int n, float beta, float *C, int ldc, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  const size_t total = (size_t)m * n;
  const int blocks = (int)((total + 255) / 256 > 8192 ? 8192 : (total + 255) / 256);
  B2_PROF("scale_matrix", s);
  scale_kernel<float><<<blocks, 256, 0, s>>>(m, n, beta, C, ldc);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int dgemm_fp64(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
               const double *B, int ldb, double beta, double *C, int ldc, cudaStream_t s,
               const Fp64Cfg *cfg_in) {
  if (m <= 0 || n <= 0) return B2_OK;
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  if (k <= 0 || alpha == 0.0) return beta == 1.0 ? B2_OK : scale_matrix_d(m, n, beta, C, ldc, s);
  Fp64Cfg cfg = cfg_in            ? *cfg_in
                : cx->fp64_override ? fp64_override_cfg()
                                    : fp64_default_cfg(m, n, k, cx->sm_count);
  const bool ak = !is_notrans(ta);  // transposed A: k contiguous
  const bool bk = is_notrans(tb);   // plain B: k contiguous
  const bool vec2 = (lda % 2 == 0) && (ldb % 2 == 0) && (((uintptr_t)A & 15) == 0) &&
                    (((uintptr_t)B & 15) == 0);
  LaunchArgs a{m, n, k, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr, 0, 1};
  int splits = cfg.split_k < 1 ? 1 : cfg.split_k;
  if (splits > 1) {
    int chunk = (k + splits - 1) / splits;
    chunk = (chunk + 15) / 16 * 16;
    splits = (k + chunk - 1) / chunk;
    a.kchunk = chunk;
    a.splits = splits;
    if (splits > 1) {
      const size_t bytes = (size_t)splits * m * n * sizeof(double);
      double *P = (double *)workspace(cx, WS_MISC, bytes);
      if (!P) return B2_ERR_NOMEM;
      a.P = P;
      a.ldp = m;
    } else {
      a.kchunk = k;
    }
  }
  cudaError_t e;
  const int mk = cfg.mmak;
  if (vec2) {
    e = mk == 16 ? launch_tile<16, 2>(cfg.tile, ak, bk, a, s)
        : mk == 8 ? launch_tile<8, 2>(cfg.tile, ak, bk, a, s)
                  : launch_tile<4, 2>(cfg.tile, ak, bk, a, s);
  } else {
    e = mk == 16 ? launch_tile<16, 1>(cfg.tile, ak, bk, a, s)
        : mk == 8 ? launch_tile<8, 1>(cfg.tile, ak, bk, a, s)
                  : launch_tile<4, 1>(cfg.tile, ak, bk, a, s);
  }
  if (e != cudaSuccess) return cuda_fail(e, "dgemm_dmma_kernel");
  if (a.P) {
    const size_t total = (size_t)m * n;
    const int blocks = (int)((total + 255) / 256 > 4096 ? 4096 : (total + 255) / 256);
    B2_PROF("dgemm_splitk_reduce", s);
    splitk_reduce_kernel<<<blocks, 256, 0, s>>>(m, n, a.splits, a.P, a.ldp, alpha, beta, C, ldc);
    B2_CUDA_TRY(cudaGetLastError());
  }
  return B2_OK;
}

}  // namespace b2

extern "C" int b2_set_fp64_config(int tile, int mmak, int split_k) {
  b2::Ctx *c = b2::ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  if (tile < 0) {
    c->fp64_override = 0;
    return B2_OK;
  }
  if (tile > 2 || !(mmak == 4 || mmak == 8 || mmak == 16) || split_k < 1 || split_k > 64)
    return B2_ERR_ARG;
  b2::Fp64Cfg &o = b2::fp64_override_cfg();
  o.tile = tile;
  o.mmak = mmak;
  o.split_k = split_k;
  c->fp64_override = 1;
  return B2_OK;
}
