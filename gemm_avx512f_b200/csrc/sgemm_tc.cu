// sgemm_tc.cu -- SGEMM on the tcgen05 tensor cores with FP32 accumulation.
//
// Replaces the reference's AVX-512 SGEMM (src/gemm_driver.c:116 built without
// -DDOUBLE, OpenBLAS-like_implementation/sgemm.c:366-412) by three tensor-core
// forms, all with FP32 accumulators in TMEM:
//   TF32    1 product:  C = tf32(A) tf32(B)                     (kind::tf32)
//   TF32X3  3 products: A = Ab + As, B = Bb + Bs (each TF32),
//                       C = Ab Bb + Ab Bs + As Bb                (kind::tf32)
//   BF16X3  3 products: A = Ah + Al, B = Bh + Bl (each BF16),
//                       C = Ah Bh + Ah Bl + Al Bh                (kind::f16, bf16 in)
// Every method is ONE GEMM over K' = terms * Kp on the engine in umma.cuh;
// the split/convert kernel is the only extra pass.  For three terms each
// operand stores two segments, [big | small], each padded with zeros to a
// 128-byte K block, and the engine's three-term interleave reads K' block j
// as term j % 3 of K block j / 3: (Bb, Ab), (Bs, Ab), (Bb, As).  The big part
// used by two terms is written once and read from DRAM once (its second load
// is an L2 hit a few K' blocks later).
#include <cuda_bf16.h>

#include "b2_methods.cuh"
#include "b2_profile.cuh"
#include "umma.cuh"

namespace b2 {
namespace {

__device__ __forceinline__ float tf32_round(float x) {  // round to nearest, ties away
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Writes `terms` K-segments per row of the operand viewed as R x K (element
// (r,k) at X[r*sr + k*sk]) into out[r][terms*kp] (elements of type T).
// pattern: which split part each segment holds (0 = big/high, 1 = small/low).
// vec (checked on the host: X 16-byte aligned and the strided dimension a
// multiple of 4 elements, unit stride along the other): 16-byte loads of 4
// consecutive rows (ROWCONT) or 4 consecutive k; otherwise scalar loads.
template <typename T, bool ROWCONT>
__global__ void __launch_bounds__(256)
    split_kernel(const float *__restrict__ X, long long sr, long long sk, int R, int K, int kp,
                 int terms, unsigned pattern, T *__restrict__ out, int vec) {
  __shared__ float tile[32][65];
  const int k0 = blockIdx.x * 64, r0 = blockIdx.y * 32;
  const int tid = threadIdx.x;
  if (vec) {
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int idx = tid + 256 * e;
      float v[4] = {0.f, 0.f, 0.f, 0.f};
      if (ROWCONT) {  // 32 rows x 64 k: 8 float4 per k column
        const int kk = idx >> 3, rr = (idx & 7) * 4;
        const int r = r0 + rr, k = k0 + kk;
        if (k < K) {
          const float *src = X + r + (long long)k * sk;
          if (r + 3 < R) {
            const float4 q = __ldg(reinterpret_cast<const float4 *>(src));
            v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (r + j < R) v[j] = __ldg(src + j);
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) tile[rr + j][kk] = v[j];
      } else {  // 32 rows x 64 k: 16 float4 per row
        const int rr = idx >> 4, kk = (idx & 15) * 4;
        const int r = r0 + rr, k = k0 + kk;
        if (r < R) {
          const float *src = X + (long long)r * sr + k;
          if (k + 3 < K) {
            const float4 q = __ldg(reinterpret_cast<const float4 *>(src));
            v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (k + j < K) v[j] = __ldg(src + j);
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) tile[rr][kk + j] = v[j];
      }
    }
  } else {
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int idx = tid + 256 * e;
      int rr, kk;
      if (ROWCONT) { rr = idx & 31; kk = idx >> 5; } else { kk = idx & 63; rr = idx >> 6; }
      const int r = r0 + rr, k = k0 + kk;
      float v = 0.f;
      if (r < R && k < K) v = __ldg(X + (long long)r * sr + (long long)k * sk);
      tile[rr][kk] = v;
    }
  }
  __syncthreads();
  const int rr = tid >> 3, q = tid & 7;
  const int r = r0 + rr;
  if (r >= R) return;
  T *row = out + (long long)r * terms * kp;
  // 16-byte stores of 16-byte groups of consecutive k: FP32 writes groups
  // k0 + 4q and k0 + 32 + 4q (the second only where kp reaches it; kp is a
  // multiple of 32), so each store instruction covers whole 128-byte lines
  // of a row; BF16 writes one group of 8 at k0 + 8q (kp is a multiple of 64).
  // Pad columns [K, kp) are written as zeros.
  constexpr int GW = sizeof(T) == 4 ? 4 : 8;   // elements per 16-byte group
  constexpr int NG = sizeof(T) == 4 ? 2 : 1;   // groups per thread
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    const int kl = (sizeof(T) == 4) ? g * 32 + 4 * q : 8 * q;  // offset within the 64-k tile
    if (k0 + kl >= kp) break;
    T big[GW], small[GW];
#pragma unroll
    for (int j = 0; j < GW; ++j) {
      const float v = (k0 + kl + j < K) ? tile[rr][kl + j] : 0.f;
      if constexpr (sizeof(T) == 4) {
        const float bv = tf32_round(v);
        big[j] = bv;
        small[j] = tf32_round(v - bv);
      } else {
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        big[j] = h;
        small[j] = __float2bfloat16_rn(v - __bfloat162float(h));
      }
    }
    for (int t = 0; t < terms; ++t) {
      const T *src = ((pattern >> t) & 1u) ? small : big;
      T *dst = row + (long long)t * kp + k0 + kl;
      if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(dst) = make_float4(src[0], src[1], src[2], src[3]);
      } else {
        uint4 p;
        p.x = (uint32_t)__bfloat16_as_ushort(src[0]) | ((uint32_t)__bfloat16_as_ushort(src[1]) << 16);
        p.y = (uint32_t)__bfloat16_as_ushort(src[2]) | ((uint32_t)__bfloat16_as_ushort(src[3]) << 16);
        p.z = (uint32_t)__bfloat16_as_ushort(src[4]) | ((uint32_t)__bfloat16_as_ushort(src[5]) << 16);
        p.w = (uint32_t)__bfloat16_as_ushort(src[6]) | ((uint32_t)__bfloat16_as_ushort(src[7]) << 16);
        *reinterpret_cast<uint4 *>(dst) = p;
      }
    }
  }
}

// FP32 epilogue: lane p = column n of C, columns q = rows m (contiguous in C).
struct F32Epi {
  float *C;
  int ldc;
  int M, N;
  float alpha, beta;
  __device__ __forceinline__ void operator()(int, int p, int q0, const uint32_t (&v)[32]) const {
    if (p >= N || q0 >= M) return;
    float *col = C + (long long)p * ldc + q0;
    const int nq = min(32, M - q0);
    const bool one = (beta == 1.f);
    if (nq == 32 && ((((uintptr_t)col) & 15) == 0)) {
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        float4 c = reinterpret_cast<float4 *>(col)[g];
        const float a0 = __uint_as_float(v[4 * g]), a1 = __uint_as_float(v[4 * g + 1]);
        const float a2 = __uint_as_float(v[4 * g + 2]), a3 = __uint_as_float(v[4 * g + 3]);
        c.x = one ? fmaf(alpha, a0, c.x) : fmaf(alpha, a0, beta * c.x);
        c.y = one ? fmaf(alpha, a1, c.y) : fmaf(alpha, a1, beta * c.y);
        c.z = one ? fmaf(alpha, a2, c.z) : fmaf(alpha, a2, beta * c.z);
        c.w = one ? fmaf(alpha, a3, c.w) : fmaf(alpha, a3, beta * c.w);
        reinterpret_cast<float4 *>(col)[g] = c;
      }
    } else {
      for (int j = 0; j < nq; ++j) {
        const float a = __uint_as_float(v[j]);
        col[j] = one ? fmaf(alpha, a, col[j]) : fmaf(alpha, a, beta * col[j]);
      }
    }
  }
};

// Split-K epilogue: the raw FP32 partial of K range ks (the engine's batch
// index) to W[ks][n][ldw]; sgemm_splitk_reduce_kernel adds the ranges in a
// fixed order.
struct F32PartialEpi {
  float *W;
  long long plane;
  int ldw;
  int M, N;
  __device__ __forceinline__ void operator()(int ks, int p, int q0, const uint32_t (&v)[32]) const {
    if (p >= N || q0 >= M) return;
    float4 *dst = reinterpret_cast<float4 *>(W + ks * plane + (long long)p * ldw + q0);
#pragma unroll
    for (int g = 0; g < 8; ++g)
      dst[g] = make_float4(__uint_as_float(v[4 * g]), __uint_as_float(v[4 * g + 1]),
                           __uint_as_float(v[4 * g + 2]), __uint_as_float(v[4 * g + 3]));
  }
};

// C(m, n) = alpha * sum_ks W[ks][n][m] + beta C (beta != 1 multiplies), the
// partials summed in FP64 in K order and rounded once.
__global__ void sgemm_splitk_reduce_kernel(const float *__restrict__ W, long long plane, int ldw,
                                           int S, int M, int N, float alpha, float beta,
                                           float *__restrict__ C, int ldc) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  for (int n = blockIdx.y; n < N; n += gridDim.y) {
    double acc = 0.0;
    for (int ks = 0; ks < S; ++ks) acc += (double)W[ks * plane + (long long)n * ldw + m];
    float *c = C + (long long)n * ldc + m;
    const float a = (float)acc;
    *c = (beta == 1.f) ? fmaf(alpha, a, *c) : fmaf(alpha, a, beta * *c);
  }
}

// K ranges for a product of `tiles` output tiles and `kblocks` K blocks: 1
// when the tiles already fill the SMs, else the count (at most 16, >= 8 K
// blocks per range) that best fills whole waves of `sms` CTAs.
int choose_ksplit(long long tiles, int kblocks, int sms) {
  if (tiles >= sms) return 1;
  int best = 1;
  double best_eff = (double)tiles / sms;
  for (int S = 2; S <= 16 && S * 8 <= kblocks; ++S) {
    const long long units = tiles * S;
    const long long waves = (units + sms - 1) / sms;
    const double eff = (double)units / (double)(waves * sms);
    if (eff > best_eff + 0.02) {
      best_eff = eff;
      best = S;
    }
  }
  return best;
}

inline long long round_up(long long x, long long a) { return (x + a - 1) / a * a; }

template <typename T>
int run_split(const float *Xp, long long sr, long long sk, int R, int K, int kp, int terms,
              unsigned pattern, T *out, cudaStream_t s) {
  dim3 grid((kp + 63) / 64, (R + 31) / 32);
  B2_PROF("sgemm_split", s);
  const bool aligned = ((uintptr_t)Xp & 15) == 0;
  if (sr == 1) {
    const int vec = aligned && (sk % 4 == 0);
    split_kernel<T, true><<<grid, 256, 0, s>>>(Xp, sr, sk, R, K, kp, terms, pattern, out, vec);
  } else {
    const int vec = aligned && sk == 1 && (sr % 4 == 0);
    split_kernel<T, false><<<grid, 256, 0, s>>>(Xp, sr, sk, R, K, kp, terms, pattern, out, vec);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

}  // namespace

int sgemm_split_tf32x3(const float *X, long long sr, long long sk, int R, int K, int kp,
                       float *out, cudaStream_t s) {
  return run_split<float>(X, sr, sk, R, K, kp, 2, 0x2u, out, s);
}

// Tensor-core engine of an SGEMM call: 0 = single CTA, 128 x 256 tile, 4
// stages; 1 = single CTA, 128 x 128 tile, 6 stages; 2 = CTA pair, 256 x 256
// tile, 6 stages.  split: K ranges (0 = chosen from the tile count).
int sgemm_tensor_cfg(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                     const float *B, int ldb, float beta, float *C, int ldc, int method,
                     const SgCfg &cfg, cudaStream_t s);

// Without selector weights: on the exhaustive sweep of 11000 shapes with M, N,
// K in [16, 1024] (B200) the 128 x 128 engine with 8 K ranges is the best
// single configuration of every method (mean regret 2.6 % TF32, 2.0 % TF32x3,
// 2.3 % BF16x3 against the per-shape best).  Larger products run on the CTA
// pair with the wave-fitting split: at 4096^3 and 8192^3 it is the fastest
// engine of every method (8192^3: TF32 688, TF32x3 267, BF16x3 463 TFLOPS,
// against 622 / 220 / 366 for the single-CTA 128 x 256 engine).
SgCfg sgemm_default_cfg(int m, int n, int k, int method) {
  (void)method;
  if (m <= 1024 && n <= 1024 && k <= 1024) return SgCfg{1, 8};
  return SgCfg{2, 0};
}

int sgemm_tensor(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                 const float *B, int ldb, float beta, float *C, int ldc, int method,
                 cudaStream_t s) {
  return sgemm_tensor_cfg(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, method,
                          sgemm_pick_cfg(ta, tb, m, n, k, beta == 0.f, method), s);
}

int sgemm_tensor_cfg(char ta, char tb, int m, int n, int k, float alpha, const float *A, int lda,
                     const float *B, int ldb, float beta, float *C, int ldc, int method,
                     const SgCfg &cfg, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B2_OK;
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  if (k <= 0 || alpha == 0.f) return beta == 1.f ? B2_OK : scale_matrix_s(m, n, beta, C, ldc, s);
  const bool tA = !(ta == 'N' || ta == 'n');
  const bool tB = !(tb == 'N' || tb == 'n');
  const long long asr = tA ? lda : 1, ask = tA ? 1 : lda;   // op(A) rows m
  const long long bsr = tB ? 1 : ldb, bsk = tB ? ldb : 1;   // op(B) columns n
  const bool bf16 = (method == B2_METHOD_BF16X3);
  const int terms = (method == B2_METHOD_TF32) ? 1 : 3;
  const int esz = bf16 ? 2 : 4;
  const int kp = (int)round_up(k, 128 / esz);
  const long long kt = (long long)terms * kp;               // K' of the one GEMM
  const int segs = terms == 3 ? 2 : 1;                      // stored segments per row
  const long long ks_ = (long long)segs * kp;
  void *Yp = workspace(cx, WS_SPLIT_Y, (size_t)m * ks_ * esz);
  void *Xp = workspace(cx, WS_SPLIT_X, (size_t)n * ks_ * esz);
  if (!Yp || !Xp) return B2_ERR_NOMEM;
  // stored segments: [big] or [big, small]; terms read (Bb, Ab), (Bs, Ab), (Bb, As)
  const unsigned pat = 0x2u;                      // segment 1 holds the small part
  const unsigned segX = 0x2u, segY = 0x4u;        // term -> segment, B side / A side
  int rc;
  if (bf16) {
    rc = run_split<__nv_bfloat16>(A, asr, ask, m, k, kp, segs, pat, (__nv_bfloat16 *)Yp, s);
    if (rc == B2_OK)
      rc = run_split<__nv_bfloat16>(B, bsr, bsk, n, k, kp, segs, pat, (__nv_bfloat16 *)Xp, s);
  } else {
    rc = run_split<float>(A, asr, ask, m, k, kp, segs, pat, (float *)Yp, s);
    if (rc == B2_OK) rc = run_split<float>(B, bsr, bsk, n, k, kp, segs, pat, (float *)Xp, s);
  }
  if (rc != B2_OK) return rc;
  const int kind = bf16 ? umma::KIND_BF16 : umma::KIND_TF32;
  const int eng = (cfg.engine >= 0 && cfg.engine <= 2) ? cfg.engine : 0;
  // tile: X rows (n side) per tile x Y rows (m side) per tile; TMA boxes per CTA
  const int tile_p = eng == 2 ? 256 : umma::BM, tile_q = eng == 1 ? 128 : 256;
  const int ybox = eng == 0 ? 256 : 128;
  CUtensorMap tmX, tmY;
  rc = umma::make_kmajor_map(&tmX, kind, Xp, ks_, n, 1, ks_ * esz, (long long)n * ks_ * esz,
                             umma::BM);
  if (rc == B2_OK)
    rc = umma::make_kmajor_map(&tmY, kind, Yp, ks_, m, 1, ks_ * esz, (long long)m * ks_ * esz, ybox);
  if (rc != B2_OK) return rc;
  const int seg_kb = terms == 3 ? (int)((long long)kp * esz / umma::KBLOCK_BYTES) : 0;
  const long long tiles = ((n + tile_p - 1) / tile_p) * (long long)((m + tile_q - 1) / tile_q);
  const int kblocks = (int)((kt * esz + umma::KBLOCK_BYTES - 1) / umma::KBLOCK_BYTES);
  const int slots = eng == 2 ? cx->sm_count / 2 : cx->sm_count;
  int S = cfg.split > 0 ? cfg.split : choose_ksplit(tiles, kblocks, slots);
  if (S > kblocks) S = kblocks > 0 ? kblocks : 1;
  if (S > 1) {
    // the engine may merge ranges; size W for S and pass the count it uses
    const int kbps = (kblocks + S - 1) / S;
    S = (kblocks + kbps - 1) / kbps;
  }
  auto run = [&](auto &&epi) -> int {
    const char *nm = bf16 ? "sgemm_umma_bf16" : "sgemm_umma_tf32";
    if (eng == 2)
      return bf16 ? umma::launch_pair<umma::KIND_BF16, 256, 6>(tmX, tmY, n, m, kt, 1, epi,
                                                               cx->device, cx->derr, s, nm,
                                                               nullptr, S, seg_kb, segX, segY)
                  : umma::launch_pair<umma::KIND_TF32, 256, 6>(tmX, tmY, n, m, kt, 1, epi,
                                                               cx->device, cx->derr, s, nm,
                                                               nullptr, S, seg_kb, segX, segY);
    if (eng == 1)
      return bf16 ? umma::launch<umma::KIND_BF16, 128, 6>(tmX, tmY, n, m, kt, 1, epi,
                                                          cx->sm_count, cx->derr, s, nm, 0,
                                                          nullptr, S, seg_kb, segX, segY)
                  : umma::launch<umma::KIND_TF32, 128, 6>(tmX, tmY, n, m, kt, 1, epi,
                                                          cx->sm_count, cx->derr, s, nm, 0,
                                                          nullptr, S, seg_kb, segX, segY);
    return bf16 ? umma::launch<umma::KIND_BF16, 256, 4>(tmX, tmY, n, m, kt, 1, epi, cx->sm_count,
                                                        cx->derr, s, nm, 0, nullptr, S, seg_kb,
                                                        segX, segY)
                : umma::launch<umma::KIND_TF32, 256, 4>(tmX, tmY, n, m, kt, 1, epi, cx->sm_count,
                                                        cx->derr, s, nm, 0, nullptr, S, seg_kb,
                                                        segX, segY);
  };
  if (S == 1) {
    F32Epi epi{C, ldc, m, n, alpha, beta};
    return run(epi);
  }
  // Split-K: S partial products of K ranges, then one fixed-order reduction.
  const int ldw = (int)round_up(m, 256);  // whole 256-column tiles stay in bounds
  const long long plane = (long long)n * ldw;
  float *W = (float *)workspace(cx, WS_MISC, (size_t)plane * S * sizeof(float));
  if (!W) return B2_ERR_NOMEM;
  F32PartialEpi pe{W, plane, ldw, m, n};
  rc = run(pe);
  if (rc != B2_OK) return rc;
  return sgemm_splitk_reduce(W, plane, ldw, S, m, n, alpha, beta, C, ldc, s);
}

int sgemm_splitk_reduce(const float *W, long long plane, int ldw, int S, int m, int n,
                        float alpha, float beta, float *C, int ldc, cudaStream_t s) {
  dim3 grid((unsigned)((m + 255) / 256), (unsigned)(n < 4096 ? n : 4096));
  B2_PROF("sgemm_splitk_reduce", s);
  sgemm_splitk_reduce_kernel<<<grid, 256, 0, s>>>(W, plane, ldw, S, m, n, alpha, beta, C, ldc);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

}  // namespace b2
