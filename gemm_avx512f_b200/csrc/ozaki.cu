// ozaki.cu -- DGEMM emulated with INT8 tensor-core products (Ozaki scheme II).
//
// Published method: Ozaki, Uchino, Imamura, "Ozaki Scheme II: A GEMM-oriented
// emulation of floating-point matrix multiplication using an integer modular
// technique" (2025), building on the error-free splitting of Ozaki, Ogita,
// Oishi & Rump (2012) and the INT8 emulation of Ootomo, Ozaki & Yokota (2024).
// Restated here in this library's own form:
//
//  1. Power-of-two scaling.  Row i of op(A) gets sigma_i and column j of op(B)
//     gets tau_j such that ||a_i||_2 * 2^sigma_i <= 2^H and ||b_j||_2 * 2^tau_j
//     <= 2^H, and the scaled entries are truncated to integers
//     A'_ik = trunc(a_ik 2^sigma_i), B'_kj = trunc(b_kj 2^tau_j).  By
//     Cauchy-Schwarz |(A'B')_ij| <= 2^2H <= P/4, where P = m_1 ... m_s is the
//     product of s pairwise-coprime moduli <= 256.
//  2. Residue slices.  For every modulus, A' mod m and B' mod m in [0, m)
//     fit in uint8; each slice product (A' mod m)(B' mod m) is an exact
//     INT32 tcgen05 GEMM on unsigned 8-bit operands (sum < K 2^16 < 2^31 for
//     K <= 32768; longer K is cut into passes whose residues are added mod m).  The GEMM epilogue keeps only
//     the product mod m (one byte per element per modulus).
//  3. Reconstruction.  The integer C' = A'B' is the unique value in (-P/2, P/2)
//     with the s residues (Chinese remainder theorem); it is rebuilt exactly in
//     42-bit-limb integer arithmetic, converted to FP64 once, and scaled by
//     2^-(sigma_i + tau_j).  alpha/beta are applied in the same pass.
//
// The only FP64 arithmetic is the norm/exponent extraction, the final
// conversion and scaling, and the alpha/beta epilogue.  Error: truncation
// contributes < 2 sqrt(K) 2^-H relative to ||a_i|| ||b_j|| per element; H
// grows by ~4 bits per added modulus.  Rows or columns holding Inf/NaN are
// computed by a direct FP64 dot product so IEEE propagation is kept.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>

#include "b2_methods.cuh"
#include "b2_profile.cuh"
#include "umma.cuh"

namespace b2 {

namespace {

constexpr int OZ_MAX = 16;
// K per exact INT32 pass: residues are below 256, so K products stay below
// 32768 * 255^2 < 2^31; longer K is cut into passes whose residues add mod m.
constexpr int OZ_KCHUNK = 1 << 15;
// Pairwise-coprime moduli <= 256 (distinct prime factors), largest first.
constexpr int kModuli[OZ_MAX] = {256, 255, 253, 251, 247, 241, 239, 233,
                                 229, 227, 223, 217, 211, 199, 197, 193};
constexpr long long LIMB = 1ll << 42;
constexpr int NONFINITE = -100000;  // exponent marker for rows/columns with Inf/NaN

struct CrtTable {
  int s;                 // modulus count
  int H;                 // scaling target: 2-norms scaled to <= 2^H
  long long W[OZ_MAX][3];  // CRT weights, 42-bit limbs (low first)
  long long Pl[3];       // P in 42-bit limbs
  double Wd[OZ_MAX][4];  // CRT weights in reconstruction limbs (limb_of)
  double Pd[4];          // P in reconstruction limbs
  double invP;
  double log2P;
};

// Modulus i as a compile-time function, so fully unrolled loops over the
// moduli fold every derived constant into an immediate.
__host__ __device__ constexpr unsigned mod_at(int i) {
  return i == 0 ? 256u : i == 1 ? 255u : i == 2 ? 253u : i == 3 ? 251u : i == 4 ? 247u
       : i == 5 ? 241u : i == 6 ? 239u : i == 7 ? 233u : i == 8 ? 229u : i == 9 ? 227u
       : i == 10 ? 223u : i == 11 ? 217u : i == 12 ? 211u : i == 13 ? 199u : i == 14 ? 197u
       : 193u;
}
constexpr bool moduli_agree() {
  for (int i = 0; i < OZ_MAX; ++i)
    if (mod_at(i) != (unsigned)kModuli[i]) return false;
  return true;
}
static_assert(moduli_agree(), "mod_at must list kModuli in order");

// Epilogue constants, indexed by the batch (= modulus) of a GEMM tile:
// m and the exact Barrett multiplier ceil(2^39 / m).
__constant__ unsigned c_mod[OZ_MAX];
__constant__ unsigned c_m39[OZ_MAX];
// CRT tables for every modulus count s = 0..OZ_MAX (index s), uploaded once per
// device so calls with different counts never re-upload or synchronise.
__constant__ double c_Wd[OZ_MAX + 1][OZ_MAX][4];  // weights in limb_of limbs (low first)
__constant__ double c_Pd[OZ_MAX + 1][4];          // P in limb_of limbs
__constant__ double c_invP[OZ_MAX + 1];

typedef unsigned __int128 u128;

// Limb l of x for the reconstruction with s moduli: 40-bit limbs (the third
// holding everything above bit 80) when s <= 15, 32-bit limbs otherwise.
double limb_of(u128 x, int l, int s) {
  if (s <= 15) {
    if (l >= 3) return 0.0;
    const u128 v = l == 2 ? (x >> 80) : ((x >> (40 * l)) & (((u128)1 << 40) - 1));
    return (double)(unsigned long long)v;
  }
  return (double)(unsigned long long)((x >> (32 * l)) & 0xFFFFFFFFu);
}

CrtTable make_table(int s) {
  CrtTable t{};
  t.s = s;
  u128 P = 1;
  double l2 = 0;
  for (int i = 0; i < s; ++i) {
    P *= (u128)kModuli[i];
    l2 += log2((double)kModuli[i]);
  }
  t.log2P = l2;
  t.H = (int)floor((l2 - 2.0) / 2.0);
  for (int i = 0; i < s; ++i) {
    const int m = kModuli[i];
    const u128 Mi = P / (u128)m;
    const int r = (int)(Mi % (u128)m);
    int inv = 0;
    for (int x = 1; x < m; ++x)
      if ((r * x) % m == 1) { inv = x; break; }
    const u128 W = Mi * (u128)inv;  // < P since inv < m
    t.W[i][0] = (long long)(W & (u128)(LIMB - 1));
    t.W[i][1] = (long long)((W >> 42) & (u128)(LIMB - 1));
    t.W[i][2] = (long long)(W >> 84);
    // limbs of the reconstruction: 3 x 40 bits for s <= 15 (P < 2^118), else 4 x 32
    for (int l = 0; l < 4; ++l) t.Wd[i][l] = limb_of(W, l, s);
  }
  for (int l = 0; l < 4; ++l) t.Pd[l] = limb_of(P, l, s);
  t.Pl[0] = (long long)(P & (u128)(LIMB - 1));
  t.Pl[1] = (long long)((P >> 42) & (u128)(LIMB - 1));
  t.Pl[2] = (long long)(P >> 84);
  t.invP = 1.0 / ((double)t.Pl[2] * 0x1p84 + (double)t.Pl[1] * 0x1p42 + (double)t.Pl[0]);
  return t;
}

// ------------------------------------------------------- norm exponents --
// Fast partial pass: plain sum of squares and max |x| per (row, K chunk).
// Exact enough whenever the row's max |x| lies in [2^-480, 2^480]: no square
// comes near overflow, and squares that underflow (|x| < 2^-511) add less
// than K 2^-1022, negligible against max^2 >= 2^-960.  Rows outside that
// range, and rows holding Inf/NaN (their sum turns non-finite), are redone
// by the finalize kernel with a power-of-two-scaled sum.
// Rows contiguous (element (r,k) at X[r + k*sk]): each thread owns 4
// consecutive rows (two 16-byte loads per column when X and sk allow), a
// 256-thread block covers 1024 rows, so every column of a block is one 8 KB
// contiguous read, with 4 columns (128 B per thread) in flight.
__global__ void __launch_bounds__(256)
    norm_partial_rows_kernel(const double *__restrict__ X, long long sk, int R, int K, int kchunk,
                             bool vec, double *__restrict__ pmax, double *__restrict__ pssq,
                             double *__restrict__ pl1) {
  const int chunk = blockIdx.y;
  const int k0 = chunk * kchunk, k1 = min(K, k0 + kchunk);
  const int r0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (r0 >= R) return;
  double sa[4] = {0.0, 0.0, 0.0, 0.0}, ma[4] = {0.0, 0.0, 0.0, 0.0}, la[4] = {0.0, 0.0, 0.0, 0.0};
  const double *p = X + r0;
  if (vec && r0 + 3 < R) {
    int k = k0;
    for (; k + 3 < k1; k += 4) {
      double2 a[4][2];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 *q = reinterpret_cast<const double2 *>(p + (long long)(k + j) * sk);
        a[j][0] = __ldg(q);
        a[j][1] = __ldg(q + 1);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double v[4] = {a[j][0].x, a[j][0].y, a[j][1].x, a[j][1].y};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          sa[e] = fma(v[e], v[e], sa[e]);
          ma[e] = fmax(ma[e], fabs(v[e]));
          la[e] += fabs(v[e]);
        }
      }
    }
    for (; k < k1; ++k) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double v = __ldg(p + (long long)k * sk + e);
        sa[e] = fma(v, v, sa[e]);
        ma[e] = fmax(ma[e], fabs(v));
        la[e] += fabs(v);
      }
    }
  } else {
    for (int e = 0; e < 4 && r0 + e < R; ++e)
      for (int k = k0; k < k1; ++k) {
        const double v = __ldg(p + (long long)k * sk + e);
        sa[e] = fma(v, v, sa[e]);
        ma[e] = fmax(ma[e], fabs(v));
        la[e] += fabs(v);
      }
  }
  for (int e = 0; e < 4 && r0 + e < R; ++e) {
    pmax[(long long)chunk * R + r0 + e] = ma[e];
    pssq[(long long)chunk * R + r0 + e] = sa[e];
    pl1[(long long)chunk * R + r0 + e] = la[e];
  }
}

// K contiguous (element (r,k) at X[r*sr + k]): one warp per row; lanes read
// 16-byte pairs (when X, sr and the chunk start allow), 4 pairs in flight.
__global__ void __launch_bounds__(256)
    norm_partial_kcont_kernel(const double *__restrict__ X, long long sr, int R, int K,
                              int kchunk, bool vec, double *__restrict__ pmax,
                              double *__restrict__ pssq, double *__restrict__ pl1) {
  const int chunk = blockIdx.y;
  const int k0 = chunk * kchunk, k1 = min(K, k0 + kchunk);
  const int warps = blockDim.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * warps + (threadIdx.x >> 5);
  if (r >= R) return;
  const double *p = X + (long long)r * sr;
  double sa[4] = {0.0, 0.0, 0.0, 0.0}, ma[4] = {0.0, 0.0, 0.0, 0.0}, la = 0.0;
  if (vec && (k0 & 1) == 0) {
    int k = k0 + 2 * lane;
    for (; k + 193 < k1; k += 256) {
      double2 a[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) a[j] = __ldg(reinterpret_cast<const double2 *>(p + k + 64 * j));
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        sa[j] = fma(a[j].x, a[j].x, sa[j]);
        sa[j] = fma(a[j].y, a[j].y, sa[j]);
        ma[j] = fmax(ma[j], fmax(fabs(a[j].x), fabs(a[j].y)));
        la += fabs(a[j].x) + fabs(a[j].y);
      }
    }
    for (; k + 1 < k1; k += 64) {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(p + k));
      sa[0] = fma(a.x, a.x, sa[0]);
      sa[0] = fma(a.y, a.y, sa[0]);
      ma[0] = fmax(ma[0], fmax(fabs(a.x), fabs(a.y)));
      la += fabs(a.x) + fabs(a.y);
    }
    if (k < k1) {
      const double v = __ldg(p + k);
      sa[0] = fma(v, v, sa[0]);
      ma[0] = fmax(ma[0], fabs(v));
      la += fabs(v);
    }
  } else {
    for (int k = k0 + lane; k < k1; k += 32) {
      const double v = __ldg(p + k);
      sa[0] = fma(v, v, sa[0]);
      ma[0] = fmax(ma[0], fabs(v));
      la += fabs(v);
    }
  }
  double s = (sa[0] + sa[1]) + (sa[2] + sa[3]);
  double mx = fmax(fmax(ma[0], ma[1]), fmax(ma[2], ma[3]));
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    la += __shfl_down_sync(0xffffffffu, la, o);
  }
  if (lane == 0) {
    pmax[(long long)chunk * R + r] = mx;
    pssq[(long long)chunk * R + r] = s;
    pl1[(long long)chunk * R + r] = la;
  }
}

// Scaled sum of squares for the rare rows outside the fast range:
// value = s * 4^e with every term scaled by the running power of two.
struct Ssq {
  int e;
  double s;
  int bad;
};
__device__ __forceinline__ void ssq_add(Ssq &a, double x) {
  if (!isfinite(x)) { a.bad = 1; return; }
  if (x == 0.0) return;
  const int ex = ilogb(x) + 1;  // |x| * 2^-ex in [0.5, 1)
  if (ex > a.e) {
    a.s = scalbn(a.s, 2 * (a.e - ex));
    a.e = ex;
  }
  const double y = scalbn(x, -a.e);
  a.s = fma(y, y, a.s);
}

// Exponent of a row outside the fast range (or holding Inf/NaN), from the
// power-of-two-scaled sum of squares.
__device__ int norm_slow_sigma(const double *p, long long sk, int K, int H) {
  Ssq a{-2000, 0.0, 0};
  for (int k = 0; k < K; ++k) ssq_add(a, p[(long long)k * sk]);
  if (a.bad) return NONFINITE;
  if (a.s == 0.0) return 0;
  int g;
  frexp(a.s * (1.0 + 0x1p-30), &g);
  return H - (a.e + ((g + 1) >> 1));
}

// sigma_r = H - ceil(log2 ||x_r||_2); NONFINITE if the row holds Inf/NaN;
// 0 for an all-zero row.  With `stat` non-null it also adds each finite
// nonzero fast-range row's flatness log2(||x_r||_1 / (sqrt(K) ||x_r||_2)) to
// stat[0] and the row count to stat[1] (the modulus-count statistic; about
// -0.2 for uniform rows, far below -2 when a few elements carry the norm).
// Block: 32 rows (lane = row) x 8 warps; warp w sums the chunks c = w mod 8,
// the eight partial sums are added in warp order (the result does not depend
// on scheduling), and warp 0 finishes the rows.
constexpr int FIN_WARPS = 8;
__global__ void __launch_bounds__(32 * FIN_WARPS)
    norm_finalize_kernel(const double *__restrict__ pmax, const double *__restrict__ pssq,
                         const double *__restrict__ pl1, int R, int chunks, int H,
                         int *__restrict__ sigma, const double *__restrict__ X, long long sr,
                         long long sk, int K, double *stat) {
  __shared__ double part[3][FIN_WARPS][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + lane;
  double mx = 0.0, ss = 0.0, l1 = 0.0;
  if (r < R) {
#pragma unroll 4
    for (int c = warp; c < chunks; c += FIN_WARPS) {
      mx = fmax(mx, pmax[(long long)c * R + r]);
      ss += pssq[(long long)c * R + r];
      l1 += pl1[(long long)c * R + r];
    }
  }
  part[0][warp][lane] = mx;
  part[1][warp][lane] = ss;
  part[2][warp][lane] = l1;
  __syncthreads();
  if (warp != 0) return;
  mx = part[0][0][lane];
  ss = part[1][0][lane];
  l1 = part[2][0][lane];
#pragma unroll
  for (int w = 1; w < FIN_WARPS; ++w) {
    mx = fmax(mx, part[0][w][lane]);
    ss += part[1][w][lane];
    l1 += part[2][w][lane];
  }
  double flat = 0.0, cnt = 0.0;
  if (r < R) {
    if (mx == 0.0 && ss == 0.0) {
      sigma[r] = 0;
    } else if (isfinite(ss) && mx >= 0x1p-480 && mx <= 0x1p480) {
      int g;
      frexp(ss * (1.0 + 0x1p-30), &g);  // ss (1+eps) < 2^g, so ||x|| < 2^ceil(g/2)
      sigma[r] = H - ((g + 1) >> 1);
      flat = log2(l1 / (sqrt((double)K) * sqrt(ss)));
      cnt = 1.0;
    } else {
      sigma[r] = norm_slow_sigma(X + (long long)r * sr, sk, K, H);
    }
  }
  if (stat) {  // every lane of warp 0 reaches this point
    for (int o = 16; o > 0; o >>= 1) {
      flat += __shfl_down_sync(0xffffffffu, flat, o);
      cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if (lane == 0 && cnt > 0.0) {
      atomicAdd(stat, flat);
      atomicAdd(stat + 1, cnt);
    }
  }
}

// Modulus count of the call, written to *s_dev for the slice, GEMM and
// reconstruction kernels.  Adaptive calls take s_hi when the mean row
// flatness of op(A) plus that of op(B) is below log2_rho_min (heavy-tailed
// rows: a few elements carry each norm, so the truncation error, relative to
// the norms, grows against |C| and against FP64's own error) and then raise
// every finite exponent by dH = H(s_hi) - H(s_base); otherwise s_base.  One
// block.
__global__ void ozaki_decide_kernel(const double *statA, const double *statB, int adaptive,
                                    int s_base, int s_hi, int dH, double log2_rho_min,
                                    int *s_dev, int *sigA, int m, int *tauB, int n,
                                    int *plan_host) {
  __shared__ int s_eff;
  if (threadIdx.x == 0) {
    int sv = s_base;
    if (adaptive && statA[1] > 0.0 && statB[1] > 0.0 &&
        statA[0] / statA[1] + statB[0] / statB[1] < log2_rho_min)
      sv = s_hi;
    s_eff = sv;
    *s_dev = sv;
    if (plan_host) *plan_host = sv;  // mapped pinned word, read after the call's event
  }
  __syncthreads();
  if (s_eff == s_base) return;
  for (int i = threadIdx.x; i < m + n; i += blockDim.x) {
    int *q = i < m ? sigA + i : tauB + (i - m);
    if (*q != NONFINITE) *q += dH;
  }
}

// --------------------------------------------------------- residue slices --
// Unsigned residues from byte dot products.  u = x + 2^62 lies in [1, 2^63)
// for |x| < 2^62; its eight bytes b_0..b_7 are its two 32-bit words.  For
// modulus m,
//   sh = sum_j b_j (2^(8j) mod m) + ((m - 2^62 mod m) mod m)
// is congruent to x modulo m and below 8*255*255 + 255 < 2^19, so two dp4a
// instructions form it (the constant rides in the accumulator).  Then
// q = floor(sh * ceil(2^32/m) / 2^32) is exactly floor(sh/m): with
// ceil(2^32/m) = 2^32/m + d, 0 <= d < 1, the excess sh d / 2^32 < 2^-13 is
// below 1/m and cannot carry the fraction of sh/m (at most 1 - 1/m) past the
// next integer.  r = sh - q m in [0, m) is the residue, one byte (uint8 for
// every modulus <= 256).  Four integer instructions per modulus, no shifts.
struct ResConst {
  unsigned lo, hi, off, mul, m;
};
__host__ __device__ constexpr unsigned pow2_mod(int e, unsigned m) {
  return (unsigned)((1ull << e) % m);
}
__host__ __device__ constexpr unsigned pack4(unsigned a, unsigned b, unsigned c, unsigned d) {
  return a | (b << 8) | (c << 16) | (d << 24);
}
__host__ __device__ constexpr ResConst res_const(int i) {
  return ResConst{pack4(pow2_mod(0, mod_at(i)), pow2_mod(8, mod_at(i)), pow2_mod(16, mod_at(i)),
                        pow2_mod(24, mod_at(i))),
                  pack4(pow2_mod(32, mod_at(i)), pow2_mod(40, mod_at(i)), pow2_mod(48, mod_at(i)),
                        pow2_mod(56, mod_at(i))),
                  (mod_at(i) - pow2_mod(62, mod_at(i))) % mod_at(i),
                  (unsigned)(((1ull << 32) + mod_at(i) - 1) / mod_at(i)), mod_at(i)};
}
static_assert(res_const(0).lo == 1u && res_const(0).hi == 0u && res_const(0).mul == (1u << 24),
              "modulus 256 keeps the low byte");

template <int I>
__device__ __forceinline__ unsigned residue_u8(unsigned lo, unsigned hi) {
  constexpr ResConst K = res_const(I);
  const unsigned sh = __dp4a(lo, K.lo, __dp4a(hi, K.hi, K.off));
  return sh - __umulhi(sh, K.mul) * K.m;
}

// Writes the 8 residue bytes of one thread's elements for modulus I.
template <int I>
__device__ __forceinline__ void store_slice(const unsigned (&lo)[8], const unsigned (&hi)[8],
                                            uint8_t *dst, int nk) {
  unsigned r[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = residue_u8<I>(lo[j], hi[j]);
  const unsigned w0 = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040),
                                  0x5410);
  const unsigned w1 = __byte_perm(__byte_perm(r[4], r[5], 0x0040), __byte_perm(r[6], r[7], 0x0040),
                                  0x5410);
  if (nk == 8) {
    *reinterpret_cast<uint2 *>(dst) = make_uint2(w0, w1);
  } else {
    for (int j = 0; j < nk; ++j) dst[j] = (uint8_t)r[j];
  }
}

template <int I>
__device__ __forceinline__ void store_slices(const unsigned (&lo)[8], const unsigned (&hi)[8],
                                             int s, uint8_t *dst, long long plane, int nk) {
  if constexpr (I < OZ_MAX) {
    if (I >= s) return;
    store_slice<I>(lo, hi, dst + (long long)I * plane, nk);
    store_slices<I + 1>(lo, hi, s, dst, plane, nk);
  }
}

__device__ __forceinline__ double pow2(int e) {  // e in [-1022, 1023]
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// Operand viewed as R x K (element (r,k) at X[r*sr + k*sk]); writes s planes
// out[i][r][k] (row pitch kp bytes, plane pitch plane bytes) of the residues
// of trunc(x * 2^sigma_r) modulo m_i.  Tile: 32 rows x 64 k, 256 threads, each
// thread 8 consecutive k of one row.
template <bool ROWCONT>
__global__ void __launch_bounds__(256)
    slice_kernel(const double *__restrict__ X, long long sr, long long sk, int R, int K,
                 const int *__restrict__ sigma, const int *__restrict__ s_dev,
                 uint8_t *__restrict__ out, long long kp, long long plane) {
  __shared__ double tile[32][65];
  const int k0 = blockIdx.x * 64, r0 = blockIdx.y * 32;
  const int tid = threadIdx.x;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int idx = tid + 256 * e;
    int rr, kk;
    if (ROWCONT) { rr = idx & 31; kk = idx >> 5; } else { kk = idx & 63; rr = idx >> 6; }
    const int r = r0 + rr, k = k0 + kk;
    double v = 0.0;
    if (r < R && k < K) v = __ldg(X + (long long)r * sr + (long long)k * sk);
    tile[rr][kk] = v;
  }
  __syncthreads();
  const int rr = tid >> 3, kg = (tid & 7) * 8;
  const int r = r0 + rr;
  if (r >= R || k0 + kg >= K) return;
  const int sg = sigma[r];
  const bool dead = (sg == NONFINITE);
  // 2^sigma as two in-range factors (sigma in [H-1024, H+1074])
  const int e1 = dead ? 0 : (sg > 1000 ? 1000 : (sg < -1000 ? -1000 : sg));
  const double f1 = pow2(e1), f2 = pow2(dead ? 0 : sg - e1);
  unsigned lo[8], hi[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const double v = dead ? 0.0 : (tile[rr][kg + j] * f1) * f2;
    const unsigned long long u = (unsigned long long)(__double2ll_rz(v) + (1ll << 62));
    lo[j] = (unsigned)u;
    hi[j] = (unsigned)(u >> 32);
  }
  const int nk = min(8, K - (k0 + kg));
  store_slices<0>(lo, hi, *s_dev, out + (long long)r * kp + k0 + kg, plane, nk);
}

// ---------------------------------------------------------- GEMM epilogue --
// D = X_b Y_b^T with X = B-slices (rows n), Y = A-slices (rows m): lane p = n,
// column q = m.  Stores D mod m_b in [0, m_b) as one byte at R[b][n][m].
struct ResidueEpi {
  uint8_t *R;
  long long plane;
  int ldr;
  int P, Q;
  int accumulate;  // add onto the stored residue (K chunks after the first)
  __device__ __forceinline__ void operator()(int b, int p, int q0, const uint32_t (&v)[32]) const {
    if (p >= P || q0 >= Q) return;
    // d mod m for 0 <= d < 2^31 (K <= 32768 products of residues <= 255):
    // floor(d * ceil(2^39/m) / 2^39) is exactly floor(d/m) because the excess
    // d d' / 2^39 (d' < 1) stays below 2^-8 <= 1/m (and is 0 for m = 256).
    const unsigned m = c_mod[b], m39 = c_m39[b];
    uint8_t *dst = R + (long long)b * plane + (long long)p * ldr + q0;
    uint32_t w[8];
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      unsigned r4[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const unsigned e = v[4 * g + j];
        r4[j] = e - (__umulhi(e, m39) >> 7) * m;
      }
      w[g] = __byte_perm(__byte_perm(r4[0], r4[1], 0x0040), __byte_perm(r4[2], r4[3], 0x0040),
                         0x5410);
    }
    const int nq = min(32, Q - q0);
    if (accumulate) {
      for (int j = 0; j < nq; ++j) {
        unsigned r = ((w[j >> 2] >> (8 * (j & 3))) & 0xFFu) + (unsigned)dst[j];
        r -= (r >= m) ? m : 0u;
        dst[j] = (uint8_t)r;
      }
    } else if (nq == 32) {
      uint4 *d4 = reinterpret_cast<uint4 *>(dst);
      d4[0] = make_uint4(w[0], w[1], w[2], w[3]);
      d4[1] = make_uint4(w[4], w[5], w[6], w[7]);
    } else {
      for (int j = 0; j < nq; ++j) dst[j] = (uint8_t)((w[j >> 2] >> (8 * (j & 3))) & 0xFF);
    }
  }
};

// ---------------------------------------------------------- reconstruction --
// (hi * 2^64 + lo) -> double, one rounding when the value fits in 64 bits,
// otherwise at most 1.5 ulp.
__device__ __forceinline__ double i128_to_double(long long hi, unsigned long long lo) {
  if ((hi == 0 && (long long)lo >= 0) || (hi == -1 && (long long)lo < 0))
    return (double)(long long)lo;
  return fma((double)hi, 0x1p64, (double)lo);
}

__device__ __forceinline__ double byte_to_double(unsigned b) {  // exact, no conversion unit
  return __hiloint2double(0x43300000, (int)b) - 4503599627370496.0;
}

// The integer C' with residues r_i (value in (-P/2, P/2)) as a double, then
// scaled: 2^-(sg + tg) C'.  S_l = sum_i r_i W_il are exact limb sums held in
// doubles (three 40-bit limbs when S <= 15: r_i W_il < 2^48, sums < 15 * 2^48
// < 2^52; four 32-bit limbs for S = 16); the quotient q = round(S/P) comes
// from one double estimate (|C'| <= P/4 keeps it exact), S_l - q P_l is exact
// per limb (q P_l < 2^52), and the carries are settled in 64-bit integers, so
// C' is rounded once (exact whenever it is representable).
template <int S>
__device__ __forceinline__ double crt_value(const double (&Sl)[S <= 15 ? 3 : 4], int sg, int tg) {
  constexpr int LIMBS = S <= 15 ? 3 : 4;
  constexpr int LB = LIMBS == 3 ? 40 : 32;
  double Sd = Sl[LIMBS - 1];
#pragma unroll
  for (int l = LIMBS - 2; l >= 0; --l) Sd = fma(Sd, (double)(1ull << LB), Sl[l]);
  const double q = rint(Sd * c_invP[S]);
  long long X[LIMBS];
#pragma unroll
  for (int l = 0; l < LIMBS; ++l) X[l] = __double2ll_rn(fma(-q, c_Pd[S][l], Sl[l]));
#pragma unroll
  for (int l = 0; l + 1 < LIMBS; ++l) {
    const long long cy = X[l] >> LB;
    X[l] -= cy * (1ll << LB);
    X[l + 1] += cy;
  }
  unsigned long long lo;
  long long hi;
  if constexpr (LIMBS == 3) {  // X0 + X1 2^40 + X2 2^80, X0, X1 in [0, 2^40)
    lo = (unsigned long long)X[0] | ((unsigned long long)X[1] << 40);
    hi = (X[1] >> 24) + X[2] * 65536ll;
  } else {  // X0 + X1 2^32 + X2 2^64 + X3 2^96, X0..X2 in [0, 2^32)
    lo = ((unsigned long long)X[1] << 32) | (unsigned long long)X[0];
    hi = X[3] * 4294967296ll + X[2];
  }
  // times 2^-(sg + tg) as two exact power-of-two factors: the first keeps the
  // value normal, so the product rounds once (|C'| < 2^118: a remaining
  // factor below 2^-1022 leaves less than the smallest subnormal, one above
  // 2^1023 overflows any nonzero C')
  const int ex = -(sg + tg);
  const int e1 = ex > 1000 ? 1000 : (ex < -1000 ? -1000 : ex);
  const int e2 = ex - e1;
  const double f2 = e2 < -1022 ? 0.0 : pow2(e2 > 1023 ? 1023 : e2);
  return (i128_to_double(hi, lo) * pow2(e1)) * f2;
}

// C(m,n) = alpha * C'(m,n) 2^-(sigma_m + tau_n) + beta C(m,n) for a modulus
// count S fixed at compile time (so every CRT weight is an immediate operand
// from the constant bank).  Each thread handles E consecutive rows m and walks
// the columns n with the grid's y stride; per column
// it issues every load first -- S residue words and the C pairs -- then
// accumulates the limb sums (one byte-to-double conversion and LIMBS fused
// multiply-adds per residue).  Rows/columns flagged NONFINITE use a direct
// FP64 dot product.  Launched for the two possible counts of a call; the one
// that is not the device-chosen count returns at once.
// Rows per thread E and resident blocks MINB: 4 and 4 up to 15 moduli (64
// registers; 0.566 ms at 8192^2 x 15 moduli on B200 against 0.622 for 8 rows
// and 2 blocks, same bits), 4 and 1 for 16 (the 4-limb form needs more).
template <int S, int E = 4, int MINB = (S <= 15 ? 4 : 1)>
__global__ void __launch_bounds__(256, MINB)
    reconstruct_kernel(const uint8_t *__restrict__ R, long long plane, int ldr,
                       const int *__restrict__ s_dev, int M, int N,
                       const int *__restrict__ sigA, const int *__restrict__ tauB, double alpha,
                       double beta, double *__restrict__ C, int ldc,
                       const double *__restrict__ A, long long asr, long long ask,
                       const double *__restrict__ B, long long bsk, long long bsc, int K) {
  constexpr int LIMBS = S <= 15 ? 3 : 4;
  static_assert(E == 4 || E == 8, "rows per thread: 4 or 8");
  constexpr int WPR = E / 4;  // 32-bit residue words per modulus
  if (*s_dev != S) return;
  const int m0 = (blockIdx.x * blockDim.x + threadIdx.x) * E;
  if (m0 >= M) return;
  // residue words and C as vectors when every row group is aligned
  const bool full = m0 + E <= M;
  const bool rvec = full && ((reinterpret_cast<uintptr_t>(R) & (4 * WPR - 1)) == 0) &&
                    ((ldr & (4 * WPR - 1)) == 0) && ((plane & (4 * WPR - 1)) == 0);
  const bool cvec = full && ((reinterpret_cast<uintptr_t>(C) & 15) == 0) && ((ldc & 1) == 0);
  int sg[E];
  bool anydead = false;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    sg[e] = m0 + e < M ? sigA[m0 + e] : 0;
    anydead |= sg[e] == NONFINITE;
  }
  for (int n = blockIdx.y; n < N; n += gridDim.y) {
    const uint8_t *rp = R + (long long)n * ldr + m0;
    unsigned w[S][WPR];
#pragma unroll
    for (int i = 0; i < S; ++i) {
      if (rvec) {
        if constexpr (WPR == 2) {
          const uint2 v = __ldg(reinterpret_cast<const uint2 *>(rp + (long long)i * plane));
          w[i][0] = v.x;
          w[i][WPR - 1] = v.y;
        } else {
          w[i][0] = __ldg(reinterpret_cast<const unsigned *>(rp + (long long)i * plane));
        }
      } else {
#pragma unroll
        for (int h = 0; h < WPR; ++h) {
          unsigned x = 0;
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (m0 + 4 * h + e < M) x |= (unsigned)rp[(long long)i * plane + 4 * h + e] << (8 * e);
          w[i][h] = x;
        }
      }
    }
    double *cp = C + (long long)n * ldc + m0;
    double cold[E];
    if (cvec) {
#pragma unroll
      for (int h = 0; h < E / 2; ++h) {
        const double2 v = *reinterpret_cast<const double2 *>(cp + 2 * h);
        cold[2 * h] = v.x;
        cold[2 * h + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) cold[e] = m0 + e < M ? cp[e] : 0.0;
    }
    const int tg = tauB[n];
    double Sl[E][LIMBS];
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int l = 0; l < LIMBS; ++l) Sl[e][l] = 0.0;
#pragma unroll
    for (int i = 0; i < S; ++i) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const double rd =
            byte_to_double(__byte_perm(w[i][e >> 2], 0u, 0x4440u | (unsigned)(e & 3)));
#pragma unroll
        for (int l = 0; l < LIMBS; ++l) Sl[e][l] = fma(rd, c_Wd[S][i][l], Sl[e][l]);
      }
    }
    double out[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      double val = crt_value<S>(Sl[e], sg[e], tg);
      if ((anydead || tg == NONFINITE) && m0 + e < M && (sg[e] == NONFINITE || tg == NONFINITE)) {
        double acc = 0.0;
        const int m = m0 + e;
        for (int k = 0; k < K; ++k) acc = fma(A[m * asr + k * ask], B[k * bsk + n * bsc], acc);
        val = acc;
      }
      out[e] = (beta == 1.0) ? fma(alpha, val, cold[e]) : fma(alpha, val, beta * cold[e]);
    }
    if (cvec) {
#pragma unroll
      for (int h = 0; h < E / 2; ++h)
        *reinterpret_cast<double2 *>(cp + 2 * h) = make_double2(out[2 * h], out[2 * h + 1]);
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (m0 + e < M) cp[e] = out[e];
    }
  }
}

// Grid: x covers the row groups (4 rows per thread, 256 threads per block);
// y strides over the columns.  ymax caps the y extent.
template <int S>
void launch_reconstruct_s(unsigned ymax, cudaStream_t st, const uint8_t *R, long long plane,
                          int ldr, const int *s_dev, int M, int N, const int *sigA,
                          const int *tauB, double alpha, double beta, double *C, int ldc,
                          const double *A, long long asr, long long ask, const double *B,
                          long long bsk, long long bsc, int K) {
  constexpr int E = 4;
  const unsigned bx = (unsigned)(((M + E - 1) / E + 255) / 256);
  unsigned by = (unsigned)N < ymax ? (unsigned)N : ymax;
  if (by < 1u) by = 1u;
  reconstruct_kernel<S><<<dim3(bx, by), 256, 0, st>>>(R, plane, ldr, s_dev, M, N, sigA, tauB,
                                                      alpha, beta, C, ldc, A, asr, ask, B, bsk,
                                                      bsc, K);
}

template <int S>
void launch_reconstruct_any(int s, unsigned ymax, cudaStream_t st, const uint8_t *R,
                            long long plane, int ldr, const int *s_dev, int M, int N,
                            const int *sigA, const int *tauB, double alpha, double beta,
                            double *C, int ldc, const double *A, long long asr, long long ask,
                            const double *B, long long bsk, long long bsc, int K) {
  if constexpr (S <= OZ_MAX) {
    if (s == S)
      launch_reconstruct_s<S>(ymax, st, R, plane, ldr, s_dev, M, N, sigA, tauB, alpha, beta, C,
                              ldc, A, asr, ask, B, bsk, bsc, K);
    else
      launch_reconstruct_any<S + 1>(s, ymax, st, R, plane, ldr, s_dev, M, N, sigA, tauB, alpha,
                                    beta, C, ldc, A, asr, ask, B, bsk, bsc, K);
  }
}

// Launch of the reconstruction for the call's possible modulus counts; each
// launch returns at once unless the device-chosen count is its own.
void launch_reconstruct(const uint8_t *R, long long plane, int ldr, const int *s_dev, int s_lo,
                        int s_hi, int M, int N,
                        const int *sigA, const int *tauB, double alpha, double beta, double *C,
                        int ldc, const double *A, long long asr, long long ask, const double *B,
                        long long bsk, long long bsc, int K, cudaStream_t st) {
  // each thread walks about four columns, so its set-up (row exponents) is
  // amortised
  const unsigned ymax = (unsigned)((N + 3) / 4 < 65535 ? (N + 3) / 4 : 65535);
  launch_reconstruct_any<2>(s_lo, ymax, st, R, plane, ldr, s_dev, M, N, sigA, tauB, alpha, beta, C,
                            ldc, A, asr, ask, B, bsk, bsc, K);
  if (s_hi != s_lo) {
    // The heavy-tail count is the rare one: this launch usually exits at
    // once, and a grid of about 8 blocks per SM (columns strided) keeps that
    // cheap.
    const unsigned bx = (unsigned)(((M + 3) / 4 + 255) / 256);
    unsigned y = 1184u / (bx > 0 ? bx : 1u);
    y = y < 1u ? 1u : (y < ymax ? y : ymax);
    launch_reconstruct_any<2>(s_hi, y, st, R, plane, ldr, s_dev, M, N, sigA, tauB, alpha, beta, C,
                              ldc, A, asr, ask, B, bsk, bsc, K);
  }
}

struct OzPlan {
  int s = 0, kchunks = 0;
  const int *word = nullptr;  // pinned copy of the device-chosen count (behind ev)
  cudaEvent_t ev = nullptr;
};
thread_local OzPlan g_last_plan;

std::mutex g_table_mu;
bool g_table_done[64] = {};

// Upload every constant table once per device (all modulus counts at once).
int upload_tables(int dev, cudaStream_t st) {
  if (dev < 0 || dev >= 64) return B2_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_table_mu);
  if (g_table_done[dev]) return B2_OK;
  unsigned mod[OZ_MAX], m39[OZ_MAX];
  for (int i = 0; i < OZ_MAX; ++i) {
    const unsigned long long m = (unsigned long long)kModuli[i];
    mod[i] = (unsigned)m;
    m39[i] = (unsigned)(((1ull << 39) + m - 1) / m);
  }
  static double wd[OZ_MAX + 1][OZ_MAX][4], pd[OZ_MAX + 1][4], ip[OZ_MAX + 1];
  memset(wd, 0, sizeof(wd));
  memset(pd, 0, sizeof(pd));
  memset(ip, 0, sizeof(ip));
  for (int s = 2; s <= OZ_MAX; ++s) {
    const CrtTable t = make_table(s);
    memcpy(wd[s], t.Wd, sizeof(t.Wd));
    memcpy(pd[s], t.Pd, sizeof(t.Pd));
    ip[s] = t.invP;
  }
  B2_CUDA_TRY(cudaMemcpyToSymbolAsync(c_mod, mod, sizeof(mod), 0, cudaMemcpyHostToDevice, st));
  B2_CUDA_TRY(cudaMemcpyToSymbolAsync(c_m39, m39, sizeof(m39), 0, cudaMemcpyHostToDevice, st));
  B2_CUDA_TRY(cudaMemcpyToSymbolAsync(c_Wd, wd, sizeof(wd), 0, cudaMemcpyHostToDevice, st));
  B2_CUDA_TRY(cudaMemcpyToSymbolAsync(c_Pd, pd, sizeof(pd), 0, cudaMemcpyHostToDevice, st));
  B2_CUDA_TRY(cudaMemcpyToSymbolAsync(c_invP, ip, sizeof(ip), 0, cudaMemcpyHostToDevice, st));
  // The constant bank is shared by every stream: finish before any launch uses it.
  B2_CUDA_TRY(cudaStreamSynchronize(st));
  g_table_done[dev] = true;
  return B2_OK;
}

inline long long round_up(long long x, long long a) { return (x + a - 1) / a * a; }

// INT8 engine shape used by the allocating Ozaki path (tuning variants):
//   0: 128 x 256 tile, 4 stages   1: 128 x 128 tile, 6 stages   2: 128 x 128, 4 stages
//   3: CTA pair, 256 x 256 tile, 6 stages   4: CTA pair, 256 x 256 tile, 7 stages
// Default 3 (measured fastest at 8192^3 x 15 moduli: 124.5 vs 117.1 TFLOPS for
// the whole Ozaki DGEMM with engine 0); B2_OZAKI_ENGINE (0..4) overrides it.
constexpr int OZ_VARIANTS = 5;
int default_oz_variant() {
  static const int v = [] {
    const char *e = getenv("B2_OZAKI_ENGINE");
    const int x = e ? atoi(e) : 3;
    return (x >= 0 && x < OZ_VARIANTS) ? x : 3;
  }();
  return v;
}
thread_local int g_oz_variant = default_oz_variant();

// Column block of the host-operand pipeline this thread is running (-1:
// none) and the rows of op(A) the next call computes.  The pipeline calls the
// Ozaki DGEMM once per block of B and C (block 0 in two row halves, the first
// starting before all of A has arrived) with the same A; each row range of A
// is cut into exponents and residue slices once, and an automatic count is
// fixed at 16 moduli for the whole pipeline (the per-block choice cannot
// change A's slices once they are cut; the extra modulus is hidden under the
// copies that bound the pipeline).
struct PipeRows {
  int block = -1;
  const double *a_full = nullptr;
  int m_full = 0, r0 = 0;
};
thread_local PipeRows g_pipe;
// A's exponents (sigA) and slices (Y) for the pipeline's whole op(A), with the
// row ranges already cut (at most 8 disjoint ranges, merged when they touch).
struct ASideCache {
  bool valid = false;
  const double *A = nullptr;
  int m = 0, k = 0, lda = 0, s = 0, H = 0;
  bool tA = false;
  const void *Y = nullptr, *sc = nullptr;
  int nr = 0;
  int lo[8], hi[8];
  bool covers(int r0, int r1) const {
    for (int i = 0; i < nr; ++i)
      if (lo[i] <= r0 && r1 <= hi[i]) return true;
    return false;
  }
  void add(int r0, int r1) {
    for (int i = 0; i < nr;) {  // absorb every range that overlaps or touches
      if (lo[i] <= r1 && r0 <= hi[i]) {
        r0 = lo[i] < r0 ? lo[i] : r0;
        r1 = hi[i] > r1 ? hi[i] : r1;
        lo[i] = lo[nr - 1], hi[i] = hi[nr - 1], --nr;
      } else {
        ++i;
      }
    }
    if (nr < 8) lo[nr] = r0, hi[nr] = r1, ++nr;
  }
};
thread_local ASideCache g_aside;

int run_i8_gemm(int variant, const uint8_t *X, const uint8_t *Y, long long kcl, int n, int m, int s,
                long long kp, long long planeX, long long planeY, const ResidueEpi &epi,
                int device, int sm_count, int *derr, cudaStream_t st, const int *s_dev) {
  const int ybox = variant == 0 ? 256 : 128;  // pair variants stage BN/2 = 128 rows per CTA
  CUtensorMap tmX, tmY;
  int rc = umma::make_kmajor_map(&tmX, umma::KIND_U8, X, kcl, n, s, kp, planeX, umma::BM);
  if (rc == B2_OK) rc = umma::make_kmajor_map(&tmY, umma::KIND_U8, Y, kcl, m, s, kp, planeY, ybox);
  if (rc != B2_OK) return rc;
  switch (variant) {
    case 1:
      return umma::launch<umma::KIND_U8, 128, 6>(tmX, tmY, n, m, kcl, s, epi, sm_count, derr, st,
                                                  "ozaki_i8_gemm", 0, s_dev);
    case 2:
      return umma::launch<umma::KIND_U8, 128, 4>(tmX, tmY, n, m, kcl, s, epi, sm_count, derr, st,
                                                  "ozaki_i8_gemm", 0, s_dev);
    case 3:
      return umma::launch_pair<umma::KIND_U8, 256, 6>(tmX, tmY, n, m, kcl, s, epi, device, derr,
                                                       st, "ozaki_i8_gemm", s_dev);
    case 4:
      return umma::launch_pair<umma::KIND_U8, 256, 7>(tmX, tmY, n, m, kcl, s, epi, device, derr,
                                                       st, "ozaki_i8_gemm", s_dev);
    default:
      return umma::launch<umma::KIND_U8, 256, 4>(tmX, tmY, n, m, kcl, s, epi, sm_count, derr, st,
                                                  "ozaki_i8_gemm", 0, s_dev);
  }
}

// Exponents for the R "rows" of an operand (element (r,k) at X[r*sr + k*sk]).
// K chunks of the norm pass.  Rows contiguous: enough 1024-row blocks x
// chunks for ~8 blocks per SM (at most 128 chunks, at least 32 columns each).
// K contiguous: rows x chunks >= 16384 warps (at most 64 chunks, at least 256
// of K each).  The chunk length is rounded up to a multiple of 8.
int norm_chunks(int R, int K, bool rowcont) {
  if (R < 1) R = 1;
  int c;
  if (rowcont) {
    const int rb = (R + 1023) / 1024;
    c = (1184 + rb - 1) / rb;
    if (c > 128) c = 128;
    const int maxc = K / 32 > 1 ? K / 32 : 1;
    if (c > maxc) c = maxc;
  } else {
    c = (16384 + R - 1) / R;
    if (c > 64) c = 64;
    const int maxc = K / 256 > 1 ? K / 256 : 1;
    if (c > maxc) c = maxc;
  }
  return c > 1 ? c : 1;
}

int norm_exponents(const double *X, long long sr, long long sk, int R, int K, int H, int *sigma,
                   void *scratch, double *stat, cudaStream_t s) {
  const bool rowcont = sr == 1;
  const int want = norm_chunks(R, K, rowcont);
  const int kchunk = K > 0 ? (int)round_up((K + want - 1) / want, 8) : 8;
  const int chunks = K > 0 ? (K + kchunk - 1) / kchunk : 1;
  double *pmax = (double *)round_up((uintptr_t)scratch, 16);
  double *pssq = pmax + (long long)chunks * R;
  double *pl1 = pssq + (long long)chunks * R;
  if (rowcont) {
    const bool vec = ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && ((sk & 1) == 0);
    dim3 grid((R + 1023) / 1024, chunks);
    B2_PROF("ozaki_norm_rowcont", s);
    norm_partial_rows_kernel<<<grid, 256, 0, s>>>(X, sk, R, K, kchunk, vec, pmax, pssq, pl1);
  } else {
    const bool vec = ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && ((sr & 1) == 0) && sk == 1;
    dim3 grid((R + 7) / 8, chunks);
    B2_PROF("ozaki_norm_kcont", s);
    if (sk == 1) {
      norm_partial_kcont_kernel<<<grid, 256, 0, s>>>(X, sr, R, K, kchunk, vec, pmax, pssq, pl1);
    } else {
      return B2_ERR_ARG;  // every operand view has one unit stride
    }
  }
  B2_CUDA_TRY(cudaGetLastError());
  {
    B2_PROF("ozaki_norm_finalize", s);
    norm_finalize_kernel<<<(R + 31) / 32, 32 * FIN_WARPS, 0, s>>>(pmax, pssq, pl1, R, chunks, H,
                                                                   sigma, X, sr, sk, K, stat);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

size_t norm_scratch_bytes(int R, int K) {
  const int a = norm_chunks(R, K, true), b = norm_chunks(R, K, false);
  return (size_t)(a > b ? a : b) * R * 24 + 64;
}

}  // namespace

void ozaki_pipeline_rows(int j, const double *a_full, int m_full, int r0) {
  g_pipe.block = j;
  g_pipe.a_full = j < 0 ? nullptr : a_full;
  g_pipe.m_full = j < 0 ? 0 : m_full;
  g_pipe.r0 = j < 0 ? 0 : r0;
  if (j < 0) g_aside.valid = false;
}

void ozaki_set_variant(int v) {
  g_oz_variant = (v >= 0 && v < OZ_VARIANTS) ? v : default_oz_variant();
}

int ozaki_auto_moduli(int k) {
  // Both the truncation error (~2^-H sqrt(K)) and FP64 rounding (~u sqrt(K))
  // grow like sqrt(K) relative to |C|, so the count that matches FP64 does not
  // depend on K; it depends on the exponent spread of the inputs, because FP64
  // rounds relative to each partial sum while the truncation is relative to
  // the row norm.  Measured on B200 at M=N=K in {2048, 8192},
  // a = u exp(phi g): 14 moduli give 2.0x / 2.7x / 9x the FP64 normwise error
  // for phi = 0.1 / 1 / 4, 15 moduli give 0.22x / 0.31x / 1.2x.  15 keeps the
  // emulation within FP64's error across that whole range.
  (void)k;
  return 15;
}

// Heavy-tail threshold of the automatic modulus count: 16 moduli instead of 15
// when the mean log2 row flatness of op(A) plus that of op(B) is below -4
// (uniform data: about -0.4; a = u exp(g): about -1.9; a = u exp(4g): about -10).
constexpr double OZ_LOG2_RHO_MIN = -4.0;


int dgemm_ozaki(char ta, char tb, int m, int n, int k, double alpha, const double *A, int lda,
                const double *B, int ldb, double beta, double *C, int ldc, int slices,
                cudaStream_t st) {
  if (m <= 0 || n <= 0) return B2_OK;
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  if (k <= 0 || alpha == 0.0) return beta == 1.0 ? B2_OK : scale_matrix_d(m, n, beta, C, ldc, st);
  // slices <= 0: automatic count, s_base or (heavy-tailed inputs) s_base + 1,
  // chosen on the device after the norm pass; buffers are sized for s_max.
  const bool piped = g_pipe.block >= 0;
  bool adaptive = slices <= 0;
  int s_base = adaptive ? ozaki_auto_moduli(k) : slices;
  if (piped && adaptive) {  // fixed count across the pipeline's blocks
    adaptive = false;
    s_base = s_base < OZ_MAX ? s_base + 1 : OZ_MAX;
  }
  if (!piped) g_aside.valid = false;
  if (s_base < 2 || s_base > OZ_MAX) return B2_ERR_ARG;
  const int s_max = adaptive && s_base < OZ_MAX ? s_base + 1 : s_base;
  int rc = upload_tables(cx->device, st);
  if (rc != B2_OK) return rc;
  const CrtTable t = make_table(s_base);
  const int dH = make_table(s_max).H - t.H;

  const bool tA = !(ta == 'N' || ta == 'n');
  const bool tB = !(tb == 'N' || tb == 'n');
  // op(A) as m x K rows: element (i,k) at A[i*asr + k*ask]
  const long long asr = tA ? lda : 1, ask = tA ? 1 : lda;
  // op(B) columns as n x K rows: element (j,k) at B[j*bsr + k*bsk]
  const long long bsr = tB ? 1 : ldb, bsk = tB ? ldb : 1;

  const int KCH = OZ_KCHUNK;  // K per INT32-exact GEMM pass
  const int kchunks = (k + KCH - 1) / KCH;
  const long long kp = round_up(k < KCH ? k : KCH, 16);
  const long long mp = round_up(m, 16);
  // Inside the pipeline, this call's rows [r0, r0 + m) of op(A) are a view
  // of the pipeline's whole op(A) (m_all rows): A's exponents and slices live
  // at their place in full-size arrays, so every block can reuse them.
  const bool rows_view = piped && kchunks == 1 && g_pipe.a_full && g_pipe.r0 >= 0 &&
                         g_pipe.r0 + m <= g_pipe.m_full &&
                         g_pipe.a_full + (long long)g_pipe.r0 * asr == A;
  if (!rows_view) g_aside.valid = false;
  const int m_all = rows_view ? g_pipe.m_full : m, r0 = rows_view ? g_pipe.r0 : 0;
  const long long planeY = (long long)m_all * kp, planeX = (long long)n * kp;
  const long long planeR = (long long)n * mp;

  uint8_t *Yall = (uint8_t *)workspace(cx, WS_OZ_Y, (size_t)planeY * s_max);
  uint8_t *X = (uint8_t *)workspace(cx, WS_OZ_X, (size_t)planeX * s_max);
  uint8_t *Rb = (uint8_t *)workspace(cx, WS_OZ_R, (size_t)planeR * s_max);
  const size_t nsA = norm_scratch_bytes(m, k), nsB = norm_scratch_bytes(n, k);
  // [sigma (m_all)|tau][stat A (2 doubles), stat B (2 doubles), modulus count][norm A][norm B]
  const size_t o_stat = round_up((m_all + n) * sizeof(int), 256);
  const size_t o_scr = o_stat + 256;
  const size_t sc_bytes = o_scr + round_up(nsA, 256) + nsB + 512;
  uint8_t *sc = (uint8_t *)workspace(cx, WS_OZ_SCALE, sc_bytes);
  if (!Yall || !X || !Rb || !sc) return B2_ERR_NOMEM;
  int *sigA = (int *)sc + r0;
  int *tauB = (int *)sc + m_all;
  uint8_t *Y = Yall + (long long)r0 * kp;
  double *stat = (double *)(sc + o_stat);
  int *s_dev = (int *)(stat + 4);
  void *scrA = sc + o_scr;
  void *scrB = (uint8_t *)scrA + round_up(nsA, 256);

  // A pipeline block reuses A's exponents (sigA) and residue slices (Y) when
  // its rows were already cut for the same A and are still in place.
  const bool same_a = rows_view && g_aside.valid && g_aside.A == g_pipe.a_full &&
                      g_aside.m == m_all && g_aside.k == k && g_aside.lda == lda &&
                      g_aside.tA == tA && g_aside.s == s_base && g_aside.H == t.H &&
                      g_aside.Y == (const void *)Yall && g_aside.sc == (const void *)sc;
  const bool reuse_a = same_a && g_aside.covers(r0, r0 + m);
  // The count actually used is known on the device only: the decide kernel
  // stores it straight into mapped pinned memory (a copy would queue behind
  // the host pipeline's large copy-outs on the same copy engine), read by
  // b2_ozaki_last_plan after plan_ev.
  int *plan_word = (int *)((uint8_t *)cx->pinned + 64);
  int *plan_dev = cx->pinned_dev ? (int *)((uint8_t *)cx->pinned_dev + 64) : nullptr;
  if (adaptive) B2_CUDA_TRY(cudaMemsetAsync(stat, 0, 4 * sizeof(double), st));
  // Large single-pass products overlap the GEMMs with the auxiliary passes on
  // a second stream (below); their two norm passes, both HBM-bound, also run
  // side by side there (separate scratch and statistics).
  const bool overlap = !piped && !rows_view && kchunks == 1 && n >= 4096 &&
                       (double)m * n * k >= 8589934592.0 && ozaki_overlap_streams(cx);
  if (overlap && !reuse_a) {
    cudaStream_t as = cx->oz_aux;
    B2_CUDA_TRY(cudaEventRecord(cx->oz_ev[33], st));
    B2_CUDA_TRY(cudaStreamWaitEvent(as, cx->oz_ev[33], 0));
    rc = norm_exponents(B, bsr, bsk, n, k, t.H, tauB, scrB, adaptive ? stat + 2 : nullptr, as);
    const int ra = norm_exponents(A, asr, ask, m, k, t.H, sigA, scrA, adaptive ? stat : nullptr, st);
    // join before anything can return, so no work of this call stays unordered
    cudaError_t e = cudaEventRecord(cx->oz_ev[34], as);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, cx->oz_ev[34], 0);
    if (rc == B2_OK) rc = ra;
    if (rc == B2_OK && e != cudaSuccess) rc = cuda_fail(e, "ozaki norm join");
  } else {
    if (!reuse_a)
      rc = norm_exponents(A, asr, ask, m, k, t.H, sigA, scrA, adaptive ? stat : nullptr, st);
    if (rc == B2_OK)
      rc = norm_exponents(B, bsr, bsk, n, k, t.H, tauB, scrB, adaptive ? stat + 2 : nullptr, st);
  }
  if (rc != B2_OK) return rc;
  {
    B2_PROF("ozaki_decide", st);
    ozaki_decide_kernel<<<1, 1024, 0, st>>>(stat, stat + 2, adaptive && s_max > s_base ? 1 : 0,
                                            s_base, s_max, dH, OZ_LOG2_RHO_MIN, s_dev, sigA, m,
                                            tauB, n, plan_dev);
    B2_CUDA_TRY(cudaGetLastError());
  }

  // Overlapped schedule for large single-pass products: B and C in J column
  // blocks; the INT8 GEMM of block j (tensor-bound, little HBM traffic) runs
  // on a high-priority stream while the slicing of later blocks and the
  // reconstruction of earlier ones (HBM- and FP64-bound) run beside it on an
  // auxiliary stream, so most of the auxiliary passes hide under the GEMMs.
  // B2_OZAKI_BLOCKS = J (1 = no overlap, up to 16) fixes the block count.
  const char *jenv = getenv("B2_OZAKI_BLOCKS");
  const int jfix = jenv ? atoi(jenv) : 0;
  // Blocks of about 4096 columns: measured at 8192^3 x 15 moduli on B200,
  // 6.62 ms with 2 blocks, 6.71 with 4, 6.98 with 8 (the auxiliary passes
  // gain little beside the persistent GEMM, which leaves them few registers
  // and little shared memory, while each block boundary adds a GEMM tail).
  int J = overlap ? (n / 4096 < 2 ? 2 : (n / 4096 > 8 ? 8 : n / 4096)) : 1;
  if (J > 1 && jfix >= 1) J = jfix > 16 ? 16 : jfix;
  if (J > 1) {
    const int nb = (int)round_up((n + J - 1) / J, 256);
    const int nblk = (n + nb - 1) / nb;
    cudaStream_t gs = cx->oz_gemm, as = cx->oz_aux;
    // events: [0, 16) block sliced, [16, 32) block multiplied, 32 fork, 33/34 joins
    cudaEvent_t *ev = cx->oz_ev;
    auto slice_b = [&](int j, cudaStream_t s2) {
      const int j0 = j * nb, nj = n - j0 < nb ? n - j0 : nb;
      dim3 grid((k + 63) / 64, (nj + 31) / 32);
      B2_PROF(bsr == 1 ? "ozaki_slice_rowcont" : "ozaki_slice_kcont", s2);
      if (bsr == 1)
        slice_kernel<true><<<grid, 256, 0, s2>>>(B + j0 * bsr, bsr, bsk, nj, k, tauB + j0, s_dev,
                                                 X + (long long)j0 * kp, kp, planeX);
      else
        slice_kernel<false><<<grid, 256, 0, s2>>>(B + j0 * bsr, bsr, bsk, nj, k, tauB + j0, s_dev,
                                                  X + (long long)j0 * kp, kp, planeX);
    };
    {
      dim3 grid((k + 63) / 64, (m + 31) / 32);
      B2_PROF(asr == 1 ? "ozaki_slice_rowcont" : "ozaki_slice_kcont", st);
      if (asr == 1)
        slice_kernel<true><<<grid, 256, 0, st>>>(A, asr, ask, m, k, sigA, s_dev, Y, kp, planeY);
      else
        slice_kernel<false><<<grid, 256, 0, st>>>(A, asr, ask, m, k, sigA, s_dev, Y, kp, planeY);
      B2_CUDA_TRY(cudaGetLastError());
    }
    slice_b(0, st);
    B2_CUDA_TRY(cudaGetLastError());
    B2_CUDA_TRY(cudaEventRecord(ev[32], st));  // exponents, count, A and block 0 sliced
    B2_CUDA_TRY(cudaStreamWaitEvent(gs, ev[32], 0));
    B2_CUDA_TRY(cudaStreamWaitEvent(as, ev[32], 0));
    for (int j = 1; j < nblk; ++j) {
      slice_b(j, as);
      B2_CUDA_TRY(cudaGetLastError());
      B2_CUDA_TRY(cudaEventRecord(ev[j], as));
    }
    for (int j = 0; j < nblk && rc == B2_OK; ++j) {
      const int j0 = j * nb, nj = n - j0 < nb ? n - j0 : nb;
      if (j > 0) B2_CUDA_TRY(cudaStreamWaitEvent(gs, ev[j], 0));
      ResidueEpi epi{Rb + (long long)j0 * mp, planeR, (int)mp, nj, m, 0};
      rc = run_i8_gemm(g_oz_variant, X + (long long)j0 * kp, Y, k, nj, m, s_max, kp, planeX,
                       planeY, epi, cx->device, cx->sm_count, cx->derr, gs, s_dev);
      if (rc == B2_OK) rc = cudaEventRecord(ev[16 + j], gs) == cudaSuccess ? B2_OK : B2_ERR_CUDA;
    }
    for (int j = 0; j < nblk && rc == B2_OK; ++j) {
      const int j0 = j * nb, nj = n - j0 < nb ? n - j0 : nb;
      B2_CUDA_TRY(cudaStreamWaitEvent(as, ev[16 + j], 0));
      B2_PROF("ozaki_reconstruct", as);
      launch_reconstruct(Rb + (long long)j0 * mp, planeR, (int)mp, s_dev, s_base, s_max, m, nj,
                         sigA, tauB + j0, alpha, beta, C + (long long)j0 * ldc, ldc, A, asr, ask,
                         B + j0 * bsr, bsk, bsr, k, as);
      B2_CUDA_TRY(cudaGetLastError());
    }
    // join: the caller's stream waits for both streams (also on an error, so
    // nothing of this call is left running unordered)
    cudaError_t e1 = cudaEventRecord(ev[33], as);
    if (e1 == cudaSuccess) e1 = cudaStreamWaitEvent(st, ev[33], 0);
    cudaError_t e2 = cudaEventRecord(ev[34], gs);
    if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(st, ev[34], 0);
    if (rc != B2_OK) return rc;
    if (e1 != cudaSuccess) return cuda_fail(e1, "ozaki overlap join");
    if (e2 != cudaSuccess) return cuda_fail(e2, "ozaki overlap join");
  }

  for (int c = 0; c < kchunks && rc == B2_OK && J == 1; ++c) {
    const int kc0 = c * KCH, kcl = (k - kc0 < KCH) ? k - kc0 : KCH;
    if (!reuse_a) {
      dim3 grid((kcl + 63) / 64, (m + 31) / 32);
      B2_PROF(asr == 1 ? "ozaki_slice_rowcont" : "ozaki_slice_kcont", st);
      if (asr == 1)
        slice_kernel<true><<<grid, 256, 0, st>>>(A + kc0 * ask, asr, ask, m, kcl, sigA, s_dev, Y,
                                                 kp, planeY);
      else
        slice_kernel<false><<<grid, 256, 0, st>>>(A + kc0 * ask, asr, ask, m, kcl, sigA, s_dev, Y,
                                                  kp, planeY);
      B2_CUDA_TRY(cudaGetLastError());
    }
    {
      dim3 grid((kcl + 63) / 64, (n + 31) / 32);
      B2_PROF(bsr == 1 ? "ozaki_slice_rowcont" : "ozaki_slice_kcont", st);
      if (bsr == 1)
        slice_kernel<true><<<grid, 256, 0, st>>>(B + kc0 * bsk, bsr, bsk, n, kcl, tauB, s_dev, X,
                                                 kp, planeX);
      else
        slice_kernel<false><<<grid, 256, 0, st>>>(B + kc0 * bsk, bsr, bsk, n, kcl, tauB, s_dev, X,
                                                  kp, planeX);
      B2_CUDA_TRY(cudaGetLastError());
    }
    ResidueEpi epi{Rb, planeR, (int)mp, n, m, c > 0 ? 1 : 0};
    rc = run_i8_gemm(g_oz_variant, X, Y, kcl, n, m, s_max, kp, planeX, planeY, epi, cx->device,
                     cx->sm_count, cx->derr, st, s_dev);
  }
  if (rc != B2_OK) return rc;
  if (J == 1) {
    B2_PROF("ozaki_reconstruct", st);
    launch_reconstruct(Rb, planeR, (int)mp, s_dev, s_base, s_max, m, n, sigA, tauB, alpha, beta, C,
                       ldc, A, asr, ask, B, bsk, bsr, k, st);
    B2_CUDA_TRY(cudaGetLastError());
  }
  if (!plan_dev)
    B2_CUDA_TRY(cudaMemcpyAsync(plan_word, s_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CUDA_TRY(cudaEventRecord(cx->plan_ev, st));
  if (rows_view && !reuse_a) {
    if (!same_a) {
      g_aside.valid = true;
      g_aside.A = g_pipe.a_full;
      g_aside.m = m_all;
      g_aside.k = k;
      g_aside.lda = lda;
      g_aside.tA = tA;
      g_aside.s = s_base;
      g_aside.H = t.H;
      g_aside.Y = Yall;
      g_aside.sc = sc;
      g_aside.nr = 0;
    }
    g_aside.add(r0, r0 + m);
  }
  g_last_plan.s = s_base;
  g_last_plan.kchunks = kchunks;
  g_last_plan.word = plan_word;
  g_last_plan.ev = cx->plan_ev;
  return B2_OK;
}

}  // namespace b2

extern "C" int b2_ozaki_last_plan(int *out, int n) {
  if (!out || n < 2) return B2_ERR_ARG;
  if (b2::g_last_plan.ev && cudaEventSynchronize(b2::g_last_plan.ev) == cudaSuccess)
    b2::g_last_plan.s = *b2::g_last_plan.word;
  out[0] = b2::g_last_plan.s;
  out[1] = b2::g_last_plan.kchunks;
  return B2_OK;
}

// ---------------------------------------------------------------------------
// Body of the allocation-free Ozaki DGEMM (the entry point, its static scratch
// array and the array's set-up live in ozaki_noalloc.cu).  Every scratch
// buffer is carved out of `base` (cap bytes, 256-byte aligned):
//   [error word][modulus count][sigma|tau][norm scratch A|B][Y][X][R]
// The call needs s*(m*kp + n*kp + n*mp) + (m + n)*4 + the norm scratch
// (24 bytes per row and K chunk) + alignment, kp = K rounded up to 16
// (K <= 32768), mp = m rounded up to 16; a larger problem is refused with
// B2_ERR_ARG before anything is launched.  Device pointers only (checked by
// the caller).  Nothing here allocates.
// ---------------------------------------------------------------------------
namespace b2 {

size_t ozaki_noalloc_bytes(int m, int n, int k, int s) {
  const long long kp = round_up(k, 16), mp = round_up(m, 16);
  size_t off = 256;
  off += round_up((long long)(m + n) * sizeof(int), 256);
  off += round_up(norm_scratch_bytes(m, k), 256);
  off += round_up(norm_scratch_bytes(n, k), 256);
  off += round_up((long long)m * kp * s, 256);
  off += round_up((long long)n * kp * s, 256);
  off += round_up((long long)n * mp * s, 256);
  return off;
}

int ozaki_noalloc_run(unsigned char *base, size_t cap, int dev, int sm_count, char transa,
                      char transb, int m, int n, int k, double alpha, const double *A, int lda,
                      const double *B, int ldb, double beta, double *C, int ldc, int slices,
                      cudaStream_t st) {
  const int s = slices > 0 ? slices : ozaki_auto_moduli(k);
  if (s < 2 || s > OZ_MAX) return B2_ERR_ARG;
  if (k > OZ_KCHUNK) return B2_ERR_ARG;  // one exact INT32 pass only
  if (ozaki_noalloc_bytes(m, n, k, s) > cap) return B2_ERR_ARG;

  const long long kp = round_up(k, 16), mp = round_up(m, 16);
  const long long planeY = (long long)m * kp, planeX = (long long)n * kp;
  const long long planeR = (long long)n * mp;
  const size_t nsA = norm_scratch_bytes(m, k), nsB = norm_scratch_bytes(n, k);
  size_t off = 256;
  const size_t o_sig = off;
  off += round_up((long long)(m + n) * sizeof(int), 256);
  const size_t o_nA = off;
  off += round_up(nsA, 256);
  const size_t o_nB = off;
  off += round_up(nsB, 256);
  const size_t o_Y = off;
  off += round_up(planeY * s, 256);
  const size_t o_X = off;
  off += round_up(planeX * s, 256);
  const size_t o_R = off;

  int *derr = (int *)base;
  int *s_dev = (int *)(base + 64);  // modulus count read by the kernels (set below)
  int *sigA = (int *)(base + o_sig);
  int *tauB = sigA + m;
  uint8_t *Y = (uint8_t *)(base + o_Y);
  uint8_t *X = (uint8_t *)(base + o_X);
  uint8_t *Rb = (uint8_t *)(base + o_R);
  // the error word is the only state that must start at zero
  B2_CUDA_TRY(cudaMemsetAsync(derr, 0, sizeof(int), st));

  int rc = upload_tables(dev, st);
  if (rc != B2_OK) return rc;
  const CrtTable t = make_table(s);
  const bool tA = !(transa == 'N' || transa == 'n');
  const bool tB = !(transb == 'N' || transb == 'n');
  const long long asr = tA ? lda : 1, ask = tA ? 1 : lda;
  const long long bsr = tB ? 1 : ldb, bsk = tB ? ldb : 1;

  rc = norm_exponents(A, asr, ask, m, k, t.H, sigA, base + o_nA, nullptr, st);
  if (rc == B2_OK) rc = norm_exponents(B, bsr, bsk, n, k, t.H, tauB, base + o_nB, nullptr, st);
  if (rc != B2_OK) return rc;
  // fixed count (no statistics): the kernel only stores s
  ozaki_decide_kernel<<<1, 32, 0, st>>>(nullptr, nullptr, 0, s, s, 0, 0.0, s_dev, sigA, m, tauB,
                                        n, nullptr);
  B2_CUDA_TRY(cudaGetLastError());
  {
    dim3 grid((k + 63) / 64, (m + 31) / 32);
    if (asr == 1)
      slice_kernel<true><<<grid, 256, 0, st>>>(A, asr, ask, m, k, sigA, s_dev, Y, kp, planeY);
    else
      slice_kernel<false><<<grid, 256, 0, st>>>(A, asr, ask, m, k, sigA, s_dev, Y, kp, planeY);
    B2_CUDA_TRY(cudaGetLastError());
  }
  {
    dim3 grid((k + 63) / 64, (n + 31) / 32);
    if (bsr == 1)
      slice_kernel<true><<<grid, 256, 0, st>>>(B, bsr, bsk, n, k, tauB, s_dev, X, kp, planeX);
    else
      slice_kernel<false><<<grid, 256, 0, st>>>(B, bsr, bsk, n, k, tauB, s_dev, X, kp, planeX);
    B2_CUDA_TRY(cudaGetLastError());
  }
  CUtensorMap tmX, tmY;
  rc = umma::make_kmajor_map(&tmX, umma::KIND_U8, X, k, n, s, kp, planeX, umma::BM);
  if (rc == B2_OK) rc = umma::make_kmajor_map(&tmY, umma::KIND_U8, Y, k, m, s, kp, planeY, 256);
  if (rc != B2_OK) return rc;
  ResidueEpi epi{Rb, planeR, (int)mp, n, m, 0};
  rc = umma::launch<umma::KIND_U8, 256, 4>(tmX, tmY, n, m, k, s, epi, sm_count, derr, st,
                                            "ozaki_i8_gemm");
  if (rc != B2_OK) return rc;
  launch_reconstruct(Rb, planeR, (int)mp, s_dev, s, s, m, n, sigA, tauB, alpha, beta, C, ldc, A,
                     asr, ask, B, bsk, bsr, k, st);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

}  // namespace b2
