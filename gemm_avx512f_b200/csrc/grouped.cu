// grouped.cu -- thousands of independent GEMMs in one persistent launch.
//
// The reference parallelises one GEMM at a time: a static N split over OpenMP
// threads (src/gemm_driver.c:136-149) or a CAS task queue of 192 x (96 k)
// tiles (OpenBLAS-like_implementation/dgemm.c:449-483, get_gemm_task).  The
// B200 form of that queue runs across a whole batch of unrelated problems:
// the host flattens every problem into 64 x 64 output tiles (problems sorted
// by K, largest first, so the longest tiles are handed out first), a
// persistent grid pulls tile indices from a device-side atomic counter, finds
// the owning problem through a tile -> problem map and runs the tile with the
// problem's own dtype, transposes, strides and alpha/beta:
//   FP64 tiles: DMMA mma.sync.m16n8k8.f64, 8 warps of 32 x 16;
//   FP32 tiles: paired FMAs (fma.rn.f32x2), 8 warps of 32 x 16, each lane 4 x 4;
//   complex tiles (zgemm3m_ / cgemm3m_ problems): 32 x 32, the three real
//   products of the 3M method on DMMA (complex128) or FFMA (complex64);
// warps whose block of a tile lies outside the problem skip their multiplies.
// A plan uploads the descriptors once and captures "reset counter + launch" in
// a CUDA graph, so replaying a batch is a single graph launch.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "b2_methods.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace {

constexpr int GT_M = 64, GT_N = 64, GT_K = 16;
constexpr int GT_NE = GT_M * GT_K / 256;  // elements of each operand panel per thread
constexpr int GT_MINB = 3;                 // resident CTAs per SM
constexpr int GT_LD = GT_M + 4;  // [k][m] stride (68 = 4 mod 16 doubles)

struct GroupDesc {
  const void *A;
  const void *B;
  void *C;
  double alpha, beta;
  int m, n, k, lda, ldb, ldc;
  int dtype;  // 0 = f64, 1 = f32, 2 = complex128 3M, 3 = complex64 3M
  int ta, tb;
  int tiles_m, tiles_n;
  long long tile_offset;
  double alpha_i, beta_i;  // complex dtypes
  int ca, cb;              // complex dtypes: operand conjugated ('C', 'R')
};

// A GT_K-deep panel: op(A) tile (64 x 16) and op(B) tile (16 x 64), 4
// elements of each per thread.  load_panel fetches it from global memory into
// registers (zero outside the problem), store_panel writes it to shared
// memory as As[k][m] and Bs[k][n] (stride GT_LD).  Tiles double-buffer the
// panels: the next panel's loads are in flight while the current one is
// multiplied.
//
// Element of a thread's e-th slot (idx = tid + 256 e, lane = idx % 32,
// w = idx / 32): an operand whose m (or n) index is contiguous in memory
// takes m = idx % 64, k = idx / 64 (one warp: 32 consecutive m of one k).  An
// operand whose k is contiguous takes KL consecutive k per row (KL = 4
// doubles or 8 floats, one 32-byte sector) over 32 / KL rows per warp:
// k = lane % KL + KL (w % (16 / KL)), m = lane / KL + (32 / KL)(w / (16 / KL)).
// Its shared-memory stores then hit every bank pair at most twice per warp
// (stride 68: bank pair (8k + 2m) mod 32 for doubles, bank (4k + m) mod 32
// for floats), where one k column of 16 k by 2 rows had hit each four times.
template <typename T, int W = GT_M>
__device__ __forceinline__ void panel_slot(int idx, bool kcont, int &mn, int &kk) {
  if (!kcont) {
    mn = idx % W;
    kk = idx / W;
    return;
  }
  constexpr int KL = 32 / (int)sizeof(T);  // 4 doubles or 8 floats: one 32-byte sector
  const int lane = idx & 31, w = idx >> 5;
  kk = lane % KL + KL * (w % (GT_K / KL));
  mn = lane / KL + (32 / KL) * (w / (GT_K / KL));
}

template <typename T>
struct PanelRegs {
  T a[GT_NE], b[GT_NE];
};

template <typename T>
__device__ __forceinline__ void load_panel(const GroupDesc &g, int m0, int n0, int k0,
                                           PanelRegs<T> &r) {
  const T *A = (const T *)g.A;
  const T *B = (const T *)g.B;
#pragma unroll
  for (int e = 0; e < GT_NE; ++e) {
    const int idx = threadIdx.x + 256 * e;
    int mm, kk;
    panel_slot<T>(idx, g.ta != 0, mm, kk);
    const int gm = m0 + mm, gk = k0 + kk;
    r.a[e] = (gm < g.m && gk < g.k)
                 ? (g.ta ? A[(long long)gm * g.lda + gk] : A[(long long)gk * g.lda + gm])
                 : (T)0;
    int nn, kb;
    panel_slot<T>(idx, g.tb == 0, nn, kb);
    const int gn = n0 + nn, gk2 = k0 + kb;
    r.b[e] = (gn < g.n && gk2 < g.k)
                 ? (g.tb ? B[(long long)gk2 * g.ldb + gn] : B[(long long)gn * g.ldb + gk2])
                 : (T)0;
  }
}

template <typename T>
__device__ __forceinline__ void store_panel(const GroupDesc &g, const PanelRegs<T> &r, T *As,
                                            T *Bs) {
#pragma unroll
  for (int e = 0; e < GT_NE; ++e) {
    const int idx = threadIdx.x + 256 * e;
    int mm, kk;
    panel_slot<T>(idx, g.ta != 0, mm, kk);
    As[kk * GT_LD + mm] = r.a[e];
    int nn, kb;
    panel_slot<T>(idx, g.tb == 0, nn, kb);
    Bs[kb * GT_LD + nn] = r.b[e];
  }
}

constexpr int GT_PANEL = GT_K * GT_LD;  // elements of one operand panel
constexpr int GT_STAGE = 2 * GT_PANEL;  // A and B panels of one stage
constexpr int GT_SMEM = 2 * GT_STAGE * (int)sizeof(double);

// Runs the K loop of one tile over two shared-memory stages; `mac(As, Bs)`
// multiplies one resident panel pair.
template <typename T, class Mac>
__device__ __forceinline__ void tile_k_loop(const GroupDesc &g, int m0, int n0, T *buf, Mac mac) {
  const int nk = (g.k + GT_K - 1) / GT_K;
  PanelRegs<T> r;
  if (nk > 0) {
    load_panel<T>(g, m0, n0, 0, r);
    store_panel<T>(g, r, buf, buf + GT_PANEL);
  }
  __syncthreads();
  for (int it = 0; it < nk; ++it) {
    T *As = buf + (it & 1) * GT_STAGE;
    const bool more = it + 1 < nk;
    if (more) load_panel<T>(g, m0, n0, (it + 1) * GT_K, r);
    mac(As, As + GT_PANEL);
    if (more) {
      T *An = buf + ((it + 1) & 1) * GT_STAGE;
      store_panel<T>(g, r, An, An + GT_PANEL);
    }
    __syncthreads();  // the stage just read is refilled two iterations later
  }
}

__device__ void tile_f64(const GroupDesc &g, int m0, int n0, double *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane >> 2, t = lane & 3;
  const int wm0 = (warp >> 2) * 32, wn0 = (warp & 3) * 16;
  double acc[2][2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
  // A warp whose 32 x 16 block lies wholly outside the problem (edge tiles of
  // small M or N) skips its multiplies: the test depends on the warp and the
  // tile only, so every lane of the warp takes the same branch.  (Skipping
  // single 16 x 8 blocks as well spills registers and was slower.)
  const bool live = m0 + wm0 < g.m && n0 + wn0 < g.n;
  // DMMA m16n8k8: A fragment rows g, g+8 x k t, t+4; B fragment k t, t+4 x column g
  tile_k_loop<double>(g, m0, n0, sm, [&](const double *As, const double *Bs) {
    if (!live) return;
#pragma unroll
    for (int kk = 0; kk < GT_K; kk += 8) {
      double af[2][4], bf[2][2];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int v1 = 0; v1 < 2; ++v1)
#pragma unroll
          for (int v0 = 0; v0 < 2; ++v0)
            af[i][v0 + 2 * v1] = As[(kk + t + 4 * v1) * GT_LD + wm0 + i * 16 + gq + 8 * v0];
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int v = 0; v < 2; ++v) bf[j][v] = Bs[(kk + t + 4 * v) * GT_LD + wn0 + j * 8 + gq];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
              "{%8,%9}, {%0,%1,%2,%3};\n"
              : "+d"(acc[i][j][0]), "+d"(acc[i][j][1]), "+d"(acc[i][j][2]), "+d"(acc[i][j][3])
              : "d"(af[i][0]), "d"(af[i][1]), "d"(af[i][2]), "d"(af[i][3]), "d"(bf[j][0]),
                "d"(bf[j][1]));
    }
  });
  double *C = (double *)g.C;
  const bool one = (g.beta == 1.0);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int m = m0 + wm0 + i * 16 + gq + 8 * (v >> 1);
        const int n = n0 + wn0 + j * 8 + 2 * t + (v & 1);
        if (m < g.m && n < g.n) {
          double *p = C + (long long)n * g.ldc + m;
          *p = one ? fma(g.alpha, acc[i][j][v], *p) : fma(g.alpha, acc[i][j][v], g.beta * *p);
        }
      }
}

// Two FP32 FMAs per issued instruction (sm_100 fma.rn.f32x2, each lane
// rounded as fmaf): c.xy += a.xy * b.xy on 64-bit register pairs.
__device__ __forceinline__ unsigned long long dup2(float a) {
  unsigned long long d;
  asm("mov.b64 %0, {%1, %1};" : "=l"(d) : "f"(a));
  return d;
}
__device__ __forceinline__ void ffma2(unsigned long long &c, unsigned long long a,
                                      unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(c) : "l"(a), "l"(b));
}

// FP32 tile: 8 warps of 32 x 16 outputs (the FP64 warp grid), each lane 4 x 4
// of them: rows 32 (warp / 4) + 4 (lane % 8) + i, columns 16 (warp % 4) +
// 4 (lane / 8) + j, accumulated as column pairs with paired FMAs.  A warp
// whose block lies wholly outside the problem skips its multiplies.
__device__ void tile_f32(const GroupDesc &g, int m0, int n0, float *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rm = (warp >> 2) * 32 + (lane & 7) * 4, cn = (warp & 3) * 16 + (lane >> 3) * 4;
  const bool live = m0 + (warp >> 2) * 32 < g.m && n0 + (warp & 3) * 16 < g.n;
  unsigned long long acc[4][2];  // row i, columns (2 jp, 2 jp + 1)
#pragma unroll
  for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = 0ull;
  tile_k_loop<float>(g, m0, n0, sm, [&](const float *As, const float *Bs) {
    if (!live) return;
#pragma unroll
    for (int kk = 0; kk < GT_K; ++kk) {
      const float4 a = *reinterpret_cast<const float4 *>(&As[kk * GT_LD + rm]);
      const ulonglong2 b = *reinterpret_cast<const ulonglong2 *>(&Bs[kk * GT_LD + cn]);
      const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const unsigned long long ai = dup2(av[i]);
        ffma2(acc[i][0], ai, b.x);
        ffma2(acc[i][1], ai, b.y);
      }
    }
  });
  float *C = (float *)g.C;
  const float al = (float)g.alpha, be = (float)g.beta;
  const bool one = (be == 1.f);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int jp = 0; jp < 2; ++jp) {
      const float2 v = *reinterpret_cast<const float2 *>(&acc[i][jp]);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int m = m0 + rm + i, n = n0 + cn + 2 * jp + e;
        if (m < g.m && n < g.n) {
          float *p = C + (long long)n * g.ldc + m;
          const float x = e ? v.y : v.x;
          *p = one ? fmaf(al, x, *p) : fmaf(al, x, be * *p);
        }
      }
    }
}

// ------------------------------------------------------------ 3M tiles --
// A complex problem's tile is 32 x 32 outputs of C.  Each K panel holds op(A)
// (32 x 16) and op(B) (16 x 32) complex elements, two of each per thread,
// de-interleaved on the way to shared memory into two real panels per
// operand: real part and imaginary part (negated for a conjugated operand).
// Every warp forms the three real products of the 3M method on one 16 x 8
// block, the pre-added operands of the third from the first two's fragments
// in registers (two shared loads fewer per product than a third panel),
//     P1 = Ar Br,  P2 = Ai Bi,  P3 = (Ar + Ai)(Br + Bi),
// and the epilogue combines Re = P1 - P2, Im = P3 - P1 - P2 with the complex
// alpha and beta.  The reference kernels (zgemm3m_kernel_2x8_skylakex.c:
// 336-351, cgemm3m_kernel_16x4_skylakex.c:415-440) take one pre-added real
// product per call; here the three share the staged panels and one queue
// entry.
constexpr int Z_T = 32;                  // tile edge
constexpr int Z_LD = Z_T + 4;            // panel row stride (36 = 4 mod 16)
constexpr int Z_PANEL = GT_K * Z_LD;     // one real panel
constexpr int Z_STAGE = 4 * Z_PANEL;     // A: re, im; B: re, im
constexpr int Z_PER = Z_T * GT_K / 256;  // complex elements per thread per operand
constexpr int GT_SMEM_3M = 2 * Z_STAGE * (int)sizeof(double);

// Slot map of a complex panel (32 wide), in complex elements (16 or 8 bytes).
// An operand whose m (or n) is contiguous takes m = idx % 32, k = idx / 32.  A
// K-contiguous one takes KL = 32 B / element consecutive k per row (one whole
// 32-byte sector) over 32 / KL rows per warp, and spreads those rows so that
// the warp's stores into the real and imaginary panels (stride 36) find every
// bank free: rows 0-3 and 8-11 in the first half-warp of a complex128 store
// (one 128-byte wavefront each), rows 0-3 and 16-19 for complex64.
template <typename CT>
__device__ __forceinline__ void panel_slot3m(int idx, bool kcont, int &mn, int &kk) {
  if (!kcont) {
    mn = idx % 32;
    kk = idx / 32;
    return;
  }
  constexpr int KL = 32 / (int)sizeof(CT);  // 2 (complex128) or 4 (complex64)
  const int lane = idx & 31, w = idx >> 5, r = lane / KL;
  kk = lane % KL + KL * (w % (GT_K / KL));
  const int row = KL == 2 ? ((r & 3) | ((r & 4) << 1) | ((r & 8) >> 1)) : ((r & 3) | ((r & 4) << 2));
  mn = row + (KL == 2 ? 16 : 4) * (w / (GT_K / KL));
}
template <typename R>
struct Cplx;
template <>
struct Cplx<double> {
  using type = double2;
};
template <>
struct Cplx<float> {
  using type = float2;
};

template <typename R>
struct Panel3M {
  R ar[Z_PER], ai[Z_PER], br[Z_PER], bi[Z_PER];
};

template <typename R>
__device__ __forceinline__ void load_panel3m(const GroupDesc &g, int m0, int n0, int k0,
                                             Panel3M<R> &r) {
  using CT = typename Cplx<R>::type;
  const R *A = (const R *)g.A;
  const R *B = (const R *)g.B;
  const R sa = g.ca ? (R)-1 : (R)1, sb = g.cb ? (R)-1 : (R)1;
#pragma unroll
  for (int e = 0; e < Z_PER; ++e) {
    const int idx = threadIdx.x + 256 * e;
    int mm, kk;
    panel_slot3m<CT>(idx, g.ta != 0, mm, kk);
    const int gm = m0 + mm, gk = k0 + kk;
    R re = 0, im = 0;
    if (gm < g.m && gk < g.k) {
      const R *q = A + 2 * (g.ta ? (long long)gm * g.lda + gk : (long long)gk * g.lda + gm);
      re = q[0];
      im = sa * q[1];
    }
    r.ar[e] = re;
    r.ai[e] = im;
    int nn, kb;
    panel_slot3m<CT>(idx, g.tb == 0, nn, kb);
    const int gn = n0 + nn, gk2 = k0 + kb;
    re = 0;
    im = 0;
    if (gn < g.n && gk2 < g.k) {
      const R *q = B + 2 * (g.tb ? (long long)gk2 * g.ldb + gn : (long long)gn * g.ldb + gk2);
      re = q[0];
      im = sb * q[1];
    }
    r.br[e] = re;
    r.bi[e] = im;
  }
}

template <typename R>
__device__ __forceinline__ void store_panel3m(const GroupDesc &g, const Panel3M<R> &r, R *S) {
  using CT = typename Cplx<R>::type;
#pragma unroll
  for (int e = 0; e < Z_PER; ++e) {
    const int idx = threadIdx.x + 256 * e;
    int mm, kk;
    panel_slot3m<CT>(idx, g.ta != 0, mm, kk);
    R *a = S + kk * Z_LD + mm;
    a[0] = r.ar[e];
    a[Z_PANEL] = r.ai[e];
    int nn, kb;
    panel_slot3m<CT>(idx, g.tb == 0, nn, kb);
    R *b = S + 2 * Z_PANEL + kb * Z_LD + nn;
    b[0] = r.br[e];
    b[Z_PANEL] = r.bi[e];
  }
}

// K loop of a 3M tile over two stages; `mac(S)` multiplies one resident stage.
template <typename R, class Mac>
__device__ __forceinline__ void tile3m_k_loop(const GroupDesc &g, int m0, int n0, R *buf,
                                              Mac mac) {
  const int nk = (g.k + GT_K - 1) / GT_K;
  Panel3M<R> r;
  if (nk > 0) {
    load_panel3m<R>(g, m0, n0, 0, r);
    store_panel3m<R>(g, r, buf);
  }
  __syncthreads();
  for (int it = 0; it < nk; ++it) {
    const bool more = it + 1 < nk;
    if (more) load_panel3m<R>(g, m0, n0, (it + 1) * GT_K, r);
    mac(buf + (it & 1) * Z_STAGE);
    if (more) store_panel3m<R>(g, r, buf + ((it + 1) & 1) * Z_STAGE);
    __syncthreads();  // the stage just read is refilled two iterations later
  }
}

// C(m, n) = alpha (Re + i Im) + beta C(m, n) with Re = P1 - P2 and
// Im = P3 - P1 - P2; C is scaled whenever beta != 1 (the reference drivers'
// rule), so a NaN in C stays even for beta = 0.
template <typename R>
__device__ __forceinline__ void store3m(const GroupDesc &g, int m, int n, R p1, R p2, R p3) {
  if (m >= g.m || n >= g.n) return;
  const R re = p1 - p2, im = p3 - p1 - p2;
  const R ar = (R)g.alpha, ai = (R)g.alpha_i, br = (R)g.beta, bi = (R)g.beta_i;
  R *c = (R *)g.C + 2 * ((long long)n * g.ldc + m);
  R cr = c[0], ci = c[1];
  if (!(br == (R)1 && bi == (R)0)) {
    const R tr = br * cr - bi * ci, ti = br * ci + bi * cr;
    cr = tr;
    ci = ti;
  }
  c[0] = cr + (ar * re - ai * im);
  c[1] = ci + (ar * im + ai * re);
}

// complex128 3M tile: 8 warps of 16 x 8 outputs (2 x 4 of them), one DMMA
// m16n8k8 block per product per K step of 8.
__device__ void tile_z3m(const GroupDesc &g, int m0, int n0, double *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane >> 2, t = lane & 3;
  const int wm0 = (warp >> 2) * 16, wn0 = (warp & 3) * 8;
  const bool live = m0 + wm0 < g.m && n0 + wn0 < g.n;
  double acc[3][4];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[p][v] = 0.0;
  tile3m_k_loop<double>(g, m0, n0, sm, [&](const double *S) {
    if (!live) return;
#pragma unroll
    for (int kk = 0; kk < GT_K; kk += 8) {
      double af[2][4], bf[2][2];  // [re, im] fragments
#pragma unroll
      for (int p = 0; p < 2; ++p) {
#pragma unroll
        for (int v1 = 0; v1 < 2; ++v1)
#pragma unroll
          for (int v0 = 0; v0 < 2; ++v0)
            af[p][v0 + 2 * v1] = S[p * Z_PANEL + (kk + t + 4 * v1) * Z_LD + wm0 + gq + 8 * v0];
#pragma unroll
        for (int v = 0; v < 2; ++v)
          bf[p][v] = S[(2 + p) * Z_PANEL + (kk + t + 4 * v) * Z_LD + wn0 + gq];
      }
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        if (p == 2) {  // (Ar + Ai), (Br + Bi)
#pragma unroll
          for (int v = 0; v < 4; ++v) af[0][v] += af[1][v];
#pragma unroll
          for (int v = 0; v < 2; ++v) bf[0][v] += bf[1][v];
        }
        const int q = p == 1 ? 1 : 0;
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+d"(acc[p][0]), "+d"(acc[p][1]), "+d"(acc[p][2]), "+d"(acc[p][3])
            : "d"(af[q][0]), "d"(af[q][1]), "d"(af[q][2]), "d"(af[q][3]), "d"(bf[q][0]),
              "d"(bf[q][1]));
      }
    }
  });

#pragma unroll
  for (int v = 0; v < 4; ++v)
    store3m<double>(g, m0 + wm0 + gq + 8 * (v >> 1), n0 + wn0 + 2 * t + (v & 1), acc[0][v],
                    acc[1][v], acc[2][v]);
}

// complex64 3M tile: the same warp grid, each lane 2 x 2 outputs of its
// warp's 16 x 8 block (rows 2 (lane % 8) + i, columns 2 (lane / 8) + j), FFMA.
__device__ void tile_c3m(const GroupDesc &g, int m0, int n0, float *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rm = (warp >> 2) * 16 + (lane & 7) * 2, cn = (warp & 3) * 8 + (lane >> 3) * 2;
  const bool live = m0 + (warp >> 2) * 16 < g.m && n0 + (warp & 3) * 8 < g.n;
  float acc[3][2][2];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) acc[p][i][j] = 0.f;
  tile3m_k_loop<float>(g, m0, n0, sm, [&](const float *S) {
    if (!live) return;
#pragma unroll
    for (int kk = 0; kk < GT_K; ++kk) {
      const float2 a1 = *reinterpret_cast<const float2 *>(&S[kk * Z_LD + rm]);
      const float2 a2 = *reinterpret_cast<const float2 *>(&S[Z_PANEL + kk * Z_LD + rm]);
      const float2 b1 = *reinterpret_cast<const float2 *>(&S[2 * Z_PANEL + kk * Z_LD + cn]);
      const float2 b2 = *reinterpret_cast<const float2 *>(&S[3 * Z_PANEL + kk * Z_LD + cn]);
      const float2 a3 = make_float2(a1.x + a2.x, a1.y + a2.y);
      const float2 b3 = make_float2(b1.x + b2.x, b1.y + b2.y);
      const float2 av[3] = {a1, a2, a3}, bv[3] = {b1, b2, b3};
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        acc[p][0][0] = fmaf(av[p].x, bv[p].x, acc[p][0][0]);
        acc[p][0][1] = fmaf(av[p].x, bv[p].y, acc[p][0][1]);
        acc[p][1][0] = fmaf(av[p].y, bv[p].x, acc[p][1][0]);
        acc[p][1][1] = fmaf(av[p].y, bv[p].y, acc[p][1][1]);
      }
    }
  });

#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
      store3m<float>(g, m0 + rm + i, n0 + cn + j, acc[0][i][j], acc[1][i][j], acc[2][i][j]);
}

// tile_prob[t] is the problem that owns flattened tile t (one load instead of
// a binary search of dependent descriptor loads).  Thread 0 fetches the next
// tile index while the current tile runs, so the counter's round trip is
// hidden too.
// CPLX: the batch holds complex (3M) problems.  Real-only batches run the
// instantiation without the complex tiles, which keeps its registers free of
// their code (compiled together the four tile kinds spill).
template <bool CPLX>
__global__ void __launch_bounds__(256, GT_MINB)
    grouped_kernel(const GroupDesc *__restrict__ d, const int *__restrict__ tile_prob,
                   long long total_tiles, unsigned long long *counter) {
  // two stages of A and B panels (GT_SMEM; GT_SMEM_3M when the batch has complex problems)
  extern __shared__ __align__(16) double sm[];
  __shared__ long long next_s;
  if (threadIdx.x == 0) next_s = (long long)atomicAdd(counter, 1ull);
  __syncthreads();
  long long t = next_s;
  while (t < total_tiles) {
    __syncthreads();  // every thread has read next_s
    if (threadIdx.x == 0) next_s = (long long)atomicAdd(counter, 1ull);
    const GroupDesc g = d[tile_prob[t]];
    const int local = (int)(t - g.tile_offset);
    const int tm = local % g.tiles_m, tn = local / g.tiles_m;
    float *smf = reinterpret_cast<float *>(sm);
    if (!CPLX || g.dtype < 2) {
      if (g.dtype == 0) tile_f64(g, tm * GT_M, tn * GT_N, sm);
      else tile_f32(g, tm * GT_M, tn * GT_N, smf);
    } else {
      if (g.dtype == 2) tile_z3m(g, tm * Z_T, tn * Z_T, sm);
      else tile_c3m(g, tm * Z_T, tn * Z_T, smf);
    }
    __syncthreads();  // thread 0's store of next_s is visible
    t = next_s;
  }
}

struct Plan {
  int device = -1;
  int count = 0;
  long long total_tiles = 0;
  bool owns = true;  // device buffers allocated for this plan (else context workspace)
  GroupDesc *d_desc = nullptr;
  int *d_map = nullptr;  // tile -> problem
  unsigned long long *d_counter = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int grid = 0;
  bool cplx = false;   // the batch holds complex problems
  int smem = GT_SMEM;  // GT_SMEM_3M when it does
};

bool is_nt(char c) { return c == 'N' || c == 'n'; }
// complex operands: 'N'/'R' keep the layout, 'C'/'R' conjugate
bool is_cnt(char c) { return c == 'N' || c == 'n' || c == 'R' || c == 'r'; }
bool is_conj(char c) { return c == 'C' || c == 'c' || c == 'R' || c == 'r'; }

int build_descs(int count, const b2_gemm_problem *pr, std::vector<GroupDesc> &out,
                std::vector<int> &map, long long *total, bool *has3m, int *info) {
  *has3m = false;
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  // largest K first: each tile costs ~K, so the long tiles are dequeued first
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pr[a].k > pr[b].k; });
  out.clear();
  long long off = 0;
  for (int idx : order) {
    const b2_gemm_problem &p = pr[idx];
    int inf = 0;
    if (p.dtype < 0 || p.dtype > 3) { *info = idx + 1; return B2_ERR_ARG; }
    const bool cplx = p.dtype >= 2;
    const bool tA = cplx ? !is_cnt(p.transa) : !is_nt(p.transa);
    const bool tB = cplx ? !is_cnt(p.transb) : !is_nt(p.transb);
    if (check_gemm(tA ? 'T' : 'N', tB ? 'T' : 'N', p.m, p.n, p.k, p.lda, p.ldb, p.ldc, p.A, p.B,
                   p.C, &inf) != B2_OK) {
      *info = idx + 1;
      return B2_ERR_ARG;
    }
    if (p.m == 0 || p.n == 0) continue;
    GroupDesc g;
    g.A = p.A;
    g.B = p.B;
    g.C = p.C;
    g.alpha = p.alpha;
    g.beta = p.beta;
    g.m = p.m;
    g.n = p.n;
    g.k = p.k;
    g.lda = p.lda;
    g.ldb = p.ldb;
    g.ldc = p.ldc;
    g.dtype = p.dtype;
    g.ta = tA ? 1 : 0;
    g.tb = tB ? 1 : 0;
    g.alpha_i = cplx ? p.alpha_i : 0.0;
    g.beta_i = cplx ? p.beta_i : 0.0;
    g.ca = cplx && is_conj(p.transa) ? 1 : 0;
    g.cb = cplx && is_conj(p.transb) ? 1 : 0;
    const int tm = cplx ? Z_T : GT_M, tn = cplx ? Z_T : GT_N;
    g.tiles_m = (p.m + tm - 1) / tm;
    g.tiles_n = (p.n + tn - 1) / tn;
    if (cplx) *has3m = true;
    g.tile_offset = off;
    off += (long long)g.tiles_m * g.tiles_n;
    if (off > (1ll << 31)) { *info = idx + 1; return B2_ERR_ARG; }
    out.push_back(g);
  }
  map.resize((size_t)off);
  for (size_t i = 0; i < out.size(); ++i) {
    const long long t1 = i + 1 < out.size() ? out[i + 1].tile_offset : off;
    for (long long t = out[i].tile_offset; t < t1; ++t) map[(size_t)t] = (int)i;
  }
  *total = off;
  return B2_OK;
}

int enqueue(const Plan &p, cudaStream_t s) {
  B2_CUDA_TRY(cudaMemsetAsync(p.d_counter, 0, sizeof(unsigned long long), s));
  if (p.total_tiles == 0) return B2_OK;
  B2_PROF("grouped_gemm", s);
  if (p.cplx)
    grouped_kernel<true><<<p.grid, 256, p.smem, s>>>(p.d_desc, p.d_map, p.total_tiles,
                                                     p.d_counter);
  else
    grouped_kernel<false><<<p.grid, 256, p.smem, s>>>(p.d_desc, p.d_map, p.total_tiles,
                                                      p.d_counter);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

void free_plan(Plan *p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->owns) {
    if (p->d_desc) cudaFree(p->d_desc);
    if (p->d_map) cudaFree(p->d_map);
    if (p->d_counter) cudaFree(p->d_counter);
  }
  delete p;
}

// A plan for graph capture owns its device buffers; the one-shot path
// (capture false) places descriptors, tile map and counter in one of the
// calling context's two descriptor slots (`*slot`), uploads them on `s` from
// pinned staging, and allocates nothing per call once the slots have grown.
int make_plan(int count, const b2_gemm_problem *problems, bool capture, cudaStream_t s, Plan **out,
              int *slot, int *info) {
  Ctx *cx = ctx();
  if (!cx) return B2_ERR_NO_DEVICE;
  std::vector<GroupDesc> descs;
  std::vector<int> map;
  long long total = 0;
  bool has3m = false;
  int rc = build_descs(count, problems, descs, map, &total, &has3m, info);
  if (rc != B2_OK) return rc;
  Plan *p = new Plan();
  p->device = cx->device;
  p->count = (int)descs.size();
  p->total_tiles = total;
  p->cplx = has3m;
  p->smem = has3m ? GT_SMEM_3M : GT_SMEM;
  int per_sm = 0;
  const void *fn = has3m ? (const void *)grouped_kernel<true> : (const void *)grouped_kernel<false>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, p->smem) !=
      cudaSuccess) {
    (void)cudaGetLastError();
    free_plan(p);
    return B2_ERR_CUDA;
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, p->smem);
  if (per_sm < 1) per_sm = 1;
  const long long want = (long long)cx->sm_count * per_sm;
  p->grid = (int)(total < want ? (total > 0 ? total : 1) : want);
  const size_t bd = sizeof(GroupDesc) * (descs.empty() ? 1 : descs.size());
  const size_t bm = sizeof(int) * (map.empty() ? 1 : map.size());
  const size_t od = 0, om = (bd + 255) / 256 * 256, oc = om + (bm + 255) / 256 * 256;
  if (capture) {
    if (cudaMalloc(&p->d_desc, bd) != cudaSuccess || cudaMalloc(&p->d_map, bm) != cudaSuccess ||
        cudaMalloc(&p->d_counter, sizeof(unsigned long long)) != cudaSuccess) {
      (void)cudaGetLastError();
      free_plan(p);
      return B2_ERR_NOMEM;
    }
  } else {
    // The slot's previous launch (two calls ago) has read its descriptors.
    const int sl = cx->grp_next;
    cx->grp_next ^= 1;
    *slot = sl;
    if (cx->grp_ev[sl]) {
      const cudaError_t e = cudaEventSynchronize(cx->grp_ev[sl]);
      if (e != cudaSuccess) {
        free_plan(p);
        return cuda_fail(e, "grouped descriptor slot");
      }
    } else if (cudaEventCreateWithFlags(&cx->grp_ev[sl], cudaEventDisableTiming) != cudaSuccess) {
      cx->grp_ev[sl] = nullptr;
      free_plan(p);
      return cuda_fail(cudaGetLastError(), "grouped descriptor event");
    }
    char *w = (char *)workspace(cx, sl ? WS_GROUP2 : WS_GROUP, oc + 256);
    if (!w) {
      free_plan(p);
      return B2_ERR_NOMEM;
    }
    if (cx->grp_host_bytes[sl] < oc) {
      if (cx->grp_host[sl]) cudaFreeHost(cx->grp_host[sl]);
      cx->grp_host[sl] = nullptr;
      cx->grp_host_bytes[sl] = 0;
      if (cudaHostAlloc(&cx->grp_host[sl], oc, cudaHostAllocDefault) != cudaSuccess) {
        (void)cudaGetLastError();
        cx->grp_host[sl] = nullptr;
        free_plan(p);
        return B2_ERR_NOMEM;
      }
      cx->grp_host_bytes[sl] = oc;
    }
    char *h = (char *)cx->grp_host[sl];
    if (!descs.empty()) memcpy(h + od, descs.data(), sizeof(GroupDesc) * descs.size());
    if (!map.empty()) memcpy(h + om, map.data(), sizeof(int) * map.size());
    p->owns = false;
    p->d_desc = (GroupDesc *)(w + od);
    p->d_map = (int *)(w + om);
    p->d_counter = (unsigned long long *)(w + oc);
    const cudaError_t e = cudaMemcpyAsync(w, h, oc, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      free_plan(p);
      return cuda_fail(e, "grouped descriptors");
    }
  }
  if (capture &&
      ((!descs.empty() && cudaMemcpy(p->d_desc, descs.data(), sizeof(GroupDesc) * descs.size(),
                                     cudaMemcpyHostToDevice) != cudaSuccess) ||
       (!map.empty() && cudaMemcpy(p->d_map, map.data(), sizeof(int) * map.size(),
                                   cudaMemcpyHostToDevice) != cudaSuccess))) {
    free_plan(p);
    return cuda_fail(cudaGetLastError(), "grouped descriptors");
  }
  if (capture) {
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
      free_plan(p);
      return cuda_fail(cudaGetLastError(), "capture stream");
    }
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      rc = enqueue(*p, cs);
      e = cudaStreamEndCapture(cs, &p->graph);
    }
    if (e == cudaSuccess && rc == B2_OK) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess || rc != B2_OK) {
      free_plan(p);
      return rc != B2_OK ? rc : cuda_fail(e, "grouped graph capture");
    }
  }
  *out = p;
  return B2_OK;
}

}  // namespace

int grouped_device(int count, const b2_gemm_problem *problems, cudaStream_t s, int *info) {
  Plan *p = nullptr;
  int slot = 0;
  int rc = make_plan(count, problems, false, s, &p, &slot, info);
  if (rc != B2_OK) return rc;
  rc = enqueue(*p, s);
  // The next call but one that takes this slot waits for this event before
  // it overwrites the descriptors (and their pinned staging).
  const cudaError_t e = cudaEventRecord(ctx()->grp_ev[slot], s);
  free_plan(p);
  if (rc == B2_OK && e != cudaSuccess) rc = cuda_fail(e, "grouped descriptor event");
  return rc;
}

int grouped_plan_create(int count, const b2_gemm_problem *problems, void **plan, int *info) {
  Plan *p = nullptr;
  int slot = 0;
  const int rc = make_plan(count, problems, true, nullptr, &p, &slot, info);
  if (rc == B2_OK) *plan = p;
  return rc;
}

int grouped_plan_launch(void *plan, cudaStream_t s) {
  Plan *p = (Plan *)plan;
  cudaError_t e = cudaGraphLaunch(p->exec, s);
  if (e != cudaSuccess) return cuda_fail(e, "grouped graph launch");
  return B2_OK;
}

int grouped_plan_destroy(void *plan) {
  free_plan((Plan *)plan);
  return B2_OK;
}

}  // namespace b2
