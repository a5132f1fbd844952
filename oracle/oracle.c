/*
 * oracle.c -- CPU restatement of the reference's dense BLAS-3 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py
 * load the library built from it.  The product (libb2blas.so) never links,
 * loads or calls anything here.
 *
 * Every function cites the reference file:line it restates (paths inside the
 * wjc404/GEMM_AVX512F project).  Parity of this restatement is pinned against
 * the reference itself, compiled from its own sources by oracle/Makefile into
 * oracle/_ref/, and against golden vectors in tests/golden/ generated from it.
 *
 * Layout conventions are the reference's: column-major, Fortran-style leading
 * dimensions, trans char 'N'/'n' = no transpose, anything else = transpose
 * (src/gemm_driver.c:18-19).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int notrans(char c) { return c == 'N' || c == 'n'; } /* src/gemm_driver.c:18-19 */

/* Blocking of the reference driver: the K dimension is cut into blocks of
 * GEMM_BLOCK_DIM_K = 384 (src/gemm_set_parameters.h:73-78 with dgemm_tune.h /
 * sgemm_tune.h: 4*4*8*3), the remainder block is processed FIRST
 * (src/gemm_driver.c:124-125,155-168), and every block is consumed in L1
 * sub-blocks of GEMM_BLOCK_L1DIM_K = 128 (src/kernel/gemm_kernel_wrapper.c:9-51),
 * each of which is accumulated from zero in registers (gemm_kernel.S:438-450,
 * vpxorq) and then added onto C. */
#define REF_BLOCK_K 384
#define REF_L1_K 128

/* ------------------------------------------------------------------------- */
/* GEMM: C <- alpha*op(A)*op(B) + beta*C  (src/gemm_driver.c:116-195)         */
/* ------------------------------------------------------------------------- */
#define DEFINE_ORACLE_GEMM(NAME, T, FMA)                                                \
  void NAME(char transa, char transb, int M, int N, int K, T alpha, const T *A,       \
            int lda, const T *B, int ldb, T beta, T *C, int ldc) {                      \
    const int nta = notrans(transa), ntb = notrans(transb);                            \
    if (M <= 0 || N <= 0) return;                                                        \
    /* beta pre-scale: C *= beta whenever beta != 1, so beta == 0 keeps NaN/Inf      \
       already in C (src/gemm_driver.c:131,104-114). */                                \
    if (beta != (T)1)                                                                   \
      for (int j = 0; j < N; j++)                                                       \
        for (int i = 0; i < M; i++) C[(int64_t)j * ldc + i] *= beta;                   \
    if (alpha == (T)0) return; /* src/gemm_driver.c:132 */                             \
    const int nblk = (K - 1) / REF_BLOCK_K + 1;                                         \
    const int edge = K - (nblk - 1) * REF_BLOCK_K; /* :125 */                           \
    _Pragma("omp parallel for schedule(static)")                                        \
    for (int j = 0; j < N; j++) {                                                       \
      for (int i = 0; i < M; i++) {                                                     \
        T c = C[(int64_t)j * ldc + i];                                                  \
        int k0 = 0;                                                                     \
        for (int blk = 0; blk < nblk && K > 0; blk++) {                                 \
          const int kb = (blk == 0) ? edge : REF_BLOCK_K;                               \
          for (int s0 = 0; s0 < kb; s0 += REF_L1_K) {                                   \
            const int s1 = (s0 + REF_L1_K < kb) ? s0 + REF_L1_K : kb;                   \
            T acc = (T)0;                                                               \
            for (int kk = k0 + s0; kk < k0 + s1; kk++) {                                \
              const T a = nta ? A[(int64_t)kk * lda + i] : A[(int64_t)i * lda + kk];    \
              /* alpha is folded into B while packing (src/gemm_copy.c:64,88) */       \
              const T b = alpha * (ntb ? B[(int64_t)j * ldb + kk]                       \
                                       : B[(int64_t)kk * ldb + j]);                     \
              acc = FMA(a, b, acc);                                                     \
            }                                                                           \
            c += acc;                                                                   \
          }                                                                             \
          k0 += kb;                                                                     \
        }                                                                               \
        C[(int64_t)j * ldc + i] = c;                                                    \
      }                                                                                 \
    }                                                                                   \
  }

DEFINE_ORACLE_GEMM(oracle_dgemm, double, fma)
DEFINE_ORACLE_GEMM(oracle_sgemm, float, fmaf)

/* ------------------------------------------------------------------------- */
/* Double-double GEMM: the error yardstick ("dd oracle").                      */
/* Error-free transformations: TwoSum (Knuth, TAOCP vol. 2, 4.2.2) and         */
/* TwoProd via fused multiply-add (Dekker 1971; exact since fma rounds once).  */
/* Output: hi + lo ~= alpha*op(A)*op(B) + beta*C0 to ~2^-104 relative, with     */
/* the reference's beta semantics (C0 scaled whenever beta != 1).               */
/* ------------------------------------------------------------------------- */
static inline void two_sum(double a, double b, double *s, double *e) {
  double x = a + b, bb = x - a;
  *s = x;
  *e = (a - (x - bb)) + (b - bb);
}
static inline void dd_add(double *h, double *l, double ph, double pl) {
  double s, e;
  two_sum(*h, ph, &s, &e);
  e += *l + pl;
  double hh = s + e;
  *l = e - (hh - s);
  *h = hh;
}
static inline void dd_mul_d(double h, double l, double b, double *oh, double *ol) {
  double p = h * b;
  double e = fma(h, b, -p) + l * b;
  double hh = p + e;
  *ol = e - (hh - p);
  *oh = hh;
}

void oracle_dgemm_dd(char transa, char transb, int M, int N, int K, double alpha,
                     const double *A, int lda, const double *B, int ldb, double beta,
                     const double *C0, int ldc, double *Chi, double *Clo, int ldo) {
  const int nta = notrans(transa), ntb = notrans(transb);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < N; j++) {
    for (int i = 0; i < M; i++) {
      double sh = 0.0, sl = 0.0;
      if (alpha != 0.0) {
        for (int kk = 0; kk < K; kk++) {
          const double a = nta ? A[(int64_t)kk * lda + i] : A[(int64_t)i * lda + kk];
          const double b = ntb ? B[(int64_t)j * ldb + kk] : B[(int64_t)kk * ldb + j];
          const double p = a * b, pe = fma(a, b, -p);
          dd_add(&sh, &sl, p, pe);
        }
        dd_mul_d(sh, sl, alpha, &sh, &sl);
      }
      const double c = C0 ? C0[(int64_t)j * ldc + i] : 0.0;
      if (beta != 1.0) {
        const double p = beta * c, pe = fma(beta, c, -p);
        dd_add(&sh, &sl, p, pe);
      } else {
        dd_add(&sh, &sl, c, 0.0);
      }
      Chi[(int64_t)j * ldo + i] = sh;
      if (Clo) Clo[(int64_t)j * ldo + i] = sl;
    }
  }
}

/* ------------------------------------------------------------------------- */
/* DTRSM solve kernels (OpenBLAS kernel ABI), restating the tester's C         */
/* reference solvers OpenBLAS-like_implementation/dtrsm_16x4/                  */
/* dtrsm_kernel_16x4_tester.c:66-199.  sa/sb are the packed panels; the        */
/* triangle's diagonal is stored pre-inverted (the kernels multiply by it).    */
/* ------------------------------------------------------------------------- */
static void tr_update_c(long M, long N, const double *sb, double *C, long LDC) { /* :66-77 */
  for (long n = 0; n < N; ++n)
    for (long m = 0; m < M; ++m) C[m + n * LDC] += sb[n + m * N];
}
static void tr_update_c_a(long M, long N, const double *sa, double *C, long LDC) { /* :79-89 */
  for (long n = 0; n < N; ++n)
    for (long m = 0; m < M; ++m) C[m + n * LDC] += sa[m + n * M];
}
static const double *tr_get_b(const double *base, unsigned long ldb, unsigned char unroll,
                              unsigned long k, unsigned long n) { /* :91-95 */
  return base + (n >> 2) * (ldb << 2) + k * unroll + (n & 3u);
}

void oracle_trsm_kernel_rn(long M, long N, double *sa, double *sb, double *C, long LDB,
                           long LDC) { /* :97-119 */
  tr_update_c_a(M, N, sa, C, LDC);
  const unsigned char un = N > 4 ? 4 : (unsigned char)N;
  for (long nk = 0; nk < N; ++nk) {
    const double b0 = *tr_get_b(sb, LDB, un, nk, nk);
    double *c = C + nk * LDC, *a = sa + nk * M;
    for (long m = 0; m < M; ++m) { c[m] *= b0; a[m] = c[m]; }
    for (long nr = nk + 1; nr < N; ++nr) {
      const double b1 = *tr_get_b(sb, LDB, un, nk, nr);
      double *cc = C + nr * LDC;
      for (long m = 0; m < M; ++m) cc[m] -= a[m] * b1;
    }
  }
}

void oracle_trsm_kernel_rt(long M, long N, double *sa, double *sb, double *C, long LDB,
                           long LDC) { /* :121-143 */
  tr_update_c_a(M, N, sa, C, LDC);
  const unsigned char un = N > 4 ? 4 : (unsigned char)N;
  for (long nk = N - 1; nk >= 0; nk--) {
    const double b0 = *tr_get_b(sb, LDB, un, nk, nk);
    double *c = C + nk * LDC, *a = sa + nk * M;
    for (long m = 0; m < M; ++m) { c[m] *= b0; a[m] = c[m]; }
    for (long nl = 0; nl < nk; ++nl) {
      const double b1 = *tr_get_b(sb, LDB, un, nk, nl);
      double *cc = C + nl * LDC;
      for (long m = 0; m < M; ++m) cc[m] -= a[m] * b1;
    }
  }
}

static void tr_solve_ln(long M, long N, const double *sa, double *sb, double *C,
                        long LDC) { /* :145-158 */
  for (long mk = M - 1; mk >= 0; mk--) {
    const double a0 = sa[mk * M + mk];
    for (long n = 0; n < N; ++n) {
      const double b0 = C[mk + n * LDC] * a0;
      sb[mk * N + n] = C[mk + n * LDC] = b0;
      for (long mu = 0; mu < mk; ++mu) C[mu + n * LDC] -= b0 * sa[mk * M + mu];
    }
  }
}
static void tr_solve_lt(long M, long N, const double *sa, double *sb, double *C,
                        long LDC) { /* :160-173 */
  for (long mk = 0; mk < M; ++mk) {
    const double a0 = sa[mk * M + mk];
    for (long n = 0; n < N; ++n) {
      const double b0 = C[mk + n * LDC] * a0;
      sb[mk * N + n] = C[mk + n * LDC] = b0;
      for (long ml = mk + 1; ml < M; ++ml) C[ml + n * LDC] -= b0 * sa[mk * M + ml];
    }
  }
}
void oracle_trsm_kernel_ln(long M, long N, double *sa, double *sb, double *C, long LDB,
                           long LDC) { /* :175-186 */
  long n = 4;
  for (; N; N -= n) {
    if (N < 4) n = N;
    tr_update_c(M, n, sb, C, LDC);
    tr_solve_ln(M, n, sa, sb, C, LDC);
    sb += n * LDB;
    C += n * LDC;
  }
}
void oracle_trsm_kernel_lt(long M, long N, double *sa, double *sb, double *C, long LDB,
                           long LDC) { /* :188-199 */
  long n = 4;
  for (; N; N -= n) {
    if (N < 4) n = N;
    tr_update_c(M, n, sb, C, LDC);
    tr_solve_lt(M, n, sa, sb, C, LDC);
    sb += n * LDB;
    C += n * LDC;
  }
}

/* ------------------------------------------------------------------------- */
/* dtrsm_: Fortran-BLAS contract.  The reference ships only the solve kernels  */
/* (above) and no dtrsm_ driver, so the BLAS definition is the spec:           */
/*   side 'L': op(A) X = alpha B      side 'R': X op(A) = alpha B              */
/* B (m x n, ldb) is overwritten by X.  'U'/'u' upper, else lower; 'N'/'n' no  */
/* transpose, else transpose; 'U'/'u' unit diagonal, else non-unit.            */
/* Left/Lower/NoTrans is restated blocked, the way a driver drives the LT      */
/* kernel (forward substitution multiplying by the inverted diagonal,          */
/* tester.c:160-173) with the trailing update through oracle_dgemm.            */
/* ------------------------------------------------------------------------- */
static int is_upper(char c) { return c == 'U' || c == 'u'; }
static int is_left(char c) { return c == 'L' || c == 'l'; }
static int is_unit(char c) { return c == 'U' || c == 'u'; }

void oracle_dtrsm(char side, char uplo, char transa, char diag, int M, int N, double alpha,
                  const double *A, int lda, double *B, int ldb, int nb) {
  if (M <= 0 || N <= 0) return;
  if (alpha == 0.0) { /* BLAS: B := 0 */
    for (int j = 0; j < N; j++)
      for (int i = 0; i < M; i++) B[(int64_t)j * ldb + i] = 0.0;
    return;
  }
  if (alpha != 1.0)
    for (int j = 0; j < N; j++)
      for (int i = 0; i < M; i++) B[(int64_t)j * ldb + i] *= alpha;
  const int left = is_left(side), up = is_upper(uplo), nt = notrans(transa), unit = is_unit(diag);
#define AEL(i, j) A[(int64_t)(j) * lda + (i)]
#define BEL(i, j) B[(int64_t)(j) * ldb + (i)]
  if (left) {
    /* effective lower = forward substitution over rows of op(A) */
    const int fwd = (!up && nt) || (up && !nt);
    if (fwd && nb > 0 && !up && nt) {
      for (int ib = 0; ib < M; ib += nb) {
        const int bs = (M - ib < nb) ? (M - ib) : nb;
        for (int mk = ib; mk < ib + bs; mk++) {
          const double inv = unit ? 1.0 : 1.0 / AEL(mk, mk);
          for (int j = 0; j < N; j++) {
            const double x = BEL(mk, j) * inv;
            BEL(mk, j) = x;
            for (int ml = mk + 1; ml < ib + bs; ml++) BEL(ml, j) -= x * AEL(ml, mk);
          }
        }
        const int rest = M - ib - bs;
        if (rest > 0)
          oracle_dgemm('N', 'N', rest, N, bs, -1.0, &AEL(ib + bs, ib), lda, &BEL(ib, 0), ldb, 1.0,
                       &BEL(ib + bs, 0), ldb);
      }
      return;
    }
#pragma omp parallel for schedule(static)
    for (int j = 0; j < N; j++) {
      if (fwd) {
        for (int k = 0; k < M; k++) {
          double s = BEL(k, j);
          for (int i = 0; i < k; i++) s -= (nt ? AEL(k, i) : AEL(i, k)) * BEL(i, j);
          BEL(k, j) = unit ? s : s / AEL(k, k);
        }
      } else {
        for (int k = M - 1; k >= 0; k--) {
          double s = BEL(k, j);
          for (int i = k + 1; i < M; i++) s -= (nt ? AEL(k, i) : AEL(i, k)) * BEL(i, j);
          BEL(k, j) = unit ? s : s / AEL(k, k);
        }
      }
    }
  } else {
    /* X op(A) = B: column k of X depends on columns processed before it. */
    const int fwd = (up && nt) || (!up && !nt);
    if (fwd) {
      for (int k = 0; k < N; k++) {
        for (int i = 0; i < k; i++) {
          const double a = nt ? AEL(i, k) : AEL(k, i);
          if (a != 0.0)
            for (int m = 0; m < M; m++) BEL(m, k) -= BEL(m, i) * a;
        }
        if (!unit) {
          const double inv = 1.0 / AEL(k, k);
          for (int m = 0; m < M; m++) BEL(m, k) *= inv;
        }
      }
    } else {
      for (int k = N - 1; k >= 0; k--) {
        for (int i = k + 1; i < N; i++) {
          const double a = nt ? AEL(i, k) : AEL(k, i);
          if (a != 0.0)
            for (int m = 0; m < M; m++) BEL(m, k) -= BEL(m, i) * a;
        }
        if (!unit) {
          const double inv = 1.0 / AEL(k, k);
          for (int m = 0; m < M; m++) BEL(m, k) *= inv;
        }
      }
    }
  }
#undef AEL
#undef BEL
}

/* ------------------------------------------------------------------------- */
/* 3M complex GEMM.  The reference's 3M kernels compute                        */
/*   C_cplx += (alpha_r + i alpha_i) * (A_real_packed . B_real_packed)          */
/* (zgemm3m_kernel_2x8_skylakex.c:336-351, cgemm3m_kernel_16x4_skylakex.c:415-  */
/* 440); the driver that calls them three times (OpenBLAS driver/level3/        */
/* gemm3m, not vendored) forms the standard 3M products                         */
/*   P1 = Ar Br,  P2 = Ai Bi,  P3 = (Ar + Ai)(Br + Bi)                          */
/*   Re(AB) = P1 - P2,  Im(AB) = P3 - P1 - P2                                   */
/* restated here with the real products through oracle_dgemm / oracle_sgemm.    */
/* trans: 'N' op(X)=X, 'T' transpose, 'C' conjugate transpose, 'R' conjugate.   */
/* Complex scalars and matrices are interleaved (re, im) pairs; ld in complex   */
/* elements.  beta follows the reference drivers: C *= beta when beta != 1.     */
/* ------------------------------------------------------------------------- */
static int tr_is_t(char c) { return !(c == 'N' || c == 'n' || c == 'R' || c == 'r'); }
static int tr_is_conj(char c) { return c == 'C' || c == 'c' || c == 'R' || c == 'r'; }

#define DEFINE_ORACLE_GEMM3M(NAME, T, RGEMM)                                              \
  void NAME(char transa, char transb, int M, int N, int K, const T *alpha, const T *A,    \
            int lda, const T *B, int ldb, const T *beta, T *C, int ldc) {                   \
    if (M <= 0 || N <= 0) return;                                                          \
    const int ta = tr_is_t(transa), tb = tr_is_t(transb);                                  \
    const T sa = tr_is_conj(transa) ? (T)-1 : (T)1, sb = tr_is_conj(transb) ? (T)-1 : (T)1; \
    const int64_t na = (int64_t)M * K, nb = (int64_t)K * N, nc = (int64_t)M * N;            \
    T *Ar = (T *)malloc(sizeof(T) * na), *Ai = (T *)malloc(sizeof(T) * na);                \
    T *As = (T *)malloc(sizeof(T) * na), *Br = (T *)malloc(sizeof(T) * nb);                \
    T *Bi = (T *)malloc(sizeof(T) * nb), *Bs = (T *)malloc(sizeof(T) * nb);                \
    T *P1 = (T *)calloc(nc, sizeof(T)), *P2 = (T *)calloc(nc, sizeof(T));                  \
    T *P3 = (T *)calloc(nc, sizeof(T));                                                    \
    for (int kk = 0; kk < K; kk++)                                                         \
      for (int i = 0; i < M; i++) {                                                        \
        const T *x = ta ? &A[2 * ((int64_t)i * lda + kk)] : &A[2 * ((int64_t)kk * lda + i)]; \
        const int64_t o = (int64_t)kk * M + i;                                             \
        Ar[o] = x[0]; Ai[o] = sa * x[1]; As[o] = Ar[o] + Ai[o];                            \
      }                                                                                    \
    for (int j = 0; j < N; j++)                                                            \
      for (int kk = 0; kk < K; kk++) {                                                     \
        const T *x = tb ? &B[2 * ((int64_t)kk * ldb + j)] : &B[2 * ((int64_t)j * ldb + kk)]; \
        const int64_t o = (int64_t)j * K + kk;                                             \
        Br[o] = x[0]; Bi[o] = sb * x[1]; Bs[o] = Br[o] + Bi[o];                            \
      }                                                                                    \
    RGEMM('N', 'N', M, N, K, (T)1, Ar, M, Br, K, (T)0, P1, M);                              \
    RGEMM('N', 'N', M, N, K, (T)1, Ai, M, Bi, K, (T)0, P2, M);                              \
    RGEMM('N', 'N', M, N, K, (T)1, As, M, Bs, K, (T)0, P3, M);                              \
    const T ar = alpha[0], ai = alpha[1], br = beta[0], bi = beta[1];                      \
    for (int j = 0; j < N; j++)                                                            \
      for (int i = 0; i < M; i++) {                                                        \
        const int64_t o = (int64_t)j * M + i;                                              \
        const T re = P1[o] - P2[o], im = P3[o] - P1[o] - P2[o];                            \
        T *c = &C[2 * ((int64_t)j * ldc + i)];                                             \
        T cr = c[0], ci = c[1];                                                            \
        if (!(br == (T)1 && bi == (T)0)) {                                                 \
          const T tr = br * cr - bi * ci, ti = br * ci + bi * cr;                          \
          cr = tr; ci = ti;                                                                \
        }                                                                                  \
        c[0] = cr + (ar * re - ai * im);                                                   \
        c[1] = ci + (ar * im + ai * re);                                                   \
      }                                                                                    \
    free(Ar); free(Ai); free(As); free(Br); free(Bi); free(Bs);                            \
    free(P1); free(P2); free(P3);                                                          \
  }

DEFINE_ORACLE_GEMM3M(oracle_zgemm3m, double, oracle_dgemm)
DEFINE_ORACLE_GEMM3M(oracle_cgemm3m, float, oracle_sgemm)

/* Kernel-level 3M step: C_cplx(i,j) += (alpha_r + i alpha_i) * sum_k A[i,k] B[j,k]
 * on unpacked real operands A (m x k, row i at A + i, column stride lda) and
 * B (n x k likewise); restates the CNAME contract of
 * zgemm3m_kernel_2x8_skylakex.c:336-351 without the panel packing. */
void oracle_gemm3m_kernel_z(long m, long n, long k, double alphar, double alphai,
                            const double *A, long lda, const double *B, long ldb, double *C,
                            long ldc) {
  for (long j = 0; j < n; j++)
    for (long i = 0; i < m; i++) {
      double s = 0.0;
      for (long kk = 0; kk < k; kk++) s = fma(A[i + kk * lda], B[j + kk * ldb], s);
      C[2 * (i + j * ldc)] += alphar * s;
      C[2 * (i + j * ldc) + 1] += alphai * s;
    }
}
