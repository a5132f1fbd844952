"""Seeded synthetic inputs of the benchmark configurations, drawn with numpy's
PCG64 generator (``numpy.random.default_rng(seed)``) in column-major element
order, so the reference's CPU call and the GPU call see identical buffers.

The reference publishes no benchmark suite; these are its configurations'
shapes, seeds and value distributions:

1. plain DGEMM NN, M=N=K=1024, alpha=1.5, beta=0.5, A, B, C ~ U[-1,1), seed 0;
2. SGEMM, M=N=K in {2048, 4096, 8192} and 8192x256x8192, all four trans
   combinations, A, B ~ U[-1,1), seed 1, alpha=1, beta=0;
3. emulated DGEMM, a = u*exp(phi*g), u ~ U[-1,1), g ~ N(0,1) (u then g, for A
   then for B), M=N=K in {4096, 8192, 16384}, phi in {0.1, 1, 4}, seed 2;
4. grouped GEMM (4096 problems, log-uniform M, N, K in [16, 1024], half FP32 /
   half FP64, random trans), seed 3, and zgemm3m 2048^3 (re, im ~ U[-1,1));
5. DTRSM L/L/N/N, n = 16384, off-diagonal U[-1,1), diagonal n + |U[0,1)|,
   4096 right-hand sides U[-1,1), seed 4.

Every matrix is returned as a Fortran-ordered numpy array.
"""
from __future__ import annotations

import numpy as np


def _fmat(rng, rows, cols, dtype=np.float64):
    return np.asfortranarray(
        rng.uniform(-1.0, 1.0, rows * cols).reshape(rows, cols, order="F").astype(dtype))


def config1(n: int = 1024, seed: int = 0):
    """A, B, C (n x n FP64), drawn in that order; alpha = 1.5, beta = 0.5."""
    rng = np.random.default_rng(seed)
    return _fmat(rng, n, n), _fmat(rng, n, n), _fmat(rng, n, n)


def config2(m: int, n: int, k: int, transa: str = "N", transb: str = "N", seed: int = 1):
    """A (m x k, or k x m for 'T') and B (k x n, or n x k for 'T'), FP32."""
    rng = np.random.default_rng(seed)
    ar, ac = (m, k) if transa in ("N", "n") else (k, m)
    br, bc = (k, n) if transb in ("N", "n") else (n, k)
    return _fmat(rng, ar, ac, np.float32), _fmat(rng, br, bc, np.float32)


def config3(n: int, phi: float, seed: int = 2):
    """A, B (n x n FP64) with entries u*exp(phi*g): u then g for A, then B."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(2):
        u = rng.uniform(-1.0, 1.0, n * n)
        g = rng.standard_normal(n * n)
        out.append(np.asfortranarray((u * np.exp(phi * g)).reshape(n, n, order="F")))
    return out[0], out[1]


def config3_flat(n: int, phi: float, seed: int = 2):
    """config3 as flat column-major vectors (no copy)."""
    a, b = config3(n, phi, seed)
    return a.reshape(-1, order="F"), b.reshape(-1, order="F")


def config4_problems(count: int = 4096, seed: int = 3):
    """Shapes of the grouped batch: (dtype, transa, transb, m, n, k) per problem,
    M, N, K log-uniform integers in [16, 1024], dtype 0 = FP64 for the first
    half and 1 = FP32 for the second, random trans."""
    rng = np.random.default_rng(seed)
    dims = np.floor(np.exp(rng.uniform(np.log(16), np.log(1025), (count, 3)))).astype(int)
    dims = np.clip(dims, 16, 1024)
    trans = rng.integers(0, 2, (count, 2))
    out = []
    for i in range(count):
        out.append((0 if i < count // 2 else 1, "NT"[trans[i, 0]], "NT"[trans[i, 1]],
                    int(dims[i, 0]), int(dims[i, 1]), int(dims[i, 2])))
    return out


def config4_complex(n: int = 2048, seed: int = 3, dtype=np.complex128):
    """A, B, C (n x n complex), real then imaginary part of each, in that order."""
    rng = np.random.default_rng(seed)
    rt = np.float64 if dtype == np.complex128 else np.float32

    def cm():
        re = rng.uniform(-1.0, 1.0, n * n).astype(rt)
        im = rng.uniform(-1.0, 1.0, n * n).astype(rt)
        return np.asfortranarray((re + 1j * im).astype(dtype).reshape(n, n, order="F"))

    return cm(), cm(), cm()


def config5(n: int = 16384, nrhs: int = 4096, seed: int = 4):
    """Lower-triangular A (n x n; strictly upper part zero), off-diagonal
    U[-1,1), diagonal n + |U[0,1)|; B (n x nrhs) U[-1,1)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1.0, 1.0, n * n).reshape(n, n, order="F")
    for j in range(1, n):  # zero the strictly upper part, column by column (in place)
        a[:j, j] = 0.0
    a[np.arange(n), np.arange(n)] = n + np.abs(rng.uniform(0.0, 1.0, n))
    b = _fmat(rng, n, nrhs)
    return a, b
