"""CPU restatement of the INT8 Ozaki-II DGEMM emulation, in exact integers.

TEST INFRASTRUCTURE ONLY (imported by tests/ only).  It restates the published
method (Ozaki, Uchino & Imamura 2025, "Ozaki Scheme II", over the error-free
splitting of Ozaki, Ogita, Oishi & Rump 2012) with the same moduli, the same
scaling rule and the same residue conventions as the library, so the GPU
pipeline can be checked stage by stage on small inputs:

    sigma_i = H - ceil(log2 ||a_i||_2),  A'_ik = trunc(a_ik 2^sigma_i)
    r_t     = A' (resp. B') mod m_t in [0, m_t)             (uint8)
    D_t     = r_t(A) r_t(B) mod m_t                           (exact)
    C'      = CRT(D_1 .. D_s) in (-P/2, P/2)
    C       = alpha * C' 2^-(sigma_i + tau_j) + beta * C

The reference itself (wjc404/GEMM_AVX512F) has no emulated DGEMM; its
dgemm_ (src/gemm_driver.c:116) is the semantics being emulated, and the
oracle's oracle_dgemm restates that bit-exactly.
"""
from __future__ import annotations

import math

import numpy as np

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193]


def h_for(s: int) -> int:
    log2p = sum(math.log2(m) for m in MODULI[:s])
    return int(math.floor((log2p - 2.0) / 2.0))


def row_sigma(x: np.ndarray, H: int) -> np.ndarray:
    """sigma_r = H - (e + ceil(g/2)) with ||x_r||^2 = s 4^e, s (1 + 2^-30) < 2^g."""
    out = np.zeros(x.shape[0], dtype=np.int64)
    for r in range(x.shape[0]):
        row = x[r]
        if not np.all(np.isfinite(row)):
            out[r] = -100000
            continue
        nz = row[row != 0]
        if nz.size == 0:
            out[r] = 0
            continue
        e = int(np.max(np.frexp(nz)[1]))
        s = float(np.sum(np.ldexp(nz, -e) ** 2))
        _, g = math.frexp(s * (1.0 + 2.0 ** -30))
        out[r] = H - (e + (g + 1) // 2)
    return out


def residue(x: int, m: int) -> int:
    """x mod m in [0, m) (Python's % is non-negative for m > 0)."""
    return x % m


def emulate(transa, transb, m, n, k, alpha, a, b, beta, c, s=14):
    """Full emulation on Fortran arrays; returns the new C (m x n)."""
    opa = a[:m, :k] if transa in "Nn" else a[:k, :m].T
    opb = b[:k, :n] if transb in "Nn" else b[:n, :k].T
    H = h_for(s)
    sig = row_sigma(np.asarray(opa, dtype=np.float64), H)
    tau = row_sigma(np.asarray(opb.T, dtype=np.float64), H)
    out = np.array(c[:m, :n], dtype=np.float64, copy=True)
    ia = [[int(np.trunc(np.ldexp(opa[i, kk], int(sig[i])))) for kk in range(k)] for i in range(m)]
    ib = [[int(np.trunc(np.ldexp(opb[kk, j], int(tau[j])))) for kk in range(k)] for j in range(n)]
    mods = MODULI[:s]
    P = math.prod(mods)
    W = []
    for mt in mods:
        Mi = P // mt
        W.append(Mi * pow(Mi % mt, -1, mt))
    for i in range(m):
        for j in range(n):
            if sig[i] == -100000 or tau[j] == -100000:
                val = float(np.dot(opa[i], opb[:, j]))
            else:
                acc = 0
                for t, mt in enumerate(mods):
                    d = sum(residue(ia[i][kk], mt) * residue(ib[j][kk], mt)
                            for kk in range(k)) % mt
                    acc += d * W[t]
                x = acc % P
                if x > P // 2:
                    x -= P
                val = math.ldexp(float(x), -int(sig[i] + tau[j]))
            if beta == 1.0:
                out[i, j] = out[i, j] + alpha * val
            else:
                out[i, j] = alpha * val + beta * out[i, j]
    return out
