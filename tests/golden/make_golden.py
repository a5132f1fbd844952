"""Generate golden vectors by running the REFERENCE itself (oracle/_ref/*.so,
compiled from the wjc404/GEMM_AVX512F sources by oracle/Makefile).

    python tests/golden/make_golden.py [fixture.npz ...]

Writes small .npz fixtures next to this script.  Each holds the seeded inputs
and the reference's outputs, so the oracle restatement and the GPU path can be
checked against the reference on machines where the reference is absent.
Needs an AVX-512F host (the reference kernels are AVX-512 code).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

GEMM_SHAPES = [(1, 1, 1), (7, 5, 3), (37, 53, 29), (17, 5, 385), (24, 8, 384), (50, 17, 1),
               (5, 3, 769)]
ALPHA_BETA = [(1.5, 0.5), (1.0, 0.0), (1.0, 1.0), (-0.7, 2.0)]


def gemm_cases(dtype, seed):
    rng = np.random.default_rng(seed)
    out = {}
    idx = 0
    for (m, n, k) in GEMM_SHAPES:
        for ta in "NT":
            for tb in "NT":
                al, be = ALPHA_BETA[idx % len(ALPHA_BETA)]
                ar, ac = (m, k) if ta == "N" else (k, m)
                br, bc = (k, n) if tb == "N" else (n, k)
                a = np.asfortranarray(rng.uniform(-1, 1, (ar + 3, ac)).astype(dtype))
                b = np.asfortranarray(rng.uniform(-1, 1, (br + 2, bc)).astype(dtype))
                c = np.asfortranarray(rng.uniform(-1, 1, (m + 1, n)).astype(dtype))
                cout = c.copy(order="F")
                O.ref_gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, cout[:m])
                key = f"c{idx}"
                out[key + "_meta"] = np.array([m, n, k, ord(ta), ord(tb)], dtype=np.int64)
                out[key + "_ab"] = np.array([al, be])
                out[key + "_a"], out[key + "_b"] = a, b
                out[key + "_c"], out[key + "_out"] = c, cout
                idx += 1
    out["count"] = np.array(idx)
    return out


def gemm8x8_cases(seed):
    """The two 8x8 DGEMM files' own serial dgemm_ drivers (kernel_avx512_opt8x8.c:821,
    kernel_avx512_standard8x8.c:843): 8-row A panels (dgemm_tcopy_8 /
    dgemm_ncopy_8, :749/:775) and 8-column B panels, K blocks of 168 (opt) or
    128 (standard), M blocks of 384 / 512; shapes cover ragged panels and
    several K and M blocks, all four trans combinations."""
    rng = np.random.default_rng(seed)
    out = {}
    idx = 0
    shapes = [(1, 1, 1), (7, 5, 3), (13, 17, 29), (17, 9, 170), (9, 10, 260), (389, 2, 16)]
    for which in ("8x8opt", "8x8std"):
        for (m, n, k) in shapes:
            for ta in "NT":
                for tb in "NT":
                    al, be = ALPHA_BETA[idx % len(ALPHA_BETA)]
                    ar, ac = (m, k) if ta == "N" else (k, m)
                    br, bc = (k, n) if tb == "N" else (n, k)
                    a = np.asfortranarray(rng.uniform(-1, 1, (ar + 3, ac)))
                    b = np.asfortranarray(rng.uniform(-1, 1, (br + 2, bc)))
                    c = np.asfortranarray(rng.uniform(-1, 1, (m + 1, n)))
                    cout = c.copy(order="F")
                    O.ref_gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, cout[:m], which=which)
                    key = f"e{idx}"
                    out[key + "_meta"] = np.array([m, n, k, ord(ta), ord(tb)], dtype=np.int64)
                    out[key + "_kind"] = np.array(which)
                    out[key + "_ab"] = np.array([al, be])
                    out[key + "_a"], out[key + "_b"] = a, b
                    out[key + "_c"], out[key + "_out"] = c, cout
                    idx += 1
    out["count"] = np.array(idx)
    return out


def trsm_cases(seed):
    rng = np.random.default_rng(seed)
    out = {}
    idx = 0
    for kind, ms, ns in [("lt", [1, 2, 4, 8, 16], [1, 2, 4, 8, 12]),
                         ("ln", [1, 2, 4, 8, 16], [1, 2, 4, 8, 12]),
                         ("rn", [8, 16], [4, 8, 12]), ("rt", [8, 16], [4, 8, 12])]:
        for M in ms:
            for N in ns:
                is_r = kind[0] == "r"
                K = N if is_r else M
                sa = rng.uniform(0, 1, M * K)
                sb = rng.uniform(0, 1, N * K)
                st = (sa if is_r else sb)[: M * N].copy()
                c = rng.uniform(0, 1, M * N)
                c_out = c.copy()
                if is_r:
                    s1, s2 = st.copy(), sb.copy()
                    O.ref_trsm_kernel(kind, M, N, s1, s2, c_out, K, M)
                    packed_out = s1
                else:
                    s1, s2 = sa.copy(), st.copy()
                    O.ref_trsm_kernel(kind, M, N, s1, s2, c_out, K, M)
                    packed_out = s2
                key = f"t{idx}"
                out[key + "_meta"] = np.array([M, N, K, ord(kind[0]), ord(kind[1])], np.int64)
                out[key + "_sa"], out[key + "_sb"], out[key + "_c"] = sa, sb, c
                out[key + "_cout"], out[key + "_packed_out"] = c_out, packed_out
                idx += 1
    out["count"] = np.array(idx)
    return out


def gemm3m_kernel_cases(seed):
    rng = np.random.default_rng(seed)
    out = {}
    idx = 0
    for (m, n, k) in [(1, 1, 5), (2, 8, 7), (12, 16, 9), (27, 45, 33)]:
        a = rng.uniform(-1, 1, (m, k))
        b = rng.uniform(-1, 1, (n, k))
        ldc = m + 1
        c = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)) + 1j * rng.uniform(-1, 1, (ldc, n)))
        ar, ai = 0.75, -1.25
        pa = O.pack_panels(a, [2, 1])  # GEMM_UNROLL_M = 2 of the 2x8 kernel
        pb = O.pack_panels(b, [8, 4, 2, 1])  # GEMM_UNROLL_N = 8
        cout = c.copy(order="F")
        O.ref_gemm3m_kernel("z2x8", m, n, k, ar, ai, pa, pb, cout)
        key = f"z{idx}"
        out[key + "_meta"] = np.array([m, n, k], np.int64)
        out[key + "_alpha"] = np.array([ar, ai])
        out[key + "_a"], out[key + "_b"], out[key + "_c"], out[key + "_out"] = a, b, c, cout
        idx += 1
    out["count"] = np.array(idx)
    return out


def gemm_kernel_cases(seed):
    """Real and 3M kernels of the OpenBLAS kernel ABI on packed panels:
    C += alpha * A B (real), C_cplx += (ar + i ai) * A B (3M, interleaved C)."""
    rng = np.random.default_rng(seed)
    out = {}
    idx = 0
    shapes = [(1, 1, 1), (3, 5, 7), (16, 2, 9), (29, 13, 33), (37, 26, 64), (8, 24, 5)]
    for which in ("d16x2", "d4x8", "s16x4", "c16x4"):
        if which == "c16x4":
            um, un, dt = 16, 4, np.float32
        else:
            _, _, _, _, um, un = O.GEMM_KERNELS[which]
            dt = np.float32 if which[0] == "s" else np.float64
        for (m, n, k) in shapes:
            a = rng.uniform(-1, 1, (m, k)).astype(dt)
            b = rng.uniform(-1, 1, (n, k)).astype(dt)
            pa = O.pack_panels(a, O.panel_widths(um))
            pb = O.pack_panels(b, O.panel_widths(un))
            ldc = m + 2
            if which == "c16x4":
                c = np.asfortranarray((rng.uniform(-1, 1, (ldc, n)) +
                                       1j * rng.uniform(-1, 1, (ldc, n))).astype(np.complex64))
                al = np.array([0.5, -1.5], dt)
                cout = c.copy(order="F")
                O.ref_gemm3m_kernel("c16x4", m, n, k, al[0], al[1], pa, pb, cout)
            else:
                c = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(dt))
                al = np.array([1.25, 0.0], dt)
                cout = c.copy(order="F")
                O.ref_gemm_kernel(which, m, n, k, al[0], pa, pb, cout)
            key = f"g{idx}"
            out[key + "_meta"] = np.array([m, n, k, um, un], np.int64)
            out[key + "_kind"] = np.array(which)
            out[key + "_alpha"] = al
            out[key + "_a"], out[key + "_b"], out[key + "_c"], out[key + "_out"] = a, b, c, cout
            idx += 1
    out["count"] = np.array(idx)
    return out


FIXTURES = {
    "dgemm_ref.npz": lambda: gemm_cases(np.float64, 11),
    "sgemm_ref.npz": lambda: gemm_cases(np.float32, 12),
    "trsm_kernels_ref.npz": lambda: trsm_cases(13),
    "zgemm3m_kernel_ref.npz": lambda: gemm3m_kernel_cases(14),
    "gemm_kernels_ref.npz": lambda: gemm_kernel_cases(15),
    "dgemm_8x8_ref.npz": lambda: gemm8x8_cases(16),
}


def main():
    """Writes every fixture, or only those named on the command line."""
    if not (O.ref_available("DGEMM.so") and O.host_has_avx512f()):
        raise SystemExit("reference libraries not built or host lacks AVX-512F")
    names = [a for a in sys.argv[1:] if a in FIXTURES] or list(FIXTURES)
    for name in names:
        np.savez_compressed(os.path.join(HERE, name), **FIXTURES[name]())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
