"""The packed-panel layout of the OpenBLAS kernel ABI, pinned on the CPU.

tests/golden/gemm_kernels_ref.npz holds the reference's own kernels run on
packed panels (dgemm.c CNAME 16x2, dgemm_kernel_4x8_skylakex_2.c 4x8,
sgemm.c CNAME 16x4, cgemm3m_kernel_16x4_skylakex.c) -- see make_golden.py.
Unpacked, the same inputs give the same products, which pins both the
packing (oracle.pack_panels / panel_widths, the layout the device entry
points read) and the accumulate semantics C += alpha * A B.
"""
import os

import numpy as np

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_golden_kernels_are_the_unpacked_product():
    z = np.load(os.path.join(GOLD, "gemm_kernels_ref.npz"))
    kinds = set()
    for i in range(int(z["count"])):
        key = f"g{i}"
        m, n, k, um, un = (int(v) for v in z[key + "_meta"])
        kind = str(z[key + "_kind"])
        kinds.add(kind)
        a, b = z[key + "_a"].astype(np.float64), z[key + "_b"].astype(np.float64)
        al = z[key + "_alpha"].astype(np.float64)
        c, out = z[key + "_c"], z[key + "_out"]
        p = a @ b.T
        if kind == "c16x4":
            want = c.astype(np.complex128)
            want[:m] += (al[0] + 1j * al[1]) * p
        else:
            want = c.astype(np.float64)
            want[:m] += al[0] * p
        u = np.finfo(np.float32 if c.dtype in (np.float32, np.complex64) else np.float64).eps
        scale = max(1.0, float(np.abs(a).max() * np.abs(b).max() * k))
        assert np.abs(out - want).max() <= 4 * u * scale, (kind, m, n, k)
        assert np.array_equal(out[m:], c[m:]), "rows beyond m of C were written"
    assert kinds == {"d16x2", "d4x8", "s16x4", "c16x4"}


def test_panel_widths_and_packing_layout():
    assert O.panel_widths(16) == [16, 8, 4, 2, 1]
    assert O.panel_widths(2) == [2, 1]
    x = np.arange(7 * 3, dtype=np.float64).reshape(7, 3)  # 7 rows, depth 3
    p = O.pack_panels(x, O.panel_widths(4))  # panels 4, 2, 1
    # full panel (rows 0..3) k-major, then rows 4..5, then row 6
    want = np.concatenate([x[0:4].T.ravel(), x[4:6].T.ravel(), x[6:7].T.ravel()])
    assert np.array_equal(p, want)
