"""GPU tests of the OpenBLAS kernel-level ABI on device pointers
(b2_dgemm_kernel, b2_sgemm_kernel, b2_zgemm3m_kernel, b2_cgemm3m_kernel,
b2_dtrsm_kernel), through the C ABI, against golden vectors made by the
reference's own kernels (tests/golden/make_golden.py).

GEMM kernels: ||C - C_ref||_F / (K u ||A||_F ||B||_F |alpha|) <= 8 with u of
the data type, rows of C beyond m untouched.  Solve kernels: the tester's own
criterion, maxdiff at rounding level (dtrsm_kernel_16x4_tester.c:256-257),
on C and on the packed right-hand side written back.
"""
import os

import numpy as np
import pytest

from gemm_avx512f_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _dev(x, cuda):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def _err(got, want, m, k, a, b, alpha, u):
    num = float(np.linalg.norm((got[:m] - want[:m]).astype(np.complex128)))
    den = max(k, 1) * u * float(np.linalg.norm(a.astype(np.float64))) * \
        float(np.linalg.norm(b.astype(np.float64))) * max(abs(alpha), 1e-300)
    return num / den


def test_real_and_3m_gemm_kernels_match_reference_golden(cuda):
    import torch

    L = _lib.lib()
    z = np.load(os.path.join(GOLD, "gemm_kernels_ref.npz"))
    for i in range(int(z["count"])):
        key = f"g{i}"
        m, n, k, um, un = (int(v) for v in z[key + "_meta"])
        kind = str(z[key + "_kind"])
        a, b, al = z[key + "_a"], z[key + "_b"], z[key + "_alpha"]
        c, want = z[key + "_c"], z[key + "_out"]
        pa = _dev(O.pack_panels(a, O.panel_widths(um)), cuda)
        pb = _dev(O.pack_panels(b, O.panel_widths(un)), cuda)
        ldc = c.shape[0]
        if kind == "c16x4":
            cd = _dev(np.asfortranarray(c).T.copy().view(np.float32).reshape(-1), cuda)
            st = L.b2_cgemm3m_kernel(um, un, m, n, k, float(al[0]), float(al[1]), pa.data_ptr(),
                                     pb.data_ptr(), cd.data_ptr(), ldc, None)
            torch.cuda.synchronize()
            got = cd.cpu().numpy().view(np.complex64).reshape(n, ldc).T
            u, alpha = np.finfo(np.float32).eps / 2, complex(al[0], al[1])
        else:
            cd = _dev(np.asfortranarray(c).T.copy().reshape(-1), cuda)
            fn = L.b2_sgemm_kernel if c.dtype == np.float32 else L.b2_dgemm_kernel
            st = fn(um, un, m, n, k, float(al[0]), pa.data_ptr(), pb.data_ptr(), cd.data_ptr(), ldc,
                    None)
            torch.cuda.synchronize()
            got = cd.cpu().numpy().reshape(n, ldc).T
            u, alpha = np.finfo(c.dtype).eps / 2, float(al[0])
        assert st == 0, (kind, st)
        assert np.array_equal(got[m:], c[m:]), (kind, "rows beyond m were written")
        assert _err(got, want, m, k, a, b, alpha, u) <= 8, (kind, m, n, k)


def test_zgemm3m_kernel_matches_reference_golden(cuda):
    import torch

    L = _lib.lib()
    z = np.load(os.path.join(GOLD, "zgemm3m_kernel_ref.npz"))
    for i in range(int(z["count"])):
        m, n, k = (int(v) for v in z[f"z{i}_meta"])
        ar, ai = (float(v) for v in z[f"z{i}_alpha"])
        a, b, c, want = z[f"z{i}_a"], z[f"z{i}_b"], z[f"z{i}_c"], z[f"z{i}_out"]
        pa = _dev(O.pack_panels(a, [2, 1]), cuda)
        pb = _dev(O.pack_panels(b, [8, 4, 2, 1]), cuda)
        ldc = c.shape[0]
        cd = _dev(np.asfortranarray(c).T.copy().view(np.float64).reshape(-1), cuda)
        assert L.b2_zgemm3m_kernel(2, 8, m, n, k, ar, ai, pa.data_ptr(), pb.data_ptr(),
                                   cd.data_ptr(), ldc, None) == 0
        torch.cuda.synchronize()
        got = cd.cpu().numpy().view(np.complex128).reshape(n, ldc).T
        assert np.array_equal(got[m:], c[m:])
        assert _err(got, want, m, k, a, b, complex(ar, ai), 2.0 ** -53) <= 8


def test_dtrsm_kernels_match_reference_golden(cuda):
    import torch

    L = _lib.lib()
    z = np.load(os.path.join(GOLD, "trsm_kernels_ref.npz"))
    worst = 0.0
    seen = set()
    for i in range(int(z["count"])):
        M, N, K, s0, s1 = (int(v) for v in z[f"t{i}_meta"])
        kind = chr(s0) + chr(s1)
        seen.add(kind)
        sa, sb, c = (_dev(z[f"t{i}_{x}"], cuda) for x in ("sa", "sb", "c"))
        side, trans = kind[0].upper(), kind[1].upper()
        assert L.b2_dtrsm_kernel(side.encode(), trans.encode(), M, N, sa.data_ptr(),
                                 sb.data_ptr(), c.data_ptr(), K, M, None) == 0
        torch.cuda.synchronize()
        packed = (sa if kind[0] == "r" else sb).cpu().numpy()[: M * N]
        worst = max(worst, np.abs(c.cpu().numpy() - z[f"t{i}_cout"]).max(),
                    np.abs(packed - z[f"t{i}_packed_out"]).max())
    assert seen == {"ln", "lt", "rn", "rt"}
    assert worst < 1e-14, worst


def test_kernel_abi_argument_checks(cuda):
    import torch

    L = _lib.lib()
    buf = torch.zeros(64, dtype=torch.float64, device=cuda)
    p = buf.data_ptr()
    assert L.b2_dgemm_kernel(3, 2, 4, 4, 4, 1.0, p, p, p, 4, None) == _lib.B2_ERR_ARG  # unroll 3
    assert L.b2_dgemm_kernel(4, 2, 4, 4, 4, 1.0, p, p, p, 2, None) == _lib.B2_ERR_ARG  # ldc < m
    host = np.zeros(64)
    assert L.b2_dgemm_kernel(4, 2, 4, 4, 4, 1.0, host.ctypes.data, p, p, 4,
                             None) == _lib.B2_ERR_ARG  # host operand
    assert L.b2_dgemm_kernel(4, 2, 0, 4, 4, 1.0, p, p, p, 4, None) == 0  # empty: no-op
