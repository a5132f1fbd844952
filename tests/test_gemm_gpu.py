"""GPU parity: the CUDA GEMM paths against the oracle (which is bit-exact with the
reference's own dgemm_/sgemm_) and the golden vectors, through the C ABI.

Bar: ||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8 (normalized error vs the
reference on the same seeded inputs), padding rows of C untouched."""
import os

import numpy as np
import pytest

from gemm_avx512f_b200 import blas
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 8.0

SHAPES = [(1, 1, 1), (7, 5, 3), (37, 53, 29), (129, 65, 385), (513, 129, 1031), (64, 64, 4096),
          (300, 1000, 17), (1, 700, 300)]
AB = [(1.5, 0.5), (1.0, 0.0), (1.0, 1.0), (-0.7, 2.0)]


def _case(rng, dtype, m, n, k, ta, tb, pad=3):
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ar + pad, ac)).astype(dtype))
    b = np.asfortranarray(rng.uniform(-1, 1, (br + pad, bc)).astype(dtype))
    c = np.asfortranarray(rng.uniform(-1, 1, (m + pad, n)).astype(dtype))
    return a, b, c, ar, br


@pytest.mark.parametrize("m,n,k", SHAPES)
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_dgemm_dropin_host_parity(cuda, m, n, k, ta, tb):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a, b, c, ar, br = _case(rng, np.float64, m, n, k, ta, tb)
    u = np.finfo(np.float64).eps / 2
    for al, be in AB:
        ref = c.copy(order="F")
        O.gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, ref[:m])
        got = c.copy(order="F")
        blas.dgemm(ta, tb, m, n, k, al, a, a.shape[0], b, b.shape[0], be, got, got.shape[0])
        assert np.array_equal(got[m:], c[m:]), "padding rows of C were written"
        e = normalized(got[:m], ref[:m], k, a[:ar], b[:br], u)
        assert e <= TOL, (m, n, k, ta, tb, al, be, e)


@pytest.mark.parametrize("method", ["fp64", "ozaki"])
def test_dgemm_dropin_matches_8x8_reference_drivers(cuda, method):
    """Golden outputs of the 8x8 files' own dgemm_ drivers
    (kernel_avx512_opt8x8.c:821, kernel_avx512_standard8x8.c:843)."""
    z = np.load(os.path.join(GOLD, "dgemm_8x8_ref.npz"))
    u = np.finfo(np.float64).eps / 2
    blas.set_dgemm_method(method, 0)
    try:
        for i in range(int(z["count"])):
            m, n, k, ta, tb = (int(v) for v in z[f"e{i}_meta"])
            ta, tb = chr(ta), chr(tb)
            al, be = (float(v) for v in z[f"e{i}_ab"])
            a, b, c, out = z[f"e{i}_a"], z[f"e{i}_b"], z[f"e{i}_c"], z[f"e{i}_out"]
            ar = m if ta == "N" else k
            br = k if tb == "N" else n
            got = np.asfortranarray(c.copy())
            blas.dgemm(ta, tb, m, n, k, al, a, a.shape[0], b, b.shape[0], be, got, got.shape[0])
            assert np.array_equal(got[m:], c[m:]), "padding rows of C were written"
            e = normalized(got[:m], out[:m], k, a[:ar], b[:br], u)
            assert e <= TOL, (str(z[f"e{i}_kind"]), m, n, k, ta, tb, e)
    finally:
        blas.set_dgemm_method("fp64", 0)


def _pinned(x):
    """A copy of the Fortran array x in page-locked host memory."""
    import torch

    t = torch.empty(x.size, dtype=torch.from_numpy(x[:1, :1].copy()).dtype).pin_memory()
    y = t.numpy().reshape(x.shape, order="F")
    y[...] = x
    return y, t  # keep t alive with y


def test_process_exits_after_pageable_copies(cuda, tmp_path):
    """Pageable operands of 8 MiB are copied into the bounce buffers by the
    library's host copy threads; a process that used them must still exit
    promptly (the threads outlive every static destructor)."""
    import subprocess
    import sys

    script = tmp_path / "pageable_exit.py"
    script.write_text(
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "from gemm_avx512f_b200 import blas\n"
        "rng = np.random.default_rng(5)\n"
        "n = 1024\n"
        "a = np.asfortranarray(rng.uniform(-1, 1, (n, n)))\n"
        "b = np.asfortranarray(rng.uniform(-1, 1, (n, n)))\n"
        "c = np.zeros((n, n), order='F')\n"
        "blas.dgemm('N', 'N', n, n, n, 1.0, a, n, b, n, 0.0, c, n)\n"
        "e = np.abs(c - a @ b).max()\n"
        "print('MAXERR', e)\n"
        "sys.exit(0 if e < 1e-10 else 1)\n")
    r = subprocess.run([sys.executable, str(script)], capture_output=True, text=True,
                       timeout=180, cwd=ROOT, env=dict(os.environ, B2_METHOD="fp64"))
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.parametrize("host", ["pinned", "pageable"])
@pytest.mark.parametrize("method,plant_nan", [("fp64", True), ("ozaki", True), ("fp64", False),
                                              ("ozaki", False)])
def test_dgemm_dropin_pipelined_host_operands(cuda, method, plant_nan, host):
    """Pinned host operands of a product >= 2^32 flops go through the
    column-block copy/compute/copy pipeline; blocks of 256-multiples leave a
    ragged last block here (n = 1800), and op(B) blocks are row blocks of B
    for 'T'.  Pageable (malloc'ed) operands go through the library's pinned
    bounce buffers in one block instead.  beta == 0 with an all-finite C skips
    copying C in (the device blocks are zeroed); a NaN in C makes the library
    copy it, and the NaN survives."""
    m, n, k = 1000, 1800, 1300
    rng = np.random.default_rng(77)
    u = np.finfo(np.float64).eps / 2
    blas.set_dgemm_method(method, 0)
    keep = []
    try:
        for ta, tb in [("N", "N"), ("T", "T")]:
            a, b, c, ar, br = _case(rng, np.float64, m, n, k, ta, tb)
            if host == "pinned":
                (a, ka), (b, kb) = _pinned(a), _pinned(b)
                keep += [ka, kb]
            if plant_nan:
                c[5, 1700] = np.nan  # beta == 0 still multiplies C: NaN survives, as in the reference
            ref = c.copy(order="F")
            O.gemm(ta, tb, m, n, k, 1.25, a[:ar], b[:br], 0.0, ref[:m])
            got = c.copy(order="F")
            if host == "pinned":
                got, kc = _pinned(got)
                keep.append(kc)
            blas.dgemm(ta, tb, m, n, k, 1.25, a, a.shape[0], b, b.shape[0], 0.0, got,
                       got.shape[0])
            assert np.array_equal(got[m:], c[m:]), "padding rows of C were written"
            assert np.isnan(got[5, 1700]) == plant_nan and np.isnan(ref[5, 1700]) == plant_nan
            fin = np.isfinite(ref[:m])
            assert fin.sum() == m * n - (1 if plant_nan else 0)
            g, r = np.where(fin, got[:m], 0.0), np.where(fin, ref[:m], 0.0)
            e = normalized(g, r, k, a[:ar], b[:br], u)
            assert e <= TOL, (method, ta, tb, e)
    finally:
        blas.set_dgemm_method("fp64", 0)


def test_sgemm_dropin_pipelined_host_operands(cuda):
    m, n, k = 900, 2100, 1500
    rng = np.random.default_rng(78)
    u = np.finfo(np.float32).eps / 2
    a, b, c, ar, br = _case(rng, np.float32, m, n, k, "N", "T")
    ref = c.copy(order="F")
    O.gemm("N", "T", m, n, k, 0.5, a[:ar], b[:br], 2.0, ref[:m])
    got = c.copy(order="F")
    blas.sgemm("N", "T", m, n, k, 0.5, a, a.shape[0], b, b.shape[0], 2.0, got, got.shape[0])
    assert np.array_equal(got[m:], c[m:])
    assert normalized(got[:m], ref[:m], k, a[:ar], b[:br], u) <= TOL


@pytest.mark.parametrize("m,n,k", [(37, 53, 29), (513, 129, 1031), (1024, 1024, 1024)])
def test_sgemm_dropin_host_parity(cuda, m, n, k):
    rng = np.random.default_rng(k)
    u = np.finfo(np.float32).eps / 2
    for ta, tb in [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")]:
        a, b, c, ar, br = _case(rng, np.float32, m, n, k, ta, tb)
        for al, be in AB:
            ref = c.copy(order="F")
            O.gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, ref[:m])
            got = c.copy(order="F")
            blas.sgemm(ta, tb, m, n, k, al, a, a.shape[0], b, b.shape[0], be, got, got.shape[0])
            assert np.array_equal(got[m:], c[m:])
            e = normalized(got[:m], ref[:m], k, a[:ar], b[:br], u)
            assert e <= TOL, (m, n, k, ta, tb, al, be, e)


@pytest.mark.parametrize("name,dtype", [("dgemm_ref.npz", np.float64),
                                        ("sgemm_ref.npz", np.float32)])
def test_gemm_matches_reference_golden(cuda, name, dtype):
    z = np.load(os.path.join(GOLD, name))
    u = np.finfo(dtype).eps / 2
    fn = blas.dgemm if dtype == np.float64 else blas.sgemm
    for i in range(int(z["count"])):
        m, n, k, ta, tb = (int(v) for v in z[f"c{i}_meta"])
        ta, tb = chr(ta), chr(tb)
        al, be = (float(v) for v in z[f"c{i}_ab"])
        a, b, c, out = z[f"c{i}_a"], z[f"c{i}_b"], z[f"c{i}_c"], z[f"c{i}_out"]
        got = np.asfortranarray(c.copy())
        fn(ta, tb, m, n, k, al, np.asfortranarray(a), a.shape[0], np.asfortranarray(b),
           b.shape[0], be, got, got.shape[0])
        ar = m if ta == "N" else k
        br = k if tb == "N" else n
        assert np.array_equal(got[m:], out[m:])
        assert normalized(got[:m], out[:m], k, a[:ar], b[:br], u) <= TOL


def test_dgemm_reference_semantics_edges(cuda):
    # beta == 0 keeps NaN already in C (src/gemm_driver.c:131)
    a = np.asfortranarray(np.ones((8, 8)))
    c = np.asfortranarray(np.full((8, 8), np.nan))
    blas.dgemm("N", "N", 8, 8, 8, 1.0, a, 8, a, 8, 0.0, c, 8)
    assert np.isnan(c).all()
    # alpha == 0 skips the product entirely (:132): NaN in A does not reach C
    an = np.asfortranarray(np.full((8, 8), np.nan))
    c2 = np.asfortranarray(np.ones((8, 8)))
    blas.dgemm("N", "N", 8, 8, 8, 0.0, an, 8, an, 8, 3.0, c2, 8)
    assert (c2 == 3.0).all()
    # K == 0: C <- beta*C
    c3 = np.asfortranarray(np.full((5, 4), 2.0))
    blas.dgemm("N", "N", 5, 4, 0, 1.0, a, 8, a, 8, 0.25, c3, 5)
    assert (c3 == 0.5).all()
    # M == 0 / N == 0: quick return, C untouched
    c4 = np.asfortranarray(np.full((5, 4), 7.0))
    blas.dgemm("N", "N", 0, 4, 3, 1.0, a, 8, a, 8, 0.0, c4, 5)
    blas.dgemm("N", "N", 5, 0, 3, 1.0, a, 8, a, 8, 0.0, c4, 5)
    assert (c4 == 7.0).all()


def test_dgemm_device_pointers_and_odd_leading_dims(cuda):
    import torch

    rng = np.random.default_rng(21)
    m, n, k = 333, 257, 511
    u = np.finfo(np.float64).eps / 2
    for lda, ldb, ldc in [(m, k, m), (m + 1, k + 3, m + 5)]:  # odd ld -> 8-byte loads
        a = np.asfortranarray(rng.uniform(-1, 1, (lda, k)))
        b = np.asfortranarray(rng.uniform(-1, 1, (ldb, n)))
        c = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)))
        ref = c.copy(order="F")
        O.gemm("N", "N", m, n, k, 1.5, a[:m], b[:k], 0.5, ref[:m])
        ta, tb, tc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))  # col-major
        blas.dgemm_device("N", "N", m, n, k, 1.5, ta, lda, tb, ldb, 0.5, tc, ldc)
        torch.cuda.synchronize()
        got = np.asfortranarray(tc.cpu().numpy().T)
        assert np.array_equal(got[m:], c[m:])
        assert normalized(got[:m], ref[:m], k, a[:m], b[:k], u) <= TOL


def test_dd_kernel_matches_cpu_dd_oracle(cuda):
    import torch

    rng = np.random.default_rng(8)
    m, n, k = 70, 45, 333
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (n, k)))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    hi_ref, lo_ref = O.gemm_dd("N", "T", m, n, k, 1.5, a, b, 0.5, c0)
    ta, tb, tc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c0))
    hi = torch.zeros((n, m), dtype=torch.float64, device=cuda)
    lo = torch.zeros_like(hi)
    blas.dgemm_dd_device("N", "T", m, n, k, 1.5, ta, m, tb, n, 0.5, tc, m, hi, lo, m)
    torch.cuda.synchronize()
    h, l = hi.cpu().numpy().T, lo.cpu().numpy().T
    # both are ~2^-100 accurate: their difference is far below one FP64 ulp
    err = np.abs((h - hi_ref) + (l - lo_ref)).max()
    assert err <= 2.0 ** -90 * np.abs(hi_ref).max()


def test_error_stats_of_fp64_path(cuda):
    import torch

    rng = np.random.default_rng(10)
    m = n = k = 512
    a, b, c = (torch.from_numpy(rng.uniform(-1, 1, (m, m))).to(cuda) for _ in range(3))
    out = c.clone()
    blas.dgemm_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, out, m)
    nw, me = blas.dgemm_error_device("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, out, m)
    assert 0 < nw < 1e-14 and 0 < me < 1e-13
