"""GPU tests of the INT8 Ozaki-II DGEMM (tcgen05 kind::i8), through the C ABI.

* stage-by-stage agreement with the exact-integer CPU restatement
  (oracle/ozaki_ref.py) to a few ulps;
* parity with the reference dgemm_ (oracle, bit-exact restatement):
  ||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8;
* size-independent properties at larger sizes: integer inputs come out exact,
  Inf/NaN propagate like FP64, K beyond one exact INT32 pass is chunked;
* equal-error claim: normwise error vs the double-double product within 2x
  of the plain FP64 path's on the exponent-spread inputs of the benchmark.
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import _lib, blas
from oracle import oracle as O
from oracle import ozaki_ref as Z
from tests._util import normalized

pytestmark = pytest.mark.gpu
U = 2.0 ** -53


def _dev(x, dev):
    import torch

    return torch.from_numpy(np.asfortranarray(x).T.copy()).to(dev)


def _host(t):
    return np.asfortranarray(t.cpu().numpy().T)


def _run(dev, ta, tb, m, n, k, alpha, a, b, beta, c, method="ozaki", slices=0):
    import torch

    da, db, dc = _dev(a, dev), _dev(b, dev), _dev(c, dev)
    blas.dgemm_device(ta, tb, m, n, k, alpha, da, a.shape[0], db, b.shape[0], beta, dc,
                      c.shape[0], method=method, slices=slices)
    torch.cuda.synchronize()
    return _host(dc)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("s", [6, 10, 14])
def test_matches_cpu_restatement(cuda, ta, tb, s):
    rng = np.random.default_rng(s)
    for (m, n, k) in [(7, 5, 33), (37, 21, 130)]:
        a = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)) *
                              np.exp(rng.standard_normal((m, k) if ta == "N" else (k, m))))
        b = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
        want = Z.emulate(ta, tb, m, n, k, 1.5, a, b, 0.5, c, s=s)
        got = _run(cuda, ta, tb, m, n, k, 1.5, a, b, 0.5, c, slices=s)
        # the final alpha*C' + beta*C rounds on the scale of its terms, which
        # can be far larger than the (cancelled) result
        opa = a if ta == "N" else a.T
        opb = b if tb == "N" else b.T
        scale = np.maximum(np.abs(1.5 * (opa @ opb)), np.abs(0.5 * c))
        tol = 4 * np.spacing(np.maximum(scale, np.abs(want)))
        assert np.all(np.abs(got - want) <= tol), (m, n, k, np.abs(got - want).max())


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (129, 65, 385), (513, 129, 1031), (300, 700, 64),
                                   (1024, 1024, 1024)])
def test_parity_with_reference_dgemm(cuda, m, n, k):
    rng = np.random.default_rng(m + n + k)
    for ta, tb in [("N", "N"), ("T", "T"), ("N", "T"), ("T", "N")]:
        a = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)))
        b = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
        ref = O.gemm(ta, tb, m, n, k, 1.5, a, b, 0.5, c.copy(order="F"))
        got = _run(cuda, ta, tb, m, n, k, 1.5, a, b, 0.5, c)
        assert normalized(got, ref, k, a, b, U) <= 8


def test_dropin_dgemm_with_ozaki_method(cuda):
    rng = np.random.default_rng(5)
    m, n, k = 200, 150, 300
    a = np.asfortranarray(rng.uniform(-1, 1, (m + 2, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k + 1, n)))
    c = np.asfortranarray(rng.uniform(-1, 1, (m + 3, n)))
    ref = O.gemm("N", "N", m, n, k, -0.7, a[:m], b[:k], 2.0, c.copy(order="F")[:m])
    blas.set_dgemm_method("ozaki", 0)
    try:
        got = c.copy(order="F")
        blas.dgemm("N", "N", m, n, k, -0.7, a, m + 2, b, k + 1, 2.0, got, m + 3)
    finally:
        blas.set_dgemm_method("fp64", 0)
    assert np.array_equal(got[m:], c[m:])
    assert normalized(got[:m], ref, k, a[:m], b[:k], U) <= 8


def test_integer_inputs_exact(cuda):
    rng = np.random.default_rng(6)
    m, n, k = 640, 384, 2000
    a = rng.integers(-1000, 1000, (m, k)).astype(np.float64)
    b = rng.integers(-1000, 1000, (k, n)).astype(np.float64)
    c = np.zeros((m, n))
    got = _run(cuda, "N", "N", m, n, k, 1.0, a, b, 0.0, c)
    assert np.array_equal(got, a @ b)


def test_nonfinite_propagates_like_fp64(cuda):
    rng = np.random.default_rng(7)
    m, n, k = 64, 48, 96
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    a[3, 5] = np.nan
    a[10, 2] = np.inf
    b[7, 9] = -np.inf
    c = rng.uniform(-1, 1, (m, n))
    f = _run(cuda, "N", "N", m, n, k, 1.0, a, b, 1.0, c, method="fp64")
    z = _run(cuda, "N", "N", m, n, k, 1.0, a, b, 1.0, c, method="ozaki")
    assert np.array_equal(np.isnan(f), np.isnan(z))
    assert np.array_equal(np.isinf(f), np.isinf(z))
    fin = np.isfinite(f)
    assert np.abs(f[fin] - z[fin]).max() < 1e-12


def test_zero_operand_and_beta_semantics(cuda):
    m, n, k = 40, 30, 20
    a = np.zeros((m, k))
    b = np.ones((k, n))
    c = np.full((m, n), np.nan)
    z = _run(cuda, "N", "N", m, n, k, 1.0, a, b, 0.0, c)
    assert np.isnan(z).all()  # beta == 0 keeps NaN (src/gemm_driver.c:131)
    c2 = np.full((m, n), 2.0)
    z2 = _run(cuda, "N", "N", m, n, k, 1.0, a, b, 0.5, c2)
    assert (z2 == 1.0).all()


def test_long_k_is_chunked(cuda):
    rng = np.random.default_rng(8)
    m, n, k = 24, 16, 70000
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    c = np.zeros((m, n), order="F")
    ref = O.gemm("N", "N", m, n, k, 1.0, a, b, 0.0, c.copy(order="F"))
    got = _run(cuda, "N", "N", m, n, k, 1.0, a, b, 0.0, c)
    plan = (__import__("ctypes").c_int * 2)()
    _lib.lib().b2_ozaki_last_plan(plan, 2)
    assert plan[1] == -(-k // 32768)  # exact INT32 passes of at most 32768
    assert normalized(got, ref, k, a, b, U) <= 8


@pytest.mark.parametrize("phi", [0.1, 1.0, 4.0])
def test_error_within_2x_of_fp64(cuda, phi):
    import torch

    n = 2048
    rng = np.random.default_rng(2)
    a = rng.uniform(-1, 1, n * n) * np.exp(phi * rng.standard_normal(n * n))
    b = rng.uniform(-1, 1, n * n) * np.exp(phi * rng.standard_normal(n * n))
    A, B = (torch.from_numpy(x).to(cuda) for x in (a, b))
    C = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    errs = {}
    plan = (__import__("ctypes").c_int * 2)()
    for meth in ("fp64", "ozaki"):
        out = C.clone()
        blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, out, n, method=meth)
        if meth == "ozaki":
            _lib.lib().b2_ozaki_last_plan(plan, 2)
        errs[meth] = blas.dgemm_error_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, out, n)
    # automatic count: 15 moduli, 16 for heavy-tailed rows (phi = 4)
    assert plan[0] == (16 if phi >= 4 else 15), (phi, plan[0])
    assert errs["ozaki"][0] <= 2.0 * errs["fp64"][0], errs
    assert _lib.lib().b2_device_error(0) == 0


def test_explicit_modulus_count_is_kept_for_heavy_tails(cuda):
    import torch

    n = 512
    rng = np.random.default_rng(12)
    a = rng.uniform(-1, 1, n * n) * np.exp(4.0 * rng.standard_normal(n * n))
    b = rng.uniform(-1, 1, n * n) * np.exp(4.0 * rng.standard_normal(n * n))
    A, B = (torch.from_numpy(x).to(cuda) for x in (a, b))
    plan = (__import__("ctypes").c_int * 2)()
    for s in (14, 15):
        out = torch.zeros(n * n, dtype=torch.float64, device=cuda)
        blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, out, n, method="ozaki",
                          slices=s)
        _lib.lib().b2_ozaki_last_plan(plan, 2)
        assert plan[0] == s


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T")])
def test_overlapped_column_blocks_ragged(cuda, ta, tb):
    """Products large enough for the overlapped schedule run C in column
    blocks of B on two streams (here 2 ragged blocks: n = 4173 -> 2304 + 1869
    columns, m = 8492 rows).  Against the plain FP64 path on the same device
    inputs, with alpha/beta and a NaN planted in one row of A and one column of
    B (recomputed by the direct dot product inside their blocks)."""
    import torch

    m, n, k = 8492, 4173, 2000
    g = torch.Generator(device=cuda).manual_seed(5)
    ar, br = (m, k) if ta == "N" else (k, m), (k, n) if tb == "N" else (n, k)
    A = (torch.rand(ar[1], ar[0], device=cuda, dtype=torch.float64, generator=g) * 2 - 1)
    B = (torch.rand(br[1], br[0], device=cuda, dtype=torch.float64, generator=g) * 2 - 1)
    C0 = torch.rand(n, m, device=cuda, dtype=torch.float64, generator=g)
    # element (row 6000 of op(A), k = 7) and (k = 11, column 3000 of op(B))
    if ta == "N":
        A[7, 6000] = float("nan")
    else:
        A[6000, 7] = float("nan")
    if tb == "N":
        B[3000, 11] = float("nan")
    else:
        B[11, 3000] = float("nan")
    out = {}
    for method in ("ozaki", "fp64"):
        C = C0.clone()
        blas.dgemm_device(ta, tb, m, n, k, 1.25, A, ar[0], B, br[0], -0.5, C, m, method=method)
        torch.cuda.synchronize()
        out[method] = C.t()  # m x n
    oz, fp = out["ozaki"], out["fp64"]
    nan_oz, nan_fp = torch.isnan(oz), torch.isnan(fp)
    assert torch.equal(nan_oz, nan_fp)
    assert bool(nan_fp[6000].all()) and bool(nan_fp[:, 3000].all())
    fin = ~nan_fp
    den = k * U * float(torch.linalg.norm(torch.nan_to_num(A))) * float(torch.linalg.norm(torch.nan_to_num(B)))
    err = float(torch.linalg.norm(torch.where(fin, oz - fp, torch.zeros_like(oz)))) / den
    assert err <= 8, (ta, tb, err)
