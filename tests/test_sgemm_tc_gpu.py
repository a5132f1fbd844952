"""GPU tests of the tensor-core SGEMM forms (1xTF32, 3xTF32, 3xBF16 on tcgen05,
FP32 accumulation in TMEM) through the C ABI.

Parity bar: ||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8 against
the reference sgemm_ (oracle, bit-exact restatement), with u the unit
roundoff of the arithmetic each method actually performs: 1xTF32 rounds the
inputs to 11 significant bits (u = 2^-11), the split forms carry ~22 (TF32)
and ~16 (BF16) bits of each input (u = 2^-21, 2^-16).  Each method also
states its accuracy against an FP64 product; the tensor core's FP32
accumulation adds an error that grows with K, so those bounds scale with K.
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import blas
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu
U_METHOD = {"tf32": 2.0 ** -11, "tf32x3": 2.0 ** -21, "bf16x3": 2.0 ** -16}
METHODS = ["tf32", "tf32x3", "bf16x3"]
# normwise error vs FP64 per method: constant part + K-proportional part
BOUND = {"tf32": (2e-3, 0.0), "tf32x3": (2e-6, 2e-8), "bf16x3": (4e-5, 1e-8)}


def _run(dev, meth, ta, tb, m, n, k, alpha, a, b, beta, c):
    import torch

    da, db, dc = (torch.from_numpy(np.asfortranarray(x).T.copy()).to(dev) for x in (a, b, c))
    blas.sgemm_device(ta, tb, m, n, k, alpha, da, a.shape[0], db, b.shape[0], beta, dc,
                      c.shape[0], method=meth)
    torch.cuda.synchronize()
    return np.asfortranarray(dc.cpu().numpy().T)


@pytest.mark.parametrize("meth", METHODS)
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (37, 53, 29), (129, 65, 385), (300, 257, 1000),
                                   (1024, 1024, 1024), (2048, 160, 1536)])
def test_parity_with_reference_sgemm(cuda, meth, m, n, k):
    # shapes with fewer output tiles than SMs run split-K (partials + reduction)
    rng = np.random.default_rng(m * 3 + k)
    for ta, tb in [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")]:
        a = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)).astype(np.float32))
        b = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)).astype(np.float32))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(np.float32))
        ref = O.gemm(ta, tb, m, n, k, np.float32(1.5), a, b, np.float32(0.5), c.copy(order="F"))
        got = _run(cuda, meth, ta, tb, m, n, k, 1.5, a, b, 0.5, c)
        assert normalized(got, ref, k, a, b, U_METHOD[meth]) <= 8, (meth, m, n, k, ta, tb)
        # method accuracy vs the FP64 product
        opa = (a if ta == "N" else a.T).astype(np.float64)
        opb = (b if tb == "N" else b.T).astype(np.float64)
        prod = 1.5 * opa @ opb
        exact = prod + 0.5 * c.astype(np.float64)
        c0, ck = BOUND[meth]
        scale = np.linalg.norm(np.abs(prod) + np.abs(0.5 * c))  # no credit for cancellation
        err = np.linalg.norm(got - exact) / scale
        assert err <= c0 + ck * k, (meth, m, n, k, ta, tb, err)


@pytest.mark.parametrize("meth", METHODS)
def test_dropin_sgemm_method_and_semantics(cuda, meth):
    rng = np.random.default_rng(3)
    m, n, k = 200, 150, 300
    a = np.asfortranarray(rng.uniform(-1, 1, (m + 1, k)).astype(np.float32))
    b = np.asfortranarray(rng.uniform(-1, 1, (k + 2, n)).astype(np.float32))
    c = np.asfortranarray(np.full((m + 3, n), np.nan, np.float32))
    blas.set_sgemm_method(meth)
    try:
        got = c.copy(order="F")
        blas.sgemm("N", "N", m, n, k, 1.0, a, m + 1, b, k + 2, 0.0, got, m + 3)
        # beta == 0 keeps NaN already in C (src/gemm_driver.c:131), padding untouched
        assert np.isnan(got[:m]).all() and np.isnan(got[m:]).all()
        c2 = np.asfortranarray(rng.uniform(-1, 1, (m + 3, n)).astype(np.float32))
        got2 = c2.copy(order="F")
        blas.sgemm("N", "N", m, n, k, 0.0, a, m + 1, b, k + 2, 2.0, got2, m + 3)
        assert np.array_equal(got2[:m], 2.0 * c2[:m]) and np.array_equal(got2[m:], c2[m:])
    finally:
        blas.set_sgemm_method("fp32")
