"""GPU tests of the blocked DTRSM (dtrsm_ / b2_dtrsm) through the C ABI.

* all 16 side/uplo/trans/diag variants against the oracle (oracle_dtrsm,
  whose Left/Lower/NoTrans path restates the reference's forward substitution
  with the inverted diagonal, dtrsm_kernel_16x4_tester.c:160-199);
* the benchmark configuration's shape family (Left/Lower/N/NonUnit, diagonal
  n + U[0,1)) with trailing updates through plain FP64 and through the INT8
  Ozaki GEMM: residual ||A X - B|| / (||A|| ||X|| n u) stated for each;
* host drop-in with padded leading dimensions, alpha semantics.
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import blas
from oracle import oracle as O

pytestmark = pytest.mark.gpu
U = 2.0 ** -53
VARIANTS = [(s, u, t, d) for s in "LR" for u in "UL" for t in "NT" for d in "NU"]


def _tri(rng, n, uplo):
    a = rng.uniform(-1, 1, (n, n))
    a[np.diag_indices(n)] = n + rng.uniform(0, 1, n)
    return np.asfortranarray(a)


@pytest.mark.parametrize("side,uplo,trans,diag", VARIANTS)
def test_dtrsm_variants_match_oracle(cuda, side, uplo, trans, diag):
    rng = np.random.default_rng(hash((side, uplo, trans, diag)) % 2**32)
    m, n = 257, 131  # several 128-leaves and ragged edges
    na = m if side == "L" else n
    a = _tri(rng, na, uplo)
    b = np.asfortranarray(rng.uniform(-1, 1, (m + 3, n)))
    ref = b.copy(order="F")
    O.trsm(side, uplo, trans, diag, m, n, 1.25, a, ref[:m], nb=0)
    got = b.copy(order="F")
    blas.dtrsm(side, uplo, trans, diag, m, n, 1.25, a, na, got, m + 3)
    assert np.array_equal(got[m:], b[m:]), "padding rows of B were written"
    err = np.linalg.norm(got[:m] - ref[:m]) / np.linalg.norm(ref[:m])
    assert err <= 64 * U * na, (side, uplo, trans, diag, err)


@pytest.mark.parametrize("update", ["fp64", "ozaki"])
def test_dtrsm_residual_left_lower(cuda, update):
    import torch

    rng = np.random.default_rng(4)
    n, nrhs = 2048, 512
    a = np.tril(rng.uniform(-1, 1, (n, n)))
    a[np.diag_indices(n)] = n + np.abs(rng.uniform(0, 1, n))
    b = rng.uniform(-1, 1, (n, nrhs))
    A = torch.from_numpy(np.ascontiguousarray(a.T)).to(cuda)  # column-major
    X = torch.from_numpy(np.ascontiguousarray(b.T)).to(cuda)
    blas.dtrsm_device("L", "L", "N", "N", n, nrhs, 1.0, A, n, X, n, update=update)
    torch.cuda.synchronize()
    x = X.cpu().numpy().T
    res = np.linalg.norm(a @ x - b) / (np.linalg.norm(a) * np.linalg.norm(x) * n * U)
    assert res <= 1.0, res
    ref = O.trsm("L", "L", "N", "N", n, nrhs, 1.0, np.asfortranarray(a),
                 np.asfortranarray(b.copy()), nb=128)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) <= 1e-13


def test_dtrsm_alpha_zero_and_one(cuda):
    rng = np.random.default_rng(5)
    m, n = 40, 30
    a = _tri(rng, m, "L")
    b = np.asfortranarray(np.full((m, n), np.nan))
    blas.dtrsm("L", "L", "N", "N", m, n, 0.0, a, m, b, m)
    assert (b == 0.0).all()  # BLAS: alpha == 0 sets B to zero
    b2 = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    x = b2.copy(order="F")
    blas.dtrsm("L", "L", "N", "U", m, n, 1.0, a, m, x, m)
    t = np.tril(a)
    t[np.diag_indices(m)] = 1.0
    np.testing.assert_allclose(t @ x, b2, rtol=0, atol=1e-12)
