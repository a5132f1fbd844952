"""CPU tests: the oracle restatement is pinned to the reference.

* against the golden vectors in tests/golden/ (reference outputs, always run);
* against the reference itself in oracle/_ref/ when it is built and the host
  has AVX-512F (bit-exact for GEMM: the restatement follows the reference's
  blocking and summation order).
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
HAVE_REF = O.ref_available("DGEMM.so") and O.host_has_avx512f()


def _gemm_golden(name, dtype):
    z = np.load(os.path.join(GOLD, name))
    for i in range(int(z["count"])):
        m, n, k, ta, tb = (int(v) for v in z[f"c{i}_meta"])
        al, be = z[f"c{i}_ab"]
        yield (m, n, k, chr(ta), chr(tb), dtype(al), dtype(be), z[f"c{i}_a"], z[f"c{i}_b"],
               z[f"c{i}_c"], z[f"c{i}_out"])


@pytest.mark.parametrize("name,dtype", [("dgemm_ref.npz", np.float64),
                                        ("sgemm_ref.npz", np.float32)])
def test_oracle_gemm_matches_golden_bitexact(name, dtype):
    n_cases = 0
    for (m, n, k, ta, tb, al, be, a, b, c, out) in _gemm_golden(name, dtype):
        ar = m if ta == "N" else k
        br = k if tb == "N" else n
        got = np.asfortranarray(c.copy())
        O.gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, got[:m])
        assert np.array_equal(got, out), (m, n, k, ta, tb)
        n_cases += 1
    assert n_cases == 28


@pytest.mark.skipif(not HAVE_REF, reason="reference not built here or no AVX-512F")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_gemm_matches_reference_bitexact(dtype):
    rng = np.random.default_rng(5)
    for (m, n, k) in [(3, 4, 5), (64, 33, 1000), (130, 70, 400), (25, 161, 383)]:
        for ta in "NnTC":
            for tb in "NT":
                ar, ac = (m, k) if ta in "Nn" else (k, m)
                br, bc = (k, n) if tb == "N" else (n, k)
                a = np.asfortranarray(rng.uniform(-1, 1, (ar + 2, ac)).astype(dtype))
                b = np.asfortranarray(rng.uniform(-1, 1, (br + 1, bc)).astype(dtype))
                c = np.asfortranarray(rng.uniform(-1, 1, (m + 3, n)).astype(dtype))
                c1, c2 = c.copy(order="F"), c.copy(order="F")
                O.gemm(ta, tb, m, n, k, 1.25, a[:ar], b[:br], -0.5, c1[:m])
                O.ref_gemm(ta, tb, m, n, k, 1.25, a[:ar], b[:br], -0.5, c2[:m])
                assert np.array_equal(c1, c2)


def _gemm8x8_golden():
    z = np.load(os.path.join(GOLD, "dgemm_8x8_ref.npz"))
    for i in range(int(z["count"])):
        m, n, k, ta, tb = (int(v) for v in z[f"e{i}_meta"])
        al, be = z[f"e{i}_ab"]
        yield (str(z[f"e{i}_kind"]), m, n, k, chr(ta), chr(tb), float(al), float(be),
               z[f"e{i}_a"], z[f"e{i}_b"], z[f"e{i}_c"], z[f"e{i}_out"])


def test_oracle_gemm_matches_8x8_reference_drivers():
    """The 8x8 files' own dgemm_ (kernel_avx512_opt8x8.c:821, _standard8x8.c:843)
    block K by 168 / 128 and M by 384 / 512 and fold alpha into the kernel,
    so they agree with the main driver's restatement to rounding only:
    ||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8, padding rows untouched."""
    u = 2.0 ** -53
    kinds = set()
    for (kind, m, n, k, ta, tb, al, be, a, b, c, out) in _gemm8x8_golden():
        ar = m if ta == "N" else k
        br = k if tb == "N" else n
        got = np.asfortranarray(c.copy())
        O.gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, got[:m])
        assert np.array_equal(got[m:], out[m:])
        den = max(k, 1) * u * np.linalg.norm(a[:ar]) * np.linalg.norm(b[:br])
        assert np.linalg.norm(got[:m] - out[:m]) / den <= 8, (kind, m, n, k, ta, tb)
        kinds.add(kind)
    assert kinds == {"8x8opt", "8x8std"}


@pytest.mark.skipif(not (O.ref_available("dgemm_8x8_opt.so") and O.host_has_avx512f()),
                    reason="8x8 reference drivers not built here or no AVX-512F")
def test_8x8_golden_regenerates_from_reference():
    for (kind, m, n, k, ta, tb, al, be, a, b, c, out) in _gemm8x8_golden():
        ar = m if ta == "N" else k
        br = k if tb == "N" else n
        got = np.asfortranarray(c.copy())
        O.ref_gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, got[:m], which=kind)
        assert np.array_equal(got, out), (kind, m, n, k, ta, tb)


def test_oracle_beta_zero_keeps_nan_and_alpha_zero_skips():
    a = np.asfortranarray(np.ones((4, 4)))
    c = np.asfortranarray(np.full((4, 4), np.nan))
    O.gemm("N", "N", 4, 4, 4, 1.0, a, a, 0.0, c)  # gemm_driver.c:131: C *= 0 keeps NaN
    assert np.isnan(c).all()
    a2 = np.asfortranarray(np.full((4, 4), np.nan))
    c2 = np.asfortranarray(np.ones((4, 4)))
    O.gemm("N", "N", 4, 4, 4, 0.0, a2, a2, 2.0, c2)  # :132: alpha == 0 skips the product
    assert (c2 == 2.0).all()


def test_trsm_kernels_match_golden():
    z = np.load(os.path.join(GOLD, "trsm_kernels_ref.npz"))
    worst = 0.0
    for i in range(int(z["count"])):
        M, N, K, s0, s1 = (int(v) for v in z[f"t{i}_meta"])
        kind = chr(s0) + chr(s1)
        sa, sb, c = z[f"t{i}_sa"].copy(), z[f"t{i}_sb"].copy(), z[f"t{i}_c"].copy()
        O.trsm_kernel(kind, M, N, sa, sb, c, K, M)
        packed = sa[: M * N] if kind[0] == "r" else sb[: M * N]
        worst = max(worst, np.abs(c - z[f"t{i}_cout"]).max(),
                    np.abs(packed - z[f"t{i}_packed_out"]).max())
    # the tester's own criterion: maxdiff at rounding level (tester.c:256-257)
    assert worst < 1e-14, worst


def test_gemm3m_kernel_matches_golden():
    z = np.load(os.path.join(GOLD, "zgemm3m_kernel_ref.npz"))
    for i in range(int(z["count"])):
        m, n, k = (int(v) for v in z[f"z{i}_meta"])
        ar, ai = z[f"z{i}_alpha"]
        a, b = np.asfortranarray(z[f"z{i}_a"]), np.asfortranarray(z[f"z{i}_b"])
        c = np.asfortranarray(z[f"z{i}_c"].copy())
        O.gemm3m_kernel_z(m, n, k, ar, ai, a, b, c)
        np.testing.assert_allclose(c, z[f"z{i}_out"], rtol=0, atol=1e-13)


def test_zgemm3m_formula_matches_complex_product():
    rng = np.random.default_rng(3)
    for ta, tb in [("N", "N"), ("T", "N"), ("C", "T"), ("R", "C")]:
        m, n, k = 13, 9, 21
        ar, ac = (m, k) if ta in "NR" else (k, m)
        br, bc = (k, n) if tb in "NR" else (n, k)
        a = np.asfortranarray(rng.uniform(-1, 1, (ar, ac)) + 1j * rng.uniform(-1, 1, (ar, ac)))
        b = np.asfortranarray(rng.uniform(-1, 1, (br, bc)) + 1j * rng.uniform(-1, 1, (br, bc)))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)) + 1j * rng.uniform(-1, 1, (m, n)))
        opa = {"N": a, "T": a.T, "C": a.conj().T, "R": a.conj()}[ta]
        opb = {"N": b, "T": b.T, "C": b.conj().T, "R": b.conj()}[tb]
        al, be = 0.5 - 1.5j, 0.25 + 0.75j
        ref = al * (opa @ opb) + be * c
        got = O.gemm3m(ta, tb, m, n, k, al, a, b, be, c.copy(order="F"))
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13)


@pytest.mark.parametrize("side,uplo,trans,diag", [
    ("L", "L", "N", "N"), ("L", "U", "N", "U"), ("L", "L", "T", "N"), ("L", "U", "T", "N"),
    ("R", "L", "N", "N"), ("R", "U", "N", "N"), ("R", "L", "T", "U"), ("R", "U", "T", "N")])
def test_oracle_dtrsm_solves(side, uplo, trans, diag):
    rng = np.random.default_rng(4)
    m, n = 37, 23
    na = m if side == "L" else n
    a = rng.uniform(-1, 1, (na, na))
    a[np.diag_indices(na)] = na + rng.uniform(0, 1, na)
    a = np.asfortranarray(a)
    b = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    x = O.trsm(side, uplo, trans, diag, m, n, 1.5, a, b.copy(order="F"), nb=8)
    t = np.tril(a) if uplo == "L" else np.triu(a)
    if diag == "U":
        t[np.diag_indices(na)] = 1.0
    opa = t if trans == "N" else t.T
    lhs = opa @ x if side == "L" else x @ opa
    np.testing.assert_allclose(lhs, 1.5 * b, rtol=0, atol=1e-12)


def test_dd_oracle_is_exact_to_double_rounding():
    rng = np.random.default_rng(7)
    a = np.asfortranarray(rng.uniform(-1, 1, (8, 40)))
    b = np.asfortranarray(rng.uniform(-1, 1, (40, 6)))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (8, 6)))
    hi, lo = O.gemm_dd("N", "N", 8, 6, 40, 1.5, a, b, 0.5, c0)
    for i, j in [(0, 0), (3, 5), (7, 2)]:
        ex = Fraction(1.5) * sum(Fraction(a[i, k]) * Fraction(b[k, j]) for k in range(40)) \
            + Fraction(0.5) * Fraction(c0[i, j])
        err = abs(Fraction(hi[i, j]) + Fraction(lo[i, j]) - ex)
        assert err <= abs(ex) * Fraction(2) ** -100


def test_comparer_flags_planted_corruption():
    """Fault injection on the host, as sgemm.c:584 plants it: one corrupted
    element of C must push the parity yardstick far past the bound of 8."""
    from tests._util import normalized

    rng = np.random.default_rng(9)
    m, n, k = 91, 45, 31
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)).astype(np.float32))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)).astype(np.float32))
    c = np.asfortranarray(np.zeros((m, n), np.float32))
    ref = O.gemm("N", "N", m, n, k, 1.0, a, b, 0.0, c.copy(order="F"))
    good = O.gemm("N", "N", m, n, k, 1.0, a, b, 0.0, c.copy(order="F"))
    bad = good.copy(order="F")
    bad.reshape(-1, order="F")[101] *= 2.0
    u = np.finfo(np.float32).eps / 2
    assert normalized(good, ref, k, a, b, u) <= 8
    assert normalized(bad, ref, k, a, b, u) > 8


def test_blas_trsm_oracle_agrees_with_reference_lt_kernel_semantics():
    """The tester's 'lt' reference (dtrsm_kernel_16x4_tester.c:160-199) solves a
    lower triangle packed with its diagonal inverted, after adding the GEMM
    update sb to C.  Unpacking that triangle and calling the BLAS-level
    oracle_dtrsm (Left/Lower/NoTrans) on C + update gives the same X."""
    rng = np.random.default_rng(11)
    M, N = 16, 12
    sa = rng.uniform(0.5, 1.5, M * M)
    # lower triangle L with L[i, i] = 1 / sa[i*M + i] and L[i, k] = sa[k*M + i] for i > k
    L = np.zeros((M, M))
    for k in range(M):
        L[k, k] = 1.0 / sa[k * M + k]
        for i in range(k + 1, M):
            L[i, k] = sa[k * M + i]
    sb = rng.uniform(-1, 1, N * M)
    C = rng.uniform(-1, 1, M * N)
    c_kern = C.copy()
    O.trsm_kernel("lt", M, N, sa.copy(), sb.copy(), c_kern, M, M)
    upd = np.zeros((M, N))
    n0 = 0
    while n0 < N:  # sb holds the update in 4-column panels, k-major within a panel
        w = min(4, N - n0)
        blk = sb[n0 * M: n0 * M + w * M].reshape(M, w)
        upd[:, n0:n0 + w] = blk
        n0 += w
    rhs = np.asfortranarray(C.reshape(N, M).T + upd)
    x = O.trsm("L", "L", "N", "N", M, N, 1.0, np.asfortranarray(L), rhs, nb=0)
    np.testing.assert_allclose(x, c_kern.reshape(N, M).T, rtol=0, atol=1e-12)
