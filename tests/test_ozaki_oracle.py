"""CPU tests of the Ozaki-II restatement: it emulates the reference dgemm_
within the scheme's stated truncation bound, the CRT step is exact, and the
error falls as moduli are added."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ozaki_ref as Z


def test_moduli_pairwise_coprime_and_table():
    for i, a in enumerate(Z.MODULI):
        for b in Z.MODULI[i + 1:]:
            assert math.gcd(a, b) == 1
    # H grows ~4 bits per modulus, and 2H + 2 <= log2(P)
    for s in range(2, 17):
        log2p = sum(math.log2(m) for m in Z.MODULI[:s])
        assert 2 * Z.h_for(s) + 2 <= log2p
    assert Z.h_for(14) == 54


def test_crt_roundtrip_is_exact():
    rng = np.random.default_rng(0)
    mods = Z.MODULI[:14]
    P = math.prod(mods)
    W = [(P // m) * pow((P // m) % m, -1, m) for m in mods]
    for _ in range(200):
        x = int(rng.integers(-2**62, 2**62)) * int(rng.integers(1, 2**40))
        if abs(x) >= P // 2:
            continue
        acc = sum((x % m) * w for m, w in zip(mods, W)) % P
        if acc > P // 2:
            acc -= P
        assert acc == x


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_emulation_matches_reference_dgemm(ta, tb):
    rng = np.random.default_rng(1)
    m, n, k = 7, 5, 33
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)) *
                          np.exp(2 * rng.standard_normal((m, k) if ta == "N" else (k, m))))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)))
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    ref = O.gemm(ta, tb, m, n, k, 1.5, a, b, 0.5, c.copy(order="F"))
    emu = Z.emulate(ta, tb, m, n, k, 1.5, a, b, 0.5, c, s=14)
    u = 2.0 ** -53
    den = k * u * np.linalg.norm(a) * np.linalg.norm(b)
    assert np.linalg.norm(emu - ref) / den <= 8


def test_error_falls_with_moduli():
    rng = np.random.default_rng(2)
    m, n, k = 4, 4, 64
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    c = np.zeros((m, n), order="F")
    hi, _ = O.gemm_dd("N", "N", m, n, k, 1.0, a, b, 0.0, c)
    errs = [np.linalg.norm(Z.emulate("N", "N", m, n, k, 1.0, a, b, 0.0, c, s=s) - hi)
            for s in (4, 6, 8, 10)]
    assert errs[0] > errs[1] > errs[2] > errs[3]
    # stated bound: per element < 2 sqrt(K) 2^-H ||a_i|| ||b_j|| (+ final rounding)
    for s in (4, 6, 8):
        emu = Z.emulate("N", "N", m, n, k, 1.0, a, b, 0.0, c, s=s)
        bound = 2 * math.sqrt(k) * 2.0 ** -Z.h_for(s) * np.outer(np.linalg.norm(a, axis=1),
                                                               np.linalg.norm(b, axis=0))
        assert np.all(np.abs(emu - hi) <= bound + 4 * np.spacing(np.abs(hi)))


def test_integer_inputs_are_exact():
    rng = np.random.default_rng(3)
    m, n, k = 6, 5, 40
    a = np.asfortranarray(rng.integers(-1000, 1000, (m, k)).astype(np.float64))
    b = np.asfortranarray(rng.integers(-1000, 1000, (k, n)).astype(np.float64))
    c = np.zeros((m, n), order="F")
    exact = a @ b  # integers < 2^53: exact in float64
    assert np.array_equal(Z.emulate("N", "N", m, n, k, 1.0, a, b, 0.0, c, s=10), exact)
