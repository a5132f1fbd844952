"""CPU restatement of the device integer arithmetic of the Ozaki DGEMM, checked
in exact Python integers before it runs on a GPU:

* slicing: u = x + 2^62 split into two 32-bit words, sh = dp4a(lo, K_lo,
  dp4a(hi, K_hi, off)), q = umulhi(sh, ceil(2^32/m)), r = sh - q m must equal
  x mod m for every modulus and every |x| < 2^62, with sh < 2^19;
* GEMM epilogue: d < 2^31 (K <= 32768 products of residues <= 255),
  r = d - (umulhi(d, ceil(2^39/m)) >> 7) m must equal d mod m.
"""
import numpy as np

from oracle import ozaki_ref as Z

MASK32 = (1 << 32) - 1


def res_const(m):
    lo = sum(((1 << (8 * j)) % m) << (8 * j) for j in range(4))
    hi = sum(((1 << (8 * (j + 4))) % m) << (8 * j) for j in range(4))
    off = (m - (1 << 62) % m) % m
    mul = ((1 << 32) + m - 1) // m
    return lo, hi, off, mul


def dp4a(a, b, c):
    """Unsigned 4-way byte dot product plus accumulator, modulo 2^32."""
    return (sum(((a >> (8 * j)) & 255) * ((b >> (8 * j)) & 255) for j in range(4)) + c) & MASK32


def residue_u8(x, m):
    lo_c, hi_c, off, mul = res_const(m)
    u = x + (1 << 62)
    assert 0 <= u < (1 << 63)
    lo, hi = u & MASK32, u >> 32
    sh = dp4a(lo, lo_c, dp4a(hi, hi_c, off))
    assert sh < (1 << 19)
    q = (sh * mul) >> 32
    return sh - q * m


def test_byte_weights_fit_a_byte():
    for m in Z.MODULI:
        lo, hi, off, mul = res_const(m)
        assert lo < (1 << 32) and hi < (1 << 32) and off < m and mul < (1 << 32)


def test_slice_residue_matches_exact_modulus():
    rng = np.random.default_rng(0)
    xs = [0, 1, -1, (1 << 62) - 1, -(1 << 62) + 1, (1 << 53), -(1 << 53), 255 * 256, -256]
    xs += [int(v) for v in rng.integers(-(1 << 62) + 1, 1 << 62, 4000, dtype=np.int64)]
    xs += [int(v) << int(e) for v, e in zip(rng.integers(-(1 << 52), 1 << 52, 500),
                                            rng.integers(0, 9, 500))]
    for m in Z.MODULI:
        xs_m = xs + [m * t for t in (1, -1, 12345, -(1 << 40))] + [m * 7 - 1, -m * 7 + 1]
        for x in xs_m:
            if abs(x) >= (1 << 62):
                continue
            assert residue_u8(x, m) == x % m, (m, x)


def test_epilogue_barrett_is_exact_below_2_31():
    rng = np.random.default_rng(1)
    ds = [0, 1, (1 << 31) - 1, 32768 * 255 * 255]
    ds += [int(v) for v in rng.integers(0, 1 << 31, 4000)]
    for m in Z.MODULI:
        m39 = ((1 << 39) + m - 1) // m
        assert m39 < (1 << 32)
        for d in ds + [m * t for t in range(1, 50)] + [(1 << 31) - 1 - t for t in range(300)]:
            q = ((d * m39) >> 32) >> 7
            assert d - q * m == d % m, (m, d)
