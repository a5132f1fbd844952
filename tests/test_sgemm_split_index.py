"""CPU restatement of the index arithmetic of the SGEMM tensor-core path
(csrc/sgemm_tc.cu split_kernel and the three-term interleave of the umma.cuh
producer), checked before any GPU run:

* split_kernel: every 16-byte vector load stays inside the operand and is
  aligned when the host enables it; every tile cell is loaded once from the
  right element; every element of the padded output rows [r][t*kp + k] is
  written exactly once, by an aligned 16-byte store inside the row.
* interleave: K' block j reads term j % 3 of K block j / 3 from segment
  bit(t) of each operand's [big | small] storage; every coordinate plus its
  box stays inside the 2*kp extent, is a multiple of 128 bytes, and the three
  (X, Y) segment pairs are (Bb, Ab), (Bs, Ab), (Bb, As) for every K block."""
import pytest


def _split(R, K, esz, terms, rowcont, ld, vec):
    kp = -(-K // (128 // esz)) * (128 // esz)
    sr, sk = (1, ld) if rowcont else (ld, 1)
    extent = ((ld * (K - 1) + R) if rowcont else (ld * (R - 1) + K)) * 4
    written = set()
    for bx in range(-(-kp // 64)):
        for by in range(-(-R // 32)):
            k0, r0 = bx * 64, by * 32
            tile = {}
            for tid in range(256):
                if vec:
                    for e in range(2):
                        idx = tid + 256 * e
                        if rowcont:
                            kk, rr = idx >> 3, (idx & 7) * 4
                            r, k = r0 + rr, k0 + kk
                            if k < K:
                                off = (r + k * sk) * 4
                                if r + 3 < R:
                                    assert off % 16 == 0 and off + 16 <= extent
                                for j in range(4):
                                    if r + j < R:
                                        assert off + 4 * j + 4 <= extent
                            cells = [((rr + j, kk), (r + j, k) if k < K and r + j < R else None)
                                     for j in range(4)]
                        else:
                            rr, kk = idx >> 4, (idx & 15) * 4
                            r, k = r0 + rr, k0 + kk
                            if r < R:
                                off = (r * sr + k) * 4
                                if k + 3 < K:
                                    assert off % 16 == 0 and off + 16 <= extent
                                for j in range(4):
                                    if k + j < K:
                                        assert off + 4 * j + 4 <= extent
                            cells = [((rr, kk + j), (r, k + j) if r < R and k + j < K else None)
                                     for j in range(4)]
                        for cell, src in cells:
                            assert cell not in tile
                            tile[cell] = src
                else:
                    for e in range(8):
                        idx = tid + 256 * e
                        rr, kk = (idx & 31, idx >> 5) if rowcont else (idx >> 6, idx & 63)
                        assert (rr, kk) not in tile
                        ok = r0 + rr < R and k0 + kk < K
                        tile[(rr, kk)] = (r0 + rr, k0 + kk) if ok else None
            assert len(tile) == 32 * 64
            gw, ng = (4, 2) if esz == 4 else (8, 1)
            for tid in range(256):
                rr, q = tid >> 3, tid & 7
                r = r0 + rr
                if r >= R:
                    continue
                for g in range(ng):
                    kl = g * 32 + 4 * q if esz == 4 else 8 * q
                    if k0 + kl >= kp:
                        break
                    for j in range(gw):
                        if k0 + kl + j < K:
                            assert tile[(rr, kl + j)] == (r, k0 + kl + j)
                    assert k0 + kl + gw <= kp
                    for t in range(terms):
                        assert ((r * terms * kp + t * kp + k0 + kl) * esz) % 16 == 0
                        for j in range(gw):
                            key = (r, t, k0 + kl + j)
                            assert key not in written
                            written.add(key)
    assert len(written) == R * terms * kp


@pytest.mark.parametrize("esz", [4, 2])
@pytest.mark.parametrize("rowcont", [True, False])
def test_split_kernel_index_math(esz, rowcont):
    for R, K in [(1, 1), (37, 53), (33, 65), (70, 130), (8, 200)]:
        for terms in (1, 2):
            n = R if rowcont else K
            _split(R, K, esz, terms, rowcont, n + 3, False)          # scalar loads
            _split(R, K, esz, terms, rowcont, -(-n // 4) * 4, True)  # 16-byte loads


@pytest.mark.parametrize("esz", [4, 2])
def test_three_term_interleave_coordinates(esz):
    kcoord = 128 // esz            # elements per 128-byte K block
    seg_x, seg_y = 0x2, 0x4        # term -> segment (B side, A side)
    for K in (1, 31, 64, 65, 1000, 8192):
        kp = -(-K // kcoord) * kcoord
        seg_kb = kp * esz // 128
        seen = set()
        for j in range(3 * seg_kb):
            kq, t = divmod(j, 3)
            kx = (((seg_x >> t) & 1) * seg_kb + kq) * kcoord
            ky = (((seg_y >> t) & 1) * seg_kb + kq) * kcoord
            for c in (kx, ky):
                assert (c * esz) % 128 == 0 and 0 <= c and c + kcoord <= 2 * kp
            seen.add((kq, (kx - kq * kcoord) // kp, (ky - kq * kcoord) // kp))
        # per K block: (Bb, Ab), (Bs, Ab), (Bb, As) -- segments 0 = big, 1 = small
        assert seen == {(kq, sx, sy) for kq in range(seg_kb)
                        for sx, sy in ((0, 0), (1, 0), (0, 1))}
