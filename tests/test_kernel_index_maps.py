"""CPU restatements of the index maps of two kernels, checked before they run on
a GPU: every output element is owned by exactly one thread, every staged
element is loaded exactly once, and every shared-memory access stays inside
its buffer.

* the paired-FMA FP32 kernel (csrc/sgemm.cu, sgemm_ffma2_kernel): 128 x 128
  tile, K blocks of 16, 256 threads, duplicated A panel;
* the one-launch 3M kernel (csrc/gemm3m.cu, zgemm3m_dmma_kernel): 64 x 64
  complex tile, K blocks of 16, 16 warps of 16 x 16, DMMA m16n8k8 fragments.
"""
import itertools

# ---------------------------------------------------------- sgemm_ffma2 ----
S2_M, S2_N, S2_K = 128, 128, 16
S2_ALD, S2_BLD = 2 * S2_M + 4, S2_N + 4
A_FLOATS, B_FLOATS = S2_K * S2_ALD, S2_K * S2_BLD  # one buffer each


def test_ffma2_outputs_owned_once():
    seen = {}
    for tid in range(256):
        tx, ty = tid & 15, tid >> 4
        for r in range(8):
            m = 2 * tx + (r & 1) + 32 * (r >> 1)
            for c in range(4):
                nb = 64 * (c >> 1) + 4 * ty + 2 * (c & 1)
                for e in range(2):
                    key = (m, nb + e)
                    assert key not in seen
                    seen[key] = tid
    assert len(seen) == S2_M * S2_N


def test_ffma2_staging_covers_panels_once_and_stays_in_bounds():
    for ta, tb in itertools.product([False, True], repeat=2):
        a_seen, b_seen = set(), set()
        for tid in range(256):
            for h in range(2):
                c = tid + 256 * h
                if not ta:
                    kk, mm = c >> 5, (c & 31) * 4
                    elems = [(mm + e, kk) for e in range(4)]
                    offs = [kk * S2_ALD + 2 * mm + j for j in range(8)]
                else:
                    mm, kk = c >> 2, (c & 3) * 4
                    elems = [(mm, kk + e) for e in range(4)]
                    offs = [(kk + e) * S2_ALD + 2 * mm + j for e in range(4) for j in range(2)]
                for x in elems:
                    assert x not in a_seen
                    a_seen.add(x)
                assert all(0 <= o < A_FLOATS for o in offs)
                if tb:
                    kk, nn = c >> 5, (c & 31) * 4
                    elems = [(kk, nn + e) for e in range(4)]
                    offs = [kk * S2_BLD + nn + e for e in range(4)]
                else:
                    nn, kk = c >> 2, (c & 3) * 4
                    elems = [(kk + e, nn) for e in range(4)]
                    offs = [(kk + e) * S2_BLD + nn for e in range(4)]
                for x in elems:
                    assert x not in b_seen
                    b_seen.add(x)
                assert all(0 <= o < B_FLOATS for o in offs)
        assert len(a_seen) == S2_M * S2_K and len(b_seen) == S2_N * S2_K


def test_ffma2_fragment_loads_in_bounds_and_match_owned_rows():
    for tid in range(256):
        tx, ty = tid & 15, tid >> 4
        for kk in range(S2_K):
            for q in range(4):
                base = kk * S2_ALD + 2 * (32 * q + 2 * tx)
                assert base % 4 == 0 and base + 3 < A_FLOATS  # 16-byte aligned load
                # floats [0,1] = dup of row 32q + 2tx, [2,3] = dup of row 32q + 2tx + 1
                assert (base - kk * S2_ALD) // 2 == 32 * q + 2 * tx
            for h in range(2):
                base = kk * S2_BLD + 64 * h + 4 * ty
                assert base % 4 == 0 and base + 3 < B_FLOATS


def test_ffma2_quarter_warp_a_loads_conflict_free():
    # 16-byte loads run in quarter-warp phases: each phase's 8 threads must
    # touch distinct 16-byte slots of a 128-byte window (lanes 16-31 repeat
    # lanes 0-15's addresses, a broadcast)
    for kk in range(S2_K):
        for q in range(4):
            for quarter in range(4):
                lanes = range(8 * quarter, 8 * quarter + 8)
                slots = {((kk * S2_ALD + 2 * (32 * q + 2 * (l & 15))) * 4 // 16) % 8
                         for l in lanes}
                assert len(slots) == len({l & 15 for l in lanes})


# ------------------------------------------------------ zgemm3m_dmma ----
Z_BM = Z_BN = 64
Z_BK, Z_NT = 16, 512


def z_stage(kc, outer):
    return outer * (Z_BK + 4) if kc else Z_BK * (outer + 2)


def test_z_tile_loads_cover_once_in_bounds():
    for kc in (False, True):
        seen = set()
        for tid in range(Z_NT):
            for i in range(Z_BM * Z_BK // Z_NT):
                c = tid + i * Z_NT
                if kc:
                    o, k = c // Z_BK, c % Z_BK
                    off = o * (Z_BK + 4) + k
                else:
                    k, o = c // Z_BM, c % Z_BM
                    off = k * (Z_BM + 2) + o
                assert (o, k) not in seen
                seen.add((o, k))
                assert 0 <= off < z_stage(kc, Z_BM)
        assert len(seen) == Z_BM * Z_BK


def test_z_fragments_in_bounds_and_outputs_owned_once():
    owned = set()
    for warp in range(16):
        wm0, wn0 = (warp // 4) * 16, (warp % 4) * 16
        for lane in range(32):
            g, t = lane >> 2, lane & 3
            for kk in (0, 8):
                for v1 in range(2):
                    for v0 in range(2):
                        m, k = wm0 + g + 8 * v0, kk + t + 4 * v1
                        assert m < Z_BM and k < Z_BK
                        assert m * (Z_BK + 4) + k < z_stage(True, Z_BM)
                        assert k * (Z_BM + 2) + m < z_stage(False, Z_BM)
                for j in range(2):
                    for v in range(2):
                        n, k = wn0 + j * 8 + g, kk + t + 4 * v
                        assert n < Z_BN and k < Z_BK
            for j in range(2):
                for v in range(4):
                    key = (wm0 + g + 8 * (v >> 1), wn0 + j * 8 + 2 * t + (v & 1))
                    assert key not in owned
                    owned.add(key)
    assert len(owned) == Z_BM * Z_BN


def test_z_fragment_loads_conflict_free():
    # 16-byte loads, quarter-warp phases of 8 lanes (g in {2p, 2p+1}, t 0..3)
    for kc in (False, True):
        for phase in range(4):
            slots = set()
            for lane in range(8 * phase, 8 * phase + 8):
                g, t = lane >> 2, lane & 3
                off = g * (Z_BK + 4) + t if kc else t * (Z_BM + 2) + g
                slots.add((off * 16 // 16) % 8)
            assert len(slots) == 8, (kc, phase)
