"""CPU restatements of the index maps of two kernels, checked before they run on
a GPU: every output element is owned by exactly one thread, every staged
element is loaded exactly once, and every shared-memory access stays inside
its buffer.

* the paired-FMA FP32 kernel (csrc/sgemm.cu, sgemm_ffma2_kernel): 128 x 128
  tile, K blocks of 16, 256 threads, 8 x 8 outputs each;
* the one-launch 3M kernel (csrc/gemm3m.cu, zgemm3m_dmma_kernel): 64 x 64
  complex tile, K blocks of 16, 16 warps of 16 x 16, DMMA m16n8k8 fragments.
"""
import itertools

# ---------------------------------------------------------- sgemm_ffma2 ----
S2_M, S2_N, S2_K = 128, 128, 16
S2_ALD, S2_BLD = S2_M + 4, S2_N + 4
A_FLOATS, B_FLOATS = S2_K * S2_ALD, S2_K * S2_BLD  # one buffer each


def test_ffma2_outputs_owned_once():
    seen = {}
    for tid in range(256):
        tx, ty = tid & 15, tid >> 4
        for r in range(8):
            m = 4 * tx + (r & 3) + 64 * (r >> 2)
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
                    offs = [kk * S2_ALD + mm + e for e in range(4)]
                    assert (kk * S2_ALD + mm) % 4 == 0  # 16-byte store
                else:
                    mm, kk = c >> 2, (c & 3) * 4
                    elems = [(mm, kk + e) for e in range(4)]
                    offs = [(kk + e) * S2_ALD + mm for e in range(4)]
                for x in elems:
                    assert x not in a_seen
                    a_seen.add(x)
                assert all(0 <= o < A_FLOATS for o in offs)
                # the stored element sits where the fragment load expects it
                for (m_, k_), o in zip(elems, offs):
                    assert o == k_ * S2_ALD + m_
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
            for hh in range(2):
                base = kk * S2_ALD + 64 * hh + 4 * tx
                assert base % 4 == 0 and base + 3 < A_FLOATS  # 16-byte aligned load
                # floats [0..3] = rows 4tx + i + 64hh, the rows r = 4hh + i of the thread
                for i in range(4):
                    assert base + i - kk * S2_ALD == 4 * tx + ((4 * hh + i) & 3) + 64 * ((4 * hh + i) >> 2)
            for h in range(2):
                base = kk * S2_BLD + 64 * h + 4 * ty
                assert base % 4 == 0 and base + 3 < B_FLOATS


def test_ffma2_quarter_warp_a_loads_conflict_free():
    # 16-byte loads run in quarter-warp phases: each phase's 8 threads must
    # touch distinct 16-byte slots of a 128-byte window
    for kk in range(S2_K):
        for hh in range(2):
            for quarter in range(4):
                lanes = range(8 * quarter, 8 * quarter + 8)
                slots = {((kk * S2_ALD + 64 * hh + 4 * (l & 15)) * 4 // 16) % 8 for l in lanes}
                assert len(slots) == 8


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


# ------------------------------------------------------ grouped panels ----
GT_M, GT_K, GT_LD = 64, 16, 68


def panel_slot(idx, kcont, esz, W=GT_M):
    if not kcont:
        return idx % W, idx // W
    kl = 32 // esz
    lane, w = idx & 31, idx >> 5
    return lane // kl + (32 // kl) * (w // (GT_K // kl)), lane % kl + kl * (w % (GT_K // kl))


def test_grouped_panel_slots_cover_the_panel_once():
    for esz in (8, 4):
        for kcont in (False, True):
            seen = {panel_slot(tid + 256 * e, kcont, esz) for tid in range(256) for e in range(4)}
            assert len(seen) == GT_M * GT_K
            assert all(0 <= mn < GT_M and 0 <= k < GT_K for mn, k in seen)
            assert all(k * GT_LD + mn < GT_K * GT_LD for mn, k in seen)


def test_grouped_panel_stores_hit_each_bank_at_most_twice():
    # per warp store: doubles occupy bank pairs (word offset 2 x element), floats one bank
    for esz in (8, 4):
        for kcont in (False, True):
            for w in range(32):
                hits = {}
                for lane in range(32):
                    mn, k = panel_slot(32 * w + lane, kcont, esz)
                    bank = ((k * GT_LD + mn) * (esz // 4)) % 32
                    hits[bank] = hits.get(bank, 0) + 1
                # 32 lanes x 8 B need 2 wavefronts anyway; floats need 1 (allow 2)
                assert max(hits.values()) <= 2, (esz, kcont, w, hits)


def test_grouped_kcont_loads_use_whole_sectors():
    # a k-contiguous warp load reads whole 32-byte sectors of each row
    for esz in (8, 4):
        for w in range(32):
            rows = {}
            for lane in range(32):
                mn, k = panel_slot(32 * w + lane, True, esz)
                rows.setdefault(mn, []).append(k)
            for ks in rows.values():
                ks.sort()
                assert len(ks) * esz == 32 and ks == list(range(ks[0], ks[0] + len(ks)))
                assert (ks[0] * esz) % 32 == 0


def test_grouped_warp_blocks_own_each_output_once_and_skip_only_outside():
    # FP64 and FP32 tiles share the warp grid: warp w owns rows 32 (w // 4) ..
    # + 31 and columns 16 (w % 4) .. + 15; FP32 lane l owns rows 4 (l % 8) + i,
    # columns 4 (l // 8) + j of it.  A warp skips its multiplies when its
    # block starts past M or N, which leaves no output of the problem behind.
    owned = {}
    for tid in range(256):
        lane, warp = tid & 31, tid >> 5
        rm, cn = (warp >> 2) * 32 + (lane & 7) * 4, (warp & 3) * 16 + (lane >> 3) * 4
        for i in range(4):
            for j in range(4):
                owned[(rm + i, cn + j)] = owned.get((rm + i, cn + j), 0) + 1
                assert (rm + i) // 32 == warp >> 2 and (cn + j) // 16 == warp & 3
    assert len(owned) == 64 * 64 and set(owned.values()) == {1}
    for m in (1, 16, 31, 32, 33, 63, 64):
        for n in (1, 15, 16, 17, 48, 64):
            for warp in range(8):
                live = (warp >> 2) * 32 < m and (warp & 3) * 16 < n
                inside = any(r < m and c < n for r in range((warp >> 2) * 32, (warp >> 2) * 32 + 32)
                             for c in range((warp & 3) * 16, (warp & 3) * 16 + 16))
                assert live == inside


def panel_slot3m(idx, kcont, esz):
    if not kcont:
        return idx % 32, idx // 32
    kl = 32 // esz
    lane, w = idx & 31, idx >> 5
    r = lane // kl
    kk = lane % kl + kl * (w % (GT_K // kl))
    row = ((r & 3) | ((r & 4) << 1) | ((r & 8) >> 1)) if kl == 2 else ((r & 3) | ((r & 4) << 2))
    return row + (16 if kl == 2 else 4) * (w // (GT_K // kl)), kk


def test_grouped_3m_panels_and_warp_blocks():
    # complex tiles: 32-wide panels of 16 k, 2 complex elements per thread per
    # operand in slot order (element size 16 B for complex128, 8 B for
    # complex64: K-contiguous rows read whole 32-byte sectors); the real and
    # imaginary panels (stride 36) are stored as doubles (complex128: each
    # half-warp is one 128-byte wavefront, so at most one lane per bank pair)
    # or floats (complex64: one lane per bank in the whole warp); warps of
    # 16 x 8 outputs on a 2 x 4 grid; complex64 lanes own 2 x 2 of them
    LD = 36
    for esz in (16, 8):
        for kcont in (False, True):
            seen = {panel_slot3m(tid + 256 * e, kcont, esz) for tid in range(256) for e in range(2)}
            assert seen == {(mn, k) for mn in range(32) for k in range(GT_K)}
            for w in range(16):
                slots = [panel_slot3m(32 * w + lane, kcont, esz) for lane in range(32)]
                if kcont:
                    rows = {}
                    for mn, k in slots:
                        rows.setdefault(mn, []).append(k)
                    for ks in rows.values():
                        ks.sort()
                        assert len(ks) * esz == 32 and ks[0] * esz % 32 == 0
                        assert ks == list(range(ks[0], ks[0] + len(ks)))
                if esz == 16:
                    for half in (slots[:16], slots[16:]):
                        pairs = [(k * LD + mn) % 16 for mn, k in half]
                        assert len(set(pairs)) == 16, (kcont, w, pairs)
                else:
                    banks = [(k * LD + mn) % 32 for mn, k in slots]
                    assert len(set(banks)) == 32, (kcont, w, banks)
    owned = set()
    for warp in range(8):
        wm0, wn0 = (warp >> 2) * 16, (warp & 3) * 8
        for lane in range(32):
            gq, t = lane >> 2, lane & 3
            for v in range(4):  # DMMA accumulator layout
                owned.add((wm0 + gq + 8 * (v >> 1), wn0 + 2 * t + (v & 1)))
    assert owned == {(m, n) for m in range(32) for n in range(32)}
    owned = set()
    for tid in range(256):
        lane, warp = tid & 31, tid >> 5
        rm, cn = (warp >> 2) * 16 + (lane & 7) * 2, (warp & 3) * 8 + (lane >> 3) * 2
        assert rm // 16 == warp >> 2 and cn // 8 == warp & 3
        owned |= {(rm + i, cn + j) for i in range(2) for j in range(2)}
    assert owned == {(m, n) for m in range(32) for n in range(32)}


# ------------------------------------------------ FP32 CUDA-core split-K ----
def ffma2_ksplit(tiles, kblocks, sms=148):
    slots = 2 * sms
    if tiles >= slots:
        return 1
    best, best_eff = 1, tiles / slots
    for S in range(2, 9):
        if S * 32 > kblocks:
            break
        units = tiles * S
        waves = -(-units // slots)
        eff = units / (waves * slots)
        if eff > best_eff + 0.02:
            best, best_eff = S, eff
    return best


def test_ffma2_split_slices_cover_k_once():
    # slices of kchunk (a multiple of the 16-deep K block) cover [0, K) once,
    # none empty; grids that fill the 296 slots stay unsplit
    for m, n, k in [(8192, 256, 8192), (2048, 160, 1536), (1024, 1024, 1024), (4096, 4096, 4096),
                    (513, 129, 1031), (100, 100, 5000), (16, 16, 16), (128, 128, 513)]:
        tiles = -(-m // 128) * -(-n // 128)
        kblocks = -(-k // 16)
        S = ffma2_ksplit(tiles, kblocks)
        assert 1 <= S <= 8 and (S == 1 or tiles < 296)
        kchunk = -(-kblocks // S) * 16
        used = -(-k // kchunk)
        ranges = [(z * kchunk, min(k, (z + 1) * kchunk)) for z in range(used)]
        assert kchunk % 16 == 0 and all(a < b for a, b in ranges)
        assert ranges[0][0] == 0 and ranges[-1][1] == k
        assert all(ranges[i][1] == ranges[i + 1][0] for i in range(used - 1))
        if S > 1:
            assert min(b - a for a, b in ranges[:-1]) >= 512
