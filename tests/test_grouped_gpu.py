"""GPU tests of the grouped GEMM (one persistent launch over many problems)
and of its CUDA-graph plan, through the C ABI.

Each problem follows the dgemm_/sgemm_ contract and is checked against the
oracle (bit-exact restatement of the reference drivers) with the parity bar
||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8.
"""
import ctypes as C

import numpy as np
import pytest

from gemm_avx512f_b200 import _lib
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu


def make_batch(cuda, count, lo, hi, seed):
    """Config-4 style batch: log-uniform M, N, K in [lo, hi], half FP32 half
    FP64, random transposes, U[-1,1) values (seed)."""
    import torch

    rng = np.random.default_rng(seed)
    probs, keep = [], []
    for i in range(count):
        m, n, k = (int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))))) for _ in range(3))
        dtype = i % 2  # 0 = f64, 1 = f32
        ta, tb = ("N", "T")[rng.integers(2)], ("N", "T")[rng.integers(2)]
        npdt = np.float64 if dtype == 0 else np.float32
        ar, ac = (m, k) if ta == "N" else (k, m)
        br, bc = (k, n) if tb == "N" else (n, k)
        a = np.asfortranarray(rng.uniform(-1, 1, (ar, ac)).astype(npdt))
        b = np.asfortranarray(rng.uniform(-1, 1, (br, bc)).astype(npdt))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(npdt))
        al, be = float(rng.choice([1.0, 1.5, -0.5])), float(rng.choice([0.0, 1.0, 0.5]))
        da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
        p = _lib.GemmProblem(dtype, ta.encode(), tb.encode(), m, n, k, al, be, da.data_ptr(), ar,
                             db.data_ptr(), br, dc.data_ptr(), m)
        probs.append(p)
        keep.append((a, b, c, da, db, dc, ta, tb, al, be))
    arr = (_lib.GemmProblem * count)(*probs)
    return arr, keep


def check(keep):
    for (a, b, c, da, db, dc, ta, tb, al, be) in keep:
        m, n = c.shape
        k = a.shape[1] if ta == "N" else a.shape[0]
        ref = O.gemm(ta, tb, m, n, k, a.dtype.type(al), a, b, a.dtype.type(be), c.copy(order="F"))
        got = np.asfortranarray(dc.cpu().numpy().T)
        u = np.finfo(a.dtype).eps / 2
        assert normalized(got, ref, k, a, b, u) <= 8, (a.dtype, m, n, k, ta, tb)


def test_grouped_one_launch_matches_oracle(cuda):
    import torch

    arr, keep = make_batch(cuda, 300, 16, 300, seed=3)
    st = torch.cuda.Stream(cuda)
    n0 = _lib.launch_count()
    assert _lib.lib().b2_gemm_grouped(len(arr), arr, st.cuda_stream) == 0
    st.synchronize()
    assert _lib.launch_count() - n0 == 1  # one persistent launch for the whole batch
    check(keep)


def test_grouped_graph_plan_replays(cuda):
    import torch

    arr, keep = make_batch(cuda, 120, 16, 200, seed=4)
    plan = C.c_void_p()
    L = _lib.lib()
    assert L.b2_grouped_plan_create(len(arr), arr, C.byref(plan)) == 0
    st = torch.cuda.Stream(cuda)
    try:
        for rep in range(2):
            for (a, b, c, da, db, dc, *_rest) in keep:  # restore C before each replay
                dc.copy_(torch.from_numpy(c.T.copy()))
            torch.cuda.synchronize()
            assert L.b2_grouped_plan_launch(plan, st.cuda_stream) == 0
            st.synchronize()
            check(keep)
    finally:
        L.b2_grouped_plan_destroy(plan)


def test_grouped_rejects_bad_problem(cuda):
    arr, keep = make_batch(cuda, 5, 16, 32, seed=5)
    arr[3].lda = 0  # invalid leading dimension in the 4th problem
    L = _lib.lib()
    assert L.b2_gemm_grouped(len(arr), arr, None) == _lib.B2_ERR_ARG
    assert L.b2_last_info() == 4


def test_grouped_edge_problems(cuda):
    """Empty problems (M or N = 0) are skipped, K = 0 and alpha = 0 only
    scale C by beta (beta = 0 keeps a NaN already in C, as dgemm_ does), and
    the tile map and next-tile prefetch still hand every remaining tile out
    once: a batch where most problems are degenerate, around ragged real ones."""
    import torch

    rng = np.random.default_rng(9)
    shapes = [(0, 5, 7), (37, 0, 9), (65, 70, 0), (64, 64, 64), (1, 1, 1), (130, 3, 257),
              (129, 65, 33), (50, 40, 0), (3, 200, 129)]
    probs, keep = [], []
    for i, (m, n, k) in enumerate(shapes * 3):
        dtype = i % 2
        npdt = np.float64 if dtype == 0 else np.float32
        ta, tb = ("N", "T")[i % 2], ("N", "T")[(i // 2) % 2]
        ar, ac = (m, k) if ta == "N" else (k, m)
        br, bc = (k, n) if tb == "N" else (n, k)
        a = np.asfortranarray(rng.uniform(-1, 1, (max(ar, 1), max(ac, 1))).astype(npdt))
        b = np.asfortranarray(rng.uniform(-1, 1, (max(br, 1), max(bc, 1))).astype(npdt))
        c = np.asfortranarray(rng.uniform(-1, 1, (max(m, 1), max(n, 1))).astype(npdt))
        al = 0.0 if i == 13 else 1.25
        be = 0.0 if i % 3 == 0 else -0.5
        if m > 0 and n > 0 and be == 0.0:
            c[0, 0] = np.nan  # beta == 0 still multiplies C: the NaN stays
        da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
        probs.append(_lib.GemmProblem(dtype, ta.encode(), tb.encode(), m, n, k, al, be,
                                      da.data_ptr(), max(ar, 1), db.data_ptr(), max(br, 1),
                                      dc.data_ptr(), max(m, 1)))
        keep.append((a, b, c, dc, ta, tb, m, n, k, al, be, da, db))  # device buffers stay alive
    arr = (_lib.GemmProblem * len(probs))(*probs)
    L = _lib.lib()
    assert L.b2_gemm_grouped(len(probs), arr, None) == 0
    torch.cuda.synchronize()
    for (a, b, c, dc, ta, tb, m, n, k, al, be, _, _) in keep:
        got = np.asfortranarray(dc.cpu().numpy().T)
        if m == 0 or n == 0:
            assert np.array_equal(got, c, equal_nan=True)
            continue
        ar = m if ta == "N" else k
        br = k if tb == "N" else n
        if k == 0 or al == 0.0:
            ref = a.dtype.type(be) * c  # only beta C (0 * NaN stays NaN)
        else:
            ref = c.copy(order="F")
            O.gemm(ta, tb, m, n, k, a.dtype.type(al), a[:ar], b[:br], a.dtype.type(be), ref)
        assert np.array_equal(np.isnan(got), np.isnan(ref)), (m, n, k, be)
        fin = ~np.isnan(ref)
        u = np.finfo(a.dtype).eps / 2
        if k == 0 or al == 0.0:
            assert np.allclose(got[fin], ref[fin], rtol=0, atol=4 * u), (m, n, k)
        else:
            g, r = np.where(fin, got, 0), np.where(fin, ref, 0)
            assert normalized(g, r, k, a[:ar], b[:br], u) <= 8, (a.dtype, m, n, k, ta, tb)


def test_grouped_skinny_tile_shapes(cuda):
    """Problems with M or N far below 64 run on the 32 x 128 and 128 x 32
    tiles, the others on 64 x 64: every shape x dtype x transpose pair, with
    ragged edges in M, N and K, against the oracle."""
    import torch

    rng = np.random.default_rng(11)
    shapes = [(17, 300, 45), (300, 21, 77), (33, 129, 16), (129, 31, 130), (16, 16, 1000),
              (64, 64, 31), (8, 1000, 9), (1000, 8, 17), (65, 33, 64)]
    probs, keep = [], []
    i = 0
    for (m, n, k) in shapes:
        for dtype in (0, 1):
            for ta in "NT":
                for tb in "NT":
                    npdt = np.float64 if dtype == 0 else np.float32
                    ar, ac = (m, k) if ta == "N" else (k, m)
                    br, bc = (k, n) if tb == "N" else (n, k)
                    a = np.asfortranarray(rng.uniform(-1, 1, (ar, ac)).astype(npdt))
                    b = np.asfortranarray(rng.uniform(-1, 1, (br, bc)).astype(npdt))
                    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(npdt))
                    al, be = (1.0, 0.0) if i % 2 else (-0.75, 1.0)
                    da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
                    probs.append(_lib.GemmProblem(dtype, ta.encode(), tb.encode(), m, n, k, al, be,
                                                  da.data_ptr(), ar, db.data_ptr(), br,
                                                  dc.data_ptr(), m))
                    keep.append((a, b, c, da, db, dc, ta, tb, al, be))
                    i += 1
    arr = (_lib.GemmProblem * len(probs))(*probs)
    st = torch.cuda.Stream(cuda)
    assert _lib.lib().b2_gemm_grouped(len(arr), arr, st.cuda_stream) == 0
    st.synchronize()
    check(keep)


def test_grouped_complex_3m_problems_in_the_same_launch(cuda):
    """zgemm3m_ / cgemm3m_ problems (dtypes 2 and 3) share the queue with real
    ones: every op() form ('N', 'T', 'C', 'R'), complex alpha and beta,
    ragged sizes, padded leading dimensions, K = 0, alpha = 0 and a NaN in C
    with beta = 0, each checked against the oracle's 3M restatement (whose
    real products are the bit-exact restatement of the reference dgemm_)."""
    import torch

    rng = np.random.default_rng(21)
    shapes = [(13, 9, 21), (33, 65, 40), (70, 31, 129), (1, 1, 1), (64, 64, 16), (5, 40, 0),
              (40, 5, 7), (100, 90, 70)]
    probs, keep = [], []
    i = 0
    for (m, n, k) in shapes:
        for dtype in (2, 3):
            for ta, tb in (("N", "N"), ("T", "C"), ("C", "R"), ("R", "T")):
                cdt = np.complex128 if dtype == 2 else np.complex64
                ar, ac = (m, k) if ta in "NR" else (k, m)
                br, bc = (k, n) if tb in "NR" else (n, k)
                pa, pb, pc = 2, 1, 3  # padded leading dimensions

                def cm(r, c, pad):
                    x = rng.uniform(-1, 1, (r + pad, max(c, 1))) + 1j * rng.uniform(-1, 1, (r + pad, max(c, 1)))
                    return np.asfortranarray(x.astype(cdt))

                a, b, c = cm(ar, ac, pa), cm(br, bc, pb), cm(m, n, pc)
                al = 0.0 if i == 5 else 0.75 - 1.25j
                be = 0.0 if i % 4 == 1 else (1.0 if i % 4 == 2 else 0.5 + 0.25j)
                if be == 0.0:
                    c[0, 0] = np.nan  # beta == 0 still multiplies C: the NaN stays
                da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
                p = _lib.GemmProblem(dtype, ta.encode(), tb.encode(), m, n, k, float(np.real(al)),
                                     float(np.real(be)), da.data_ptr(), a.shape[0], db.data_ptr(),
                                     b.shape[0], dc.data_ptr(), c.shape[0])
                p.alpha_i, p.beta_i = float(np.imag(al)), float(np.imag(be))
                probs.append(p)
                keep.append((a, b, c, da, db, dc, ta, tb, m, n, k, al, be))
                i += 1
    real_arr, real_keep = make_batch(cuda, 40, 16, 150, seed=22)
    arr = (_lib.GemmProblem * (len(probs) + len(real_arr)))(*probs, *real_arr)
    st = torch.cuda.Stream(cuda)
    n0 = _lib.launch_count()
    assert _lib.lib().b2_gemm_grouped(len(arr), arr, st.cuda_stream) == 0
    st.synchronize()
    assert _lib.launch_count() - n0 == 1  # real and 3M problems in one launch
    check(real_keep)
    for (a, b, c, da, db, dc, ta, tb, m, n, k, al, be) in keep:
        got = np.asfortranarray(dc.cpu().numpy().T)
        ar = m if ta in "NR" else k
        br = k if tb in "NR" else n
        ref = c.copy(order="F")
        if k > 0 and al != 0.0:
            O.gemm3m(ta, tb, m, n, k, al, a[:ar], b[:br], be, ref[:m])
        elif not (be == 1.0):
            ref[:m, :n] = be * c[:m, :n]
        assert np.array_equal(got[m:], c[m:], equal_nan=True), "padding rows of C were written"
        assert np.array_equal(np.isnan(got[:m]), np.isnan(ref[:m])), (m, n, k, be)
        fin = ~np.isnan(ref[:m])
        u = np.finfo(a.dtype).eps / 2
        g, r = np.where(fin, got[:m], 0), np.where(fin, ref[:m], 0)
        den = max(k, 1) * u * np.linalg.norm(a[:ar]) * np.linalg.norm(b[:br]) + u * np.linalg.norm(r)
        if den == 0.0:  # K = 0 and beta = 0: C is exactly zero (NaN kept above)
            assert np.array_equal(g, r), (m, n, k, ta, tb)
            continue
        err = np.linalg.norm((g - r).astype(np.complex128)) / den
        assert err <= 8, (a.dtype, m, n, k, ta, tb, err)


def test_grouped_back_to_back_calls_reuse_descriptor_slots(cuda):
    """One-shot calls return once enqueued and alternate two descriptor
    slots: five batches issued back to back on one stream, with no
    synchronisation in between, all come out right."""
    import torch

    batches = [make_batch(cuda, 60, 16, 200, seed=40 + i) for i in range(5)]
    st = torch.cuda.Stream(cuda)
    L = _lib.lib()
    for arr, _keep in batches:
        assert L.b2_gemm_grouped(len(arr), arr, st.cuda_stream) == 0
    st.synchronize()
    for _arr, keep in batches:
        check(keep)
