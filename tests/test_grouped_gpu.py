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
