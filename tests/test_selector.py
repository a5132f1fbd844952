"""The learned configuration selector.

GPU: the library's CUDA forward/backward kernels agree with the numpy
restatement (oracle/mlp_ref.py) -- gradients checked element by element --
training lowers the loss, and B2_METHOD_AUTO runs the selected configuration
with reference parity.

CPU: on the committed timing database (exhaustive autotuner sweep on B200),
the trained network's picks on the 2000 held-out shapes are within 5 % of the
exhaustive best (arithmetic and geometric mean of the time ratios), and beat
the fixed rule the library uses without the network.  Uses the library's host inference (b2_selector_predict), which
needs no device.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from gemm_avx512f_b200 import _lib
from oracle import mlp_ref as R

DATA = os.path.join(os.path.dirname(os.path.dirname(__file__)), "gemm_avx512f_b200", "data")
KEY = "nvidia_b200"
NP = R.IN * R.H + R.H + R.H * R.H + R.H + R.H * R.OUT + R.OUT


def _rand_weights(seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(NP) * 0.2).astype(np.float32)


def test_param_count_matches_restatement():
    assert _lib.lib().b2_mlp_param_count() == NP


@pytest.mark.gpu
def test_gradients_match_cpu_oracle(cuda):
    rng = np.random.default_rng(1)
    w = _rand_weights(2)
    X = rng.standard_normal((50, R.IN)).astype(np.float32)
    T = rng.standard_normal((50, R.OUT)).astype(np.float32)
    T[rng.random(T.shape) < 0.1] = np.nan  # masked (untimed) targets
    g = np.zeros(NP, np.float32)
    loss = C.c_float()
    assert _lib.lib().b2_mlp_gradient(w.ctypes.data, 50, X.ctypes.data, T.ctypes.data,
                                      C.byref(loss), g.ctypes.data) == 0
    l_ref, g_ref = R.loss_and_grad(w, X, T)
    assert abs(loss.value - l_ref) <= 1e-4 * abs(l_ref)
    assert np.abs(g - g_ref).max() <= 1e-4 * np.abs(g_ref).max()


@pytest.mark.gpu
def test_forward_kernel_matches_oracle_and_host_inference(cuda):
    rng = np.random.default_rng(3)
    w = _rand_weights(4)
    X = rng.standard_normal((300, R.IN)).astype(np.float32)
    Y = np.zeros((300, R.OUT), np.float32)
    L = _lib.lib()
    assert L.b2_mlp_forward(w.ctypes.data, 300, X.ctypes.data, Y.ctypes.data) == 0
    Yr, _ = R.forward(w, X.astype(np.float64))
    assert np.abs(Y - Yr).max() <= 1e-4 * max(1.0, np.abs(Yr).max())
    # the per-call host inference computes the same function of the features
    L.b2_selector_set(w.ctypes.data)
    try:
        p = np.zeros(R.OUT, np.float32)
        L.b2_selector_predict(b"N", b"T", 300, 40, 777, 1, p.ctypes.data)
        x = R.features(300, 40, 777, 0, 1, 1)
        yr, _ = R.forward(w, x[None, :].astype(np.float64))
        assert np.abs(p - yr[0]).max() <= 1e-4 * max(1.0, np.abs(yr).max())
    finally:
        L.b2_selector_set(None)


@pytest.mark.gpu
def test_training_lowers_loss(cuda):
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (2000, R.IN)).astype(np.float32)
    T = np.stack([np.sin(X[:, 0] * (1 + j % 3)) + X[:, 1] * X[:, 2] * (j % 5) for j in range(R.OUT)],
                 axis=1).astype(np.float32)
    L = _lib.lib()
    w0 = np.zeros(NP, np.float32)
    l0 = C.c_float()
    L.b2_mlp_train(2000, X.ctypes.data, T.ctypes.data, 0, 256, C.c_float(3e-3), 9, None,
                   w0.ctypes.data, C.byref(l0))
    w = np.zeros(NP, np.float32)
    l1 = C.c_float()
    assert L.b2_mlp_train(2000, X.ctypes.data, T.ctypes.data, 60, 256, C.c_float(3e-3), 9, None,
                          w.ctypes.data, C.byref(l1)) == 0
    assert l1.value < 0.1 * l0.value


@pytest.mark.gpu
def test_auto_method_runs_the_selected_config(cuda):
    import torch

    from oracle import oracle as O
    from tests._util import normalized

    path = os.path.join(DATA, f"selector_{KEY}.f32")
    if not os.path.exists(path):
        pytest.skip("no trained selector in this tree")
    w = np.fromfile(path, np.float32)
    L = _lib.lib()
    L.b2_selector_set(w.ctypes.data)
    try:
        rng = np.random.default_rng(6)
        for (m, n, k) in [(33, 700, 129), (640, 48, 1000), (512, 512, 512)]:
            a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
            b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
            c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
            cfg = L.b2_selector_choose(b"N", b"N", m, n, k, 0, 15)
            assert 0 <= cfg < 48
            da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
            assert L.b2_dgemm(b"N", b"N", m, n, k, 1.5, da.data_ptr(), m, db.data_ptr(), k, 0.5,
                              dc.data_ptr(), m, _lib.METHODS["auto"], 0, None) == 0
            torch.cuda.synchronize()
            ref = O.gemm("N", "N", m, n, k, 1.5, a, b, 0.5, c.copy(order="F"))
            assert normalized(dc.cpu().numpy().T, ref, k, a, b, 2.0 ** -53) <= 8
    finally:
        L.b2_selector_set(None)


def test_heldout_regret_within_5_percent():
    db = os.path.join(DATA, f"tune_db_{KEY}.npz")
    wp = os.path.join(DATA, f"selector_{KEY}.f32")
    if not (os.path.exists(db) and os.path.exists(wp)):
        pytest.skip("no committed timing database / selector")
    z = np.load(db)
    shapes, T, ntr = z["shapes"], z["log2ms"].astype(np.float64), int(z["train"])
    ms = np.exp2(T)
    w = np.fromfile(wp, np.float32)
    L = _lib.lib()
    allowed = np.array([c < 36 or 13 + (c - 36) // 3 >= 15 for c in range(48)])
    hold = shapes[ntr:]
    ms_h = ms[ntr:]
    best = np.where(allowed[None, :], ms_h, np.inf).min(1)
    L.b2_selector_set(w.ctypes.data)
    try:
        pick = np.array([L.b2_selector_choose(b"T" if s[3] else b"N", b"T" if s[4] else b"N",
                                              int(s[0]), int(s[1]), int(s[2]), int(s[5]), 15)
                         for s in hold])
    finally:
        L.b2_selector_set(None)
    heur = np.array([L.b2_selector_choose(b"T" if s[3] else b"N", b"T" if s[4] else b"N",
                                          int(s[0]), int(s[1]), int(s[2]), int(s[5]), 15)
                     for s in hold])
    r_mlp = ms_h[np.arange(len(hold)), pick] / best - 1
    r_heur = ms_h[np.arange(len(hold)), heur] / best - 1
    geo = np.exp(np.log1p(r_mlp).mean()) - 1
    assert geo <= 0.05, (geo, r_mlp.mean())
    assert r_mlp.mean() <= 0.05, r_mlp.mean()  # arithmetic mean too
    assert r_mlp.mean() < r_heur.mean() and np.median(r_mlp) < np.median(r_heur)
    rep = os.path.join(DATA, f"selector_{KEY}.json")
    if os.path.exists(rep):
        with open(rep) as fh:
            assert json.load(fh)["heldout"] == len(hold)


def test_sgemm_heldout_regret_within_5_percent_per_method():
    """The network chooses the engine and split-K of the tensor-core SGEMM
    methods too (dtype input 1): on the held-out SGEMM shapes of the committed
    timing database its pick is within 5 % of the exhaustive best of the
    method, for each method, and no worse than the library default."""
    db = os.path.join(DATA, f"tune_db_{KEY}.npz")
    wp = os.path.join(DATA, f"selector_{KEY}.f32")
    if not (os.path.exists(db) and os.path.exists(wp)):
        pytest.skip("no committed timing database / selector")
    z = np.load(db)
    if "shapes_s" not in z:
        pytest.skip("timing database without SGEMM sweep")
    shapes, ntr = z["shapes_s"], int(z["train_s"])
    ms = np.exp2(z["log2ms_s"].astype(np.float64))
    hold, ms_h = shapes[ntr:], ms[ntr:]
    w = np.fromfile(wp, np.float32)
    L = _lib.lib()
    for b, code in enumerate((_lib.METHODS["tf32"], _lib.METHODS["tf32x3"],
                              _lib.METHODS["bf16x3"])):
        valid = np.zeros(48, bool)
        valid[16 * b:16 * b + 12] = True
        best = np.where(valid[None, :], ms_h, np.inf).min(1)

        def picks():
            return np.array([L.b2_sgemm_selector_choose(code, b"T" if s[3] else b"N",
                                                        b"T" if s[4] else b"N", int(s[0]),
                                                        int(s[1]), int(s[2]), int(s[5]))
                             for s in hold])

        L.b2_selector_set(w.ctypes.data)
        try:
            pick = picks()
        finally:
            L.b2_selector_set(None)
        dflt = picks()
        assert valid[pick].all()
        r = ms_h[np.arange(len(hold)), pick] / best - 1
        rd = ms_h[np.arange(len(hold)), dflt] / best - 1
        assert r.mean() <= 0.05, (b, r.mean())
        assert np.exp(np.log1p(r).mean()) - 1 <= 0.05, (b, r.mean())
        assert r.mean() <= rd.mean(), (b, r.mean(), rd.mean())


@pytest.mark.gpu
def test_every_sgemm_configuration_matches_the_oracle(cuda):
    """Every engine / split-K slot of every tensor-core method (the space the
    selector chooses from) computes the product: parity with the oracle, for
    shapes that give the CTA pair both full and ragged tiles and several K
    ranges."""
    import torch

    from oracle import oracle as O
    from tests._util import normalized

    L = _lib.lib()
    U = {0: 2.0 ** -11, 1: 2.0 ** -21, 2: 2.0 ** -16}
    rng = np.random.default_rng(17)
    for (m, n, k, ta, tb) in [(300, 520, 700, "N", "T"), (512, 256, 1536, "T", "N")]:
        a = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)).astype(np.float32))
        b = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)).astype(np.float32))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(np.float32))
        ref = O.gemm(ta, tb, m, n, k, np.float32(1.25), a, b, np.float32(-0.5), c.copy(order="F"))
        da, db = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b))
        for cfg in range(48):
            if cfg % 16 >= 12:
                assert L.b2_sgemm_config(ta.encode(), tb.encode(), m, n, k, 1.0, da.data_ptr(),
                                         a.shape[0], db.data_ptr(), b.shape[0], 0.0,
                                         da.data_ptr(), m, cfg, None) == _lib.B2_ERR_ARG
                continue
            dc = torch.from_numpy(c.T.copy()).to(cuda)
            torch.cuda.synchronize()
            assert L.b2_sgemm_config(ta.encode(), tb.encode(), m, n, k, 1.25, da.data_ptr(),
                                     a.shape[0], db.data_ptr(), b.shape[0], -0.5, dc.data_ptr(),
                                     m, cfg, None) == 0
            torch.cuda.synchronize()
            got = np.asfortranarray(dc.cpu().numpy().T)
            assert normalized(got, ref, k, a, b, U[cfg // 16]) <= 8, (cfg, m, n, k, ta, tb)
