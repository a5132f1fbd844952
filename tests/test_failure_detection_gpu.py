"""Failure detection of the tensor-core engines, made to happen without a GPU
fault: a test hook shortens every bounded device wait to about a millisecond
and makes the next launch post its first K-block's byte count without issuing
the copy.  The wait for that copy then runs out: the kernel records
B2_ERR_TIMEOUT in its error word, every role drains (the copies that were
issued are waited for, bounded), TMEM is freed and the kernel returns.

Checked for the single-CTA engine (1xTF32 SGEMM, the allocation-free Ozaki
entry point) and the CTA-pair engine (the allocating Ozaki DGEMM): the
synchronous drop-in symbols report B2_ERR_TIMEOUT through b2_last_error(),
the asynchronous b2_* calls through b2_device_error(), the allocation-free
entry point through its own error word; the context stays usable and the next
normal call passes parity against the oracle.  The reference's own waits spin
forever (src/gemm_driver.c:21-31, OpenBLAS-like_implementation/dgemm.c:436-448).
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import _lib, blas
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu
WAIT_NS = 1_000_000  # 1 ms


def _inputs(rng, dtype, m, n, k):
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)).astype(dtype))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)).astype(dtype))
    c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(dtype))
    return a, b, c


def _stall_next(launches=1):
    assert _lib.lib().b2_test_bounded_wait(WAIT_NS, launches) == 0


def _restore():
    assert _lib.lib().b2_test_bounded_wait(0, 0) == 0


def _dropin(fn, a, b, c, m, n, k, dtype):
    ct = np.float64 if dtype == np.float64 else np.float32
    got = c.copy(order="F")
    L = _lib.lib()
    import ctypes as C

    cty = C.c_double if ct == np.float64 else C.c_float
    ip = lambda v: C.byref(C.c_int(v))
    getattr(L, fn)(b"N", b"N", ip(m), ip(n), ip(k), C.byref(cty(1.5)), a.ctypes.data, ip(m),
                   b.ctypes.data, ip(k), C.byref(cty(0.5)), got.ctypes.data, ip(m))
    return L.b2_last_error(), got


@pytest.mark.parametrize("engine", ["single_cta_tf32", "cta_pair_ozaki"])
def test_dropin_reports_timeout_then_recovers(cuda, engine):
    rng = np.random.default_rng(91)
    m, n, k = 640, 520, 700
    if engine == "single_cta_tf32":
        dtype, fn, u = np.float32, "sgemm_", 2.0 ** -11
        blas.set_sgemm_method("tf32")
    else:
        dtype, fn, u = np.float64, "dgemm_", 2.0 ** -53
        blas.set_dgemm_method("ozaki", 15)
    a, b, c = _inputs(rng, dtype, m, n, k)
    try:
        _stall_next()
        try:
            st, _ = _dropin(fn, a, b, c, m, n, k, dtype)
        finally:
            _restore()
        assert st == _lib.B2_ERR_TIMEOUT, st
        assert _lib.lib().b2_device_error(0) == 0  # the drop-in read and cleared it
        # the kernel returned and the context is usable: a normal call passes parity
        st, got = _dropin(fn, a, b, c, m, n, k, dtype)
        assert st == 0
        ref = O.gemm("N", "N", m, n, k, dtype(1.5), a, b, dtype(0.5), c.copy(order="F"))
        assert normalized(got, ref, k, a, b, u) <= 8
    finally:
        blas.set_sgemm_method("fp32")
        blas.set_dgemm_method("fp64", 0)


def test_async_call_reports_timeout_through_device_error(cuda):
    import torch

    rng = np.random.default_rng(92)
    m, n, k = 512, 384, 640
    a, b, c = _inputs(rng, np.float64, m, n, k)
    da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
    L = _lib.lib()
    stream = torch.cuda.Stream(cuda)
    _stall_next()
    try:
        st = L.b2_dgemm(b"N", b"N", m, n, k, 1.5, da.data_ptr(), m, db.data_ptr(), k, 0.5,
                        dc.data_ptr(), m, _lib.METHODS["ozaki"], 15, stream.cuda_stream)
        stream.synchronize()
    finally:
        _restore()
    assert st == 0  # asynchronous: the launch itself succeeded
    assert L.b2_device_error(1) == _lib.B2_ERR_TIMEOUT
    assert L.b2_device_error(0) == 0  # cleared
    out = torch.from_numpy(c.T.copy()).to(cuda)
    assert L.b2_dgemm(b"N", b"N", m, n, k, 1.5, da.data_ptr(), m, db.data_ptr(), k, 0.5,
                      out.data_ptr(), m, _lib.METHODS["ozaki"], 15, stream.cuda_stream) == 0
    stream.synchronize()
    assert L.b2_device_error(0) == 0
    ref = O.gemm("N", "N", m, n, k, 1.5, a, b, 0.5, c.copy(order="F"))
    assert normalized(out.cpu().numpy().T, ref, k, a, b, 2.0 ** -53) <= 8


def test_noalloc_entry_reports_timeout_through_its_error_word(cuda):
    import torch

    rng = np.random.default_rng(93)
    m, n, k = 300, 260, 400
    a, b, c = _inputs(rng, np.float64, m, n, k)
    da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
    L = _lib.lib()
    stream = torch.cuda.Stream(cuda)
    # set-up call first (resolves the static array), then the stalled call
    assert L.b2_dgemm_ozaki_noalloc(b"N", b"N", m, n, k, 1.5, da.data_ptr(), m, db.data_ptr(),
                                    k, 0.5, dc.clone().data_ptr(), m, 15,
                                    stream.cuda_stream) == 0
    assert L.b2_dgemm_ozaki_noalloc_error(0, stream.cuda_stream) == 0
    _stall_next()
    try:
        st = L.b2_dgemm_ozaki_noalloc(b"N", b"N", m, n, k, 1.5, da.data_ptr(), m,
                                      db.data_ptr(), k, 0.5, dc.clone().data_ptr(), m, 15,
                                      stream.cuda_stream)
    finally:
        _restore()
    assert st == 0
    assert L.b2_dgemm_ozaki_noalloc_error(1, stream.cuda_stream) == _lib.B2_ERR_TIMEOUT
    assert L.b2_dgemm_ozaki_noalloc_error(0, stream.cuda_stream) == 0
    out = dc.clone()
    assert L.b2_dgemm_ozaki_noalloc(b"N", b"N", m, n, k, 1.5, da.data_ptr(), m, db.data_ptr(),
                                    k, 0.5, out.data_ptr(), m, 15, stream.cuda_stream) == 0
    assert L.b2_dgemm_ozaki_noalloc_error(0, stream.cuda_stream) == 0
    ref = O.gemm("N", "N", m, n, k, 1.5, a, b, 0.5, c.copy(order="F"))
    assert normalized(out.cpu().numpy().T, ref, k, a, b, 2.0 ** -53) <= 8
