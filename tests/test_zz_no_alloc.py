"""The allocation-free Ozaki DGEMM entry point, b2_dgemm_ozaki_noalloc.

It exists for callers that cannot allocate device memory when they call the
library -- real-time loops that must stay out of the allocator for their
latency, or processes whose device memory another framework reserved up
front, where an allocation during the call would fail or stall.  Instead of
the per-thread workspace it uses one static device array of
B2_NOALLOC_SCRATCH_BYTES (64 MiB) that every call shares.

Checked here through the C ABI: two calls in a row (different shapes and
data, so the second one runs over the first one's leftovers in the shared
array) agree with the allocating entry point b2_dgemm(..., B2_METHOD_OZAKI)
within the parity tolerance used everywhere else
(||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8); transposed operands (the
other slicing layout) agree with the oracle, which is bit-exact with the
reference's dgemm_; and a problem whose scratch exceeds the maximum is refused
with B2_ERR_ARG without touching C.  This file is named to be collected last
and needs nothing from the other tests.
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import _lib
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu
OZAKI = _lib.METHODS["ozaki"]


def _case(cuda, rng, m, n, k):
    import torch

    a = torch.from_numpy(rng.uniform(-1, 1, (k, m)) * np.exp(rng.standard_normal((k, m))))
    b = torch.from_numpy(rng.uniform(-1, 1, (n, k)))
    c = torch.from_numpy(rng.uniform(-1, 1, (n, m)))
    return a.to(cuda), b.to(cuda), c.to(cuda)  # column-major m x k, k x n, m x n


def test_noalloc_matches_allocating_entry_point(cuda):
    import torch

    L = _lib.lib()
    rng = np.random.default_rng(123)
    stream = torch.cuda.Stream(cuda)
    u = 2.0 ** -53
    for (m, n, k, slices) in [(700, 520, 900, 15), (333, 1100, 257, 14)]:
        a, b, c = _case(cuda, rng, m, n, k)
        ref = c.clone()
        got = c.clone()
        assert L.b2_dgemm(b"N", b"N", m, n, k, 1.5, a.data_ptr(), m, b.data_ptr(), k, 0.5,
                          ref.data_ptr(), m, OZAKI, slices, stream.cuda_stream) == 0
        assert L.b2_dgemm_ozaki_noalloc(b"N", b"N", m, n, k, 1.5, a.data_ptr(), m, b.data_ptr(),
                                        k, 0.5, got.data_ptr(), m, slices,
                                        stream.cuda_stream) == 0
        stream.synchronize()
        A, B = a.cpu().numpy().T, b.cpu().numpy().T
        err = normalized(got.cpu().numpy().T, ref.cpu().numpy().T, k, A, B, u)
        assert err <= 8, (m, n, k, err)


def test_noalloc_transposed_operands_match_the_oracle(cuda):
    import torch

    L = _lib.lib()
    rng = np.random.default_rng(321)
    stream = torch.cuda.Stream(cuda)
    for (m, n, k) in [(450, 380, 610), (1200, 1200, 1200)]:  # the largest square size it takes
        a = np.asfortranarray(rng.uniform(-1, 1, (k, m)))  # op(A) = A^T
        b = np.asfortranarray(rng.uniform(-1, 1, (n, k)))  # op(B) = B^T
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
        da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
        assert L.b2_dgemm_ozaki_noalloc(b"T", b"T", m, n, k, -0.75, da.data_ptr(), k,
                                        db.data_ptr(), n, 1.25, dc.data_ptr(), m, 15,
                                        stream.cuda_stream) == 0
        stream.synchronize()
        ref = O.gemm("T", "T", m, n, k, -0.75, a, b, 1.25, c.copy(order="F"))
        err = normalized(dc.cpu().numpy().T, ref, k, a, b, 2.0 ** -53)
        assert err <= 8, (m, n, k, err)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch

    L = _lib.lib()
    m = n = k = 1201  # one past the largest square size that fits the 64 MiB array at 15 moduli
    a = torch.zeros(m * k, dtype=torch.float64, device=cuda)
    b = torch.zeros(k * n, dtype=torch.float64, device=cuda)
    c = torch.full((m * n,), 7.0, dtype=torch.float64, device=cuda)
    st = L.b2_dgemm_ozaki_noalloc(b"N", b"N", m, n, k, 1.0, a.data_ptr(), m, b.data_ptr(), k,
                                  0.0, c.data_ptr(), m, 15, None)
    torch.cuda.synchronize()
    assert st == _lib.B2_ERR_ARG
    assert bool((c == 7.0).all())
