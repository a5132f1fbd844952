"""The allocation-free Ozaki DGEMM entry point, b2_dgemm_ozaki_noalloc.

It exists for callers that cannot allocate device memory when they call the
library -- code running during CUDA graph capture, real-time loops that must
stay out of the allocator, or processes whose device memory another framework
reserved up front.  Instead of the per-thread workspace it uses one static
device array of B2_NOALLOC_SCRATCH_BYTES (64 MiB) that every call shares.

Checked here through the C ABI: two calls in a row (different shapes and
data, so the second one runs over the first one's leftovers in the shared
array) agree with the allocating entry point b2_dgemm(..., B2_METHOD_OZAKI)
within the parity tolerance used everywhere else
(||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8), and a problem whose scratch
exceeds the maximum is refused with B2_ERR_ARG without touching C.  This file
is named to be collected last and needs nothing from the other tests.
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import _lib
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


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch

    L = _lib.lib()
    m = n = k = 2048  # needs ~189 MB of scratch at 15 moduli, above the 64 MiB array
    a = torch.zeros(m * k, dtype=torch.float64, device=cuda)
    b = torch.zeros(k * n, dtype=torch.float64, device=cuda)
    c = torch.full((m * n,), 7.0, dtype=torch.float64, device=cuda)
    st = L.b2_dgemm_ozaki_noalloc(b"N", b"N", m, n, k, 1.0, a.data_ptr(), m, b.data_ptr(), k,
                                  0.0, c.data_ptr(), m, 15, None)
    torch.cuda.synchronize()
    assert st == _lib.B2_ERR_ARG
    assert bool((c == 7.0).all())
