"""GPU tests of the library's own tracing (b2_launch_count, b2_profile_*):
the per-kernel report and the per-launch timeline of an overlapped Ozaki
DGEMM, whose GEMM and auxiliary kernels run on two streams."""
import numpy as np
import pytest

from gemm_avx512f_b200 import _lib, blas

pytestmark = pytest.mark.gpu


def test_report_and_timeline_of_an_overlapped_ozaki_call(cuda):
    import torch

    n = 4096  # large enough for the column-block schedule (two blocks)
    g = torch.Generator(device=cuda).manual_seed(4)
    A = torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g)
    B = torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g)
    C = torch.zeros(n, n, device=cuda, dtype=torch.float64)
    blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, method="ozaki")
    torch.cuda.synchronize()
    _lib.profile_report()  # drop anything recorded before
    _lib.profile_enable(True)
    try:
        n0 = _lib.launch_count()
        blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, method="ozaki")
        torch.cuda.synchronize()
        launches = _lib.launch_count() - n0
        tl = _lib.profile_timeline()
    finally:
        _lib.profile_enable(False)
    names = [t[0] for t in tl]
    assert len(tl) == launches, (len(tl), launches)
    assert names.count("ozaki_i8_gemm") == 2  # one INT8 GEMM per column block
    assert names.count("ozaki_reconstruct") == 2
    assert names[0].startswith("ozaki_norm")
    assert min(a for _, a, _ in tl) == 0.0  # times count from the earliest start
    assert all(0.0 <= a <= b for _, a, b in tl)
    gemms = [(a, b) for nm, a, b in tl if nm == "ozaki_i8_gemm"]
    assert gemms[0][1] <= gemms[1][0] + 1e-3  # the GEMMs run one after another
    # the slicing of the second block runs beside the first GEMM (two streams)
    slices = [(a, b) for nm, a, b in tl if nm.startswith("ozaki_slice")]
    assert any(a < gemms[0][1] and b > gemms[0][0] for a, b in slices[1:])
    # the per-kernel report sums the same records
    blas.dgemm_device("N", "N", 256, 256, 256, 1.0, A, n, B, n, 0.0, C, n, method="fp64")
    torch.cuda.synchronize()
    assert _lib.profile_report() == {}  # recording is off again: nothing new
    np.testing.assert_array_equal(np.isfinite(C[:256, :256].cpu().numpy()), True)
