"""B200-native (sm_100a) dense BLAS-3: a drop-in for the sgemm_/dgemm_ hot path of
wjc404/GEMM_AVX512F, plus dtrsm_, zgemm3m_/cgemm3m_, INT8 Ozaki-emulated DGEMM,
split-precision SGEMM, grouped GEMM, an autotuner and a learned config selector.

The compute lives in ``lib/libb2blas.so`` (CUDA, C ABI in include/b2blas.h);
this package is the Python host mirror of that interface.
"""
from ._lib import B2Error, lib  # noqa: F401
from .blas import *  # noqa: F401,F403

__version__ = "0.1.0"
