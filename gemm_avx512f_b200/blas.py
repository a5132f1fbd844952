"""Python mirror of the reference's Fortran-BLAS interface, over libb2blas.so.

Same names, argument order and meaning as the C symbols the reference exports
(``dgemm_``/``sgemm_`` of src/gemm_driver.c:116): column-major matrices with
explicit leading dimensions, trans chars where 'N'/'n' means no transpose and
anything else means transpose, ``beta != 1`` scaling C (so a NaN in C survives
``beta == 0``), ``alpha == 0`` skipping the product.  Matrices may be numpy
arrays (host memory; staged through the device by the library), torch CUDA
tensors (used in place) or raw integer addresses.  Errors raise ``B2Error``
carrying the library status and the BLAS argument position.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import METHODS, B2Error, check, lib

__all__ = [
    "dgemm", "sgemm", "dtrsm", "zgemm3m", "cgemm3m", "set_dgemm_method", "set_sgemm_method",
    "dgemm_device", "sgemm_device", "dgemm_dd_device", "dgemm_error_device", "dtrsm_device",
    "zgemm3m_device", "cgemm3m_device", "last_error", "B2Error", "load_selector",
]


def _addr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    raise TypeError(f"unsupported buffer type {type(x)!r}")


def _c(ch) -> bytes:
    return ch.encode() if isinstance(ch, str) else bytes(ch)


def _ip(v: int):
    return C.byref(C.c_int(int(v)))


def _stream(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return getattr(stream, "cuda_stream", None)


def last_error() -> tuple[int, int]:
    L = lib()
    return L.b2_last_error(), L.b2_last_info()


def _raise_if_failed(what: str) -> None:
    st, info = last_error()
    if st != 0:
        raise B2Error(st, info, what)


# ------------------------------------------------------- drop-in mirror ----
def dgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """``dgemm_`` (src/gemm_driver.c:116): C <- alpha*op(A)*op(B) + beta*C."""
    al, be = C.c_double(alpha), C.c_double(beta)
    lib().dgemm_(_c(transa), _c(transb), _ip(m), _ip(n), _ip(k), C.byref(al), _addr(a), _ip(lda),
                 _addr(b), _ip(ldb), C.byref(be), _addr(c), _ip(ldc))
    _raise_if_failed("dgemm_")
    return c


def dgemm_multi(devices, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                method="default", slices=0):
    """``dgemm_`` on host arrays split by columns of C over the GPUs in
    ``devices`` (an index may repeat); see b2_dgemm_multi."""
    dv = (C.c_int * len(devices))(*[int(d) for d in devices])
    check(lib().b2_dgemm_multi(len(devices), C.addressof(dv), _c(transa), _c(transb), m, n, k,
                               alpha, _addr(a), lda, _addr(b), ldb, beta, _addr(c), ldc,
                               METHODS[method], int(slices)), "b2_dgemm_multi")
    return c


def sgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """``sgemm_`` (src/gemm_driver.c:116 without -DDOUBLE)."""
    al, be = C.c_float(alpha), C.c_float(beta)
    lib().sgemm_(_c(transa), _c(transb), _ip(m), _ip(n), _ip(k), C.byref(al), _addr(a), _ip(lda),
                 _addr(b), _ip(ldb), C.byref(be), _addr(c), _ip(ldc))
    _raise_if_failed("sgemm_")
    return c


def dtrsm(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """``dtrsm_``: op(A) X = alpha B (side 'L') or X op(A) = alpha B; B <- X."""
    al = C.c_double(alpha)
    lib().dtrsm_(_c(side), _c(uplo), _c(transa), _c(diag), _ip(m), _ip(n), C.byref(al), _addr(a),
                 _ip(lda), _addr(b), _ip(ldb))
    _raise_if_failed("dtrsm_")
    return b


def _cplx(v, dt):
    return (dt * 2)(complex(v).real, complex(v).imag)


def zgemm3m(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """``zgemm3m_``: complex128 3M product (ld in complex elements)."""
    al, be = _cplx(alpha, C.c_double), _cplx(beta, C.c_double)
    lib().zgemm3m_(_c(transa), _c(transb), _ip(m), _ip(n), _ip(k), al, _addr(a), _ip(lda),
                   _addr(b), _ip(ldb), be, _addr(c), _ip(ldc))
    _raise_if_failed("zgemm3m_")
    return c


def cgemm3m(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """``cgemm3m_``: complex64 3M product (ld in complex elements)."""
    al, be = _cplx(alpha, C.c_float), _cplx(beta, C.c_float)
    lib().cgemm3m_(_c(transa), _c(transb), _ip(m), _ip(n), _ip(k), al, _addr(a), _ip(lda),
                   _addr(b), _ip(ldb), be, _addr(c), _ip(ldc))
    _raise_if_failed("cgemm3m_")
    return c


def set_dgemm_method(method: str = "fp64", slices: int = 0) -> None:
    check(lib().b2_set_dgemm_method(METHODS[method], int(slices)), "b2_set_dgemm_method")


def load_selector(path: str | None = None) -> bool:
    """Install the learned configuration selector used by method="auto"
    (default: the weights trained on B200 shipped in gemm_avx512f_b200/data)."""
    import os

    if path is None:
        path = os.path.join(os.path.dirname(__file__), "data", "selector_nvidia_b200.f32")
    if not os.path.exists(path):
        return False
    w = np.fromfile(path, np.float32)
    if w.size != lib().b2_mlp_param_count():
        raise ValueError(f"{path}: expected {lib().b2_mlp_param_count()} parameters, got {w.size}")
    check(lib().b2_selector_set(w.ctypes.data), "b2_selector_set")
    return True


def set_sgemm_method(method: str = "fp32") -> None:
    check(lib().b2_set_sgemm_method(METHODS[method]), "b2_set_sgemm_method")


# ------------------------------------------------------ device entries ----
def dgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, method="fp64",
                 slices=0, stream=None):
    check(lib().b2_dgemm(_c(transa), _c(transb), m, n, k, alpha, _addr(a), lda, _addr(b), ldb,
                         beta, _addr(c), ldc, METHODS[method], slices, _stream(stream)),
          "b2_dgemm")
    return c


def sgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, method="fp32",
                 stream=None):
    check(lib().b2_sgemm(_c(transa), _c(transb), m, n, k, alpha, _addr(a), lda, _addr(b), ldb,
                         beta, _addr(c), ldc, METHODS[method], _stream(stream)), "b2_sgemm")
    return c


def dgemm_dd_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c0, ldc, hi, lo, ldo,
                    stream=None):
    check(lib().b2_dgemm_dd(_c(transa), _c(transb), m, n, k, alpha, _addr(a), lda, _addr(b), ldb,
                            beta, _addr(c0), ldc, _addr(hi), _addr(lo), ldo, _stream(stream)),
          "b2_dgemm_dd")
    return hi, lo


def dgemm_error_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c0, c, ldc,
                       stream=None):
    """(normwise, max-elementwise) error of c vs the double-double product."""
    nw, me = C.c_double(0.0), C.c_double(0.0)
    check(lib().b2_dgemm_error(_c(transa), _c(transb), m, n, k, alpha, _addr(a), lda, _addr(b),
                               ldb, beta, _addr(c0), _addr(c), ldc, C.addressof(nw),
                               C.addressof(me), _stream(stream)), "b2_dgemm_error")
    return nw.value, me.value


def dtrsm_device(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, update="fp64", block=0,
                 stream=None):
    check(lib().b2_dtrsm(_c(side), _c(uplo), _c(transa), _c(diag), m, n, alpha, _addr(a), lda,
                         _addr(b), ldb, METHODS[update], block, _stream(stream)), "b2_dtrsm")
    return b


def zgemm3m_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    al, be = _cplx(alpha, C.c_double), _cplx(beta, C.c_double)
    check(lib().b2_zgemm3m(_c(transa), _c(transb), m, n, k, C.addressof(al), _addr(a), lda,
                           _addr(b), ldb, C.addressof(be), _addr(c), ldc, _stream(stream)),
          "b2_zgemm3m")
    return c


def cgemm3m_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=None):
    al, be = _cplx(alpha, C.c_float), _cplx(beta, C.c_float)
    check(lib().b2_cgemm3m(_c(transa), _c(transb), m, n, k, C.addressof(al), _addr(a), lda,
                           _addr(b), ldb, C.addressof(be), _addr(c), ldc, _stream(stream)),
          "b2_cgemm3m")
    return c
