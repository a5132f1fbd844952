"""ctypes bindings for the CPU checker.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the
cpu_baseline leg of ``bench.py`` import this module.  The product library
never does.

Two libraries are exposed:

* ``liboracle.so`` -- the C restatement in ``oracle.c`` (always built).
* ``_ref/*.so``    -- the reference itself, compiled from its own sources by
  ``oracle/Makefile`` (present wherever it was built; the GPU host receives
  the prebuilt files).  The main-library ``dgemm_``/``sgemm_`` need AVX-512F
  on the host that runs them.

All matrices are numpy arrays in Fortran (column-major) order; leading
dimensions are their first stride in elements.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_lib = None
_ref = {}


def reference_dir() -> str | None:
    """The reference's source tree: $B2_REFERENCE_DIR, else a directory named
    ``reference`` beside this repository's root, when it exists; None
    otherwise (then only the prebuilt _ref/ files, if any, are used)."""
    cand = os.environ.get("B2_REFERENCE_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "reference")
    return cand if os.path.isdir(cand) else None


def build(reference: str | None = None, quiet: bool = True) -> None:
    """Compile liboracle.so and, when the reference sources exist, _ref/."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "all"], check=True, stdout=out, stderr=out)
    ref = reference or reference_dir()
    if ref and os.path.isdir(ref):
        subprocess.run(["make", "-C", HERE, "ref", f"REF={ref}"], check=True, stdout=out,
                       stderr=out)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        d, f, i, l, p, ch = C.c_double, C.c_float, C.c_int, C.c_long, C.c_void_p, C.c_char
        _lib.oracle_dgemm.argtypes = [ch, ch, i, i, i, d, p, i, p, i, d, p, i]
        _lib.oracle_sgemm.argtypes = [ch, ch, i, i, i, f, p, i, p, i, f, p, i]
        _lib.oracle_dgemm_dd.argtypes = [ch, ch, i, i, i, d, p, i, p, i, d, p, i, p, p, i]
        for nm in ("rn", "rt", "ln", "lt"):
            getattr(_lib, f"oracle_trsm_kernel_{nm}").argtypes = [l, l, p, p, p, l, l]
        _lib.oracle_dtrsm.argtypes = [ch, ch, ch, ch, i, i, d, p, i, p, i, i]
        _lib.oracle_zgemm3m.argtypes = [ch, ch, i, i, i, p, p, i, p, i, p, p, i]
        _lib.oracle_cgemm3m.argtypes = [ch, ch, i, i, i, p, p, i, p, i, p, p, i]
        _lib.oracle_gemm3m_kernel_z.argtypes = [l, l, l, d, d, p, l, p, l, p, l]
    return _lib


def ref_available(name: str = "DGEMM.so") -> bool:
    return os.path.exists(os.path.join(REF_DIR, name))


def host_has_avx512f() -> bool:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    return " avx512f" in line
    except OSError:
        pass
    return False


def ref_lib(name: str) -> C.CDLL:
    if name not in _ref:
        _ref[name] = C.CDLL(os.path.join(REF_DIR, name))
    return _ref[name]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _ld(a) -> int:
    return max(1, a.strides[1] // a.itemsize) if a.ndim == 2 else max(1, a.shape[0])


def _ch(c) -> bytes:
    return c.encode() if isinstance(c, str) else c


# ---------------------------------------------------------------- GEMM ----
def gemm(transa, transb, m, n, k, alpha, a, b, beta, c):
    """oracle_dgemm / oracle_sgemm on Fortran-ordered arrays, in place on c."""
    f = lib().oracle_dgemm if c.dtype == np.float64 else lib().oracle_sgemm
    f(_ch(transa), _ch(transb), m, n, k, alpha, _ptr(a), _ld(a), _ptr(b), _ld(b), beta,
      _ptr(c), _ld(c))
    return c


def gemm_dd(transa, transb, m, n, k, alpha, a, b, beta, c0):
    """Double-double oracle: returns (hi, lo), each m x n Fortran order."""
    hi = np.zeros((m, n), order="F")
    lo = np.zeros((m, n), order="F")
    lib().oracle_dgemm_dd(_ch(transa), _ch(transb), m, n, k, alpha, _ptr(a), _ld(a), _ptr(b),
                          _ld(b), beta, _ptr(c0), _ld(c0) if c0 is not None else 1, _ptr(hi),
                          _ptr(lo), max(1, m))
    return hi, lo


def ref_gemm(transa, transb, m, n, k, alpha, a, b, beta, c, which="main"):
    """The reference's own dgemm_/sgemm_ (Fortran ABI, all by pointer):
    which = "main" (src/gemm_driver.c:116), "oblike" (OpenBLAS-like dgemm.c:484 /
    sgemm.c:579), "8x8opt" / "8x8std" (kernel_avx512_opt8x8.c:821 /
    kernel_avx512_standard8x8.c:843, serial, FP64)."""
    dbl = c.dtype == np.float64
    if which == "main":
        fn = ref_lib("DGEMM.so").dgemm_ if dbl else ref_lib("SGEMM.so").sgemm_
    elif which in ("8x8opt", "8x8std"):  # kernel_avx512_{opt,standard}8x8.c:821/843 (FP64 only)
        fn = ref_lib("dgemm_8x8_opt.so" if which == "8x8opt" else "dgemm_8x8_std.so").dgemm_
    else:
        fn = ref_lib("oblike_dgemm.so").dgemm_ if dbl else ref_lib("oblike_sgemm.so").SGEMM_
    ct = C.c_double if dbl else C.c_float
    i = lambda v: C.byref(C.c_int(v))
    fn(C.c_char_p(_ch(transa)), C.c_char_p(_ch(transb)), i(m), i(n), i(k), C.byref(ct(alpha)),
       _ptr(a), i(_ld(a)), _ptr(b), i(_ld(b)), C.byref(ct(beta)), _ptr(c), i(_ld(c)))
    return c


# ---------------------------------------------------------------- TRSM ----
def trsm(side, uplo, transa, diag, m, n, alpha, a, b, nb=128):
    lib().oracle_dtrsm(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n, alpha, _ptr(a),
                       _ld(a), _ptr(b), _ld(b), nb)
    return b


def trsm_kernel(kind, M, N, sa, sb, C_, LDB, LDC):
    getattr(lib(), f"oracle_trsm_kernel_{kind}")(M, N, _ptr(sa), _ptr(sb), _ptr(C_), LDB, LDC)


def ref_trsm_kernel(kind, M, N, sa, sb, C_, LDB, LDC):
    fn = getattr(ref_lib("dtrsm_kernels.so"), f"dtrsm_solve_{kind}_m{M}n{N}")
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_long]
    fn(_ptr(sa), _ptr(sb), _ptr(C_), LDB, LDC)


# ------------------------------------------------------------------ 3M ----
def gemm3m(transa, transb, m, n, k, alpha, a, b, beta, c):
    """oracle_zgemm3m / oracle_cgemm3m on complex Fortran arrays, in place on c."""
    dbl = c.dtype == np.complex128
    rt = np.float64 if dbl else np.float32
    al = np.array([alpha.real, alpha.imag], dtype=rt)
    be = np.array([beta.real, beta.imag], dtype=rt)
    f = lib().oracle_zgemm3m if dbl else lib().oracle_cgemm3m
    f(_ch(transa), _ch(transb), m, n, k, _ptr(al), _ptr(a), _ld(a), _ptr(b), _ld(b), _ptr(be),
      _ptr(c), _ld(c))
    return c


def gemm3m_kernel_z(m, n, k, alphar, alphai, a, b, c):
    """Unpacked restatement of the zgemm3m kernel contract; a: m x k, b: n x k real."""
    lib().oracle_gemm3m_kernel_z(m, n, k, alphar, alphai, _ptr(a), _ld(a), _ptr(b), _ld(b),
                                 _ptr(c), _ld(c))
    return c


def ref_gemm3m_kernel(which, m, n, k, alphar, alphai, pa, pb, c):
    """The reference 3M kernel (packed panels) -- 'z2x8' or 'c16x4'."""
    dbl = which == "z2x8"
    lb = ref_lib("zgemm3m_2x8.so" if dbl else "cgemm3m_16x4.so")
    ct = C.c_double if dbl else C.c_float
    lb.kern.argtypes = [C.c_long, C.c_long, C.c_long, ct, ct, C.c_void_p, C.c_void_p, C.c_void_p,
                        C.c_long]
    lb.kern(m, n, k, alphar, alphai, _ptr(pa), _ptr(pb), _ptr(c), _ld(c))


# Reference real GEMM kernels of the OpenBLAS kernel ABI:
# C(m x n, ldc) += alpha * A_packed * B_packed.  name -> (library, symbol,
# integer type of m/n/k/ldc, scalar type, A panel width, B panel width).
GEMM_KERNELS = {
    "d16x2": ("oblike_dgemm.so", "CNAME", C.c_int, C.c_double, 16, 2),   # dgemm.c:247-263
    "d4x8": ("dgemm_4x8.so", "kern", C.c_long, C.c_double, 4, 8),        # dgemm_kernel_4x8_skylakex_2.c:661
    "s16x4": ("oblike_sgemm.so", "CNAME", C.c_int, C.c_float, 16, 4),    # sgemm.c:397-412
}


def panel_widths(unroll: int):
    """Panel widths a packing of the given unroll produces: full panels, then
    the remainder in halving widths (the tcopy/ncopy routines, dgemm.c:304-403)."""
    w, out = unroll, []
    while w >= 1:
        out.append(w)
        w //= 2
    return out


def ref_gemm_kernel(which, m, n, k, alpha, pa, pb, c):
    """The reference kernel `which` on packed panels, in place on c (Fortran)."""
    libname, sym, it, st, _, _ = GEMM_KERNELS[which]
    fn = getattr(ref_lib(libname), sym)
    fn.argtypes = [it, it, it, st, C.c_void_p, C.c_void_p, C.c_void_p, it]
    fn(m, n, k, alpha, _ptr(pa), _ptr(pb), _ptr(c), _ld(c))


def pack_panels(x: np.ndarray, widths) -> np.ndarray:
    """Greedy panel packing used by the OpenBLAS kernel ABI: rows of x (dim x k)
    cut into panels of the given widths (largest first), each stored k-major."""
    out, i, dim = [], 0, x.shape[0]
    for w in widths:
        while dim - i >= w:
            out.append(np.ascontiguousarray(x[i:i + w].T).reshape(-1))
            i += w
    return np.ascontiguousarray(np.concatenate(out)) if out else np.zeros(0, x.dtype)


# ------------------------------------------------------------ metrics ----
def normalized_error(c, c_ref, k, a_norm, b_norm, unit_roundoff):
    """||C - C_ref||_F / (K * u * ||A||_F * ||B||_F) -- the parity yardstick."""
    den = max(k, 1) * unit_roundoff * a_norm * b_norm
    num = float(np.linalg.norm((c - c_ref).astype(np.float64)))
    return num / den if den > 0 else num
