"""Loader for libb2blas.so (the C ABI declared in include/b2blas.h).

The library is built in-tree (``gemm_avx512f_b200/lib/libb2blas.so``).  There
is no fallback of any kind: if the shared library is missing or fails to load,
every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libb2blas.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "b2blas.h")

B2_OK = 0
B2_ERR_ARG = 1
B2_ERR_CUDA = 2
B2_ERR_NOMEM = 3
B2_ERR_TIMEOUT = 4
B2_ERR_UNSUPPORTED = 5
B2_ERR_NO_DEVICE = 6

METHODS = {
    "default": 0, "fp64": 1, "ozaki": 2, "auto": 3,
    "fp32": 10, "tf32": 11, "tf32x3": 12, "bf16x3": 13,
}

_lib: C.CDLL | None = None


class GemmProblem(C.Structure):
    """Mirror of b2_gemm_problem (include/b2blas.h)."""
    _fields_ = [("dtype", C.c_int), ("transa", C.c_char), ("transb", C.c_char),
                ("m", C.c_int), ("n", C.c_int), ("k", C.c_int),
                ("alpha", C.c_double), ("beta", C.c_double),
                ("A", C.c_void_p), ("lda", C.c_int), ("B", C.c_void_p), ("ldb", C.c_int),
                ("C", C.c_void_p), ("ldc", C.c_int),
                ("alpha_i", C.c_double), ("beta_i", C.c_double)]


class B2Error(RuntimeError):
    def __init__(self, status: int, info: int = 0, what: str = ""):
        self.status, self.info = status, info
        msg = f"{what}: status {status}" + (f" (argument {info})" if info else "")
        try:
            msg += f" [{lib().b2_status_string(status).decode()}]"
        except Exception:  # pragma: no cover - message decoration only
            pass
        super().__init__(msg)


def declared_symbols() -> list[str]:
    """Function names declared in include/b2blas.h."""
    with open(HEADER) as fh:
        text = fh.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^B2_API\s+[^(]*?\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text,
                                 flags=re.M)))


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libb2blas.so is not built ({LIB_PATH}); run "
                           "`python -m gemm_avx512f_b200.build`")
    L = C.CDLL(LIB_PATH)
    i, d, f, p, ch = C.c_int, C.c_double, C.c_float, C.c_void_p, C.c_char
    pi, pd, pf, pc = C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_char_p
    L.b2_last_error.restype = i
    L.b2_last_info.restype = i
    L.b2_status_string.restype = C.c_char_p
    L.b2_status_string.argtypes = [i]
    L.b2_device_count.restype = i
    L.b2_version.restype = i
    L.b2_set_dgemm_method.argtypes = [i, i]
    L.b2_set_sgemm_method.argtypes = [i]
    L.b2_set_arg_mode.argtypes = [i]
    gemm_ptrs = [pc, pc, pi, pi, pi, p, p, pi, p, pi, p, p, pi]
    for nm in ("dgemm_", "sgemm_", "SGEMM_", "zgemm3m_", "cgemm3m_"):
        getattr(L, nm).argtypes = gemm_ptrs
        getattr(L, nm).restype = None
    L.dtrsm_.argtypes = [pc, pc, pc, pc, pi, pi, p, p, pi, p, pi]
    L.dtrsm_.restype = None
    L.b2_dgemm.argtypes = [ch, ch, i, i, i, d, p, i, p, i, d, p, i, i, i, p]
    L.b2_dgemm_multi.argtypes = [i, p, ch, ch, i, i, i, d, p, i, p, i, d, p, i, i, i]
    L.b2_sgemm.argtypes = [ch, ch, i, i, i, f, p, i, p, i, f, p, i, i, p]
    L.b2_dgemm_dd.argtypes = [ch, ch, i, i, i, d, p, i, p, i, d, p, i, p, p, i, p]
    L.b2_dtrsm.argtypes = [ch, ch, ch, ch, i, i, d, p, i, p, i, i, i, p]
    L.b2_zgemm3m.argtypes = [ch, ch, i, i, i, p, p, i, p, i, p, p, i, p]
    L.b2_cgemm3m.argtypes = [ch, ch, i, i, i, p, p, i, p, i, p, p, i, p]
    lg = C.c_long
    L.b2_dgemm_kernel.argtypes = [i, i, lg, lg, lg, d, p, p, p, lg, p]
    L.b2_sgemm_kernel.argtypes = [i, i, lg, lg, lg, f, p, p, p, lg, p]
    L.b2_zgemm3m_kernel.argtypes = [i, i, lg, lg, lg, d, d, p, p, p, lg, p]
    L.b2_cgemm3m_kernel.argtypes = [i, i, lg, lg, lg, f, f, p, p, p, lg, p]
    L.b2_dtrsm_kernel.argtypes = [ch, ch, lg, lg, p, p, p, lg, lg, p]
    L.b2_dgemm_error.argtypes = [ch, ch, i, i, i, d, p, i, p, i, d, p, p, i, pd, pd, p]
    L.b2_device_error.argtypes = [i]
    L.b2_dgemm_ozaki_noalloc.argtypes = [ch, ch, i, i, i, d, p, i, p, i, d, p, i, i, p]
    L.b2_dgemm_ozaki_noalloc.restype = i
    L.b2_dgemm_ozaki_noalloc_error.argtypes = [i, p]
    L.b2_dgemm_ozaki_noalloc_error.restype = i
    L.b2_test_bounded_wait.argtypes = [C.c_longlong, i]
    L.b2_test_bounded_wait.restype = i
    L.b2_gemm_grouped.argtypes = [i, p, p]
    L.b2_grouped_plan_create.argtypes = [i, p, C.POINTER(C.c_void_p)]
    L.b2_grouped_plan_launch.argtypes = [p, p]
    L.b2_grouped_plan_destroy.argtypes = [p]
    for nm in ("b2_gemm_grouped", "b2_grouped_plan_create", "b2_grouped_plan_launch",
               "b2_grouped_plan_destroy"):
        getattr(L, nm).restype = i
    L.b2_tune_config_count.restype = i
    L.b2_mlp_param_count.restype = i
    L.b2_dgemm_config.argtypes = [ch, ch, i, i, i, d, p, i, p, i, d, p, i, i, p]
    L.b2_sgemm_config.argtypes = [ch, ch, i, i, i, f, p, i, p, i, f, p, i, i, p]
    L.b2_tune_sweep_sgemm.argtypes = [i, p, i, p]
    L.b2_sgemm_selector_choose.argtypes = [i, ch, ch, i, i, i, i]
    L.b2_tune_sweep.argtypes = [i, p, i, p]
    L.b2_mlp_train.argtypes = [i, p, p, i, i, f, i, p, p, p]
    L.b2_mlp_forward.argtypes = [p, i, p, p]
    L.b2_mlp_gradient.argtypes = [p, i, p, p, p, p]
    L.b2_selector_set.argtypes = [p]
    L.b2_selector_choose.argtypes = [ch, ch, i, i, i, i, i]
    L.b2_selector_predict.argtypes = [ch, ch, i, i, i, i, p]
    for nm in ("b2_dgemm_config", "b2_tune_sweep", "b2_sgemm_config", "b2_tune_sweep_sgemm",
               "b2_sgemm_selector_choose", "b2_mlp_train", "b2_mlp_forward",
               "b2_mlp_gradient", "b2_selector_set", "b2_selector_choose", "b2_selector_predict"):
        getattr(L, nm).restype = i
    L.b2_set_fp64_config.argtypes = [i, i, i]
    L.b2_set_fp64_config.restype = i
    L.b2_launch_count.restype = C.c_longlong
    L.b2_profile_enable.argtypes = [i]
    L.b2_profile_report.argtypes = [C.c_char_p, i]
    L.b2_profile_timeline.argtypes = [C.c_char_p, i]
    for nm in ("b2_dgemm", "b2_dgemm_multi", "b2_sgemm", "b2_dgemm_dd", "b2_dtrsm", "b2_zgemm3m", "b2_cgemm3m",
               "b2_dgemm_error", "b2_device_error", "b2_set_dgemm_method", "b2_set_sgemm_method"):
        getattr(L, nm).restype = i
    _lib = L
    return L


def profile_enable(on: bool = True) -> None:
    lib().b2_profile_enable(1 if on else 0)


def profile_report() -> dict[str, tuple[int, float]]:
    """{kernel name: (launches, total ms)} since the last report (synchronizes)."""
    buf = C.create_string_buffer(1 << 16)
    lib().b2_profile_report(buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


def profile_timeline() -> list[tuple[str, float, float]]:
    """[(kernel name, start ms, end ms)] per launch since the last report, in
    issue order, relative to the first launch's start (synchronizes)."""
    buf = C.create_string_buffer(1 << 20)
    lib().b2_profile_timeline(buf, len(buf))
    out = []
    for line in buf.value.decode().splitlines():
        name, a, b = line.split()
        out.append((name, float(a), float(b)))
    return out


def launch_count() -> int:
    return int(lib().b2_launch_count())


def check(status: int, what: str) -> None:
    if status != B2_OK:
        raise B2Error(status, lib().b2_last_info(), what)
