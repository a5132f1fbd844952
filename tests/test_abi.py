"""CPU tests of the C ABI: the library loads, exports every symbol the header
declares, and the host-side argument checks behave like BLAS xerbla without
touching C (no GPU is needed for any of this: argument checks run before the
library looks for a device)."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from gemm_avx512f_b200 import _lib
from gemm_avx512f_b200 import blas


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _lib.declared_symbols()
    assert {"dgemm_", "sgemm_", "dtrsm_", "zgemm3m_", "cgemm3m_", "b2_dgemm"} <= set(declared)
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported
    # nothing else leaks out of the library (internal symbols are hidden)
    assert exported - set(declared) <= {"_init", "_fini"}


def test_drop_in_signature_matches_reference_abi():
    # dgemm_(const char*, const char*, const int* x3, const double*, const double*,
    #        const int*, const double*, const int*, const double*, double*, const int*)
    fn = _lib.lib().dgemm_
    assert len(fn.argtypes) == 13 and fn.restype is None


@pytest.mark.parametrize("args,info", [
    (dict(m=-1), 3), (dict(n=-2), 4), (dict(k=-1), 5), (dict(lda=3), 8), (dict(ldb=2), 10),
    (dict(ldc=4), 13)])
def test_dgemm_argument_errors_leave_c_untouched(args, info):
    m, n, k = args.get("m", 5), args.get("n", 6), args.get("k", 7)
    lda, ldb, ldc = args.get("lda", 5), args.get("ldb", 7), args.get("ldc", 5)
    a = np.ones((7, 7), order="F")
    b = np.ones((7, 7), order="F")
    c = np.full((7, 7), 3.0, order="F")
    before = c.copy()
    with pytest.raises(_lib.B2Error) as ei:
        blas.dgemm("N", "N", m, n, k, 1.0, a, lda, b, ldb, 0.0, c, ldc)
    assert ei.value.status == _lib.B2_ERR_ARG and ei.value.info == info
    assert np.array_equal(c, before)


def test_transposed_leading_dimension_rules():
    a = np.ones((7, 7), order="F")
    c = np.zeros((7, 7), order="F")
    # transA='T': A is k x m, so lda must be >= k (=7), 5 is invalid -> info 8
    with pytest.raises(_lib.B2Error) as ei:
        blas.dgemm("T", "N", 5, 5, 7, 1.0, a, 5, a, 7, 0.0, c, 7)
    assert ei.value.info == 8
    # transB='X' (any non-N char) means transpose: B is n x k, ldb >= n (=6)
    with pytest.raises(_lib.B2Error) as ei:
        blas.dgemm("N", "X", 7, 6, 5, 1.0, a, 7, a, 5, 0.0, c, 7)
    assert ei.value.info == 10


def test_null_c_is_rejected():
    L = _lib.lib()
    one = C.c_double(1.0)
    i5 = C.c_int(5)
    L.dgemm_(b"N", b"N", C.byref(i5), C.byref(i5), C.byref(i5), C.byref(one), None,
             C.byref(i5), None, C.byref(i5), C.byref(one), None, C.byref(i5))
    assert blas.last_error() == (_lib.B2_ERR_ARG, 12)


def test_status_strings():
    L = _lib.lib()
    for s in range(7):
        assert L.b2_status_string(s)


@pytest.mark.parametrize("args,info", [
    (dict(side="X"), 1), (dict(uplo="Q"), 2), (dict(transa="Z"), 3), (dict(diag="W"), 4),
    (dict(m=-1), 5), (dict(n=-1), 6), (dict(lda=3), 9), (dict(ldb=2), 11)])
def test_dtrsm_argument_errors_leave_b_untouched(args, info):
    a = np.eye(8, order="F")
    b = np.full((8, 8), 5.0, order="F")
    before = b.copy()
    kw = dict(side="L", uplo="L", transa="N", diag="N", m=6, n=5, lda=8, ldb=8)
    kw.update(args)
    with pytest.raises(_lib.B2Error) as ei:
        blas.dtrsm(kw["side"], kw["uplo"], kw["transa"], kw["diag"], kw["m"], kw["n"], 1.0, a,
                   kw["lda"], b, kw["ldb"])
    assert ei.value.status == _lib.B2_ERR_ARG and ei.value.info == info
    assert np.array_equal(b, before)


def test_openblas_argument_mode(capfd):
    """B2_ARGS_OPENBLAS: the OpenBLAS-like dgemm_ checks (dgemm.c:488-498) --
    M < 1 or N < 1 returns silently, a short LDA / LDB prints the reference's
    message on stdout and returns, C untouched either way."""
    L = _lib.lib()
    assert L.b2_set_arg_mode(7) == -1  # unknown mode: nothing changes
    prev = L.b2_set_arg_mode(1)
    try:
        a = np.ones((7, 7), order="F")
        c = np.full((7, 7), 3.0, order="F")
        before = c.copy()
        blas.dgemm("N", "N", -1, 5, 5, 1.0, a, 7, a, 7, 0.0, c, 7)  # silent quick return
        blas.dgemm("N", "N", 5, 0, 5, 1.0, a, 7, a, 7, 0.0, c, 7)
        assert np.array_equal(c, before)
        cases = [("N", "N", 7, 5, 5, 5, 7, "LDA < M with column-major matrix A"),
                 ("T", "N", 5, 5, 7, 5, 7, "LDA < K with row-major matrix A"),
                 ("N", "N", 5, 5, 7, 7, 5, "LDB < K with column-major matrix B"),
                 ("N", "T", 5, 7, 5, 7, 5, "LDB < N with row-major matrix B")]
        for ta, tb, m, n, k, lda, ldb, text in cases:
            capfd.readouterr()
            with pytest.raises(_lib.B2Error) as ei:
                blas.dgemm(ta, tb, m, n, k, 1.0, a, lda, a, ldb, 0.0, c, 7)
            assert ei.value.status == _lib.B2_ERR_ARG
            out = capfd.readouterr().out
            assert out == f"ERROR: {text}. Please check input parameters.\n", out
            assert np.array_equal(c, before)
        af = a.astype(np.float32)
        cf = c.astype(np.float32)
        capfd.readouterr()
        with pytest.raises(_lib.B2Error):
            blas.sgemm("N", "N", 7, 5, 5, 1.0, af, 5, af, 7, 0.0, cf, 7)
        assert "LDA < M" in capfd.readouterr().out
    finally:
        assert L.b2_set_arg_mode(prev) == 1


@pytest.mark.parametrize("ndev,devs,args,info", [
    (0, [0], {}, 0), (65, [0] * 65, {}, 0), (2, [0, 0], dict(m=-1), 3), (2, [0, 0], dict(ldc=4), 13)])
def test_dgemm_multi_argument_errors(ndev, devs, args, info):
    # checked before any device is looked at
    m, n, k = args.get("m", 5), args.get("n", 6), 7
    ldc = args.get("ldc", 5)
    a, b = np.ones((5, 7), order="F"), np.ones((7, 6), order="F")
    c = np.full((5, 6), 3.0, order="F")
    dv = (C.c_int * len(devs))(*devs)
    st = _lib.lib().b2_dgemm_multi(ndev, C.addressof(dv), b"N", b"N", m, n, k, 1.0,
                                   a.ctypes.data, 5, b.ctypes.data, 7, 0.0, c.ctypes.data, ldc,
                                   0, 0)
    assert st == _lib.B2_ERR_ARG
    assert _lib.lib().b2_last_info() == info
    assert (c == 3.0).all()


def test_problem_struct_layout_matches_the_header(tmp_path):
    """b2_gemm_problem as a C compiler lays it out from include/b2blas.h (gcc
    here) and the ctypes mirror the Python bindings pass to
    b2_gemm_grouped: same size and the same offset for every field."""
    import os

    hdr = os.path.dirname(_lib.HEADER)
    fields = [f[0] for f in _lib.GemmProblem._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"b2blas.h\"\n"
                   "int main(void) {\n  printf(\"size %zu\\n\", sizeof(b2_gemm_problem));\n"
                   + "".join(f"  printf(\"{f} %zu\\n\", offsetof(b2_gemm_problem, {f}));\n"
                             for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", hdr, str(src), "-o", str(exe)], check=True)
    out = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.splitlines())
    assert int(out["size"]) == C.sizeof(_lib.GemmProblem)
    for f in fields:
        assert int(out[f]) == getattr(_lib.GemmProblem, f).offset, f


def test_unchanged_c_caller_links_against_the_library(tmp_path):
    """A C program written against the reference's dgemm_ (the prototype of
    src/gemm_driver.c:116) links against libb2blas.so as the integration
    notes show, and sees BLAS argument checking through b2_last_error /
    b2_last_info (no device is needed before the arguments are valid)."""
    import os

    libdir = os.path.dirname(_lib.LIB_PATH)
    src = tmp_path / "app.c"
    src.write_text(r"""
#include <stdio.h>
extern void dgemm_(const char*, const char*, const int*, const int*, const int*,
                   const double*, const double*, const int*, const double*, const int*,
                   const double*, double*, const int*);
extern int b2_last_error(void);
extern int b2_last_info(void);
int main(void) {
  double a[4] = {1, 2, 3, 4}, b[4] = {1, 0, 0, 1}, c[4] = {7, 7, 7, 7};
  double alpha = 1.0, beta = 0.0;
  int m = -1, n = 2, k = 2, lda = 2, ldb = 2, ldc = 2;
  dgemm_("N", "N", &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
  printf("bad_m %d %d %g\n", b2_last_error(), b2_last_info(), c[0]);
  m = 2; lda = 1;
  dgemm_("N", "N", &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
  printf("bad_lda %d %d %g\n", b2_last_error(), b2_last_info(), c[0]);
  return 0;
}
""")
    exe = tmp_path / "app"
    subprocess.run(["gcc", str(src), "-o", str(exe), f"-L{libdir}", "-lb2blas",
                    f"-Wl,-rpath,{libdir}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    assert out[0].split() == ["bad_m", str(_lib.B2_ERR_ARG), "3", "7"]
    assert out[1].split() == ["bad_lda", str(_lib.B2_ERR_ARG), "8", "7"]
