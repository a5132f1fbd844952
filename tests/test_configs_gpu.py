"""Parity on the benchmark configurations themselves: the same seeded inputs
(gemm_avx512f_b200/inputs.py, numpy PCG64 in column-major order) go to the
reference's own CPU routine and to the GPU path, at the configured sizes.

The CPU side is the reference's dgemm_/sgemm_ built from its sources into
oracle/_ref/ (src/gemm_driver.c:116) when this host runs AVX-512F code, else
the oracle's C port, which is bit-exact with it.  Bar for every GEMM:
||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8 with u the unit roundoff of the
arithmetic the method performs.  Errors against the double-double product
(computed on the GPU by the dd yardstick kernel, itself checked against the
CPU dd oracle elsewhere) are stated and bounded.

Config 1: DGEMM NN 1024^3, alpha 1.5, beta 0.5, seed 0; FP64, Ozaki, auto.
Config 2: SGEMM 2048^3 in all four trans combinations and 8192x256x8192 NN
          and TT, alpha 1, beta 0, seed 1; FP32, 1xTF32, 3xTF32, 3xBF16.
Config 3: Ozaki and FP64 DGEMM 4096^3 on a = u exp(phi g), phi 0.1 / 1 / 4,
          seed 2; Ozaki's error vs the dd product within 2x FP64's.
Config 4: the 4096-problem grouped batch (seed 3) in one launch, a strided
          sample checked per problem; zgemm3m 2048^3 against the 3M formula
          with its three real products through the reference dgemm_.
Config 5: DTRSM L/L/N/NonUnit n = 16384 with 4096 right-hand sides (seed 4),
          FP64 and Ozaki trailing updates, residual asserted for each.
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import _lib, blas, inputs
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu
U64, U32 = 2.0 ** -53, 2.0 ** -24
# unit roundoff of the arithmetic each SGEMM method performs
U_SGEMM = {"fp32": U32, "tf32": 2.0 ** -11, "tf32x3": 2.0 ** -21, "bf16x3": 2.0 ** -16}
# normwise error bound vs the FP64 product: constant + K-proportional part
# (the tensor core accumulates in FP32, an error that grows with K)
BOUND_SGEMM = {"fp32": (1e-5, 0.0), "tf32": (2e-3, 0.0), "tf32x3": (2e-6, 2e-8),
               "bf16x3": (4e-5, 1e-8)}


def ref_gemm(ta, tb, m, n, k, alpha, a, b, beta, c):
    """The reference's own dgemm_/sgemm_ where this host runs it, else the
    bit-exact C port."""
    lib = "DGEMM.so" if c.dtype == np.float64 else "SGEMM.so"
    if O.ref_available(lib) and O.host_has_avx512f():
        return O.ref_gemm(ta, tb, m, n, k, alpha, a, b, beta, c)
    return O.gemm(ta, tb, m, n, k, alpha, a, b, beta, c)


def to_dev(x, cuda):
    """Column-major copy on the device, complete on return (the library's own
    stream does not wait for torch's stream)."""
    import torch

    t = torch.from_numpy(np.asfortranarray(x).T).to(cuda)
    torch.cuda.synchronize()
    return t


def from_dev(t):
    """Host copy once every stream has finished (the library's default stream
    is a non-blocking stream, which torch's copy would not wait for)."""
    import torch

    torch.cuda.synchronize()
    return np.asfortranarray(t.cpu().numpy().T)


def dd_product(cuda, ta, tb, m, n, k, alpha, da, lda, db, ldb, beta, dc0, ldc):
    import torch

    hi = torch.empty(m * n, dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    blas.dgemm_dd_device(ta, tb, m, n, k, alpha, da, lda, db, ldb, beta, dc0, ldc, hi, None, m)
    torch.cuda.synchronize()
    return hi


def rel(x, ref):
    import torch

    return float(torch.linalg.vector_norm(x.reshape(-1) - ref.reshape(-1)) /
                 torch.linalg.vector_norm(ref.reshape(-1)))


# ------------------------------------------------------------- config 1 ----
@pytest.mark.parametrize("method", ["fp64", "ozaki", "auto"])
def test_config1_dgemm_1024_seed0(cuda, method):
    n = 1024
    a, b, c = inputs.config1()
    ref = ref_gemm("N", "N", n, n, n, 1.5, a, b, 0.5, c.copy(order="F"))
    blas.set_dgemm_method(method, 0)
    try:
        got = blas.dgemm("N", "N", n, n, n, 1.5, a, n, b, n, 0.5, c.copy(order="F"), n)
    finally:
        blas.set_dgemm_method("fp64", 0)
    err = normalized(got, ref, n, a, b, U64)
    assert err <= 8, (method, err)
    hi = dd_product(cuda, "N", "N", n, n, n, 1.5, to_dev(a, cuda), n, to_dev(b, cuda), n, 0.5,
                    to_dev(c, cuda), n)
    e_dd = rel(to_dev(got, cuda), hi)
    assert e_dd < 4e-15, (method, e_dd)  # FP64-class against the dd product


# ------------------------------------------------------------- config 2 ----
def _sgemm_case(cuda, ta, tb, m, n, k):
    a, b = inputs.config2(m, n, k, ta, tb)
    zero = np.zeros((m, n), dtype=np.float32, order="F")
    ref = ref_gemm(ta, tb, m, n, k, np.float32(1.0), a, b, np.float32(0.0), zero.copy(order="F"))
    opa = (a if ta == "N" else a.T).astype(np.float64)
    opb = (b if tb == "N" else b.T).astype(np.float64)
    exact = opa @ opb
    da, db = to_dev(a, cuda), to_dev(b, cuda)
    for meth in ("fp32", "tf32", "tf32x3", "bf16x3"):
        dc = to_dev(zero, cuda)
        blas.sgemm_device(ta, tb, m, n, k, 1.0, da, a.shape[0], db, b.shape[0], 0.0, dc, m,
                          method=meth)
        got = from_dev(dc)
        err = normalized(got, ref, k, a, b, U_SGEMM[meth])
        assert err <= 8, (meth, ta, tb, m, n, k, err)
        c0, ck = BOUND_SGEMM[meth]
        e64 = np.linalg.norm(got - exact) / np.linalg.norm(exact)
        assert e64 <= c0 + ck * k, (meth, ta, tb, m, n, k, e64)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_config2_sgemm_2048_seed1(cuda, ta, tb):
    _sgemm_case(cuda, ta, tb, 2048, 2048, 2048)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T")])
def test_config2_sgemm_rect_8192x256x8192_seed1(cuda, ta, tb):
    _sgemm_case(cuda, ta, tb, 8192, 256, 8192)


# ------------------------------------------------------------- config 3 ----
@pytest.mark.parametrize("phi", [0.1, 1.0, 4.0])
def test_config3_ozaki_4096_seed2(cuda, phi):
    import torch

    n = 4096
    a, b = inputs.config3(n, phi)
    ref = ref_gemm("N", "N", n, n, n, 1.0, a, b, 0.0, np.zeros((n, n), order="F"))
    da, db = to_dev(a, cuda), to_dev(b, cuda)
    hi = dd_product(cuda, "N", "N", n, n, n, 1.0, da, n, db, n, 0.0, None, n)
    errs = {}
    for meth in ("fp64", "ozaki"):
        dc = torch.zeros(n * n, dtype=torch.float64, device=cuda)
        torch.cuda.synchronize()
        blas.dgemm_device("N", "N", n, n, n, 1.0, da, n, db, n, 0.0, dc, n, method=meth)
        torch.cuda.synchronize()
        got = dc.cpu().numpy().reshape(n, n, order="F")
        e = normalized(got, ref, n, a, b, U64)
        assert e <= 8, (meth, phi, e)
        errs[meth] = rel(dc, hi)
    assert errs["ozaki"] <= 2.0 * errs["fp64"], (phi, errs)


# ------------------------------------------------------------- config 4 ----
def test_config4_grouped_4096_problems_seed3(cuda):
    import torch

    probs = inputs.config4_problems()
    arr, keep = [], []
    for i, (dt, ta, tb, m, n, k) in enumerate(probs):
        rng = np.random.default_rng([3, i])
        npdt = np.float64 if dt == 0 else np.float32
        ar, ac = (m, k) if ta == "N" else (k, m)
        br, bc = (k, n) if tb == "N" else (n, k)
        a = np.asfortranarray(rng.uniform(-1, 1, (ar, ac)).astype(npdt))
        b = np.asfortranarray(rng.uniform(-1, 1, (br, bc)).astype(npdt))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(npdt))
        da, db, dc = to_dev(a, cuda), to_dev(b, cuda), to_dev(c, cuda)
        arr.append(_lib.GemmProblem(dt, ta.encode(), tb.encode(), m, n, k, 1.0, 0.5,
                                    da.data_ptr(), ar, db.data_ptr(), br, dc.data_ptr(), m))
        checked = i % 16 == 0
        keep.append((da, db, dc) + ((a, b, c, ta, tb) if checked else ()))
    carr = (_lib.GemmProblem * len(arr))(*arr)
    stream = torch.cuda.Stream(cuda)
    _lib.check(_lib.lib().b2_gemm_grouped(len(arr), carr, stream.cuda_stream), "b2_gemm_grouped")
    stream.synchronize()
    for i, kp in enumerate(keep):
        if len(kp) == 3:
            continue
        _, _, dc, a, b, c, ta, tb = kp
        m, n = c.shape
        k = a.shape[1] if ta == "N" else a.shape[0]
        dt = a.dtype.type
        ref = ref_gemm(ta, tb, m, n, k, dt(1.0), a, b, dt(0.5), c.copy(order="F"))
        u = U64 if a.dtype == np.float64 else U32
        assert normalized(from_dev(dc), ref, k, a, b, u) <= 8, (i, a.dtype, m, n, k, ta, tb)


def test_config4_zgemm3m_2048_seed3(cuda):
    n = 2048
    a, b, c = inputs.config4_complex(n)
    al, be = 1.0 + 0.0j, 0.0 + 0.0j
    # the 3M formula (P1 = Ar Br, P2 = Ai Bi, P3 = (Ar+Ai)(Br+Bi); Cr = P1 - P2,
    # Ci = P3 - P1 - P2) with its real products through the reference dgemm_
    ar, ai = np.asfortranarray(a.real), np.asfortranarray(a.imag)
    br, bi = np.asfortranarray(b.real), np.asfortranarray(b.imag)
    z = lambda: np.zeros((n, n), order="F")
    p1 = ref_gemm("N", "N", n, n, n, 1.0, ar, br, 0.0, z())
    p2 = ref_gemm("N", "N", n, n, n, 1.0, ai, bi, 0.0, z())
    p3 = ref_gemm("N", "N", n, n, n, 1.0, np.asfortranarray(ar + ai), np.asfortranarray(br + bi),
                  0.0, z())
    ref = al * ((p1 - p2) + 1j * (p3 - p1 - p2)) + be * c
    got = blas.zgemm3m("N", "N", n, n, n, al, a, n, b, n, be, c.copy(order="F"), n)
    den = n * U64 * np.linalg.norm(a) * np.linalg.norm(b)
    assert np.linalg.norm(got - ref) / den <= 8


# ------------------------------------------------------------- config 5 ----
@pytest.mark.parametrize("update", ["fp64", "ozaki"])
def test_config5_dtrsm_16384x4096_seed4(cuda, update):
    import torch

    n, nrhs = 16384, 4096
    a, b = inputs.config5(n, nrhs)
    da, db = to_dev(a, cuda), to_dev(b, cuda)
    del a
    x = db.clone()
    torch.cuda.synchronize()
    blas.dtrsm_device("L", "L", "N", "N", n, nrhs, 1.0, da, n, x, n, update=update)
    torch.cuda.synchronize()
    r = db.clone()
    torch.cuda.synchronize()
    # R = A X - B in FP64 on the device
    blas.dgemm_device("N", "N", n, nrhs, n, 1.0, da, n, x, n, -1.0, r, n, method="fp64")
    torch.cuda.synchronize()
    nr = float(torch.linalg.vector_norm(r))
    na, nx = float(torch.linalg.vector_norm(da)), float(torch.linalg.vector_norm(x))
    scaled = nr / (na * nx * n * U64)
    assert np.isfinite(scaled) and scaled <= 1.0, (update, scaled)
