"""GPU tests of the fused 3M complex GEMMs (zgemm3m_ on FP64 DMMA, cgemm3m_ on
FP32 FFMA), through the C ABI.

* parity with the CPU 3M restatement (oracle_zgemm3m / oracle_cgemm3m, whose
  real products run through the bit-exact restatement of the reference dgemm_):
  ||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8 on complex Frobenius norms;
* pinned to the reference's own zgemm3m kernel (zgemm3m_kernel_2x8_skylakex.c:
  C_cplx += alpha * A_real B_real^T) through the golden vectors: real
  operands passed as complex with zero imaginary part and beta = 1;
* all four op() forms ('N', 'T', 'C' conjugate-transpose, 'R' conjugate),
  padded leading dimensions left untouched, reference beta semantics.
"""
import os

import numpy as np
import pytest

from gemm_avx512f_b200 import _lib, blas
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _op(x, t):
    return {"N": x, "T": x.T, "C": x.conj().T, "R": x.conj()}[t]


def _cmat(rng, r, c, dtype, pad=0):
    x = rng.uniform(-1, 1, (r + pad, c)) + 1j * rng.uniform(-1, 1, (r + pad, c))
    return np.asfortranarray(x.astype(dtype))


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (13, 9, 21), (65, 33, 129), (200, 150, 300),
                                   (512, 512, 512)])
def test_gemm3m_parity(cuda, dtype, m, n, k):
    rng = np.random.default_rng(m + 2 * n + 3 * k)
    u = np.finfo(dtype).eps / 2
    fn = blas.zgemm3m if dtype == np.complex128 else blas.cgemm3m
    for ta, tb in [("N", "N"), ("T", "C"), ("C", "N"), ("R", "T")]:
        ar, ac = (m, k) if ta in "NR" else (k, m)
        br, bc = (k, n) if tb in "NR" else (n, k)
        a = _cmat(rng, ar, ac, dtype, pad=2)
        b = _cmat(rng, br, bc, dtype, pad=1)
        c = _cmat(rng, m, n, dtype, pad=3)
        al, be = 0.75 - 1.25j, 0.5 + 0.25j
        ref = c.copy(order="F")
        O.gemm3m(ta, tb, m, n, k, al, a[:ar], b[:br], be, ref[:m])
        got = c.copy(order="F")
        fn(ta, tb, m, n, k, al, a, a.shape[0], b, b.shape[0], be, got, got.shape[0])
        assert np.array_equal(got[m:], c[m:]), "padding rows of C were written"
        den = k * u * np.linalg.norm(a[:ar]) * np.linalg.norm(b[:br])
        err = np.linalg.norm((got[:m] - ref[:m]).astype(np.complex128)) / den
        assert err <= 8, (dtype, m, n, k, ta, tb, err)
        # and it is the complex product
        exact = al * _op(a[:ar].astype(np.complex128), ta) @ _op(b[:br].astype(np.complex128), tb) \
            + be * c[:m].astype(np.complex128)
        assert np.linalg.norm(got[:m] - exact) <= 64 * den


def test_pinned_to_reference_3m_kernel_golden(cuda):
    z = np.load(os.path.join(GOLD, "zgemm3m_kernel_ref.npz"))
    for i in range(int(z["count"])):
        m, n, k = (int(v) for v in z[f"z{i}_meta"])
        ar, ai = (float(v) for v in z[f"z{i}_alpha"])
        a = np.asfortranarray(z[f"z{i}_a"].astype(np.complex128))   # m x k, imag 0
        b = np.asfortranarray(z[f"z{i}_b"].astype(np.complex128))   # n x k, imag 0
        c = np.asfortranarray(z[f"z{i}_c"].copy())                 # (m+1) x n
        blas.zgemm3m("N", "T", m, n, k, complex(ar, ai), a, m, b, n, 1.0, c, c.shape[0])
        np.testing.assert_allclose(c, z[f"z{i}_out"], rtol=0, atol=1e-13)


def test_gemm3m_beta_semantics_and_device_api(cuda):
    import torch

    m, n, k = 40, 30, 20
    rng = np.random.default_rng(0)
    a = _cmat(rng, m, k, np.complex128)
    b = _cmat(rng, k, n, np.complex128)
    c = np.asfortranarray(np.full((m, n), np.nan + 0j))
    blas.zgemm3m("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m)
    assert np.isnan(c.real).all()  # beta == 0 keeps NaN (reference beta rule)
    # alpha == 0 skips the product: C <- beta C exactly
    c2 = _cmat(rng, m, n, np.complex128)
    got = c2.copy(order="F")
    blas.zgemm3m("N", "N", m, n, k, 0.0, a, m, b, k, 2.0, got, m)
    assert np.array_equal(got, 2.0 * c2)
    # device pointers through b2_zgemm3m
    da = torch.from_numpy(np.ascontiguousarray(a.T)).to(cuda)  # column-major complex
    db = torch.from_numpy(np.ascontiguousarray(b.T)).to(cuda)
    dc = torch.zeros((n, m), dtype=torch.complex128, device=cuda)
    blas.zgemm3m_device("N", "N", m, n, k, 1.0, da, m, db, k, 0.0, dc, m)
    torch.cuda.synchronize()
    np.testing.assert_allclose(dc.cpu().numpy().T, a @ b, rtol=0, atol=1e-12)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "T")])
def test_zgemm3m_three_gemm_path_large(cuda, ta, tb):
    """From 2^35 multiply-adds zgemm3m runs three FP64 DMMA GEMMs between a
    pre-add and a combine pass: 4096^3 against the complex128 product of
    torch on the same device (plain FP64 reference of the same op)."""
    import torch

    n = 4096
    g = torch.Generator(device=cuda).manual_seed(11)
    A = torch.complex(torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1,
                      torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1)
    B = torch.complex(torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1,
                      torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1)
    C0 = torch.complex(torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g),
                       torch.zeros(n, n, device=cuda, dtype=torch.float64))
    # storage is column-major: the tensors hold the transposes of the matrices
    Am, Bm = A.t(), B.t()
    op = {"N": lambda x: x, "T": lambda x: x.t(), "C": lambda x: x.conj().t()}
    al, be = 0.75 - 1.25j, 0.5 + 0.25j
    ref = al * (op[ta](Am) @ op[tb](Bm)) + be * C0.t()
    C = C0.clone()
    blas.zgemm3m_device(ta, tb, n, n, n, al, A, n, B, n, be, C, n)
    torch.cuda.synchronize()
    got = C.t()
    u = 2.0 ** -53
    den = n * u * float(torch.linalg.norm(A)) * float(torch.linalg.norm(B)) * abs(al)
    err = float(torch.linalg.norm(got - ref)) / den
    assert err <= 8, (ta, tb, err)


def test_zgemm3m_config4_size_in_one_launch(cuda):
    """The configured zgemm3m size, 2048^3 complex128, runs its three real
    products and the pre/post additions in one launch (the library counts
    every kernel it launches), against the complex128 product of torch."""
    import torch

    n = 2048
    g = torch.Generator(device=cuda).manual_seed(12)
    A = torch.complex(torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1,
                      torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1)
    B = torch.complex(torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1,
                      torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1)
    C = torch.zeros(n, n, device=cuda, dtype=torch.complex128)
    torch.cuda.synchronize()
    n0 = _lib.launch_count()
    blas.zgemm3m_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n)
    torch.cuda.synchronize()
    assert _lib.launch_count() - n0 == 1
    ref = A.t() @ B.t()
    den = n * 2.0 ** -53 * float(torch.linalg.norm(A)) * float(torch.linalg.norm(B))
    assert float(torch.linalg.norm(C.t() - ref)) / den <= 8


_FUSED_SCRIPT = """
import os, sys
sys.path.insert(0, ROOT)
import torch
from gemm_avx512f_b200 import _lib, blas
cuda = torch.device("cuda:0")
_lib.profile_enable(True)
op = {"N": lambda x: x, "T": lambda x: x.t(), "C": lambda x: x.conj().t(), "R": lambda x: x.conj()}
for ta, tb, m, n, k in [("N", "N", 2048, 2048, 256), ("C", "T", 1100, 2100, 333),
                        ("R", "C", 4096, 640, 96)]:
    g = torch.Generator(device=cuda).manual_seed(m + n + k)
    ar_, ac_ = (m, k) if ta in "NR" else (k, m)
    br_, bc_ = (k, n) if tb in "NR" else (n, k)
    def cplx(r, c):
        return torch.complex(torch.rand(c, r, device=cuda, generator=g) * 2 - 1,
                             torch.rand(c, r, device=cuda, generator=g) * 2 - 1)
    A, B, C0 = cplx(ar_, ac_), cplx(br_, bc_), cplx(m, n)
    al, be = 0.75 - 1.25j, 0.5 + 0.25j
    Am, Bm = A.t().to(torch.complex128), B.t().to(torch.complex128)
    ref = al * (op[ta](Am) @ op[tb](Bm)) + be * C0.t().to(torch.complex128)
    C = C0.clone()
    blas.cgemm3m_device(ta, tb, m, n, k, al, A, ar_, B, br_, be, C, m)
    torch.cuda.synchronize()
    got = C.t().to(torch.complex128)
    den = k * 2.0 ** -24 * float(torch.linalg.norm(Am)) * float(torch.linalg.norm(Bm)) * abs(al)
    print("ERR", ta, tb, m, n, k, float(torch.linalg.norm(got - ref)) / den, flush=True)
print("KERNELS", " ".join(sorted(_lib.profile_report())), flush=True)
"""


def test_cgemm3m_one_tensor_core_launch(cuda, tmp_path):
    """With B2_C3M_FUSED=1 (read once per process, so in a child process) and
    128 x 128 tiles that fill the SMs, cgemm3m runs its three 3xTF32 products
    in one tcgen05 launch with three TMEM accumulators and combines them in
    the epilogue: ragged tiles, conjugated and transposed operands, complex
    alpha and beta, against the complex128 product of torch on the device,
    FP32-class error."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = tmp_path / "c3m_fused.py"
    script.write_text(f"ROOT = {root!r}\n" + _FUSED_SCRIPT)
    env = dict(os.environ, B2_C3M_FUSED="1")
    r = subprocess.run([sys.executable, str(script)], capture_output=True, text=True,
                       timeout=300, cwd=root, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    errs = [line.split() for line in r.stdout.splitlines() if line.startswith("ERR")]
    assert len(errs) == 3, r.stdout
    for e in errs:
        assert float(e[-1]) <= 8, e
    kernels = [line for line in r.stdout.splitlines() if line.startswith("KERNELS")][0].split()
    assert "cgemm3m_umma" in kernels and "sgemm_umma_tf32" not in kernels, kernels
