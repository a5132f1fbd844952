"""GPU parity of the sharded DGEMM (b2_dgemm_multi, and dgemm_ with
B2_DEVICES): C's columns split over a device list, each shard through the
drop-in host path on its device.  The box has one GPU, so the lists repeat
device 0: two or three shards on one GPU exercise the splitting, the
per-(device, occurrence) worker threads and their contexts; the shards never
wait on each other.  Bar: ||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8,
padding rows of C untouched."""
import os
import subprocess
import sys

import numpy as np
import pytest

from gemm_avx512f_b200 import blas
from gemm_avx512f_b200._lib import B2Error
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu
TOL = 8.0
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case(rng, m, n, k, ta, tb, pad=3):
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ar + pad, ac)))
    b = np.asfortranarray(rng.uniform(-1, 1, (br + pad, bc)))
    c = np.asfortranarray(rng.uniform(-1, 1, (m + pad, n)))
    return a, b, c, ar, br


@pytest.mark.parametrize("devices", [[0], [0, 0], [0, 0, 0]])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T"), ("N", "T")])
def test_sharded_dgemm_matches_oracle(cuda, devices, ta, tb):
    rng = np.random.default_rng(len(devices) * 10 + ord(ta) + 2 * ord(tb))
    u = np.finfo(np.float64).eps / 2
    for (m, n, k), method in [((700, 1201, 900), "fp64"), ((333, 5, 257), "ozaki"),
                              ((1024, 4096, 1024), "ozaki")]:  # last: each shard pipelined
        a, b, c, ar, br = _case(rng, m, n, k, ta, tb)
        for al, be in [(1.5, 0.5), (1.0, 0.0)]:
            ref = c.copy(order="F")
            O.gemm(ta, tb, m, n, k, al, a[:ar], b[:br], be, ref[:m])
            got = c.copy(order="F")
            blas.dgemm_multi(devices, ta, tb, m, n, k, al, a, a.shape[0], b, b.shape[0], be, got,
                             got.shape[0], method=method)
            assert np.array_equal(got[m:], c[m:]), "padding rows of C were written"
            e = normalized(got[:m], ref[:m], k, a[:ar], b[:br], u)
            assert e <= TOL, (devices, ta, tb, m, n, k, method, al, be, e)


def test_sharded_dgemm_rejects_device_memory(cuda):
    import torch

    a = torch.zeros((8, 8), dtype=torch.float64, device=cuda)
    c = np.zeros((8, 8), order="F")
    with pytest.raises(B2Error):
        blas.dgemm_multi([0, 0], "N", "N", 8, 8, 8, 1.0, a.data_ptr(), 8, c, 8, 0.0, c, 8)


def test_dgemm_drop_in_shards_with_env_devices(cuda, tmp_path):
    """dgemm_ reads B2_DEVICES once per process: run it in child processes.  A
    list naming a missing device makes the large call fail (so the sharded
    path is the one taken); a valid list gives the oracle's result."""
    script = tmp_path / "shard_env.py"
    script.write_text(
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "from gemm_avx512f_b200 import blas\n"
        "from oracle import oracle as O\n"
        "from tests._util import normalized\n"
        "rng = np.random.default_rng(3)\n"
        "m, n, k = 1024, 3000, 1500\n"
        "a = np.asfortranarray(rng.uniform(-1, 1, (m, k)))\n"
        "b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))\n"
        "c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))\n"
        "ref = c.copy(order='F'); O.gemm('N', 'N', m, n, k, 0.5, a, b, 2.0, ref)\n"
        "got = c.copy(order='F'); blas.dgemm('N', 'N', m, n, k, 0.5, a, m, b, k, 2.0, got, m)\n"
        "e = normalized(got, ref, k, a, b, np.finfo(np.float64).eps / 2)\n"
        "print('ERR', e)\n"
        "sys.exit(0 if e <= 8.0 else 1)\n")
    env = dict(os.environ, B2_DEVICES="0,0", B2_METHOD="fp64")
    r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True,
                       timeout=240, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    env["B2_DEVICES"] = "0,99"
    r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True,
                       timeout=240, cwd=ROOT)
    assert r.returncode != 0 and "B2Error" in r.stderr, r.stdout + r.stderr
