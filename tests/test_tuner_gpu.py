"""Every configuration of the autotuner's DGEMM space gives reference parity.

b2_dgemm_config runs one DGEMM with configuration c of b2_tune_config_count():
plain-FP64 DMMA tiles / DMMA K shapes / split-K factors and the INT8 Ozaki
engine shapes with 13..16 moduli.  Each must match the reference dgemm_
(oracle/oracle.c, the bit-exact restatement) to the parity bound
||C - C_ref||_F / (K u ||A||_F ||B||_F) <= 8 on ragged shapes (no dimension a
multiple of any tile), all four transpose combinations across the space.
"""
import numpy as np
import pytest

from gemm_avx512f_b200 import _lib
from oracle import oracle as O
from tests._util import normalized

pytestmark = pytest.mark.gpu
U = 2.0 ** -53


def test_every_config_has_reference_parity(cuda):
    import torch

    L = _lib.lib()
    ncfg = L.b2_tune_config_count()
    assert ncfg == 48
    rng = np.random.default_rng(11)
    m, n, k = 300, 257, 515
    trans = [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")]
    for cfg in range(ncfg):
        ta, tb = trans[cfg % 4]
        a = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)))
        b = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)))
        c = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
        ref = O.gemm(ta, tb, m, n, k, -1.25, a, b, 0.5, c.copy(order="F"))
        da, db, dc = (torch.from_numpy(x.T.copy()).to(cuda) for x in (a, b, c))
        st = L.b2_dgemm_config(ta.encode(), tb.encode(), m, n, k, -1.25, da.data_ptr(),
                               a.shape[0], db.data_ptr(), b.shape[0], 0.5, dc.data_ptr(), m, cfg,
                               None)
        assert st == 0, (cfg, st)
        torch.cuda.synchronize()
        got = dc.cpu().numpy().T
        assert normalized(got, ref, k, a, b, U) <= 8, cfg
    assert L.b2_device_error(0) == 0
