"""Shared helpers for the parity tests (seeded inputs, error yardsticks)."""
from __future__ import annotations

import numpy as np


def fmat(rng, rows, cols, dtype=np.float64, pad=0, lo=-1.0, hi=1.0):
    """Column-major rows x cols matrix inside a (rows+pad) x cols buffer."""
    buf = np.asfortranarray(rng.uniform(lo, hi, (rows + pad, cols)).astype(dtype))
    return buf


def op_dims(trans, rows, cols):
    return (rows, cols) if trans in ("N", "n") else (cols, rows)


def normalized(c, c_ref, k, a, b, u):
    """||C - C_ref||_F / (K u ||A||_F ||B||_F) -- the parity yardstick (<= 8)."""
    den = max(k, 1) * u * float(np.linalg.norm(a.astype(np.float64))) * float(
        np.linalg.norm(b.astype(np.float64)))
    num = float(np.linalg.norm((c.astype(np.float64) - c_ref.astype(np.float64))))
    return num / den if den > 0 else num
