"""Autotuner and learned-selector training driver.

    python -m gemm_avx512f_b200.tune [--train 20000] [--heldout 2000] [--reps 2]
                                     [--out gemm_avx512f_b200/data] [--epochs 300]

1. Exhaustive sweep: every DGEMM configuration (b2_tune_config_count() = 48)
   of every seeded shape (M, N, K log-uniform integers in [16, 1024], random
   transposes and beta == 0 flag), timed by the library's own CUDA-event loop
   (b2_tune_sweep), and every tensor-core SGEMM configuration (3 methods x
   engine x split-K, b2_tune_sweep_sgemm) of a second seeded shape set.
   Progress is checkpointed after every chunk; rerunning resumes from the
   last completed shape.
2. Training: the 7-64-64-48 MLP learns, per configuration, the log2 slowdown
   against the shape's best (for SGEMM: the best of the same method) on the
   training shapes of both dtypes at once (the dtype input selects which
   configuration space the 48 outputs mean), on the GPU, with the library's
   forward/backward/Adam kernels (b2_mlp_train).
3. Evaluation on the --heldout shapes: the configuration the selector picks
   (batched CUDA inference, b2_mlp_forward) versus the exhaustive best, as
   regret = t(chosen) / t(best) - 1, next to the regret of the fixed rule the
   library uses without the network.  Only configurations meeting the accuracy
   rule are eligible (plain FP64, or Ozaki with >= 15 moduli).

Outputs (in --out): selector_<gpu>.f32 (weights), tune_db_<gpu>.npz (shapes
and log2 timings), selector_<gpu>.json (report).  The timing database is
keyed by GPU name and driver version.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import time

import numpy as np

from ._lib import lib

NCFG = 48
MIN_SLICES = 15


def allowed_mask() -> np.ndarray:
    m = np.ones(NCFG, bool)
    for c in range(36, 48):
        slices = 13 + (c - 36) // 3
        m[c] = slices >= MIN_SLICES
    return m


def make_shapes(count: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lo, hi = np.log(16), np.log(1024)
    mnk = np.rint(np.exp(rng.uniform(lo, hi, (count, 3)))).astype(np.int32)
    flags = rng.integers(0, 2, (count, 3)).astype(np.int32)
    return np.concatenate([mnk, flags], axis=1)  # m, n, k, ta, tb, beta0


def features(shapes: np.ndarray, dtype: int = 0) -> np.ndarray:
    """MLP inputs: log2 sizes centred on 2^7 and scaled by 1/3, transposes,
    dtype (0 = FP64 configurations, 1 = FP32 tensor-core configurations),
    beta == 0."""
    m, n, k, ta, tb, b0 = (shapes[:, i].astype(np.float64) for i in range(6))
    return np.stack([(np.log2(m) - 7) / 3, (np.log2(n) - 7) / 3, (np.log2(k) - 7) / 3, ta, tb,
                     np.full_like(m, float(dtype)), b0], axis=1).astype(np.float32)


# SGEMM slots (dtype 1): method block b = slot // 16 (TF32, TF32X3, BF16X3),
# slots b*16 .. b*16+11 valid (engine x split-K), b*16+12 .. b*16+15 unused.
SG_METHODS = (("tf32", 11), ("tf32x3", 12), ("bf16x3", 13))


def sgemm_block_mask(b: int) -> np.ndarray:
    m = np.zeros(NCFG, bool)
    m[16 * b:16 * b + 12] = True
    return m


def sweep_sgemm(shapes: np.ndarray, reps: int, ckpt: str, chunk: int = 250) -> np.ndarray:
    L = lib()
    ms = np.full((len(shapes), NCFG), np.nan, np.float32)
    done = 0
    if os.path.exists(ckpt):
        z = np.load(ckpt)
        if z["shapes"].shape == shapes.shape and np.array_equal(z["shapes"], shapes):
            ms[:] = z["ms"]
            done = int(z["done"])
    while done < len(shapes):
        end = min(len(shapes), done + chunk)
        part = np.ascontiguousarray(shapes[done:end])
        out = np.zeros((end - done, NCFG), np.float32)
        st = L.b2_tune_sweep_sgemm(end - done, part.ctypes.data, reps, out.ctypes.data)
        if st != 0:
            raise RuntimeError(f"b2_tune_sweep_sgemm failed with status {st}")
        ms[done:end] = out
        done = end
        np.savez(ckpt, shapes=shapes, ms=ms, done=done)
    return ms


def sgemm_targets(T: np.ndarray, clip) -> np.ndarray:
    """log2 slowdown of each slot relative to the fastest slot of its own
    method block (the choice is made within the method the caller asked for);
    unused slots NaN (masked in training)."""
    out = np.full_like(T, np.nan, dtype=np.float32)
    for b in range(len(SG_METHODS)):
        mk = sgemm_block_mask(b)
        best = np.where(mk[None, :], T, np.inf).min(axis=1, keepdims=True)
        rel = T[:, mk] - best
        out[:, mk] = np.minimum(rel, clip) if clip else rel
    return out


def sgemm_regret(ms: np.ndarray, pred: np.ndarray, b: int) -> np.ndarray:
    mk = sgemm_block_mask(b)
    choice = np.where(mk[None, :], pred, np.inf).argmin(1)
    best = np.where(mk[None, :], ms, np.inf).min(1)
    return ms[np.arange(len(ms)), choice] / best - 1.0


def sgemm_default_regret(shapes: np.ndarray, ms: np.ndarray, b: int) -> np.ndarray:
    """Regret of the configuration the library runs without the network."""
    L = lib()
    L.b2_selector_set(None)
    code = SG_METHODS[b][1]
    pick = np.array([L.b2_sgemm_selector_choose(code, b"T" if ta else b"N", b"T" if tb else b"N",
                                                int(m), int(n), int(k), int(b0))
                     for (m, n, k, ta, tb, b0) in shapes])
    mk = sgemm_block_mask(b)
    best = np.where(mk[None, :], ms, np.inf).min(1)
    return ms[np.arange(len(ms)), pick] / best - 1.0


def gpu_key() -> str:
    try:
        import torch

        name = torch.cuda.get_device_name(0)
    except Exception:
        name = "gpu"
    return re.sub(r"[^A-Za-z0-9]+", "_", name).strip("_").lower()


def sweep(shapes: np.ndarray, reps: int, ckpt: str, chunk: int = 250) -> np.ndarray:
    L = lib()
    ms = np.full((len(shapes), NCFG), np.nan, np.float32)
    done = 0
    if os.path.exists(ckpt):
        z = np.load(ckpt)
        if z["shapes"].shape == shapes.shape and np.array_equal(z["shapes"], shapes):
            ms[:] = z["ms"]
            done = int(z["done"])
    while done < len(shapes):
        end = min(len(shapes), done + chunk)
        part = np.ascontiguousarray(shapes[done:end])
        out = np.zeros((end - done, NCFG), np.float32)
        st = L.b2_tune_sweep(end - done, part.ctypes.data, reps, out.ctypes.data)
        if st != 0:
            raise RuntimeError(f"b2_tune_sweep failed with status {st}")
        ms[done:end] = out
        done = end
        np.savez(ckpt, shapes=shapes, ms=ms, done=done)
    return ms


def train(X: np.ndarray, T: np.ndarray, epochs: int, lr: float, seed: int):
    L = lib()
    w = np.zeros(L.b2_mlp_param_count(), np.float32)
    loss = C.c_float(0.0)
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    st = L.b2_mlp_train(len(X), X.ctypes.data, T.ctypes.data, epochs, 256, C.c_float(lr), seed,
                        None, w.ctypes.data, C.byref(loss))
    if st != 0:
        raise RuntimeError(f"b2_mlp_train failed with status {st}")
    return w, float(loss.value)


def predict(w: np.ndarray, X: np.ndarray) -> np.ndarray:
    L = lib()
    X = np.ascontiguousarray(X, np.float32)
    Y = np.zeros((len(X), NCFG), np.float32)
    st = L.b2_mlp_forward(w.ctypes.data, len(X), X.ctypes.data, Y.ctypes.data)
    if st != 0:
        raise RuntimeError(f"b2_mlp_forward failed with status {st}")
    return Y


def regret(ms: np.ndarray, choice: np.ndarray) -> np.ndarray:
    ok = allowed_mask()
    best = np.where(ok[None, :], ms, np.inf).min(1)
    return ms[np.arange(len(ms)), choice] / best - 1.0


def heuristic_choices(shapes: np.ndarray) -> np.ndarray:
    L = lib()
    L.b2_selector_set(None)
    out = np.zeros(len(shapes), np.int64)
    for i, (m, n, k, ta, tb, b0) in enumerate(shapes):
        out[i] = L.b2_selector_choose(b"T" if ta else b"N", b"T" if tb else b"N", int(m), int(n),
                                      int(k), int(b0), MIN_SLICES)
    return out


def summarize(r: np.ndarray) -> dict:
    return {"mean": float(r.mean()), "median": float(np.median(r)),
            "p90": float(np.quantile(r, 0.9)), "max": float(r.max()),
            "geomean_ratio": float(np.exp(np.log1p(r).mean()) - 1.0)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--heldout", type=int, default=2000)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "data"))
    ap.add_argument("--db", default=None, help="reuse a timing database instead of sweeping")
    ap.add_argument("--select", action="store_true",
                    help="pick clip/epochs/lr/seed on a validation split of the training shapes")
    ap.add_argument("--clips", default="none,1.5,1.0", help="validation grid: target clips")
    ap.add_argument("--epochs-grid", default="600,1000", help="validation grid: epochs")
    ap.add_argument("--lrs", default="1e-3,3e-3", help="validation grid: learning rates")
    ap.add_argument("--seeds", default="", help="validation grid: training seeds (default: one)")
    ap.add_argument("--sgemm-train", type=int, default=10000)
    ap.add_argument("--sgemm-heldout", type=int, default=1000)
    args = ap.parse_args(argv)
    os.makedirs(args.out, exist_ok=True)
    key = gpu_key()
    ntr = args.train
    t0 = time.time()
    zdb = np.load(args.db) if args.db else None
    if zdb is not None:
        shapes = zdb["shapes"]
        T = zdb["log2ms"].astype(np.float32)
        ms = np.exp2(T.astype(np.float64))
        ntr = int(zdb["train"])
    else:
        shapes = make_shapes(args.train + args.heldout, args.seed)
        ms = sweep(shapes, args.reps, os.path.join(args.out, f"tune_ckpt_{key}.npz"))
        T = np.log2(np.maximum(ms, 1e-6)).astype(np.float32)
    # FP32 tensor-core configurations (dtype 1): their own seeded shapes
    if zdb is not None and "shapes_s" in zdb:
        shapes_s = zdb["shapes_s"]
        T_s = zdb["log2ms_s"].astype(np.float32)
        ntr_s = int(zdb["train_s"])
    else:
        shapes_s = make_shapes(args.sgemm_train + args.sgemm_heldout, args.seed + 100)
        ms_s0 = sweep_sgemm(shapes_s, args.reps, os.path.join(args.out, f"tune_ckpt_s_{key}.npz"))
        T_s = np.log2(np.maximum(ms_s0, 1e-6)).astype(np.float32)  # NaN slots stay NaN
        ntr_s = args.sgemm_train
    ms_s = np.exp2(T_s.astype(np.float64))
    t_sweep = time.time() - t0
    X = features(shapes)
    X_s = features(shapes_s, 1)
    # Selection needs only each shape's ranking of configurations, so the
    # network learns log2 slowdown relative to the shape's fastest
    # configuration, clipped at `clip` (how much slower a hopeless
    # configuration is does not matter for the choice).
    Tbest = np.where(allowed_mask()[None, :], T, np.inf).min(axis=1, keepdims=True)

    def targets(clip):
        rel = T - Tbest
        return (np.minimum(rel, clip) if clip else rel).astype(np.float32)

    ok = allowed_mask()
    trials = []
    epochs, lr, clip, tseed = args.epochs, args.lr, None, args.seed + 4
    if args.select:
        nv = ntr // 10
        clips = [None if c == "none" else float(c) for c in args.clips.split(",")]
        seeds = [int(v) for v in args.seeds.split(",")] if args.seeds else [args.seed + 4]
        for cl in clips:
            Tt = targets(cl)
            for ep in (int(v) for v in args.epochs_grid.split(",")):
                for lrc in (float(v) for v in args.lrs.split(",")):
                    for sd in seeds:
                        wv, _ = train(X[:ntr - nv], Tt[:ntr - nv], ep, lrc, sd)
                        pv = predict(wv, X[ntr - nv:ntr])
                        rv = regret(ms[ntr - nv:ntr],
                                    np.where(ok[None, :], pv, np.inf).argmin(1))
                        trials.append({"clip": cl, "epochs": ep, "lr": lrc, "seed": sd,
                                       "val_regret_mean": float(rv.mean())})
        best = min(trials, key=lambda t: t["val_regret_mean"])
        epochs, lr, clip, tseed = best["epochs"], best["lr"], best["clip"], best["seed"]
    t0 = time.time()
    Xtr = np.concatenate([X[:ntr], X_s[:ntr_s]])
    Ttr = np.concatenate([targets(clip)[:ntr], sgemm_targets(T_s, clip)[:ntr_s]])
    w, loss = train(Xtr, Ttr, epochs, lr, tseed)
    t_train = time.time() - t0
    pred = predict(w, X[ntr:])
    choice = np.where(ok[None, :], pred, np.inf).argmin(1)
    r_mlp = regret(ms[ntr:], choice)
    r_heur = regret(ms[ntr:], heuristic_choices(shapes[ntr:]))
    pred_s = predict(w, X_s[ntr_s:])
    sg_report = {}
    for b, (name, _) in enumerate(SG_METHODS):
        sg_report[name] = {
            "regret_mlp": summarize(sgemm_regret(ms_s[ntr_s:], pred_s, b)),
            "regret_default": summarize(sgemm_default_regret(shapes_s[ntr_s:], ms_s[ntr_s:], b))}
    w.tofile(os.path.join(args.out, f"selector_{key}.f32"))
    np.savez_compressed(os.path.join(args.out, f"tune_db_{key}.npz"), shapes=shapes,
                        log2ms=T.astype(np.float16), train=ntr, shapes_s=shapes_s,
                        log2ms_s=T_s.astype(np.float16), train_s=ntr_s)
    report = {"gpu": key, "shapes": len(shapes), "train": ntr, "heldout": args.heldout,
              "configs": NCFG, "sweep_seconds": t_sweep, "train_seconds": t_train,
              "epochs": epochs, "lr": lr, "seed": tseed, "validation_trials": trials,
              "target": "log2(ms / fastest allowed ms) per shape", "clip": clip,
              "final_train_mse_log2": loss, "regret_mlp": summarize(r_mlp),
              "regret_heuristic": summarize(r_heur),
              "chosen_ozaki_fraction": float((choice >= 36).mean()),
              "sgemm_shapes": len(shapes_s), "sgemm_train": ntr_s,
              "sgemm_heldout": len(shapes_s) - ntr_s, "regret_sgemm": sg_report}
    with open(os.path.join(args.out, f"selector_{key}.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
