"""Measurement suite for every workload of the hot path, on one B200.

    python -m gemm_avx512f_b200.suite [--only dgemm,sgemm,ozaki,grouped,complex,trsm,select]
                                      [--sgemm-shape MxNxK ...]
                                      [--quick] [--out results.jsonl]

One JSON line per measurement.  Each line names the workload (shapes, seed,
value distribution), the method, the device time per call (CUDA events on the
launching stream, after warm-up, inputs resident in HBM), the algorithmic rate,
the roofline it is bound by and the fraction reached, and the accuracy of the
result (normwise error against a double-double or FP64 yardstick computed on
the GPU).  Inputs are seeded synthetic data with the shapes of the reference's
workloads:

  dgemm    DGEMM NN M=N=K=1024, alpha=1.5, beta=0.5, U[-1,1) (seed 0); plain
           FP64 (DMMA), INT8 Ozaki and the learned selector ("auto").
  sgemm    SGEMM, 4 transpose pairs x M=N=K in {2048, 4096, 8192} and
           8192x256x8192, U[-1,1) (seed 1), alpha=1, beta=0: FP32 SIMT,
           1xTF32, 3xTF32, 3xBF16.
  ozaki    DGEMM a = u exp(phi g) (u ~ U[-1,1), g ~ N(0,1), seed 2),
           phi in {0.1, 1, 4}, M=N=K in {4096, 8192, 16384}: Ozaki and FP64,
           both errors against the double-double product.
  grouped  4096 problems, M, N, K log-uniform in [16, 1024] (seed 3), half
           FP32 half FP64, random transposes: one grouped launch, its CUDA
           graph plan, and one call per problem.
  complex  zgemm3m / cgemm3m, M=N=K=2048, real and imaginary parts U[-1,1): three
           real GEMMs (FP64 DMMA / 3xTF32) between pre-add and combine passes.
  trsm     DTRSM L/L/N/N, n=16384, 4096 right-hand sides (seed 4), diagonal
           n + U[0,1): FP64 and Ozaki trailing updates, scaled residual.
  select   learned configuration selector on the committed timing database:
           held-out regret and per-call inference time.

Peaks (the roofline denominators): HBM and dense BF16 from the measured
MEASURED_PEAKS.json beside the repository when present, else the stated
fallbacks; INT8 = 2 x BF16 and TF32 = BF16 / 2 (the B200 tensor-core ratios);
FP64 and FP32 SIMT are nominal (148 SMs x 128 FP64 or 256 FP32 FLOP/clk x
1.965 GHz), as no measured figure exists for them.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import _lib, blas, inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SM = 148
CLK = 1.965e9


def peaks() -> dict:
    p = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            m = json.load(fh)
        p = {"hbm_gbs": float(m["hbm_gbs"]), "bf16_tflops": float(m["bf16_tflops"]),
             "source": "measured"}
    p["int8_tops"] = 2.0 * p["bf16_tflops"]
    p["tf32_tflops"] = 0.5 * p["bf16_tflops"]
    p["fp64_tflops"] = SM * 128 * CLK / 1e12
    p["fp32_tflops"] = SM * 256 * CLK / 1e12
    return p


class Timer:
    def __init__(self, torch, stream):
        self.torch, self.stream = torch, stream

    def __call__(self, fn, reps=5, warmup=3) -> float:
        torch = self.torch
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for _ in range(reps):
            fn()
        e1.record(self.stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps


def upload(x, dev):
    """A Fortran-ordered host matrix as a flat column-major device tensor."""
    import torch

    t = torch.from_numpy(np.asfortranarray(x).reshape(-1, order="F")).to(dev)
    torch.cuda.synchronize()
    return t


def emit(out, rec):
    line = json.dumps(rec)
    print(line, flush=True)
    if out:
        out.write(line + "\n")
        out.flush()


def run_dgemm(ctx, out, quick):
    torch, dev, T, P = ctx["torch"], ctx["dev"], ctx["timer"], ctx["peaks"]
    st = ctx["stream"]
    n = 1024
    A, B, C0 = (upload(x, dev) for x in inputs.config1(n))
    blas.load_selector()
    for method in ("fp64", "ozaki", "auto"):
        Cm = C0.clone()
        ms = T(lambda: blas.dgemm_device("N", "N", n, n, n, 1.5, A, n, B, n, 0.5, Cm, n,
                                         method=method, stream=st), reps=20)
        Cm = C0.clone()
        blas.dgemm_device("N", "N", n, n, n, 1.5, A, n, B, n, 0.5, Cm, n, method=method,
                          stream=st)
        nw, me = blas.dgemm_error_device("N", "N", n, n, n, 1.5, A, n, B, n, 0.5, C0, Cm, n,
                                         stream=st)
        tf = 2.0 * n ** 3 / ms / 1e9
        rec = {"workload": "dgemm NN 1024^3 alpha=1.5 beta=0.5 U[-1,1) seed 0", "method": method,
               "ms": ms, "tflops": tf, "err_vs_dd_normwise": nw, "err_vs_dd_max": me}
        if method == "fp64":
            rec.update(bound="fp64 tensor (nominal)", peak=P["fp64_tflops"],
                       frac=tf / P["fp64_tflops"])
        emit(out, rec)


def run_sgemm(ctx, out, quick):
    torch, dev, T, P = ctx["torch"], ctx["dev"], ctx["timer"], ctx["peaks"]
    st = ctx["stream"]
    shapes = [(2048, 2048, 2048), (4096, 4096, 4096), (8192, 8192, 8192), (8192, 256, 8192)]
    if quick:
        shapes = [(4096, 4096, 4096), (8192, 256, 8192)]
    if ctx.get("sgemm_shapes"):
        shapes = ctx["sgemm_shapes"]
    bound = {"fp32": ("fp32 SIMT (nominal)", P["fp32_tflops"], 1),
             "tf32": ("tf32 tensor", P["tf32_tflops"], 1),
             "tf32x3": ("tf32 tensor, 3 MMAs per product", P["tf32_tflops"], 3),
             "bf16x3": ("bf16 tensor, 3 MMAs per product", P["bf16_tflops"], 3)}
    for (m, n, k) in shapes:
        for ta, tb in (("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")):
            ha, hb = inputs.config2(m, n, k, ta, tb)
            A, B = upload(ha, dev), upload(hb, dev)
            del ha, hb
            lda, ldb = (m if ta == "N" else k), (k if tb == "N" else n)
            Am = A.view(-1, lda).t()  # column-major lda x cols
            Bm = B.view(-1, ldb).t()
            opA = (Am if ta == "N" else Am.t()).double()
            opB = (Bm if tb == "N" else Bm.t()).double()
            ref = opA @ opB
            for method in ("fp32", "tf32", "tf32x3", "bf16x3"):
                Cm = torch.zeros(m * n, dtype=torch.float32, device=dev)
                ms = T(lambda: blas.sgemm_device(ta, tb, m, n, k, 1.0, A, lda, B, ldb, 0.0, Cm, m,
                                                 method=method, stream=st), reps=5)
                got = Cm.view(n, m).t().double()
                err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
                tf = 2.0 * m * n * k / ms / 1e9
                name, peak, mmas = bound[method]
                emit(out, {"workload": f"sgemm {ta}{tb} {m}x{n}x{k} U[-1,1) seed 1",
                           "method": method, "ms": ms, "tflops": tf, "bound": name,
                           "peak": peak, "frac": tf * mmas / peak,
                           "err_vs_fp64_normwise": err})
            del A, B, ref, opA, opB


def run_ozaki(ctx, out, quick):
    torch, dev, T, P = ctx["torch"], ctx["dev"], ctx["timer"], ctx["peaks"]
    st = ctx["stream"]
    L = _lib.lib()
    sizes = [4096, 8192, 16384] if not quick else [4096]
    for n in sizes:
        for phi in (0.1, 1.0, 4.0):
            ha, hb = inputs.config3(n, phi)
            A, B = upload(ha, dev), upload(hb, dev)
            del ha, hb
            res, moduli = {}, 0
            for method in ("ozaki", "fp64"):
                Cm = torch.zeros(n * n, dtype=torch.float64, device=dev)
                reps = 3 if n >= 16384 else 5
                ms = T(lambda: blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, Cm, n,
                                                 method=method, stream=st), reps=reps, warmup=2)
                if method == "ozaki":
                    plan = (C.c_int * 2)()
                    L.b2_ozaki_last_plan(plan, 2)
                    moduli = int(plan[0])
                # beta == 0: no C0 operand (None)
                nw, me = blas.dgemm_error_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, None,
                                                 Cm, n, stream=st)
                res[method] = (ms, nw, me)
                del Cm
            ms_o, nw_o, me_o = res["ozaki"]
            ms_f, nw_f, me_f = res["fp64"]
            emit(out, {"workload": f"dgemm NN {n}^3 a=u*exp({phi}*g) seed 2", "method": "ozaki",
                       "moduli": moduli, "ms": ms_o,
                       "tflops": 2.0 * n ** 3 / ms_o / 1e9, "fp64_ms": ms_f,
                       "fp64_tflops": 2.0 * n ** 3 / ms_f / 1e9, "speedup_vs_fp64": ms_f / ms_o,
                       "err_vs_dd_normwise": nw_o, "fp64_err_vs_dd_normwise": nw_f,
                       "err_ratio_vs_fp64": nw_o / nw_f if nw_f else None,
                       "err_vs_dd_max": me_o, "fp64_err_vs_dd_max": me_f})
            del A, B
            torch.cuda.empty_cache()


def run_grouped(ctx, out, quick):
    torch, dev, T = ctx["torch"], ctx["dev"], ctx["timer"]
    st = ctx["stream"]
    L = _lib.lib()
    count = 4096
    probs, keep, flops = [], [], 0.0
    for i, (dt, ta, tb, m, n, k) in enumerate(inputs.config4_problems(count)):
        rng = np.random.default_rng([3, i])
        npdt = np.float64 if dt == 0 else np.float32
        tdt = torch.float64 if dt == 0 else torch.float32
        ar, br = (m if ta == "N" else k), (k if tb == "N" else n)
        A = upload(rng.uniform(-1, 1, (ar, m * k // ar)).astype(npdt), dev)
        B = upload(rng.uniform(-1, 1, (br, k * n // br)).astype(npdt), dev)
        Cm = torch.zeros(m * n, dtype=tdt, device=dev)
        probs.append(_lib.GemmProblem(dt, ta.encode(), tb.encode(), m, n, k, 1.0, 0.0,
                                      A.data_ptr(), ar, B.data_ptr(), br, Cm.data_ptr(), m))
        keep.append((A, B, Cm, dt, ta, tb, m, n, k, ar, br))
        flops += 2.0 * m * n * k
    arr = (_lib.GemmProblem * count)(*probs)
    ms1 = T(lambda: L.b2_gemm_grouped(count, arr, st.cuda_stream), reps=5)
    plan = C.c_void_p()
    assert L.b2_grouped_plan_create(count, arr, C.byref(plan)) == 0
    ms2 = T(lambda: L.b2_grouped_plan_launch(plan, st.cuda_stream), reps=10)
    L.b2_grouped_plan_destroy(plan)

    def loop():
        for (A, B, Cm, dt, ta, tb, m, n, k, ar, br) in keep:
            if dt == 0:
                L.b2_dgemm(ta.encode(), tb.encode(), m, n, k, 1.0, A.data_ptr(), ar, B.data_ptr(),
                           br, 0.0, Cm.data_ptr(), m, _lib.METHODS["fp64"], 0, st.cuda_stream)
            else:
                L.b2_sgemm(ta.encode(), tb.encode(), m, n, k, 1.0, A.data_ptr(), ar, B.data_ptr(),
                           br, 0.0, Cm.data_ptr(), m, _lib.METHODS["fp32"], st.cuda_stream)

    ms3 = T(loop, reps=2, warmup=1)
    emit(out, {"workload": "grouped 4096 problems, M,N,K log-uniform [16,1024] seed 3, "
                           "half FP32 half FP64", "gflop": flops / 1e9,
               "grouped_ms": ms1, "grouped_tflops": flops / ms1 / 1e9,
               "graph_plan_ms": ms2, "graph_plan_tflops": flops / ms2 / 1e9,
               "per_problem_calls_ms": ms3, "speedup_vs_per_problem": ms3 / ms1})

    # the same batch plus the zgemm3m 2048^3 product as 3M problem in the queue
    n = 2048
    ha, hb, _ = inputs.config4_complex(n)
    Az, Bz = upload(ha, dev), upload(hb, dev)
    del ha, hb
    Cz = torch.zeros(n * n, dtype=torch.complex128, device=dev)
    pz = _lib.GemmProblem(2, b"N", b"N", n, n, n, 1.0, 0.0, Az.data_ptr(), n, Bz.data_ptr(), n,
                          Cz.data_ptr(), n)
    arr2 = (_lib.GemmProblem * (count + 1))(pz, *probs)
    plan = C.c_void_p()
    assert L.b2_grouped_plan_create(count + 1, arr2, C.byref(plan)) == 0
    ms4 = T(lambda: L.b2_grouped_plan_launch(plan, st.cuda_stream), reps=5)
    L.b2_grouped_plan_destroy(plan)
    ref = Az.view(n, n).t() @ Bz.view(n, n).t()
    err = float(torch.linalg.norm(Cz.view(n, n).t() - ref) / torch.linalg.norm(ref))
    zal = (C.c_double * 2)(1.0, 0.0)
    zbe = (C.c_double * 2)(0.0, 0.0)
    ms5 = T(lambda: L.b2_zgemm3m(b"N", b"N", n, n, n, C.addressof(zal), Az.data_ptr(), n,
                                 Bz.data_ptr(), n, C.addressof(zbe), Cz.data_ptr(), n,
                                 st.cuda_stream), reps=5)
    emit(out, {"workload": "grouped 4096 problems + zgemm3m 2048^3 (3M problem) in one launch",
               "graph_plan_ms": ms4, "zgemm3m_err_normwise": err,
               "separate_ms": ms2 + ms5, "zgemm3m_alone_ms": ms5,
               "gflop_real_issued": (flops + 6.0 * n ** 3) / 1e9})


def run_complex(ctx, out, quick):
    torch, dev, T, P = ctx["torch"], ctx["dev"], ctx["timer"], ctx["peaks"]
    st = ctx["stream"]
    n = 2048
    ha, hb, _ = inputs.config4_complex(n)
    A, B = upload(ha, dev), upload(hb, dev)
    del ha, hb
    ref = A.view(n, n).t() @ B.view(n, n).t()
    for name, fn, dt in (("zgemm3m", blas.zgemm3m_device, torch.complex128),
                         ("cgemm3m", blas.cgemm3m_device, torch.complex64)):
        a, b = A.to(dt), B.to(dt)
        Cm = torch.zeros(n * n, dtype=dt, device=dev)
        ms = T(lambda: fn("N", "N", n, n, n, 1.0, a, n, b, n, 0.0, Cm, n, stream=st), reps=5)
        err = float(torch.linalg.norm(Cm.view(n, n).t().to(torch.complex128) - ref) /
                    torch.linalg.norm(ref))
        rec = {"workload": f"{name} NN {n}^3 re,im U[-1,1)", "ms": ms,
               "tflops_effective_8n3": 8.0 * n ** 3 / ms / 1e9,
               "tflops_issued_6n3": 6.0 * n ** 3 / ms / 1e9, "err_normwise": err}
        if name == "zgemm3m":
            rec.update(bound="fp64 tensor (nominal), 6n^3 issued", peak=P["fp64_tflops"],
                       frac=6.0 * n ** 3 / ms / 1e9 / P["fp64_tflops"])
        else:  # three 3xTF32 tensor-core products: 3 MMAs per issued product
            rec.update(bound="tf32 tensor, 3 MMAs per product, 6n^3 issued",
                       peak=P["tf32_tflops"], frac=3 * 6.0 * n ** 3 / ms / 1e9 / P["tf32_tflops"])
        emit(out, rec)


def run_trsm(ctx, out, quick):
    torch, dev, T, P = ctx["torch"], ctx["dev"], ctx["timer"], ctx["peaks"]
    st = ctx["stream"]
    n, nrhs = (16384, 4096) if not quick else (8192, 2048)
    ha, hb = inputs.config5(n, nrhs)
    Acm = upload(ha, dev)  # column-major storage of the lower triangle L
    Lm = Acm.view(n, n).t()
    B0 = upload(hb, dev).view(nrhs, n)
    del ha, hb
    for upd in ("fp64", "ozaki"):
        X = B0.clone()

        def call():
            X.copy_(B0)
            blas.dtrsm_device("L", "L", "N", "N", n, nrhs, 1.0, Acm, n, X, n, update=upd,
                              stream=st)

        ms_copy = T(lambda: X.copy_(B0), reps=5)
        ms = T(call, reps=3, warmup=1) - ms_copy
        Xm = X.t()
        R = Lm @ Xm - B0.t()
        res = float(torch.linalg.norm(R) /
                    (torch.linalg.norm(Lm) * torch.linalg.norm(Xm) * n * 2.0 ** -53))
        tf = float(n) * n * nrhs / ms / 1e9
        emit(out, {"workload": f"dtrsm L/L/N/N n={n} nrhs={nrhs} seed 4", "update": upd,
                   "ms": ms, "tflops": tf, "bound": "fp64 tensor (nominal)",
                   "peak": P["fp64_tflops"], "frac": tf / P["fp64_tflops"],
                   "scaled_residual": res})
        del X, R


def run_select(ctx, out, quick):
    L = _lib.lib()
    data = os.path.join(os.path.dirname(__file__), "data")
    z = np.load(os.path.join(data, "tune_db_nvidia_b200.npz"))
    shapes, ntr = z["shapes"], int(z["train"])
    ms = np.exp2(z["log2ms"].astype(np.float64))
    w = np.fromfile(os.path.join(data, "selector_nvidia_b200.f32"), np.float32)
    allowed = np.array([c < 36 or 13 + (c - 36) // 3 >= 15 for c in range(48)])
    hold, ms_h = shapes[ntr:], ms[ntr:]
    best = np.where(allowed[None, :], ms_h, np.inf).min(1)
    L.b2_selector_set(w.ctypes.data)
    t0 = time.perf_counter()
    pick = np.array([L.b2_selector_choose(b"T" if s[3] else b"N", b"T" if s[4] else b"N",
                                          int(s[0]), int(s[1]), int(s[2]), int(s[5]), 15)
                     for s in hold])
    us = (time.perf_counter() - t0) / len(hold) * 1e6
    L.b2_selector_set(None)
    heur = np.array([L.b2_selector_choose(b"T" if s[3] else b"N", b"T" if s[4] else b"N",
                                          int(s[0]), int(s[1]), int(s[2]), int(s[5]), 15)
                     for s in hold])
    r = ms_h[np.arange(len(hold)), pick] / best - 1
    rh = ms_h[np.arange(len(hold)), heur] / best - 1
    emit(out, {"workload": f"selector on {len(hold)} held-out shapes (M,N,K log-uniform "
                           "[16,1024], seed 3)", "regret_mean": float(r.mean()),
               "regret_geomean": float(np.exp(np.log1p(r).mean()) - 1),
               "regret_median": float(np.median(r)), "fixed_rule_regret_mean": float(rh.mean()),
               "choose_us_per_call_incl_python": us})


RUNNERS = {"dgemm": run_dgemm, "sgemm": run_sgemm, "ozaki": run_ozaki, "grouped": run_grouped,
           "complex": run_complex, "trsm": run_trsm, "select": run_select}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=",".join(RUNNERS))
    ap.add_argument("--quick", action="store_true", help="smaller sizes (a smoke run)")
    ap.add_argument("--out", default=None)
    ap.add_argument("--sgemm-shape", action="append", default=[],
                    help="MxNxK for the sgemm runner (repeatable; default: the config-2 shapes)")
    args = ap.parse_args(argv)
    import torch

    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = {"torch": torch, "dev": dev, "stream": stream, "timer": Timer(torch, stream),
           "peaks": peaks(),
           "sgemm_shapes": [tuple(int(v) for v in sh.lower().split("x")) for sh in args.sgemm_shape]}
    out = open(args.out, "w") if args.out else None
    emit(out, {"peaks": ctx["peaks"], "gpu": torch.cuda.get_device_name(0)})
    for name in args.only.split(","):
        RUNNERS[name](ctx, out, args.quick)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    if out:
        out.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
