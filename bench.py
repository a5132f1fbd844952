#!/usr/bin/env python
"""Headline benchmark: DGEMM TFLOPS on one B200, INT8-emulated (Ozaki, tcgen05
kind::i8) vs plain FP64 (DMMA), at M=N=K=8192 on exponent-spread inputs
a = u*exp(phi*g) (u ~ U[-1,1), g ~ N(0,1), seed 2), errors stated against the
double-double product.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                    [--method ozaki|fp64] [--size 8192] [--phi 1.0] [--slices 0]

Prints ONE JSON line (rank 0).  ``value`` is device-timed whole-job TFLOPS with
inputs resident in HBM; ``e2e`` is the same metric through the drop-in
``dgemm_`` C symbol with pinned host buffers (H2D + D2H inside the timed
region).  Each 8192^2 FP64 operand is 512 MiB, larger than the 126 MB L2, so
no flush is needed between steps.  With N > 1 each rank runs an independent
replica (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DGEMM TFLOPS: INT8-emulated vs plain FP64 at equal oracle error, one B200"
SM_COUNT_B200 = 148


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--method", default="ozaki", choices=["ozaki", "fp64"])
    p.add_argument("--size", "--n", dest="n", type=int, default=8192)
    p.add_argument("--phi", type=float, default=1.0)
    p.add_argument("--slices", type=int, default=0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-error", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    return p.parse_args()


def make_inputs(n: int, phi: float, seed: int = 2):
    """Emulated-DGEMM inputs a = u*exp(phi*g): u then g for A, then u then g for
    B, flat column-major (gemm_avx512f_b200.inputs.config3)."""
    from gemm_avx512f_b200 import inputs

    return inputs.config3_flat(n, phi, seed)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, \
            "fallback"


def physical_cores() -> int:
    try:
        import psutil

        return psutil.cpu_count(logical=False) or os.cpu_count() or 1
    except Exception:
        return os.cpu_count() or 1


class Clocks:
    """SM clock and clock-event reasons sampled during the timed region.

    Read-only NVML queries every 10 ms from a background thread (so even a
    sub-second timed region gets dozens of samples); nvidia-smi -lms 200 when
    NVML cannot be loaded."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.thread = None
        self.samples = []
        self.max_mhz = None
        self.stop_flag = False

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def poll():
                while not self.stop_flag:
                    try:
                        mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h) \
                            if hasattr(nv, "nvmlDeviceGetCurrentClocksEventReasons") \
                            else nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                        self.samples.append((float(mhz), int(rs)))
                    except Exception:
                        pass
                    time.sleep(0.01)

            import threading

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag = True
            self.thread.join(timeout=2)
            if not self.samples:
                return None
            reasons = sorted({nm for _, rs in self.samples for nm, bit in self.BITS.items()
                              if rs & bit})
            return {"sm_mhz": statistics.median(m for m, _ in self.samples),
                    "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(self.samples), "source": "nvml 10 ms"}
        if self.proc is None:
            return None
        time.sleep(0.3)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sms:
            return None
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms), "source": "nvidia-smi 200 ms"}


# ------------------------------------------------------------ CPU legs ----
def cpu_dgemm_rate(a: np.ndarray, b: np.ndarray, n: int, seconds: float):
    """Time the reference's dgemm_ (oracle/_ref/DGEMM.so) on this host when it
    runs here (AVX-512F), else the oracle's C port, on a column sample of the
    same product: M = K = n, N = ncols chosen for ~`seconds` of work."""
    from oracle import oracle as O

    kind = "reference" if (O.ref_available("DGEMM.so") and O.host_has_avx512f()) else "port"
    A = a.reshape(n, n, order="F")
    B = b.reshape(n, n, order="F")

    def run(cols):
        c = np.zeros((n, cols), order="F")
        bs = B[:, :cols]
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_gemm("N", "N", n, cols, n, 1.0, A, bs, 0.0, c)
        else:
            O.gemm("N", "N", n, cols, n, 1.0, A, bs, 0.0, c)
        return time.perf_counter() - t0

    probe = 16 if kind == "port" else 64
    run(probe)  # thread pool spin-up and first-touch pages
    dt = run(probe)
    rate = 2.0 * n * n * probe / dt
    cols = int(max(probe, min(n, seconds * rate / (2.0 * n * n))))
    dt = run(cols)
    return {"value": 2.0 * n * n * cols / dt / 1e12, "unit": "TFLOPS",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
            "kind": kind,
            "sample": f"dgemm_ NN M=K={n}, N={cols} columns of the same B, alpha=1 beta=0, "
                      f"{dt:.1f} s"}


def max_over_ranks(ms: float, dist, device=None) -> float:
    """The slowest rank's time: every rank passes its own device-timed ms and
    gets the maximum (the job is as slow as its slowest replica)."""
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_tflops(world: int, flops_per_step: float, steps: int, ms: float) -> float:
    """Whole-job rate: every replica ran `steps` products of `flops_per_step`
    (weak scaling) in `ms`, the max over ranks."""
    return world * flops_per_step * steps / (ms / 1e3) / 1e12


def reference_arm(args, rank: int, world: int = 1):
    if rank != 0:
        return None
    os.environ.setdefault("OMP_NUM_THREADS", str(physical_cores()))
    a, b = make_inputs(args.n, args.phi)
    steps = []
    res = None
    for i in range(args.warmup + args.steps):
        res = cpu_dgemm_rate(a, b, args.n, seconds=max(2.0, args.cpu_seconds / 2))
        if i >= args.warmup:
            steps.append(res["value"])
    val = statistics.median(steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_block(args),
        "cpu_baseline": {"value": val, "unit": "TFLOPS", "cores": res["cores"],
                         "kind": res["kind"], "sample": res["sample"]},
        "e2e": {"value": val, "unit": "TFLOPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    return line


def config_block(args):
    return {"workload": f"DGEMM NN M=N=K={args.n}, a=u*exp(phi*g) phi={args.phi}, "
                        f"alpha=1 beta=0, seed 2",
            "M": args.n, "N": args.n, "K": args.n, "phi": args.phi, "method": args.method,
            "parallelism": f"replicas x{args.gpus}",
            "l2": "inputs larger than L2 (512 MiB per operand), no flush"}


# ------------------------------------------------------------- GPU arm ----
def gpu_arm(args, rank: int, world: int):
    import torch

    from gemm_avx512f_b200 import _lib, blas

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    L = _lib.lib()
    n = args.n
    a_h, b_h = make_inputs(n, args.phi)
    A = torch.from_numpy(a_h).to(dev)
    B = torch.from_numpy(b_h).to(dev)
    Cd = torch.zeros(n * n, dtype=torch.float64, device=dev)
    # An explicit stream: handle 0 (torch's legacy default stream) would mean
    # "the library's own stream" to libb2blas and escape the events below.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    method = _lib.METHODS[args.method]
    flops = 2.0 * n * n * n

    def step(meth=method, slices=args.slices):
        st = L.b2_dgemm(b"N", b"N", n, n, n, 1.0, A.data_ptr(), n, B.data_ptr(), n, 0.0,
                        Cd.data_ptr(), n, meth, slices, sptr)
        if st != 0:
            raise _lib.B2Error(st, L.b2_last_info(), "b2_dgemm")

    dist = None
    if world > 1:
        import torch.distributed as dist

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(dev.index)
    clocks.start()
    _lib.profile_enable(True)
    _lib.profile_report()  # drop warm-up records
    n0 = _lib.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - n0
    prof = _lib.profile_report()
    _lib.profile_enable(False)
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    if dist:
        ms = max_over_ranks(ms, dist, dev)
    ms_step = ms / args.steps
    value = job_tflops(world, flops, args.steps, ms)

    # ---- dominant kernel roofline (live CUDA-event durations over the timed region)
    peaks, peak_src = load_peaks()
    roof = None
    if prof:
        # the dominant kernel is the step's GEMM (the auxiliary passes of the
        # Ozaki schedule run beside it on another stream, so their summed
        # durations say nothing about the step); one step may issue it as
        # several column-block launches, so the rate is the step's work over
        # the GEMM's summed launch time per step
        names = [k for k in prof if k.startswith(("ozaki_i8_gemm", "dgemm_dmma"))]
        kname = names[0] if names else max(prof.items(), key=lambda kv: kv[1][1])[0]
        kcnt, kms = prof[kname]
        kstep_s = kms / args.steps / 1e3
        if kname.startswith("ozaki_i8_gemm"):
            ops = flops * ozaki_info(L)["moduli"]
            peak = 2.0 * peaks["bf16_tflops"]
            roof = {"bound": "tensor", "kernel": kname, "unit": "TFLOP/s",
                    "achieved": ops / kstep_s / 1e12, "peak": peak,
                    "peak_source": f"INT8 dense = 2 x {peak_src} bf16 ({peaks['bf16_tflops']})"}
        elif kname.startswith("dgemm_dmma"):
            peak = SM_COUNT_B200 * 128 * 1.965e9 / 1e12
            roof = {"bound": "tensor", "kernel": kname, "unit": "TFLOP/s",
                    "achieved": flops / kstep_s / 1e12, "peak": peak,
                    "peak_source": "nominal FP64 dense (148 SM x 128 FLOP/clk x 1.965 GHz); "
                                   "no measured FP64 peak"}
        if roof:
            roof["frac"] = roof["achieved"] / roof["peak"]
            roof["per"] = "step (the GEMM's launches of one step summed)"
            roof["launches_per_step"] = kcnt / args.steps
            roof["traffic"] = profile_traffic(kname)
            roof["kernel_share"] = kms / ms if ms else None
            roof["launches_timed"] = kcnt

    out = {
        "metric": METRIC, "value": value, "unit": "TFLOPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_block(args), "roofline": roof,
        "gpu_launches": launches, "clocks": ck,
        "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()},
    }
    if args.method == "ozaki":
        out["ozaki"] = ozaki_info(L)

    # ---- plain FP64 on the same inputs (the comparison the metric names)
    if args.method == "ozaki":
        for _ in range(2):
            step(_lib.METHODS["fp64"], 0)
        torch.cuda.synchronize()
        e0.record(stream)
        k2 = max(2, min(args.steps, 5))
        for _ in range(k2):
            step(_lib.METHODS["fp64"], 0)
        e1.record(stream)
        torch.cuda.synchronize()
        out["fp64_tflops"] = flops * k2 / (e0.elapsed_time(e1) / 1e3) / 1e12
        out["speedup_vs_fp64"] = value / world / out["fp64_tflops"]

    # ---- errors vs the double-double product (computed once, outside timing)
    if not args.no_error and rank == 0:
        errs = {}
        hi = torch.empty(n * n, dtype=torch.float64, device=dev)
        blas.dgemm_dd_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, None, n, hi, None, n,
                             stream=stream)
        meths = ["fp64", "ozaki"] if args.method == "ozaki" else ["fp64"]
        for mth in meths:
            step(_lib.METHODS[mth], args.slices if mth == "ozaki" else 0)
            torch.cuda.synchronize()
            d = Cd - hi
            errs[mth] = {"normwise": float(torch.linalg.vector_norm(d) /
                                           torch.linalg.vector_norm(hi)),
                         "max_elementwise": float(d.abs().max() / hi.abs().max())}
        if "ozaki" in errs:
            errs["ozaki_over_fp64_normwise"] = errs["ozaki"]["normwise"] / \
                errs["fp64"]["normwise"]
        out["errors_vs_dd"] = errs
        del hi

    # ---- end to end through the drop-in dgemm_: pinned host buffers (the
    # headline e2e), then plain malloc'ed (pageable) ones as a BLAS caller has
    if not args.no_e2e:
        out["e2e"] = e2e_leg(args, L, a_h, b_h, method, dist, dev, world)
        out["e2e_pageable"] = e2e_pageable_leg(args, L, a_h, b_h, method, dist, dev, world)

    # ---- CPU baseline (reference on the host cores), rank 0 at N=1 only
    if not args.no_cpu and rank == 0 and world == 1:
        try:
            out["cpu_baseline"] = cpu_dgemm_rate(a_h, b_h, n, args.cpu_seconds)
        except Exception as exc:  # keep the GPU line even if the CPU leg cannot run
            out["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    return out


def ozaki_info(L) -> dict:
    info = {}
    try:
        L.b2_ozaki_last_plan.argtypes = [C.c_void_p, C.c_int]
        buf = (C.c_int * 8)()
        L.b2_ozaki_last_plan(buf, 8)
        info = {"moduli": int(buf[0]), "k_chunks": int(buf[1])}
    except AttributeError:
        info = {"moduli": 0}
    return info


def profile_traffic(kname: str):
    """DRAM bytes of `kname` per step (its launches of one step summed) from the
    committed ncu summary, if any."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".md"):
            continue
        with open(os.path.join(pdir, fn)) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_step:") and kname.split("<")[0] in fn:
                    try:
                        return float(line.split(":", 1)[1].split()[0])
                    except ValueError:
                        return None
    return None


def e2e_leg(args, L, a_h, b_h, method, dist=None, dev=None, world=1):
    import torch

    n = args.n
    pa = torch.from_numpy(a_h).pin_memory()
    pb = torch.from_numpy(b_h).pin_memory()
    pc = torch.zeros(n * n, dtype=torch.float64).pin_memory()
    L.b2_set_dgemm_method(method, args.slices)
    ip = lambda v: C.byref(C.c_int(v))
    one, zero = C.c_double(1.0), C.c_double(0.0)

    def call():
        L.dgemm_(b"N", b"N", ip(n), ip(n), ip(n), C.byref(one), pa.data_ptr(), ip(n),
                 pb.data_ptr(), ip(n), C.byref(zero), pc.data_ptr(), ip(n))
        if L.b2_last_error() != 0:
            raise RuntimeError(f"dgemm_ failed: {L.b2_last_error()}")

    call()
    steps = max(2, min(args.steps, 5))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        call()  # synchronous: C is back in host memory when it returns
    dt = (time.perf_counter() - t0) / steps
    if dist:  # the job is as slow as its slowest replica; count every replica's work
        dt = max_over_ranks(dt * 1e3, dist, dev) / 1e3
    L.b2_set_dgemm_method(_lib_fp64(), 0)
    # the copy bound: these bytes at this box's pinned copy rates -- copy-in
    # alone, and copy-in plus copy-out run at the same time (the pipeline's
    # steady state)
    h2d_bytes, d2h_bytes = 2 * 8 * n * n, 8 * n * n
    h2d_gbs, duplex_gbs = pinned_copy_gbs(pa, pc, dev)
    bound_ms = None
    if h2d_gbs and duplex_gbs:
        bound_ms = max(h2d_bytes / (h2d_gbs * 1e9), (h2d_bytes + d2h_bytes) / (duplex_gbs * 1e9)) * 1e3
    return {"value": world * 2.0 * n ** 3 / dt / 1e12, "unit": "TFLOPS",
            "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
            "ms_per_step": dt * 1e3, "pcie_h2d_gbs": h2d_gbs,
            "pcie_h2d_plus_d2h_gbs": duplex_gbs, "copy_bound_ms": bound_ms,
            "frac_of_copy_bound": (bound_ms / (dt * 1e3)) if bound_ms else None,
            "note": "drop-in dgemm_ on pinned host A, B, C: A and B copied in, C copied out; "
                    "with beta == 0 C is scanned on the host (all finite, so not copied in)"}


def e2e_pageable_leg(args, L, a_h, b_h, method, dist=None, dev=None, world=1):
    """The same drop-in dgemm_ call on pageable host memory (numpy buffers, not
    pinned): the driver stages every copy through its own pinned bounce
    buffers, so the copies run slower and overlap the GPU work less."""
    n = args.n
    c_h = np.zeros(n * n)
    L.b2_set_dgemm_method(method, args.slices)
    ip = lambda v: C.byref(C.c_int(v))
    one, zero = C.c_double(1.0), C.c_double(0.0)

    def call():
        L.dgemm_(b"N", b"N", ip(n), ip(n), ip(n), C.byref(one), a_h.ctypes.data, ip(n),
                 b_h.ctypes.data, ip(n), C.byref(zero), c_h.ctypes.data, ip(n))
        if L.b2_last_error() != 0:
            raise RuntimeError(f"dgemm_ failed: {L.b2_last_error()}")

    call()
    steps = max(2, min(args.steps, 3))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    dt = (time.perf_counter() - t0) / steps
    if dist:
        dt = max_over_ranks(dt * 1e3, dist, dev) / 1e3
    L.b2_set_dgemm_method(_lib_fp64(), 0)
    return {"value": world * 2.0 * n ** 3 / dt / 1e12, "unit": "TFLOPS",
            "h2d_bytes_per_step": 2 * 8 * n * n, "d2h_bytes_per_step": 8 * n * n,
            "ms_per_step": dt * 1e3,
            "note": "drop-in dgemm_ on pageable (malloc'ed) host A, B, C, same call"}


def pinned_copy_gbs(pin_src, pin_dst, dev):
    """This box's pinned copy rates (GB/s): host-to-device alone, and
    host-to-device plus device-to-host on two streams at once (bytes of both
    directions per second).  512 MiB per direction, best of 3, CUDA events."""
    import torch

    try:
        nel = min(64 * 1024 * 1024, pin_src.numel(), pin_dst.numel())
        src, hdst = pin_src[:nel], pin_dst[:nel]
        d_in = torch.empty(nel, dtype=src.dtype, device=dev)
        d_out = torch.zeros(nel, dtype=src.dtype, device=dev)
        s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        nbytes = nel * src.element_size()
        best_in = best_both = None
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s_in):
                e0.record()
                d_in.copy_(src, non_blocking=True)
                e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            best_in = t if best_in is None else min(best_in, t)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s_in):
                e0.record()
                d_in.copy_(src, non_blocking=True)
            s_out.wait_event(e0)
            with torch.cuda.stream(s_out):
                hdst.copy_(d_out, non_blocking=True)
            s_in.wait_stream(s_out)
            with torch.cuda.stream(s_in):
                e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            best_both = t if best_both is None else min(best_both, t)
        return nbytes / (best_in / 1e3) / 1e9, 2 * nbytes / (best_both / 1e3) / 1e9
    except Exception:
        return None, None


def _lib_fp64():
    from gemm_avx512f_b200 import _lib

    return _lib.METHODS["fp64"]


def launcher_command(argv, gpus: int, port: int):
    """torchrun command that runs this script as `gpus` ranks on this node.
    `--n` is passed on as `--size` (torchrun's own parser would take `--n` for
    an abbreviation of one of its options)."""
    fwd = ["--size" if a == "--n" else ("--size=" + a[4:] if a.startswith("--n=") else a)
           for a in argv]
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={gpus}", "--master-addr", "127.0.0.1", f"--master-port={port}",
            os.path.abspath(__file__), *fwd]


def free_port() -> int:
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def main():
    args = parse()
    if args.gpus > 1 and "RANK" not in os.environ:
        # asked for N GPUs without a launcher: start the N ranks here (one
        # process per GPU), never time one replica under an N-GPU label
        return subprocess.call(launcher_command(sys.argv[1:], args.gpus, free_port()))
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        line = reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        out = gpu_arm(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
