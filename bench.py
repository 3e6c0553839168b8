#!/usr/bin/env python
"""Benchmark: RK4 steps/s of Tarang's forced isotropic Navier-Stokes configuration at 256^3
(FOUR basis, nu = 1e-3, dt = 5e-4, constant energy supply on 2 < k <= 3 at eps = 0.1, 2/3
dealiasing), FP64 form (the headline `value`) and FP32-mixed form, on synthetic seeded
random-phase initial data with E(k) ~ k^4 exp(-2 (k/4)^2), E = 0.5.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One process per GPU (torchrun for N > 1); every rank advances its own independent solve
(replicas: the single 256^3 solve fits one GPU), so scaling is weak and the reported value is
the steps of all ranks divided by the slowest rank's device time.  Inputs (~2 GB of working
set) exceed the 126 MB L2, so no L2 flush is needed between steps.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 256
FORCE = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
NU, DT = 1e-3, 5e-4
METRIC = "RK4 steps/s 256^3 FP64 vs FP32-mixed (<=1e-6 rel); batched p50/p99 latency"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="own", choices=["own", "reference"])
    p.add_argument("--size", type=int, default=N_DEFAULT)
    p.add_argument("--err-steps", type=int, default=100)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    return p.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            j = json.load(fh)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel, workload):
    """ncu DRAM bytes per launch of `kernel` from the committed summary, or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# --------------------------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return
    import numpy as np  # noqa: F401
    from oracle import tarang_oracle as o
    from tarang_b200 import ic
    n = args.size
    N = (n, n, n)
    V = ic.random_phase_field(N, seed=20261202)
    s = o.FluidSolver(N, (1.0, 1.0, 1.0), NU, DT, force=FORCE)
    warm = min(args.warmup, 1)
    steps = max(1, min(args.steps, 3))
    for _ in range(warm):
        V, _ = s.step(V)
    t0 = time.perf_counter()
    for _ in range(steps):
        V, _ = s.step(V)
    el = time.perf_counter() - t0
    v = steps / el
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"forced isotropic NS {n}^3 FOUR, RK4, nu=1e-3, dt=5e-4, energy supply 2<k<=3 eps=0.1",
                   "grid": N, "parallelism": "replicas"},
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"{steps} RK4 steps at {n}^3 after {warm} warm-up (oracle: numpy + scipy.fft pocketfft, workers={cores}); the reference's FFTW/MPI build cannot be built on this image"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------- own arm
def run_form(torch, lib_mod, N, precision, steps, warmup, stream, V, dist):
    import ctypes as C
    from tarang_b200 import _lib as L
    from tarang_b200.solver import IncFluid
    # the context queues on the torch stream so the CUDA events see its kernels
    s = IncFluid(N, nu=NU, dt=DT, force=FORCE, precision=precision, stream=stream.cuda_stream)
    s.set_V(V)
    s.step(warmup)
    s.lib.tg_profile_enable(s.h, 1)
    s.lib.tg_profile_read(s.h, None, 0, None)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    s.lib.tg_step(s.h, steps, None)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    ms = ev0.elapsed_time(ev1)
    stats = (L.tg_kernel_stat * 32)()
    n = C.c_int()
    s.lib.tg_profile_read(s.h, stats, 32, C.byref(n))
    s.lib.tg_profile_enable(s.h, 0)
    kern = [{"name": stats[i].name.decode(), "launches": stats[i].launches, "total_ms": stats[i].total_ms,
             "bytes_per_launch": stats[i].bytes_per_launch} for i in range(n.value)]
    return s, ms, kern


def rel_l2(a, b):
    import numpy as np
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def e2e_measure(s, V, steps):
    """Drop-in use with host arrays: every step uploads the three velocity fields from pinned
    host memory, advances one RK4 step through the C ABI (energy read back), and downloads
    the fields again."""
    import ctypes as C
    import numpy as np
    import torch
    from tarang_b200 import _lib as L
    pinned = [torch.empty(s.ndoubles, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    for i in range(3):
        pinned[i].numpy()[:] = V[i].view(np.float64).ravel()
    ptrs = [C.cast(C.c_void_p(p.data_ptr()), C.POINTER(C.c_double)) for p in pinned]
    e = (C.c_double * 1)()
    s.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for i in range(3):
            s._ck(s.lib.tg_field_upload(s.h, L.TG_V1 + i, ptrs[i], s.ndoubles), "upload")
        s._ck(s.lib.tg_step(s.h, 1, e), "step")
        for i in range(3):
            s._ck(s.lib.tg_field_download(s.h, L.TG_V1 + i, ptrs[i], s.ndoubles), "download")
    el = time.perf_counter() - t0
    per = 3 * s.ndoubles * 8
    return {"value": steps / el, "unit": "steps/s", "h2d_bytes_per_step": per,
            "d2h_bytes_per_step": per + 8, "steps": steps,
            "path": "tg_field_upload x3 (pinned host) + tg_step(1, energy) + tg_field_download x3 per step"}


def run_own(args, rank, world, local):
    import numpy as np
    import torch
    dist = world > 1
    if dist:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    from tarang_b200 import _lib as L
    from tarang_b200 import ic
    L.load()
    n = args.size
    N = (n, n, n)
    V = ic.random_phase_field(N, seed=20261202 + rank)
    stream = torch.cuda.Stream()
    out = {}
    with torch.cuda.stream(stream):
        with Clocks(dev) as clk:
            s64, ms64, k64 = run_form(torch, L, N, "FP64", args.steps, args.warmup, stream, V, dist)
            s32, ms32, k32 = run_form(torch, L, N, "FP32", args.steps, args.warmup, stream, V, dist)
        clocks = clk.summary()
    t = torch.tensor([ms64, ms32], dtype=torch.float64, device="cuda")
    if dist:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms64, ms32 = float(t[0]), float(t[1])
    # FP32-mixed error against the FP64 form after err_steps steps (outside the timed region)
    err = None
    if args.err_steps > 0:
        s64.set_V(V)
        s32.set_V(V)
        s64.step(args.err_steps, energies=False)
        s32.step(args.err_steps, energies=False)
        a, b = s32.get_V(), s64.get_V()
        err = rel_l2(a, b)
        E64 = s64.CV_Compute_totalenergy_diss()[0]
        E32 = s32.CV_Compute_totalenergy_diss()[0]
    e2e = None
    if not args.no_e2e:
        e2e = e2e_measure(s64, V, max(3, min(args.steps, 20)))
    if rank != 0:
        if dist:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    hbm, peak_kind = peaks()

    def roof(kern, ms, steps, workload):
        dom = max(kern, key=lambda k: k["total_ms"])
        avg = dom["total_ms"] / dom["launches"]
        ach = dom["bytes_per_launch"] / (avg * 1e-3) / 1e9
        return {"kernel": dom["name"], "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "peak_kind": peak_kind,
                "traffic": profile_traffic(dom["name"], workload),
                "share": dom["total_ms"] / sum(k["total_ms"] for k in kern),
                "avg_launch_ms": avg, "launches_per_step": dom["launches"] / steps}

    steps = args.steps
    v64 = world * steps / (ms64 * 1e-3)
    v32 = world * steps / (ms32 * 1e-3)
    launches = sum(k["launches"] for k in k64) // steps
    # convention bytes per step (B_step = V_fft 2T + V64 14c, T = 36, c = 3)
    V64 = n * n * (n // 2 + 1) * 16
    b64 = V64 * 72 + V64 * 42
    b32 = V64 * 36 + V64 * 42
    line = {
        "metric": METRIC, "value": v64, "unit": "steps/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms64 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"forced isotropic NS {n}^3 FOUR, RK4, nu=1e-3, dt=5e-4, energy supply 2<k<=3 eps=0.1",
                   "grid": N, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "working set ~2 GB > 126 MB L2; no flush"},
        "gpu_launches": launches * steps,
        "roofline": roof(k64, ms64, steps, f"fluid{n}_fp64"),
        "fp32_mixed": {"value": v32, "ms_per_step": ms32 / steps, "speedup_vs_fp64": v32 / v64,
                       "rel_l2_err_vs_fp64": err, "err_steps": args.err_steps,
                       "energy_rel_err_vs_fp64": (abs(E32 - E64) / abs(E64)) if err is not None else None,
                       "roofline": roof(k32, ms32, steps, f"fluid{n}_fp32")},
        "step_bandwidth": {"convention_bytes_per_step_fp64": b64, "convention_bytes_per_step_fp32": b32,
                           "fp64_GBps": b64 * v64 / world / 1e9, "fp32_GBps": b32 * v32 / world / 1e9},
        "kernels_fp64": k64, "kernels_fp32": k32,
        "clocks": clocks,
    }
    if e2e:
        line["e2e"] = e2e
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n)
    print(json.dumps(line), flush=True)
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def cpu_baseline(n):
    from oracle import tarang_oracle as o
    from tarang_b200 import ic
    N = (n, n, n)
    V = ic.random_phase_field(N, seed=20261202)
    s = o.FluidSolver(N, (1.0, 1.0, 1.0), NU, DT, force=FORCE)
    t0 = time.perf_counter()
    V, _ = s.step(V)
    el = time.perf_counter() - t0
    cores = os.cpu_count()
    return {"value": 1.0 / el, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"1 RK4 step at {n}^3 of the oracle (numpy + scipy.fft pocketfft, workers={cores})"}


def main():
    args = parse()
    rank, world, local = dist_info()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_own(args, rank, world, local)


if __name__ == "__main__":
    main()
