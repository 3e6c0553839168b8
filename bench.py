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


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="own", choices=["own", "reference"])
    p.add_argument("--size", type=int, default=N_DEFAULT)
    p.add_argument("--err-steps", type=int, default=100)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the MHD and convection sections")
    p.add_argument("--serve-requests", type=int, default=512,
                   help="requests of the serving ensemble (0: skip it)")
    p.add_argument("--serve-steps", type=int, default=200)
    p.add_argument("--serve-rate", type=float, default=200.0, help="mean arrivals per second")
    p.add_argument("--serve-budget", type=float, default=150e9)
    return p.parse_args(argv)


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def shard(n, rank, world):
    """Indices of the n independent units (requests) that rank serves: every world-th one."""
    return list(range(rank, n, world))


def max_over_ranks(vals, dist, device="cuda"):
    """Element-wise maximum over ranks (all ranks call it; identity with one rank)."""
    if not dist:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def gather_all(obj, dist):
    """The objects of every rank, in rank order (all ranks call it)."""
    if not dist:
        return [obj]
    import torch
    out = [None] * torch.distributed.get_world_size()
    torch.distributed.all_gather_object(out, obj)
    return out


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
def set_fields(s, fields):
    """V, then W (MHD) or T (scalar, convection)."""
    s.set_V(fields[:3])
    if len(fields) == 6:
        s.set_W(fields[3:])
    elif len(fields) == 4:
        s.set_T(fields[3])


def get_fields(s, n):
    out = s.get_V()
    if n == 6:
        out += s.get_W()
    elif n == 4:
        out.append(s.get_T())
    return out


def run_form(torch, N, steps, warmup, stream, fields, dist, **kw):
    """Device time of `steps` RK4 steps (one CUDA graph each) of one solve, CUDA events on the
    context's stream, barriers around it; then the same number of steps again with per-launch
    events (eager) for the per-kernel breakdown, outside the timed region."""
    import ctypes as C
    from tarang_b200 import _lib as L
    from tarang_b200.solver import IncFluid
    # the context queues on the torch stream so the CUDA events see its kernels
    s = IncFluid(N, stream=stream.cuda_stream, **kw)
    set_fields(s, fields)
    s.step(warmup)
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
    s.lib.tg_profile_enable(s.h, 1)
    s.lib.tg_profile_read(s.h, None, 0, None)
    s.lib.tg_step(s.h, steps, None)
    stats = (L.tg_kernel_stat * 32)()
    n = C.c_int()
    s.lib.tg_profile_read(s.h, stats, 32, C.byref(n))
    s.lib.tg_profile_enable(s.h, 0)
    kern = [{"name": stats[i].name.decode(), "launches": stats[i].launches, "total_ms": stats[i].total_ms,
             "bytes_per_launch": stats[i].bytes_per_launch} for i in range(n.value)]
    return s, ms, kern


def kernel_roofline(kern):
    """Per pass kernel of a step: average launch time (live CUDA events), algorithmic bytes per
    launch and their rate against the measured HBM copy bandwidth, and the share of the step."""
    peak = peaks()[0]
    total = sum(k["total_ms"] for k in kern) or 1.0
    out = []
    for k in kern:
        if not k["launches"]:
            continue
        ms = k["total_ms"] / k["launches"]
        gbs = k["bytes_per_launch"] / (ms * 1e-3) / 1e9 if ms > 0 and k["bytes_per_launch"] else 0.0
        out.append({"name": k["name"], "avg_us": 1e3 * ms, "bytes_per_launch": k["bytes_per_launch"],
                    "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak if peak else None,
                    "share": k["total_ms"] / total})
    return out


def rel_max(a, b):
    """max |a - b| / max |b| (0 when both vanish)."""
    import numpy as np
    a, b = np.asarray(a), np.asarray(b)
    d = float(np.abs(b).max())
    return float(np.abs(a - b).max()) / d if d > 0 else float(np.abs(a).max())


def diag_errors(s32, s64, groups=(0,), et_kinds=(0,), force_feed=False):
    """FP32-mixed against FP64 for the diagnostics of the current fields: energy per group,
    shell spectra (energy, dissipation), fluxes and shell-to-shell tables per transfer kind."""
    from tarang_b200 import _lib as L
    out = {}
    for g in groups:
        e32, d32 = s32.CV_Compute_totalenergy_diss(g)
        e64, d64 = s64.CV_Compute_totalenergy_diss(g)
        out[f"energy_g{g}"] = abs(e32 - e64) / abs(e64)
        out[f"dissipation_g{g}"] = abs(d32 - d64) / abs(d64)
        k32, dk32 = s32.CV_Compute_shell_spectrum(g)
        k64, dk64 = s64.CV_Compute_shell_spectrum(g)
        out[f"spectrum_g{g}_max_shell_rel"] = rel_max(k32, k64)
        out[f"dissipation_spectrum_g{g}_max_shell_rel"] = rel_max(dk32, dk64)
    names = {L.TG_ET_UU: "UU", L.TG_ET_BB: "BB", L.TG_ET_UB: "UB", L.TG_ET_BU: "BU"}
    for k in et_kinds:
        out[f"flux_{names[k]}_max_shell_rel"] = rel_max(s32.Compute_flux(k), s64.Compute_flux(k))
        out[f"shell_to_shell_{names[k]}_max_rel"] = rel_max(s32.Compute_shell_tr(k), s64.Compute_shell_tr(k))
    if force_feed:
        out["force_feed_max_shell_rel"] = rel_max(s32.Compute_force_feed_shell(), s64.Compute_force_feed_shell())
    return out


def et_timing(s, kinds, reps=3):
    """Wall time of the flux and shell-to-shell tables of every kind (synchronous calls)."""
    s.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        for k in kinds:
            s.Compute_flux(k)
            s.Compute_shell_tr(k)
    return 1e3 * (time.perf_counter() - t0) / reps


def rel_l2(a, b):
    import numpy as np
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def e2e_measure(s, V, steps):
    """Drop-in use with host arrays: every step uploads the three velocity fields from pinned
    host memory, advances one RK4 step through the C ABI (energy read back), and downloads
    the fields again.  Upload and tg_field_download_stored move the stored (2/3-dealiased)
    modes only; the host arrays hold zeros elsewhere, as the reference's dealiased fields do."""
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
            s._ck(s.lib.tg_field_download_stored(s.h, L.TG_V1 + i, ptrs[i], s.ndoubles), "download")
    el = time.perf_counter() - t0
    # bytes that cross the bus: the stored modes (the 2/3 support) of the 3 fields
    from tarang_b200 import ic
    per = 3 * int(ic.keep_mask(s.N).sum()) * 16
    return {"value": steps / el, "unit": "steps/s", "h2d_bytes_per_step": per,
            "d2h_bytes_per_step": per + 8, "steps": steps,
            "path": "tg_field_upload x3 (pinned host, stored modes) + tg_step(1, energy) + "
                    "tg_field_download_stored x3 per step"}


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
            kw = dict(nu=NU, dt=DT, force=FORCE, n_shells=16)
            s64, ms64, k64 = run_form(torch, N, args.steps, args.warmup, stream, V, dist, precision="FP64", **kw)
            s32, ms32, k32 = run_form(torch, N, args.steps, args.warmup, stream, V, dist, precision="FP32", **kw)
        clocks = clk.summary()
    ms64, ms32 = max_over_ranks([ms64, ms32], dist)
    # FP32-mixed error against the FP64 form after err_steps steps (outside the timed region)
    err = None
    diag_err, et_ms = None, None
    if args.err_steps > 0:
        s64.set_V(V)
        s32.set_V(V)
        s64.step(args.err_steps, energies=False)
        s32.step(args.err_steps, energies=False)
        a, b = s32.get_V(), s64.get_V()
        err = rel_l2(a, b)
        E64 = s64.CV_Compute_totalenergy_diss()[0]
        E32 = s32.CV_Compute_totalenergy_diss()[0]
        diag_err = diag_errors(s32, s64, force_feed=True)
        et_ms = {"fp64": et_timing(s64, (0,)), "fp32": et_timing(s32, (0,))}
    e2e = None
    if not args.no_e2e:
        e2e = e2e_measure(s64, V, max(3, min(args.steps, 20)))
        # whole job: the steps of all ranks over the slowest rank's wall time
        (el,) = max_over_ranks([e2e["steps"] / e2e["value"]], dist)
        e2e["value"] = world * e2e["steps"] / el
    s64.close()
    s32.close()
    configs = None
    if rank == 0 and not args.no_configs:
        with torch.cuda.stream(stream):
            configs = run_configs(args, torch, stream)
    serving = None
    if args.serve_requests > 0:
        serving = run_serving(args, rank, world, dist)
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
                       "diagnostics_err_vs_fp64": diag_err,
                       "roofline": roof(k32, ms32, steps, f"fluid{n}_fp32")},
        "step_bandwidth": {"convention_bytes_per_step_fp64": b64, "convention_bytes_per_step_fp32": b32,
                           "fp64_GBps": b64 * v64 / world / 1e9, "fp32_GBps": b32 * v32 / world / 1e9},
        "energy_transfer_ms": ({"shells": 16, "what": "flux + shell-to-shell tables (UU), one call each",
                                **et_ms} if et_ms else None),
        "kernels_fp64": k64, "kernels_fp32": k32,
        "clocks": clocks,
    }
    if e2e:
        line["e2e"] = e2e
    if configs is not None:
        line["configs"] = configs
    if serving is not None:
        line["serving"] = serving
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n)
    print(json.dumps(line), flush=True)
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# --------------------------------------------------------------------------------- other configs
def run_configs(args, torch, stream):
    """The MHD (256^3) and Rayleigh-Benard (SCFT, N1 = 129 and 128 by 256 x 256) workloads on one
    GPU: device-timed steps/s of the FP64 and FP32-mixed forms and the FP32-mixed error of every
    field, spectrum and transfer after err_steps steps (synthetic seeded initial fields)."""
    import numpy as np
    from tarang_b200 import _lib as L
    from tarang_b200 import ic
    out = {}
    steps, warm = max(3, min(args.steps, 20)), args.warmup
    es = max(1, min(args.err_steps, 100))
    # MHD 256^3: u, b random phase E(k) ~ k^4 exp(-2 (k/3)^2), E_u = E_b = 0.5; nu = eta = 1e-3
    n = args.size
    N = (n, n, n)
    f = ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261203) + \
        ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261204)
    kw = dict(physics="MHD", nu=1e-3, eta=1e-3, dt=5e-4, n_shells=16)
    s64, ms64, k64 = run_form(torch, N, steps, warm, stream, f, False, precision="FP64", **kw)
    s32, ms32, k32 = run_form(torch, N, steps, warm, stream, f, False, precision="FP32", **kw)
    for s_ in (s64, s32):
        set_fields(s_, f)
        s_.step(es, energies=False)
    kinds = (L.TG_ET_UU, L.TG_ET_BB, L.TG_ET_UB, L.TG_ET_BU)
    out["mhd"] = {
        "workload": f"incompressible MHD {n}^3 FOUR, u and b random phase k^4 exp(-2 (k/3)^2), E_u = E_b = 0.5, "
                    "nu = eta = 1e-3, dt = 5e-4, RK4; fluxes U->U, B->B, U<->B over 16 shells",
        "steps_per_s_fp64": 1e3 * steps / ms64, "steps_per_s_fp32": 1e3 * steps / ms32,
        "fp32_speedup": ms64 / ms32, "err_steps": es,
        "rel_l2_err_vs_fp64": {"u": rel_l2(s32.get_V(), s64.get_V()), "b": rel_l2(s32.get_W(), s64.get_W())},
        "diagnostics_err_vs_fp64": diag_errors(s32, s64, groups=(0, 1), et_kinds=kinds),
        "energy_transfer_ms": {"fp64": et_timing(s64, kinds, 1), "fp32": et_timing(s32, kinds, 1),
                               "what": "flux + shell-to-shell tables of the 4 kinds"},
        "kernel_roofline_fp64": kernel_roofline(k64), "kernel_roofline_fp32": kernel_roofline(k32),
    }
    s64.close()
    s32.close()
    # Rayleigh-Benard: SCFT, aspect 1 : 2 sqrt 2 : 2 sqrt 2, Ra = 1e6, Pr = 1, dt = 1e-4, at rest
    # plus a temperature perturbation of amplitude 1e-3 in the lowest 8 modes
    for n1 in (129, 128):
        N = (n1, 2 * (n // 2), 2 * (n // 2))
        shape = (N[0], N[1], N[2] // 2 + 1)
        f = [np.zeros(shape, dtype=np.complex128) for _ in range(3)] + [ic.rb_perturbation(N, seed=20261205)]
        kw = dict(basis="SCFT", physics="RB", Ra=1e6, Pr=1.0, dt=1e-4, kfactor=KF_RB)
        s64, ms64, k64 = run_form(torch, N, steps, warm, stream, f, False, precision="FP64", **kw)
        s32, ms32, k32 = run_form(torch, N, steps, warm, stream, f, False, precision="FP32", **kw)
        for s_ in (s64, s32):
            set_fields(s_, f)
            s_.step(es, energies=False)
        nu64, nu32 = s64.Get_Nusselt_no(), s32.Get_Nusselt_no()
        t32, _ = s32.CV_Compute_shell_spectrum(2)
        t64, _ = s64.CV_Compute_shell_spectrum(2)
        out[f"rb_{n1}"] = {
            "workload": f"Rayleigh-Benard SCFT {N[0]}x{N[1]}x{N[2]}, Ra = 1e6, Pr = 1, dt = 1e-4, RK4",
            "steps_per_s_fp64": 1e3 * steps / ms64, "steps_per_s_fp32": 1e3 * steps / ms32,
            "fp32_speedup": ms64 / ms32, "err_steps": es,
            "rel_l2_err_vs_fp64": {"u": rel_l2(s32.get_V(), s64.get_V()), "theta": rel_l2([s32.get_T()], [s64.get_T()])},
            "nusselt": {"fp64": nu64, "fp32": nu32, "rel_err": abs(nu32 - nu64) / abs(nu64)},
            "theta_spectrum_max_shell_rel": rel_max(t32, t64),
            "kernel_roofline_fp64": kernel_roofline(k64), "kernel_roofline_fp32": kernel_roofline(k32),
        }
        s64.close()
        s32.close()
    return out


# --------------------------------------------------------------------------------- serving
KF_RB = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
SERVE_MAX_BATCH = 128   # request slots per batch: every type of the ensemble fits one batch
SERVE_TYPES = [  # name, configuration, initial condition kind
    ("fluid32", dict(N=(32, 32, 32)), "fluid"),
    ("fluid64", dict(N=(64, 64, 64)), "fluid"),
    ("fluid128", dict(N=(128, 128, 128)), "fluid"),
    ("mhd64", dict(N=(64, 64, 64), physics="MHD"), "mhd"),
    ("rb65x128x128", dict(N=(65, 128, 128), basis="SCFT", physics="RB", kfactor=KF_RB), "rb"),
]


def serve_ic(kind, N, seed):
    """Packed initial fields (n_fields, N1, N2, N3/2+1): random-phase k^4 exp(-2 (k/k0)^2)
    velocity (k0 = 4, E = 0.5); MHD adds a magnetic field of the same shape (k0 = 3, E_u = E_b =
    0.5); convection starts from rest with a temperature perturbation in the lowest 8 modes."""
    import numpy as np
    from tarang_b200 import ic
    if kind == "fluid":
        f = ic.random_phase_field(N, k0=4.0, energy=0.5, seed=seed)
    elif kind == "mhd":
        f = ic.random_phase_field(N, k0=3.0, energy=0.5, seed=seed) + \
            ic.random_phase_field(N, k0=3.0, energy=0.5, seed=seed + 1)
    else:
        shape = (N[0], N[1], N[2] // 2 + 1)
        f = [np.zeros(shape, dtype=np.complex128) for _ in range(3)] + [ic.rb_perturbation(N, seed=seed)]
    return np.ascontiguousarray(np.stack(f))


def serve_request_config(base, nu, dt_fluid=DT, dt_rb=1e-4):
    c = dict(base, precision="FP32")
    if c.get("physics") == "RB":
        c.update(Ra=1.0 / (nu * nu), Pr=1.0, dt=dt_rb)     # nu = sqrt(Pr/Ra)
    elif c.get("physics") == "MHD":
        c.update(nu=nu, eta=nu, dt=dt_fluid)
    else:
        c.update(nu=nu, dt=dt_fluid)
    return c


def lone_run(cfg, init, steps):
    """One request as a lone context: create, upload, `steps` RK4 steps, download, destroy."""
    from tarang_b200.solver import IncFluid
    c = dict(cfg)
    N = c.pop("N")
    s = IncFluid(N, **c)
    s.set_V(init[:3])
    if init.shape[0] == 6:
        s.set_W(init[3:])
    elif init.shape[0] == 4:
        s.set_T(init[3])
    s.step(steps, energies=False)
    out = s.get_V()
    if init.shape[0] == 6:
        out += s.get_W()
    elif init.shape[0] == 4:
        out.append(s.get_T())
    s.close()
    return out


def serve_workload(args):
    """The serving ensemble, identical on every rank: (type, configuration, packed fields) per
    request and the arrival times of a seeded Poisson stream."""
    import numpy as np
    n_req = args.serve_requests
    rng = np.random.Generator(np.random.PCG64(20261203))
    kinds = rng.integers(0, len(SERVE_TYPES), n_req)
    nus = np.exp(rng.uniform(math.log(1e-3), math.log(1e-2), n_req))
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n_req))
    pool = {}
    for t, (name, base, kind) in enumerate(SERVE_TYPES):
        pool[t] = [serve_ic(kind, base["N"], 7000 + 10 * t + j) for j in range(2)]
    reqs = [(int(k), serve_request_config(SERVE_TYPES[k][1], float(nu)), pool[int(k)][i % 2])
            for i, (k, nu) in enumerate(zip(kinds, nus))]
    return reqs, arrivals


class pinned_in_place:
    """Page-locks the distinct numpy arrays given (cudaHostRegister) for the duration of a with
    block; no-op where registration is refused."""

    def __init__(self, arrays):
        uniq = {}
        for a in arrays:
            uniq.setdefault(a.__array_interface__["data"][0], a)
        self.arrays = list(uniq.values())
        self.done = []

    def __enter__(self):
        import torch
        cr = torch.cuda.cudart()
        for a in self.arrays:
            ptr, n = a.__array_interface__["data"][0], a.nbytes
            if int(cr.cudaHostRegister(ptr, n, 0)) == 0:
                self.done.append(ptr)
        return self

    def __exit__(self, *exc):
        import torch
        cr = torch.cuda.cudart()
        for ptr in self.done:
            cr.cudaHostUnregister(ptr)
        return False


def serve_loop(srv, reqs, arrivals, mine, steps, keep):
    """Submit requests `mine` at their arrival times, pump until all finish; returns
    (finish records by request index, kept results, pump round times, clock origin).  Each round
    is launched first (pump_begin) and the requests that have arrived are submitted while its
    steps run on the device; pump_end admits them and waits for the round."""
    ids, fin, results, round_ms = {}, {}, {}, []
    t_base = srv.clock()
    sub = 0
    active = 0

    def submit_arrived():
        nonlocal sub
        now = srv.clock() - t_base
        while sub < len(mine) and arrivals[mine[sub]] <= now:
            i = mine[sub]
            ids[srv.submit(reqs[i][1], reqs[i][2], steps)] = i
            sub += 1
        return now

    while True:
        if active == 0:
            now = submit_arrived()
            if len(ids) == len(fin):          # nothing in the server: wait for the next arrival
                time.sleep(min(max(arrivals[mine[sub]] - now, 0.0), 0.05))
                continue
        r0 = time.perf_counter()
        srv.pump_begin()
        submit_arrived()
        active = srv.pump_end()
        round_ms.append(1e3 * (time.perf_counter() - r0))
        for rid in srv.take_finished():
            i = ids[rid]
            fin[i] = srv.poll(rid)
            if i in keep and fin[i]["state"] == "done":
                results[i] = srv.result(rid)
            srv.release(rid)
        if sub == len(mine) and active == 0:
            return fin, results, round_ms, t_base


def sequential_solves(batch, steps):
    """Mean seconds per request of solving `batch` (same shape) one after another on one
    reused context: upload the fields, run the steps, download the fields."""
    from tarang_b200.solver import IncFluid
    c = dict(batch[0][1])
    N = c.pop("N")
    s = IncFluid(N, **c)
    el = []
    for j, (_, cfg, init) in enumerate(batch):
        t0 = time.perf_counter()
        s.set_V(init[:3])
        if init.shape[0] == 6:
            s.set_W(init[3:])
        elif init.shape[0] == 4:
            s.set_T(init[3])
        s.step(steps, energies=False)
        s.get_V()
        if init.shape[0] == 6:
            s.get_W()
        elif init.shape[0] == 4:
            s.get_T()
        if j > 0:                    # the first solve pays the one-time graph capture
            el.append(time.perf_counter() - t0)
    s.close()
    return statistics.mean(el) if el else float("nan")


def serving_shapes(n_batch=64, steps=20):
    """Per request type (FP32-mixed, nu = 3e-3): the device time of one request-step on a lone
    context (graph replay, CUDA events on its stream) and in a batch of n_batch requests of that
    type alone on a server (the batch step's event time / n_batch); the algorithmic bytes of one
    request-step (sum over the step's kernels of bytes per launch x launches, the convention of
    the per-kernel roofline) and both rates against the measured HBM copy bandwidth."""
    import torch
    from tarang_b200.serving import Server
    hbm, peak_kind = peaks()
    out = {}
    stream = torch.cuda.Stream()
    for name, base, kind in SERVE_TYPES:
        cfg = serve_request_config(base, 3e-3)
        init = serve_ic(kind, base["N"], 7000)
        c = dict(cfg)
        N = c.pop("N")
        with torch.cuda.stream(stream):
            s, ms, kern = run_form(torch, N, steps, 3, stream, init, False, **c)
        s.close()
        lone = ms / steps
        bstep = sum(k["bytes_per_launch"] * k["launches"] for k in kern) / steps
        srv = Server(hbm_budget=150e9, max_batch=n_batch, keep_results=False)
        for _ in range(n_batch):
            srv.submit(cfg, init, steps)
        srv.drain()
        timed = [b for b in srv.batch_stats() if b["step_ms"] > 0]
        srv.close()
        b = max(timed, key=lambda b: b["step_ms_n_active"])
        per = b["step_ms"] / b["step_ms_n_active"]
        out[name] = {"grid": list(N), "bytes_per_request_step": bstep,
                     "lone_ms_per_step": lone, "lone_frac_of_hbm": bstep / (lone * 1e-3) / 1e9 / hbm,
                     "batched_requests": b["step_ms_n_active"], "batched_ms_per_request_step": per,
                     "batched_frac_of_hbm": bstep / (per * 1e-3) / 1e9 / hbm,
                     "batched_speedup_vs_lone": lone / per}
    return {"per_type": out, "peak_gbs": hbm, "peak_kind": peak_kind,
            "method": f"lone: {steps} graph-replayed steps of one context, CUDA events; batched: {n_batch} "
                      f"requests of the type alone on a server, {steps} steps, the batch step's CUDA-event time "
                      f"(average over rounds at that active count) / {n_batch}"}


def run_serving(args, rank=0, world=1, dist=False):
    """A seeded Poisson stream of independent solves (sizes and physics drawn uniformly from
    SERVE_TYPES, viscosity log-uniform in [1e-3, 1e-2], FP32-mixed) through tg_server, one
    server per GPU serving every world-th request, against the same requests solved one after
    another on lone contexts (rank 0's GPU).  Returns the aggregate on rank 0, None elsewhere."""
    import numpy as np
    from tarang_b200.serving import Server, request_bytes
    n_req, steps = args.serve_requests, args.serve_steps
    reqs, arrivals = serve_workload(args)
    mine = shard(n_req, rank, world)
    first_of_type = {}
    for i in range(n_req):
        first_of_type.setdefault(reqs[i][0], i)
    keep = {i for i in first_of_type.values() if i in set(mine)}
    lone_run(reqs[0][1], reqs[0][2], 2)          # module load and first-launch costs
    if dist:
        import torch
        torch.distributed.barrier()
    # the request fields are the workload's own arrays, alive for the whole run: the server reads
    # them at admission instead of copying them at submission, and they are page-locked in place
    # once (the client keeps its input buffers pinned), so admission's uploads are plain
    # asynchronous copies
    with pinned_in_place([f for _, _, f in reqs]):
        srv = Server(hbm_budget=args.serve_budget, max_batch=SERVE_MAX_BATCH, keep_results=True, borrow_inputs=True)
        fin, results, round_ms, t_base = serve_loop(srv, reqs, arrivals, mine, steps, keep)
        st = srv.stats()
        srv.close()
    done = [i for i in fin if fin[i]["state"] == "done"]
    local = {
        "comp": [fin[i]["finish_s"] - t_base - arrivals[i] for i in done],
        "per_step": [(fin[i]["finish_s"] - fin[i]["start_s"]) / steps for i in done],
        "failed": len(fin) - len(done),
        "makespan": max(f["finish_s"] for f in fin.values()) - t_base - arrivals[0] if fin else 0.0,
        "round_ms": round_ms, "bytes_peak": st["bytes_peak"], "graph_launches": st["graph_launches"],
        "eager_steps": st["eager_steps"], "errs": {},
    }
    # FP32-mixed error of the first served request of each type against its FP64 lone solve
    for i in sorted(results):
        c64 = dict(reqs[i][1], precision="FP64")
        local["errs"][SERVE_TYPES[reqs[i][0]][0]] = rel_l2(results[i], lone_run(c64, reqs[i][2], steps))
    # sequential baseline on rank 0: per type, the same solves one after another on one context
    # of that shape, created once beforehand (upload, steps, download per request)
    # and, as the reference runs solves (one program run each), every request on a context of
    # its own: create, upload, steps, download, release
    seq_s, fresh_s = {}, {}
    shapes = serving_shapes() if rank == 0 else None
    if rank == 0:
        for t in range(len(SERVE_TYPES)):
            idx = [i for i in range(n_req) if reqs[i][0] == t][:3]
            if idx:
                seq_s[t] = sequential_solves([reqs[i] for i in idx], steps)
                # context set-up time swings from run to run (tens to hundreds of ms): the median of
                # five solves
                el = []
                for i in (idx * 2)[:5]:
                    t0 = time.perf_counter()
                    lone_run(reqs[i][1], reqs[i][2], steps)
                    el.append(time.perf_counter() - t0)
                fresh_s[t] = statistics.median(el)
    parts = gather_all(local, dist)
    if rank != 0:
        return None
    comp = np.array([x for p in parts for x in p["comp"]])
    per_step = np.array([x for p in parts for x in p["per_step"]])
    rounds = np.array([x for p in parts for x in p["round_ms"]])
    makespan = max(p["makespan"] for p in parts)
    errs = {}
    for p in parts:
        errs.update(p["errs"])
    total_steps = n_req * steps
    seq_total = sum(seq_s[k] for k, _, _ in reqs)
    fresh_total = sum(fresh_s[k] for k, _, _ in reqs)
    points = sum(float(np.prod(cfg["N"])) for _, cfg, _ in reqs) * steps
    agg = total_steps / makespan
    return {
        "workload": f"{n_req} requests, Poisson {args.serve_rate:g}/s, {steps} RK4 steps each, FP32-mixed; "
                    "types uniform over " + ", ".join(n for n, _, _ in SERVE_TYPES) +
                    "; nu log-uniform [1e-3, 1e-2] (convection: Ra = Pr/nu^2, Pr = 1)",
        "gpus": world, "placement": "request i on rank i mod n_gpus, one server per GPU",
        "hbm_budget_bytes_per_gpu": args.serve_budget, "max_batch": SERVE_MAX_BATCH,
        "requests_done": int(len(comp)), "requests_failed": sum(p["failed"] for p in parts),
        "aggregate_request_steps_per_s": agg,
        "aggregate_grid_point_steps_per_s": points / makespan,
        "makespan_s": makespan,
        "completion_latency_s": {"p50": float(np.percentile(comp, 50)), "p99": float(np.percentile(comp, 99)),
                                 "max": float(comp.max())},
        "step_latency_ms": {"p50": 1e3 * float(np.percentile(per_step, 50)),
                            "p99": 1e3 * float(np.percentile(per_step, 99))},
        "round_ms": {"p50": float(np.percentile(rounds, 50)), "p99": float(np.percentile(rounds, 99)),
                     "rounds": int(len(rounds))},
        "sequential": {"request_steps_per_s": total_steps / fresh_total, "est_total_s": fresh_total,
                       "per_request_s": {SERVE_TYPES[t][0]: v for t, v in fresh_s.items()},
                       "method": "each request solved alone on a context of its own (create, upload, 200 steps, download, release), as the reference runs one solve per program run; median of 5 per type, x the type's count; one GPU"},
        "sequential_reused_context": {
            "request_steps_per_s": total_steps / seq_total, "est_total_s": seq_total,
            "per_request_s": {SERVE_TYPES[t][0]: v for t, v in seq_s.items()},
            "method": "per type, solves one after another on one reused context of that shape created beforehand (upload, 200 steps, download); mean of the 2nd and 3rd solve, x the type's count; one GPU"},
        "speedup_vs_sequential": agg / (total_steps / fresh_total),
        "speedup_vs_sequential_reused_context": agg / (total_steps / seq_total),
        "speedup_vs_sequential_per_gpu": agg / world / (total_steps / fresh_total),
        "rel_l2_err_vs_fp64": errs,
        "per_type_step": shapes,
        "bytes_peak": max(p["bytes_peak"] for p in parts),
        "graph_launches": sum(p["graph_launches"] for p in parts),
        "eager_steps": sum(p["eager_steps"] for p in parts),
        "request_bytes": {n: request_bytes(serve_request_config(b, 1e-3)) for n, b, _ in SERVE_TYPES},
    }


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
