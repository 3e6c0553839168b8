"""Run a few RK4 steps of a configuration for an external profiler (ncu).

    python -m tarang_b200.profile_step --n 256 --precision FP64 --steps 1 --warmup 0
    python -m tarang_b200.profile_step --physics RB --n1 129 --n 256 --precision FP64
    python -m tarang_b200.profile_step --serve 64 --n 128 --precision FP32 --steps 3

Workloads: forced fluid n^3 (energy supply on 2 < k <= 3), MHD n^3 (random-phase u and b), or
Rayleigh-Benard convection in the SCFT basis on (n1, n, n) (aspect 1 : 2 sqrt 2 : 2 sqrt 2,
Ra = 1e6, Pr = 1, dt = 1e-4, the seeded temperature perturbation).  Every step runs eagerly (profiling mode keeps graph replay off) so each kernel is a separate
launch; with --warmup 0 and --steps 1 a fluid step launches each pass kernel 4 times.

--serve B: B requests of the chosen workload (unforced; nu = 3e-3) submitted at once to one
server (one batch of B slots), run for --steps steps: the first step eager, the rest as one
captured CUDA graph per step.  Prints the batch's step time (CUDA events) per request.
"""

from __future__ import annotations

import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=256)
    p.add_argument("--n1", type=int, default=129, help="RB: points along the wall normal")
    p.add_argument("--precision", default="FP64")
    p.add_argument("--physics", default="FLUID")
    p.add_argument("--steps", type=int, default=1)
    p.add_argument("--warmup", type=int, default=0)
    p.add_argument("--serve", type=int, default=0, help="batched: this many requests on one server")
    a = p.parse_args()
    from tarang_b200 import _lib as L
    from tarang_b200 import ic
    from tarang_b200.solver import IncFluid
    if a.serve:
        serve(a, ic)
        return
    if a.physics == "RB":
        import math

        import numpy as np
        N = (a.n1, a.n, a.n)
        kf = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
        s = IncFluid(N, basis="SCFT", physics="RB", Ra=1e6, Pr=1.0, dt=1e-4, kfactor=kf, precision=a.precision)
        T = ic.rb_perturbation(N, seed=20261205)
        s.set_V([np.zeros_like(T) for _ in range(3)])
        s.set_T(T)
    else:
        N = (a.n, a.n, a.n)
        force = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0) if a.physics == "FLUID" else None
        s = IncFluid(N, nu=1e-3, dt=5e-4, force=force, precision=a.precision, physics=a.physics)
        s.set_V(ic.random_phase_field(N, seed=20261202))
        if a.physics == "MHD":
            s.set_W(ic.random_phase_field(N, k0=3.0, seed=20261204))
    s.lib.tg_profile_enable(s.h, 1)   # eager launches
    if a.warmup:
        s.step(a.warmup)
    E = s.step(a.steps)
    s.synchronize()
    print(f"ok {a.physics} {a.n}^3 {a.precision}: {a.steps} steps, E = {E[-1]:.12e}")
    s.lib.tg_profile_read(s.h, None, 0, None)
    s.close()


def serve(a, ic):
    import math

    import numpy as np
    from tarang_b200.serving import Server
    if a.physics == "RB":
        N = (a.n1, a.n, a.n)
        kf = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
        cfg = dict(N=N, basis="SCFT", physics="RB", Ra=1.0 / 9e-6, Pr=1.0, dt=1e-4, kfactor=kf)
        T = ic.rb_perturbation(N, seed=7000)
        f = [np.zeros_like(T) for _ in range(3)] + [T]
    else:
        N = (a.n, a.n, a.n)
        cfg = dict(N=N, physics=a.physics, nu=3e-3, dt=5e-4)
        if a.physics == "MHD":
            cfg["eta"] = 3e-3
        f = ic.random_phase_field(N, k0=4.0, energy=0.5, seed=7000)
        if a.physics == "MHD":
            f = f + ic.random_phase_field(N, k0=3.0, energy=0.5, seed=7001)
    cfg["precision"] = a.precision
    init = np.ascontiguousarray(np.stack(f))
    srv = Server(hbm_budget=150e9, max_batch=a.serve, keep_results=False)
    for _ in range(a.serve):
        srv.submit(cfg, init, a.steps)
    srv.drain()
    for b in srv.batch_stats():
        if b["step_ms_n_active"]:
            print(f"ok served {a.physics} {N} {a.precision}: {b['step_ms_n_active']} requests, "
                  f"{b['step_ms']:.3f} ms per batch step, {b['step_ms'] / b['step_ms_n_active']:.4f} ms per request-step")
    srv.close()


if __name__ == "__main__":
    main()
