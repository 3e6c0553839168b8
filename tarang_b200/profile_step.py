"""Run a few RK4 steps of a configuration for an external profiler (ncu).

    python -m tarang_b200.profile_step --n 256 --precision FP64 --steps 1 --warmup 0
    python -m tarang_b200.profile_step --physics RB --n1 129 --n 256 --precision FP64

Workloads: forced fluid n^3 (energy supply on 2 < k <= 3), MHD n^3 (random-phase u and b), or
Rayleigh-Benard convection in the SCFT basis on (n1, n, n) (aspect 1 : 2 sqrt 2 : 2 sqrt 2,
Ra = 1e6, Pr = 1, dt = 1e-4, the seeded temperature perturbation).  Every step runs eagerly (profiling mode keeps graph replay off) so each kernel is a separate
launch; with --warmup 0 and --steps 1 a fluid step launches each pass kernel 4 times.
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
    a = p.parse_args()
    from tarang_b200 import _lib as L
    from tarang_b200 import ic
    from tarang_b200.solver import IncFluid
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


if __name__ == "__main__":
    main()
