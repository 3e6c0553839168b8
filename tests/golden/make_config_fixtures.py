"""Golden outputs of the oracle on the full-size workloads, for the GPU parity tests at those sizes.

The oracle needs 25 s per 256^3 RK4 step and about a minute per energy-transfer table on 8
cores, too slow to run inside every GPU test, so this script runs it once and writes what the
tests compare against into tests/golden/config_<name>.json:

  fluid256  forced isotropic Navier-Stokes 256^3 FOUR (random phase k^4 exp(-2 (k/4)^2),
            E = 0.5, seed 20261202; nu = 1e-3, dt = 5e-4, energy supply on 2 < k <= 3 at
            eps = 0.1), 10 RK4 steps: energy and dt per step, the velocity's sketch
            (oracle.sketch: 64 seeded random projections and the norm), its shell spectra and
            dissipation spectrum, the flux and shell-to-shell tables over 16 shells.
  mhd256    incompressible MHD 256^3 (u, b random phase k^4 exp(-2 (k/3)^2), E_u = E_b = 0.5,
            seeds 20261203 / 20261204; nu = eta = 1e-3, dt = 5e-4), 10 steps: energies per
            step, sketches of u and b, their spectra, the U->U, B->B, U<->B and B<->U fluxes
            and the U->U, B->B, U->B shell-to-shell tables over 16 shells.
  rb129     Rayleigh-Benard convection SCFT (129, 256, 256), aspect 1 : 2 sqrt 2 : 2 sqrt 2,
            Ra = 1e6, Pr = 1, dt = 1e-4, at rest plus the seeded temperature perturbation
            (seed 20261205), 10 steps: Nusselt number and temperature energy per step,
            sketches of u and theta, the theta shell spectrum.

The inputs are the synthetic seeded fields of tarang_b200.ic, as in bench.py.  Run:

    python tests/golden/make_config_fixtures.py fluid256 mhd256 rb129
"""

import json
import math
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from oracle import tarang_oracle as o  # noqa: E402
from tarang_b200 import ic  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
KF = (1.0, 1.0, 1.0)
KF_RB = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
STEPS = 10
S = 16
# energy-transfer kinds of the MHD tables: (helper, giver, receiver, sign), as tg_flux defines them
MHD_KINDS = {"UU": ("U", "U", "U", -1.0), "BB": ("U", "B", "B", -1.0), "UB": ("B", "U", "B", 1.0),
             "BU": ("U", "B", "U", 1.0)}


def _sk(fields):
    p, n = o.sketch(fields)
    return {"p": p.tolist(), "norm": n}


def fluid256():
    N = (256, 256, 256)
    force = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    V = ic.random_phase_field(N, seed=20261202)
    ref = o.FluidSolver(N, KF, 1e-3, 5e-4, force=force)
    E, dts = [], []
    for _ in range(STEPS):
        V, dt = ref.step(V)
        dts.append(dt)
        E.append(sum(o.total_energy_four(v) for v in V))
    return {
        "N": N, "steps": STEPS, "n_shells": S, "energy": E, "dt": dts, "V": _sk(V),
        "ek": [o.shell_spectrum(v, 0, KF).tolist() for v in V],
        "dk": (2 * sum(o.shell_spectrum(v, 2, KF) for v in V)).tolist(),
        "flux": {"UU": o.compute_flux(V, KF, S).tolist()},
        "shell_tr": {"UU": o.compute_shell_tr(V, KF, S).tolist()},
    }


def mhd256():
    N = (256, 256, 256)
    U = ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261203)
    B = ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261204)
    ref = o.MHDSolver(N, KF, 1e-3, 1e-3, 5e-4)
    Eu, Eb, dts = [], [], []
    for _ in range(STEPS):
        U, B, dt = ref.step2(U, B)
        dts.append(dt)
        Eu.append(sum(o.total_energy_four(v) for v in U))
        Eb.append(sum(o.total_energy_four(v) for v in B))
    fields = {"U": U, "B": B}
    flux, tr = {}, {}
    for k, (h, f, r, sg) in MHD_KINDS.items():
        flux[k] = o.compute_flux_generic(fields[h], fields[f], fields[r], sg, KF, S).tolist()
        if k != "BU":
            tr[k] = o.compute_shell_tr_generic(fields[h], fields[f], fields[r], sg, KF, S).tolist()
    return {
        "N": N, "steps": STEPS, "n_shells": S, "energy_u": Eu, "energy_b": Eb, "dt": dts,
        "U": _sk(U), "B": _sk(B),
        "ek_u": [o.shell_spectrum(v, 0, KF).tolist() for v in U],
        "ek_b": [o.shell_spectrum(v, 0, KF).tolist() for v in B],
        "flux": flux, "shell_tr": tr,
    }


def rb129():
    N = (129, 256, 256)
    T = ic.rb_perturbation(N, seed=20261205)
    V = [np.zeros_like(T) for _ in range(3)]
    ref = o.RBSolver(N, KF_RB, 1e6, 1.0, 1e-4)
    nus, Et, dts = [], [], []
    for _ in range(STEPS):
        V, T, dt = ref.step(V, T)
        dts.append(dt)
        nus.append(ref.nusselt(V, T))
        Et.append(o.total_energy(T, "SCFT"))
    return {
        "N": N, "steps": STEPS, "nusselt": nus, "energy_t": Et, "dt": dts, "V": _sk(V), "T": _sk([T]),
        "ek_t": o.shell_spectrum(T, 0, KF_RB, basis="SCFT").tolist(),
    }


def main(names):
    for name in names:
        t0 = time.time()
        out = {"what": name, "made_by": "tests/golden/make_config_fixtures.py"}
        out.update(globals()[name]())
        with open(os.path.join(HERE, f"config_{name}.json"), "w") as fh:
            json.dump(out, fh)
        print(f"{name}: {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["fluid256", "mhd256", "rb129"])
