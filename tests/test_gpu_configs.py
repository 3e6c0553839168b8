"""Parity at the sizes and step counts of the benchmark workloads (FP64 form).

Taylor-Green 64^3 runs the oracle live for all 100 steps.  The 256^3 fluid and MHD runs and
the (129, 256, 256) convection run compare with golden outputs of the oracle
(tests/golden/config_*.json, written by tests/golden/make_config_fixtures.py, because the oracle
needs minutes per step there): 10 steps each.

Bars:
  * fields: relative L2 error <= 1e-12 (at 256^3 estimated from 64 seeded random projections,
    oracle.sketch / rel_from_sketch);
  * energies, Nusselt numbers and dt per step: relative 1e-12;
  * spectra, fluxes and shell-to-shell tables per shell:
        |gpu - oracle| <= 1e-10 |oracle| + 1e-13 max|oracle|
    (the absolute floor covers the shells whose content is at round-off level, e.g. the
    empty rows of a shell-to-shell table and the far spectral tail).
Also the FP32-mixed form against the FP64 form after 100 steps at the same sizes: relative
L2 <= 1e-6 for every field.
"""

import json
import math
import os

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KF = (1.0, 1.0, 1.0)
KF_RB = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
REL, FLOOR = 1e-10, 1e-13


def per_shell(got, want, what, rel=REL, floor=FLOOR):
    want = np.asarray(want, dtype=float)
    got = np.asarray(got, dtype=float).reshape(-1)[: want.size].reshape(want.shape)
    tol = rel * np.abs(want) + floor * np.abs(want).max()
    bad = np.argwhere(np.abs(got - want) > tol)
    assert bad.size == 0, (f"{what}: {len(bad)} shells off, first {bad[:4].tolist()}; "
                           f"max |d|/|w| = {np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)):.3e}")


def rel_l2(a, b):
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def close_rel(got, want, tol, what):
    got, want = np.asarray(got, dtype=float), np.asarray(want, dtype=float)
    err = np.abs(got - want) / np.abs(want)
    assert err.max() <= tol, f"{what}: max rel err {err.max():.3e}"


def gold(name):
    with open(os.path.join(GOLD, f"config_{name}.json")) as fh:
        return json.load(fh)


def sketch_err(fields, g):
    p, _ = o.sketch(fields)
    return o.rel_from_sketch(p, g["p"], g["norm"])


def solver(N, **kw):
    from tarang_b200.solver import IncFluid
    return IncFluid(N, **kw)


def test_taylor_green_64_100_steps(lib):
    """Taylor-Green 64^3, nu = 0.01, dt = 1e-3, 100 steps; energy per step, the spectrum's 38
    shells and the 12-shell flux and shell-to-shell tables, against the oracle run live."""
    N = (64, 64, 64)
    V0 = ic.taylor_green(N)
    s = solver(N, nu=0.01, dt=1e-3, n_shells=12)
    try:
        s.set_V(V0)
        E = s.step(100)
        ref = o.FluidSolver(N, KF, 0.01, 1e-3)
        V, Ew = V0, []
        for _ in range(100):
            V, dt = ref.step(V)
            assert dt == 1e-3
            Ew.append(sum(o.total_energy_four(v) for v in V))
        assert rel_l2(s.get_V(), V) <= 1e-12
        close_rel(E, Ew, 1e-12, "energy per step")
        ek, dk = s.CV_Compute_shell_spectrum()
        assert ek.shape[1] == 38
        for i in range(3):
            per_shell(ek[i], o.shell_spectrum(V[i], 0, KF), f"ek[{i}]")
        per_shell(dk, 2 * sum(o.shell_spectrum(v, 2, KF) for v in V), "dissipation spectrum")
        per_shell(s.Compute_flux(), o.compute_flux(V, KF, 12), "flux")
        per_shell(s.Compute_shell_tr(), o.compute_shell_tr(V, KF, 12), "shell-to-shell")
    finally:
        s.close()


def test_forced_fluid_256_10_steps(lib):
    g = gold("fluid256")
    N = tuple(g["N"])
    force = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    s = solver(N, nu=1e-3, dt=5e-4, force=force, n_shells=g["n_shells"])
    try:
        s.set_V(ic.random_phase_field(N, seed=20261202))
        E, dts = [], []
        for _ in range(g["steps"]):
            dts.append(s.Get_dt())
            E.extend(s.step(1))
        close_rel(E, g["energy"], 1e-12, "energy per step")
        close_rel(dts, g["dt"], 1e-12, "dt per step")
        V = s.get_V()
        err = sketch_err(V, g["V"])
        assert err <= 1e-12, f"velocity rel L2 ~ {err:.3e}"
        ek, dk = s.CV_Compute_shell_spectrum()
        for i in range(3):
            per_shell(ek[i], g["ek"][i], f"ek[{i}]")
        per_shell(dk, g["dk"], "dissipation spectrum")
        per_shell(s.Compute_flux(), g["flux"]["UU"], "flux")
        per_shell(s.Compute_shell_tr(), g["shell_tr"]["UU"], "shell-to-shell")
    finally:
        s.close()


def test_mhd_256_10_steps(lib):
    g = gold("mhd256")
    N = tuple(g["N"])
    s = solver(N, physics="MHD", nu=1e-3, eta=1e-3, dt=5e-4, n_shells=g["n_shells"])
    try:
        s.set_V(ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261203))
        s.set_W(ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261204))
        Eu, Eb = [], []
        for _ in range(g["steps"]):
            s.step(1)
            Eu.append(s.CV_Compute_totalenergy_diss(0)[0])
            Eb.append(s.CV_Compute_totalenergy_diss(1)[0])
        close_rel(Eu, g["energy_u"], 1e-12, "E_u per step")
        close_rel(Eb, g["energy_b"], 1e-12, "E_b per step")
        for name, fields in (("U", s.get_V()), ("B", s.get_W())):
            err = sketch_err(fields, g[name])
            assert err <= 1e-12, f"{name} rel L2 ~ {err:.3e}"
        eu, _ = s.CV_Compute_shell_spectrum(0)
        eb, _ = s.CV_Compute_shell_spectrum(1)
        for i in range(3):
            per_shell(eu[i], g["ek_u"][i], f"ek_u[{i}]")
            per_shell(eb[i], g["ek_b"][i], f"ek_b[{i}]")
        kinds = {"UU": L.TG_ET_UU, "BB": L.TG_ET_BB, "UB": L.TG_ET_UB, "BU": L.TG_ET_BU}
        for k, kind in kinds.items():
            per_shell(s.Compute_flux(kind), g["flux"][k], f"flux {k}")
            if k in g["shell_tr"]:
                per_shell(s.Compute_shell_tr(kind), g["shell_tr"][k], f"shell-to-shell {k}")
    finally:
        s.close()


def test_convection_129x256x256_10_steps(lib):
    g = gold("rb129")
    N = tuple(g["N"])
    T0 = ic.rb_perturbation(N, seed=20261205)
    s = solver(N, basis="SCFT", physics="RB", Ra=1e6, Pr=1.0, dt=1e-4, kfactor=KF_RB)
    try:
        s.set_V([np.zeros_like(T0) for _ in range(3)])
        s.set_T(T0)
        nus, Et = [], []
        for _ in range(g["steps"]):
            s.step(1)
            nus.append(s.Get_Nusselt_no())
            Et.append(s.CV_Compute_totalenergy_diss(2)[0])
        close_rel(nus, g["nusselt"], 1e-12, "Nusselt number per step")
        close_rel(Et, g["energy_t"], 1e-12, "theta energy per step")
        errT = sketch_err([s.get_T()], g["T"])
        errV = sketch_err(s.get_V(), g["V"])
        assert errT <= 1e-12 and errV <= 1e-12, (errT, errV)
        et, _ = s.CV_Compute_shell_spectrum(2)
        per_shell(et[0], g["ek_t"], "theta spectrum")
    finally:
        s.close()


@pytest.mark.parametrize("case", ["fluid256", "mhd256", "rb129"])
def test_fp32_mixed_against_fp64_100_steps(lib, case):
    """The FP32-mixed form (FP32 transforms and products, FP64 RK state, projection and
    reductions) after 100 steps at the workload sizes: every field within 1e-6 (relative L2)
    of the FP64 form."""
    if case == "fluid256":
        N = (256, 256, 256)
        kw = dict(nu=1e-3, dt=5e-4, force=dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0))
        init = dict(V=ic.random_phase_field(N, seed=20261202))
    elif case == "mhd256":
        N = (256, 256, 256)
        kw = dict(physics="MHD", nu=1e-3, eta=1e-3, dt=5e-4)
        init = dict(V=ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261203),
                    W=ic.random_phase_field(N, k0=3.0, energy=0.5, seed=20261204))
    else:
        N = (129, 256, 256)
        kw = dict(basis="SCFT", physics="RB", Ra=1e6, Pr=1.0, dt=1e-4, kfactor=KF_RB)
        T0 = ic.rb_perturbation(N, seed=20261205)
        init = dict(V=[np.zeros_like(T0) for _ in range(3)], T=T0)
    out = {}
    for prec in ("FP64", "FP32"):
        s = solver(N, precision=prec, **kw)
        try:
            s.set_V(init["V"])
            if "W" in init:
                s.set_W(init["W"])
            if "T" in init:
                s.set_T(init["T"])
            s.step(100, energies=False)
            out[prec] = {"V": s.get_V()}
            if "W" in init:
                out[prec]["W"] = s.get_W()
            if "T" in init:
                out[prec]["T"] = [s.get_T()]
        finally:
            s.close()
    for name in out["FP64"]:
        err = rel_l2(out["FP32"][name], out["FP64"][name])
        assert err <= 1e-6, f"{case} {name}: FP32-mixed vs FP64 rel L2 {err:.3e}"
