"""Parity of the CUDA energy-transfer diagnostics with the oracle's restatement of the
reference's sphere/shell loops (compute_flux.cc, compute_shell_tr.cc), per shell:
|gpu - oracle| <= tol |oracle| + 1e-13 max |oracle| for every entry (FP64 form; tol = 1e-10
unless a test states another); the absolute floor covers the entries at round-off level, such as
the empty rows of a shell-to-shell table."""

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu
KF = (1.0, 1.0, 1.0)


def close(a, b, tol, floor=1e-13):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = max(np.abs(b).max(), 1e-300)
    return bool(np.all(np.abs(a - b) <= tol * np.abs(b) + floor * scale))


@pytest.mark.parametrize("N,S", [((32, 32, 32), 8), ((64, 64, 64), 12)])
def test_fluid_flux_and_shell_to_shell(lib, N, S):
    from tarang_b200.solver import IncFluid
    V = ic.random_phase_field(N, seed=31)
    s = IncFluid(N, n_shells=S)
    s.set_V(V)
    assert np.allclose(s.ET_radii(), o.et_radii(N, KF, S), rtol=0, atol=1e-13)
    f = s.Compute_flux()
    fw = o.compute_flux(V, KF, S)
    assert close(f, fw, 1e-10)
    t = s.Compute_shell_tr()
    tw = o.compute_shell_tr(V, KF, S)
    assert close(t, tw, 1e-10)


def test_taylor_green_flux_64(lib):
    """Config 1's diagnostics: TG 64^3 with 12 shells."""
    from tarang_b200.solver import IncFluid
    N = (64, 64, 64)
    V = ic.taylor_green(N)
    s = IncFluid(N, n_shells=12)
    s.set_V(V)
    s.step(3)
    V3 = s.get_V()
    assert close(s.Compute_flux(), o.compute_flux(V3, KF, 12), 1e-10)
    assert close(s.Compute_shell_tr(), o.compute_shell_tr(V3, KF, 12), 1e-10)


@pytest.mark.parametrize("kind,spec", [(L.TG_ET_UU, ("U", "U", "U", -1)), (L.TG_ET_BB, ("U", "B", "B", -1)),
                                       (L.TG_ET_UB, ("B", "U", "B", +1)), (L.TG_ET_BU, ("U", "B", "U", +1))])
def test_mhd_fluxes(lib, kind, spec):
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    U = ic.random_phase_field(N, k0=3.0, seed=20261203)
    B = ic.random_phase_field(N, k0=3.0, seed=20261204)
    s = IncFluid(N, physics="MHD", nu=1e-3, eta=1e-3, dt=5e-4, n_shells=8)
    s.set_V(U)
    s.set_W(B)
    fields = {"U": U, "B": B}
    H, F, R, sign = (fields[spec[0]], fields[spec[1]], fields[spec[2]], spec[3])
    assert close(s.Compute_flux(kind), o.compute_flux_generic(H, F, R, sign, KF, 8), 1e-10)
    if kind != L.TG_ET_BU:
        assert close(s.Compute_shell_tr(kind), o.compute_shell_tr_generic(H, F, R, sign, KF, 8), 1e-10)


@pytest.mark.parametrize("N,S", [((32, 32, 32), 12), ((64, 64, 64), 16)])
def test_force_feed_shell(lib, N, S):
    """forceV_shell of Output_flux: 2 mult Re(F . V*) per energy-transfer shell, with the
    constant-energy-supply force of the current field; zero without forcing."""
    from tarang_b200.solver import IncFluid
    V = ic.random_phase_field(N, seed=41)
    force = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    s = IncFluid(N, nu=1e-3, dt=5e-4, force=force, n_shells=S)
    s.set_V(V)
    s.Compute_force()
    got = s.Compute_force_feed_shell()
    F = o.force_const_energy_supply(V, N, KF, 2.0, 3.0, 0.1, 0.0)
    want = o.force_feed_shell(F, V, KF, S)
    assert close(got, want, 1e-12)
    assert np.count_nonzero(want) >= 1
    d = IncFluid(N, nu=1e-3, dt=5e-4, n_shells=S)
    d.set_V(V)
    assert np.all(d.Compute_force_feed_shell() == 0)


def test_tables_are_deterministic(lib):
    """The flux and shell-to-shell tables and the shell spectrum are the same bits on a second
    call and on a second context (their shell sums run in a fixed order)."""
    from tarang_b200.solver import IncFluid
    N, S = (32, 32, 32), 10
    V = ic.random_phase_field(N, seed=7)
    out = []
    for _ in range(2):
        s = IncFluid(N, nu=1e-3, dt=1e-3, n_shells=S)
        s.set_V(V)
        out.append((s.Compute_flux(), s.Compute_shell_tr(), s.Compute_flux(), s.CV_Compute_shell_spectrum()))
        s.close()
    (f0, t0, f1, e0), (g0, u0, _, e1) = out
    assert np.array_equal(f0, f1) and np.array_equal(f0, g0) and np.array_equal(t0, u0)
    # and the shell spectrum (energy, dissipation) likewise
    for a, b in zip(e0, e1):
        assert np.array_equal(a, b)
