"""Parity of the CUDA fluid time-step path with the oracle (FOUR basis, FP64 form):
nonlinear term, pressure, forcing, Get_dt, energies and spectra, and 10-step trajectories of
the Taylor-Green and forced random-phase configurations (relative L2 error <= 1e-12)."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

KF = (1.0, 1.0, 1.0)


def rel_l2(a, b):
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def make(N, **kw):
    from tarang_b200.solver import IncFluid
    return IncFluid(N, **kw)


@pytest.mark.parametrize("N", [(16, 16, 16), (32, 32, 32), (64, 64, 64), (32, 16, 64), (64, 32, 128),
                               (32, 32, 256), (16, 16, 512), (128, 128, 128)])
def test_nlin_and_pressure(lib, N):
    V = ic.random_phase_field(N, seed=21)
    s = make(N, nu=0.01, dt=1e-3)
    s.set_V(V)
    s.Compute_nlin()
    got = s.get_nlin()
    want = o.nlin_fluid(V, KF)
    assert rel_l2(got, want) < 1e-13
    s.Compute_pressure()
    p = s.get_pressure()
    pw = o.pressure(want, KF)
    assert np.abs(p - pw).max() < 1e-13 * np.abs(pw).max()


def test_taylor_green_nlin(lib):
    N = (64, 64, 64)
    V = ic.taylor_green(N)
    s = make(N)
    s.set_V(V)
    s.Compute_nlin()
    assert rel_l2(s.get_nlin(), o.nlin_fluid(V, KF)) < 1e-13


def test_energy_dissipation_spectrum(lib):
    N = (64, 64, 64)
    V = ic.random_phase_field(N, seed=4)
    s = make(N)
    s.set_V(V)
    E, D = s.CV_Compute_totalenergy_diss()
    Ew = sum(o.total_energy_four(v) for v in V)
    Dw = 2 * sum(o.total_Sn(v, 2, KF) for v in V)
    assert abs(E - Ew) < 1e-13 * Ew and abs(D - Dw) < 1e-13 * Dw
    ek, dk = s.CV_Compute_shell_spectrum()
    for i in range(3):
        w = o.shell_spectrum(V[i], 0, KF)
        assert np.abs(ek[i] - w).max() < 1e-12 * np.abs(w).max()
    dw = 2 * sum(o.shell_spectrum(v, 2, KF) for v in V)
    assert np.abs(dk - dw).max() < 1e-12 * np.abs(dw).max()


def test_spectrum_partial_shells(lib):
    """Energy out to the corners of the dealiased cube: the shells beyond kmax_inside are
    rescaled by Approx_number_modes_in_shell / count, with counts over the whole grid."""
    N = (64, 64, 64)
    V = ic.random_phase_field(N, k0=40.0, seed=14)
    s = make(N)
    s.set_V(V)
    ek, dk = s.CV_Compute_shell_spectrum()
    for i in range(3):
        w = o.shell_spectrum(V[i], 0, KF)
        assert np.abs(ek[i] - w).max() < 1e-12 * np.abs(w).max()
        assert w[25] > 1e-3 * np.abs(w).max()   # the partial shells carry energy here


def test_get_dt(lib):
    N = (64, 64, 64)
    V = ic.random_phase_field(N, seed=5, energy=50.0)   # large energy: the CFL bound is active
    s = make(N, dt=1.0)
    s.set_V(V)
    E = sum(o.total_energy_four(v) for v in V)
    assert abs(s.Get_dt() - o.get_dt(E, N, KF, 1.0)) < 1e-15


def test_forcing_field(lib):
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=6)
    force = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    s = make(N, force=force)
    s.set_V(V)
    s.Compute_force()
    got = s.get_force()
    want = o.force_const_energy_supply(V, N, KF, 2.0, 3.0, 0.1, 0.0)
    assert rel_l2(got, want) < 1e-12


def test_taylor_green_10_steps(lib):
    N = (64, 64, 64)
    V = ic.taylor_green(N)
    s = make(N, nu=0.01, dt=1e-3)
    s.set_V(V)
    E = s.step(10)
    ref = o.FluidSolver(N, KF, 0.01, 1e-3)
    Vw = V
    Ew = []
    for _ in range(10):
        Vw, dt = ref.step(Vw)
        assert dt == 1e-3
        Ew.append(sum(o.total_energy_four(v) for v in Vw))
    assert rel_l2(s.get_V(), Vw) < 1e-12
    assert np.abs(np.array(E) - np.array(Ew)).max() < 1e-13
    t, n = s.time()
    assert n == 10 and abs(t - 10e-3) < 1e-15


@pytest.mark.parametrize("precision,tol", [("FP64", 1e-12), ("FP32", 1e-6)])
def test_forced_random_phase_10_steps(lib, precision, tol):
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=20261202)
    force = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    s = make(N, nu=1e-3, dt=5e-4, force=force, precision=precision)
    s.set_V(V)
    s.step(10)
    ref = o.FluidSolver(N, KF, 1e-3, 5e-4, force=force)
    Vw = V
    for _ in range(10):
        Vw, _ = ref.step(Vw)
    assert rel_l2(s.get_V(), Vw) < tol


def test_fine_grained_calls_match_fused_step(lib):
    """The loop body of Ifluid_main.cc:261-278 called method by method equals tg_step."""
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=9)
    force = dict(inner=2.0, outer=3.0, eps=0.1)
    a = make(N, nu=1e-3, dt=5e-4, force=force)
    b = make(N, nu=1e-3, dt=5e-4, force=force)
    a.set_V(V)
    b.set_V(V)
    for _ in range(3):
        a.Compute_force()
        a.Compute_nlin()
        a.Add_force()
        a.Compute_pressure()
        a.Get_dt()
        a.Time_advance()
    b.step(3)
    assert rel_l2(a.get_V(), b.get_V()) < 1e-14


def test_graph_replay_is_deterministic(lib):
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=10)
    outs = []
    for _ in range(2):
        s = make(N, nu=1e-3, dt=5e-4)
        s.set_V(V)
        s.step(5)
        outs.append(s.get_V())
    for x, y in zip(*outs):
        assert np.array_equal(x, y)
