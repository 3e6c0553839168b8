"""The band forcings (force_field_proc 1, constant energy supply, and 2, constant energy and
helicity) in the SCFT basis: the basis_type == "SCFT" branches of
Compute_force_const_energy_helicity_supply and Compute_force_const_energy_helicity
(compute_force_ek_hk_supply.cc:51-289, compute_force_const_ek_hk.cc:53-293): modes with kx >= 0,
the SCFT modal energy, helicity and vorticity of (-i V1, V2, V3), Force_alpha_beta's SCFT form
(force_alpha_beta.cc:90-110), the SCFT mode count and reality condition.  The CUDA path against
the oracle: the force fields, 10-step trajectories of a forced fluid and a forced passive scalar
(relative L2 <= 1e-12), and the force feed per shell."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o

pytestmark = pytest.mark.gpu

KF = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
N = (24, 16, 32)


def rel_l2(a, b):
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def scft_state(seed, amp=1.0):
    """Dealiased SCFT fields: u1 (sine), u2, u3 (cosine) made divergence-free, theta (sine)."""
    rng = np.random.default_rng(seed)
    out = [amp * o.dealias(o.forward_scft(rng.standard_normal(N), p), "SCFT") for p in (1, 0, 0, 1)]
    V = out[:3]
    p = o.pressure(V, KF, "SCFT")
    V = [V[0] + o.xderiv(p, KF, "SCFT", 0), V[1] + o.yderiv(p, KF), V[2] + o.zderiv(p, KF)]
    return V, out[3]


def solver(**kw):
    from tarang_b200.solver import IncFluid
    return IncFluid(N, basis="SCFT", kfactor=KF, **kw)


@pytest.mark.parametrize("kind,eps_h", [("energy_supply", 0.0), ("energy_supply", 0.3), ("energy_helicity", 0.2)])
def test_scft_band_force_field(lib, kind, eps_h):
    V, _ = scft_state(1)
    force = dict(kind=kind, inner=2.0, outer=6.0, eps=0.1, eps_h=eps_h)
    s = solver(nu=2e-3, dt=5e-4, force=force)
    try:
        s.set_V(V)
        s.Compute_force()
        got = s.get_force()
    finally:
        s.close()
    mode = 1 if kind == "energy_supply" else 2
    want = o.force_band(V, N, KF, 2.0, 6.0, 0.1, eps_h, mode=mode, gate=(mode == 2), basis="SCFT")
    assert sum(np.count_nonzero(w) for w in want) > 10
    assert rel_l2(got, want) <= 1e-12


def test_scft_forced_fluid_10_steps(lib):
    V, _ = scft_state(2)
    force = dict(kind="energy_supply", inner=2.0, outer=6.0, eps=0.1, eps_h=0.25)
    s = solver(nu=2e-3, dt=5e-4, force=force)
    try:
        s.set_V(V)
        s.step(10)
        got = s.get_V()
    finally:
        s.close()
    ref = o.FluidSolver(N, KF, 2e-3, 5e-4, basis="SCFT", force=force)
    W = V
    for _ in range(10):
        W, dt = ref.step(W)
        assert dt == 5e-4
    assert rel_l2(got, W) <= 1e-12
    # the force changed the trajectory
    free = o.FluidSolver(N, KF, 2e-3, 5e-4, basis="SCFT")
    X = V
    for _ in range(10):
        X, _ = free.step(X)
    assert rel_l2(X, W) > 1e-6


def test_scft_forced_passive_scalar_10_steps(lib):
    V, T = scft_state(3)
    force = dict(kind="energy_helicity", inner=2.0, outer=6.0, eps=0.1, eps_h=0.1, eps_T=0.05)
    s = solver(physics="SCALAR", nu=2e-3, kappa=3e-3, dt=5e-4, force=force)
    try:
        s.set_V(V)
        s.set_T(T)
        s.step(10)
        gv, gt = s.get_V(), s.get_T()
    finally:
        s.close()
    ref = o.ScalarSolver(N, KF, 2e-3, 3e-3, 5e-4, basis="SCFT", force=force)
    v, t = V, T
    for _ in range(10):
        v, t, _ = ref.step(v, t)
    assert rel_l2(gv, v) <= 1e-12
    assert rel_l2([gt], [t]) <= 1e-12


def test_scft_band_force_feed(lib):
    V, T = scft_state(4)
    S = 8
    force = dict(kind="energy_supply", inner=2.0, outer=6.0, eps=0.1, eps_h=0.0, eps_T=0.05)
    s = solver(physics="SCALAR", nu=2e-3, kappa=3e-3, dt=5e-4, force=force, n_shells=S)
    try:
        s.set_V(V)
        s.set_T(T)
        s.Compute_force()
        fu, ft = s.Compute_force_feed_shell(0), s.Compute_force_feed_shell(2)
    finally:
        s.close()
    FU = o.force_band(V, N, KF, 2.0, 6.0, 0.1, 0.0, mode=1, gate=True, basis="SCFT")
    FT = o.force_band_scalar(T, N, KF, 2.0, 6.0, 0.05, mode=1, basis="SCFT")
    wu = o.force_feed_shell(FU, V, KF, S, basis="SCFT")
    wt = o.force_feed_shell([FT], [T], KF, S, basis="SCFT")
    assert np.count_nonzero(wu) >= 1 and np.count_nonzero(wt) >= 1
    assert np.abs(fu - wu).max() <= 1e-12 * np.abs(wu).max()
    assert np.abs(ft - wt).max() <= 1e-12 * np.abs(wt).max()
