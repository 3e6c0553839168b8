"""Parity of the fixed-mode forcings (Taylor-Green, ABC, given modes: force_field_proc 3, 4, 5)
and the Coriolis force (proc 21) on the CUDA path with the oracle: 10-step trajectories of fluid
(FOUR and SCFT) and MHD runs (relative L2 error <= 1e-12 in FP64, 1e-6 in FP32-mixed), the
method-by-method calls and the force fields they leave, the force feed, batched Coriolis
requests, and the errors of tg_set_force_modes."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import forcing, ic

pytestmark = pytest.mark.gpu

KF = (1.0, 1.0, 1.0)


def rel_l2(a, b):
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def make(N, **kw):
    from tarang_b200.solver import IncFluid
    return IncFluid(N, **kw)


def dense_cols(k, F, N, basis="FOUR"):
    N1, N2, N3 = N
    out = []
    for c in range(F.shape[1]):
        A = np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128)
        for (kx, ky, kz), f in zip(k, F[:, c]):
            A[kx if (basis == "SCFT" or kx >= 0) else kx + N1, ky % N2, kz] = f
        out.append(A)
    return out


@pytest.mark.parametrize("basis,precision,tol", [("FOUR", "FP64", 1e-12), ("SCFT", "FP64", 1e-12),
                                                 ("FOUR", "FP32", 1e-6)])
def test_taylor_green_forced_10_steps(lib, basis, precision, tol):
    N = (32, 32, 32)
    if basis == "FOUR":
        V = ic.random_phase_field(N, seed=31)
    else:
        # SCFT velocity: V1 a sine series in x, V2 and V3 cosine series (dealiased)
        rng = np.random.default_rng(31)
        V = [0.3 * o.dealias(o.forward_scft(rng.standard_normal(N), p), "SCFT") for p in (1, 0, 0)]
    k, F = forcing.taylor_green_modes(N, 2, 0.8, basis)
    s = make(N, basis=basis, nu=5e-3, dt=5e-4, force=dict(kind="modes"), precision=precision)
    s.set_force_modes(k, F)
    s.set_V(V)
    s.step(10)
    ref = o.FluidSolver(N, KF, 5e-3, 5e-4, basis=basis, force=dict(kind="static", F=o.taylor_green_force(N, 2, 0.8, basis)))
    Vw = V
    for _ in range(10):
        Vw, _ = ref.step(Vw)
    assert rel_l2(s.get_V(), Vw) < tol


def test_abc_forced_mhd_10_steps(lib):
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=32)
    W = ic.random_phase_field(N, seed=33, energy=0.2)
    k, F = forcing.abc_modes(N, 1, 0.5, 1.0, 0.7, 0.3, physics="MHD", ampW=0.25)
    s = make(N, physics="MHD", nu=4e-3, eta=6e-3, dt=5e-4, force=dict(kind="modes"))
    s.set_force_modes(k, F)
    s.set_V(V)
    s.set_W(W)
    s.step(10)
    ref = o.MHDSolver(N, KF, 4e-3, 6e-3, 5e-4, force=dict(kind="static", F=dense_cols(k, F, N)))
    Vw, Ww = V, W
    for _ in range(10):
        Vw, Ww, _ = ref.step2(Vw, Ww)
    assert rel_l2(s.get_V(), Vw) < 1e-12
    assert rel_l2(s.get_W(), Ww) < 1e-12


def test_given_modes_fine_grained_calls(lib):
    """Compute_force / Compute_nlin / Add_force with given modes: nlin = N(u) - F, the force
    field downloads as set, and the method-by-method loop equals the fused step."""
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=34)
    k, F = forcing.given_modes([(1, 2, 3, 0.3 + 0.1j, -0.2 + 0.4j), (2, 1, 0, 0.5 + 0.2j, 0.1 - 0.3j)], N)
    Fd = dense_cols(k, F, N)
    a = make(N, nu=2e-3, dt=5e-4, force=dict(kind="modes"))
    b = make(N, nu=2e-3, dt=5e-4, force=dict(kind="modes"))
    for s in (a, b):
        s.set_force_modes(k, F)
        s.set_V(V)
    a.Compute_force()
    f = a.get_force()
    assert all(np.array_equal(x, y) for x, y in zip(f, Fd))
    a.Compute_nlin()
    a.Add_force()
    nl = a.get_nlin()
    want = [x - y for x, y in zip(o.nlin_fluid(V, KF), Fd)]
    assert rel_l2(nl, want) < 1e-13
    a.Compute_pressure()
    a.Get_dt()
    a.Time_advance()
    for _ in range(2):
        a.Compute_force()
        a.Compute_nlin()
        a.Add_force()
        a.Compute_pressure()
        a.Get_dt()
        a.Time_advance()
    b.step(3)
    assert rel_l2(a.get_V(), b.get_V()) < 1e-14


def test_force_modes_reset_between_graph_steps(lib):
    """A new mode set after graph-replayed steps is used by the following steps (the captured
    step is rebuilt), and n = 0 clears the force."""
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=35)
    k1, F1 = forcing.taylor_green_modes(N, 1, 0.5)
    k2, F2 = forcing.abc_modes(N, 2, 0.5, 1.0, 1.0, 1.0)
    s = make(N, nu=5e-3, dt=5e-4, force=dict(kind="modes"))
    s.set_force_modes(k1, F1)
    s.set_V(V)
    s.step(4)
    s.set_force_modes(k2, F2)
    s.step(4)
    s.set_force_modes(np.zeros((0, 3)), np.zeros((0, 3)))
    s.step(2)
    r1 = o.FluidSolver(N, KF, 5e-3, 5e-4, force=dict(kind="static", F=dense_cols(k1, F1, N)))
    r2 = o.FluidSolver(N, KF, 5e-3, 5e-4, force=dict(kind="static", F=dense_cols(k2, F2, N)))
    r3 = o.FluidSolver(N, KF, 5e-3, 5e-4)
    Vw = V
    for r, n in ((r1, 4), (r2, 4), (r3, 2)):
        for _ in range(n):
            Vw, _ = r.step(Vw)
    assert rel_l2(s.get_V(), Vw) < 1e-12


def test_force_feed_of_fixed_modes(lib):
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=36)
    k, F = forcing.taylor_green_modes(N, 2, 0.8)
    s = make(N, nu=5e-3, dt=5e-4, force=dict(kind="modes"), n_shells=12)
    s.set_force_modes(k, F)
    s.set_V(V)
    got = s.Compute_force_feed_shell()
    want = o.force_feed_shell(dense_cols(k, F, N), V, KF, 12)
    assert np.abs(np.asarray(got) - np.asarray(want)).max() <= 1e-14 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("physics", ["FLUID", "MHD"])
def test_coriolis_10_steps(lib, physics):
    N = (32, 32, 32)
    om = (0.3, -0.5, 2.0)
    V = ic.random_phase_field(N, seed=37)
    kw = dict(nu=4e-3, dt=5e-4, force=dict(kind="coriolis", omega=om))
    if physics == "FLUID":
        s = make(N, **kw)
        s.set_V(V)
        s.step(10)
        ref = o.FluidSolver(N, KF, 4e-3, 5e-4, force=dict(kind="coriolis", omega=om))
        Vw = V
        for _ in range(10):
            Vw, _ = ref.step(Vw)
        assert rel_l2(s.get_V(), Vw) < 1e-12
    else:
        W = ic.random_phase_field(N, seed=38, energy=0.2)
        s = make(N, physics="MHD", eta=6e-3, **kw)
        s.set_V(V)
        s.set_W(W)
        s.step(10)
        ref = o.MHDSolver(N, KF, 4e-3, 6e-3, 5e-4, force=dict(kind="coriolis", omega=om))
        Vw, Ww = V, W
        for _ in range(10):
            Vw, Ww, _ = ref.step2(Vw, Ww)
        assert rel_l2(s.get_V(), Vw) < 1e-12
        assert rel_l2(s.get_W(), Ww) < 1e-12


def test_coriolis_fine_grained_and_force_field(lib):
    N = (32, 32, 32)
    om = (0.0, 0.0, 3.0)
    V = ic.random_phase_field(N, seed=39)
    s = make(N, nu=4e-3, dt=5e-4, force=dict(kind="coriolis", omega=om))
    s.set_V(V)
    s.Compute_force()
    f = s.get_force()
    want = o.force_coriolis(V, om)
    assert rel_l2(f, want) < 1e-15
    s.Compute_nlin()
    s.Add_force()
    want_nl = [x - y for x, y in zip(o.nlin_fluid(V, KF), want)]
    assert rel_l2(s.get_nlin(), want_nl) < 1e-13
    # Re(F . V*) = 0: a rotating frame feeds no energy
    assert np.abs(s.Compute_force_feed_shell()).max() == 0.0


def test_coriolis_requests_batch_alone_equals_mixed(lib):
    """Coriolis requests with the same Omega share a batch; each result equals a lone context's
    run bit for bit."""
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    om = (0.0, 1.0, 2.0)
    Vs = [ic.random_phase_field(N, seed=40 + i) for i in range(3)]
    cfgs = [dict(N=N, nu=3e-3 * (1 + i), dt=5e-4, force=dict(kind="coriolis", omega=om)) for i in range(3)]
    with Server(hbm_budget=8e9, max_batch=4) as srv:
        ids = [srv.submit(c, V, 6) for c, V in zip(cfgs, Vs)]
        srv.drain()
        for i, (rid, V) in enumerate(zip(ids, Vs)):
            got = srv.result(rid)
            s = make(N, nu=3e-3 * (1 + i), dt=5e-4, force=dict(kind="coriolis", omega=om))
            s.set_V(V)
            s.step(6)
            assert all(np.array_equal(x.view(np.float64), y.view(np.float64)) for x, y in zip(got, s.get_V()))
        assert srv.stats()["n_batches"] >= 1
        # a request carries no force modes
        with pytest.raises(L.TarangError) as e:
            srv.submit(dict(N=N, nu=1e-3, dt=5e-4, force=dict(kind="modes")), Vs[0], 2)
        assert e.value.code == L.TG_ERR_UNSUPPORTED


def test_set_force_modes_errors(lib):
    N = (32, 32, 32)
    s = make(N, nu=1e-3, dt=5e-4, force=dict(kind="modes"))
    k, F = forcing.taylor_green_modes(N, 11, 1.0)        # |k| = 11 > N/3: not stored
    with pytest.raises(L.TarangError) as e:
        s.set_force_modes(k, F)
    assert e.value.code == L.TG_ERR_ARG
    with pytest.raises(L.TarangError):
        s.set_force_modes([(1, 1, -1)], np.zeros((1, 3)))
    with pytest.raises(L.TarangError):
        s.set_force_modes([(1, 1, 1)], np.full((1, 3), np.nan))
    with pytest.raises(ValueError):
        s.set_force_modes([(1, 1, 1)], np.zeros((1, 6)))
    d = make(N, nu=1e-3, dt=5e-4)
    with pytest.raises(L.TarangError) as e:
        d.set_force_modes(*forcing.taylor_green_modes(N, 1, 1.0))
    assert e.value.code == L.TG_ERR_STATE
    with pytest.raises(L.TarangError) as e:
        make(N, physics="RB", basis="SCFT", Ra=1e4, Pr=1.0, dt=1e-4, force=dict(kind="coriolis", omega=(0, 0, 1)))
    assert e.value.code == L.TG_ERR_UNSUPPORTED


BAND = [
    ("FLUID", "energy_helicity", dict(eps=0.1, eps_h=0.3), "FP64", 1e-12),
    ("FLUID", "energy_helicity", dict(eps=0.1, eps_h=0.3), "FP32", 1e-6),
    ("MHD", "energy_supply", dict(eps=0.1, eps_h=0.2, eps_W=0.05, eps_hW=-0.4), "FP64", 1e-12),
    ("MHD", "energy_helicity", dict(eps=0.1, eps_h=0.0, eps_W=0.05, eps_hW=0.5), "FP64", 1e-12),
    ("SCALAR", "energy_supply", dict(eps=0.1, eps_h=0.0, eps_T=0.02), "FP64", 1e-12),
    ("SCALAR", "energy_helicity", dict(eps=0.1, eps_h=0.1, eps_T=0.02), "FP64", 1e-12),
]


@pytest.mark.parametrize("physics,kind,par,precision,tol", BAND)
def test_band_forcing_10_steps(lib, physics, kind, par, precision, tol):
    """force_field_proc 1 (energy-helicity supply) and 2 (constant energy and helicity) on the
    velocity, and on B (MHD) or the passive scalar with their own parameters: 10 steps against
    the oracle's loops (MHDSolver, ScalarSolver)."""
    N = (32, 32, 32)
    force = dict(kind=kind, inner=2.0, outer=3.0, **par)
    U = ic.random_phase_field(N, seed=51)
    s = make(N, physics=physics, nu=2e-3, eta=3e-3, kappa=4e-3, dt=5e-4, force=force, precision=precision)
    s.set_V(U)
    if physics == "FLUID":
        s.step(10)
        ref = o.FluidSolver(N, KF, 2e-3, 5e-4, force=force)
        Uw = U
        for _ in range(10):
            Uw, _ = ref.step(Uw)
        assert rel_l2(s.get_V(), Uw) < tol
    elif physics == "MHD":
        W = ic.random_phase_field(N, seed=52, energy=0.3)
        s.set_W(W)
        s.step(10)
        ref = o.MHDSolver(N, KF, 2e-3, 3e-3, 5e-4, force=force)
        Uw, Ww = U, W
        for _ in range(10):
            Uw, Ww, _ = ref.step2(Uw, Ww)
        assert rel_l2(s.get_V(), Uw) < tol
        assert rel_l2(s.get_W(), Ww) < tol
        # the magnetic force is on: without it B differs
        ref0 = o.MHDSolver(N, KF, 2e-3, 3e-3, 5e-4, force=dict(force, eps_W=0.0))
        U0, W0 = U, W
        for _ in range(10):
            U0, W0, _ = ref0.step2(U0, W0)
        assert rel_l2(W0, Ww) > 1e-6
    else:
        T = ic.random_phase_field(N, k0=2.0, seed=53)[0]
        s.set_T(T)
        s.step(10)
        ref = o.ScalarSolver(N, KF, 2e-3, 4e-3, 5e-4, force=force)
        Uw, Tw = U, T
        for _ in range(10):
            Uw, Tw, _ = ref.step(Uw, Tw)
        assert rel_l2(s.get_V(), Uw) < tol
        assert rel_l2([s.get_T()], [Tw]) < tol
        ref0 = o.ScalarSolver(N, KF, 2e-3, 4e-3, 5e-4, force=dict(force, eps_T=0.0))
        U0, T0 = U, T
        for _ in range(10):
            U0, T0, _ = ref0.step(U0, T0)
        assert rel_l2([T0], [Tw]) > 1e-6


@pytest.mark.parametrize("precision,tol", [("FP64", 1e-12), ("FP32", 1e-6)])
def test_passive_scalar_decay_10_steps(lib, precision, tol):
    """The passive-scalar loop (Iscalar_main.cc:272-300) without forcing: u and T after 10 steps,
    and the scalar's energy and dissipation."""
    N = (32, 32, 64)
    U = ic.random_phase_field(N, seed=54)
    T = ic.random_phase_field(N, k0=3.0, seed=55)[0]
    s = make(N, physics="SCALAR", nu=2e-3, kappa=5e-3, dt=5e-4, precision=precision)
    s.set_V(U)
    s.set_T(T)
    s.step(10)
    ref = o.ScalarSolver(N, KF, 2e-3, 5e-3, 5e-4)
    Uw, Tw = U, T
    for _ in range(10):
        Uw, Tw, _ = ref.step(Uw, Tw)
    assert rel_l2(s.get_V(), Uw) < tol
    assert rel_l2([s.get_T()], [Tw]) < tol


@pytest.mark.parametrize("precision,tol", [("FP64", 1e-12), ("FP32", 1e-6)])
def test_liquid_metal_10_steps(lib, precision, tol):
    """force_field_proc 101 for a fluid (Compute_force_Liquid_metal): Force = -(B0 . K)^2/K^2 V
    from each RK stage's velocity; 10 steps against the oracle, and the damping it adds."""
    N = (32, 32, 32)
    B0 = (0.0, 0.5, 2.0)
    V = ic.random_phase_field(N, seed=61)
    s = make(N, nu=4e-3, dt=5e-4, force=dict(kind="liquid_metal", B0=B0), precision=precision)
    s.set_V(V)
    s.step(10)
    ref = o.FluidSolver(N, KF, 4e-3, 5e-4, force=dict(kind="liquid_metal", B0=B0))
    Vw = V
    for _ in range(10):
        Vw, _ = ref.step(Vw)
    assert rel_l2(s.get_V(), Vw) < tol
    free = o.FluidSolver(N, KF, 4e-3, 5e-4)
    Vf = V
    for _ in range(10):
        Vf, _ = free.step(Vf)
    assert sum(o.total_energy(v) for v in Vw) < sum(o.total_energy(v) for v in Vf)


def test_liquid_metal_fine_grained_and_force_field(lib):
    N = (32, 32, 32)
    B0 = (1.0, 0.0, 0.5)
    V = ic.random_phase_field(N, seed=62)
    s = make(N, nu=4e-3, dt=5e-4, force=dict(kind="liquid_metal", B0=B0))
    s.set_V(V)
    s.Compute_force()
    want = o.force_liquid_metal(V, KF, B0)
    assert rel_l2(s.get_force(), want) < 1e-15
    s.Compute_nlin()
    s.Add_force()
    want_nl = [x - y for x, y in zip(o.nlin_fluid(V, KF), want)]
    assert rel_l2(s.get_nlin(), want_nl) < 1e-13


def test_force_feed_of_every_field(lib):
    """Compute_force_feed_shell for B (MHD, W.forceV_shell) and the passive scalar (forceSF_shell)
    under the band forcing, and the velocity's feed under the liquid-metal force, against the
    oracle's shell sums of 2 mult Re(F . X*)."""
    N, S = (32, 32, 32), 10
    force = dict(kind="energy_supply", inner=2.0, outer=3.0, eps=0.1, eps_h=0.0, eps_W=0.05, eps_hW=0.3)
    U = ic.random_phase_field(N, seed=71)
    W = ic.random_phase_field(N, seed=72, energy=0.3)
    s = make(N, physics="MHD", nu=2e-3, eta=3e-3, dt=5e-4, force=force, n_shells=S)
    s.set_V(U)
    s.set_W(W)
    s.Compute_force()
    FW = o.force_band(W, N, KF, 2.0, 3.0, 0.05, 0.3, mode=1, gate=True)
    want = o.force_feed_shell(FW, W, KF, S)
    assert np.count_nonzero(want) >= 1
    assert np.abs(s.Compute_force_feed_shell(1) - want).max() <= 1e-12 * np.abs(want).max()
    FU = o.force_band(U, N, KF, 2.0, 3.0, 0.1, 0.0, mode=1, gate=True)
    want = o.force_feed_shell(FU, U, KF, S)
    assert np.abs(s.Compute_force_feed_shell(0) - want).max() <= 1e-12 * np.abs(want).max()
    T = ic.random_phase_field(N, k0=2.0, seed=73)[0]
    fs = dict(kind="energy_helicity", inner=2.0, outer=3.0, eps=0.1, eps_T=0.02)
    c = make(N, physics="SCALAR", nu=2e-3, kappa=4e-3, dt=5e-4, force=fs, n_shells=S)
    c.set_V(U)
    c.set_T(T)
    c.Compute_force()
    FT = o.force_band_scalar(T, N, KF, 2.0, 3.0, 0.02, mode=2)
    want = o.force_feed_shell([FT], [T], KF, S)
    assert np.abs(c.Compute_force_feed_shell(2) - want).max() <= 1e-12 * np.abs(want).max()
    B0 = (0.0, 0.5, 2.0)
    m = make(N, nu=2e-3, dt=5e-4, force=dict(kind="liquid_metal", B0=B0), n_shells=S)
    m.set_V(U)
    m.Compute_force()
    want = o.force_feed_shell(o.force_liquid_metal(U, KF, B0), U, KF, S)
    assert np.all(want[1:] <= 0) and want.min() < 0
    assert np.abs(m.Compute_force_feed_shell() - want).max() <= 1e-12 * np.abs(want).max()


def test_ring_force_feed(lib):
    """Compute_force_feed_ring / Compute_force_feed_cylinder_ring: the force feed of U, B and a
    passive scalar binned by receiver ring and cylinder ring, and the liquid-metal feed, against
    the oracle's Ring_mult_all / Cyl_ring_mult_all restatement."""
    N = (32, 32, 32)
    U = ic.random_phase_field(N, seed=81)
    W = ic.random_phase_field(N, seed=82, energy=0.3)
    force = dict(kind="energy_helicity", inner=1.0, outer=3.0, eps=0.1, eps_h=0.2, eps_W=0.05, eps_hW=-0.3)
    s = make(N, physics="MHD", nu=2e-3, eta=3e-3, dt=5e-4, force=force)
    s.set_V(U)
    s.set_W(W)
    s.Compute_force()
    FU = o.force_band(U, N, KF, 1.0, 3.0, 0.1, 0.2, mode=2, gate=True)
    FW = o.force_band(W, N, KF, 1.0, 3.0, 0.05, -0.3, mode=2, gate=True)
    for group, F, X in ((0, FU, U), (1, FW, W)):
        for cyl, axis, n, ns in ((False, 3, 6, 3), (True, 1, 5, 4)):
            got = s.Compute_force_feed_ring(n, ns, axis, group, cyl)
            want = o.ring_mult_all(F, X, KF, axis, n, ns, cylinder=cyl)
            assert np.count_nonzero(want) >= 1
            assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), (group, cyl)
    T = ic.random_phase_field(N, k0=2.0, seed=83)[0]
    c = make(N, physics="SCALAR", nu=2e-3, kappa=4e-3, dt=5e-4,
             force=dict(kind="energy_supply", inner=1.0, outer=3.0, eps=0.1, eps_T=0.02))
    c.set_V(U)
    c.set_T(T)
    c.Compute_force()
    FT = o.force_band_scalar(T, N, KF, 1.0, 3.0, 0.02, mode=1)
    got = c.Compute_force_feed_ring(6, 2, 2, 2)
    want = o.ring_mult_all([FT], [T], KF, 2, 6, 2)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    B0 = (0.3, 0.0, 1.0)
    m = make(N, nu=2e-3, dt=5e-4, force=dict(kind="liquid_metal", B0=B0))
    m.set_V(U)
    got = m.Compute_force_feed_ring(6, 3, 3, 0, True)
    want = o.ring_mult_all(o.force_liquid_metal(U, KF, B0), U, KF, 3, 6, 3, cylinder=True)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
