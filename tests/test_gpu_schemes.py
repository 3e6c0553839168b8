"""The integration schemes of IncFluid::Time_advance (time_advance.cc:60-163) other than RK4 --
integrating-factor EULER and RK2 -- and the hyper-dissipation / hyper-diffusion term
(exp(-(nu + nu_h K^2) K^2 dt), mult_exp_visc.cc:56-165), for fluid, MHD, passive scalar and SCFT
convection: 10 steps against the oracle at <= 1e-12 relative L2 (FP64), the FP32-mixed form
against FP64 at <= 1e-6; the method-by-method loop equals tg_step; a served request equals its
lone run bit for bit."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic

pytestmark = pytest.mark.gpu
KF = (1.0, 1.0, 1.0)
KF_RB = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))


def rel_l2(a, b):
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def make(N, **kw):
    from tarang_b200.solver import IncFluid
    return IncFluid(N, **kw)


# a hyper coefficient that damps the largest kept wavenumbers noticeably in 10 steps
HYPER = 2e-6


@pytest.mark.parametrize("scheme,nu_h", [("EULER", 0.0), ("RK2", 0.0), ("RK4", HYPER), ("EULER", HYPER),
                                         ("RK2", HYPER)])
def test_fluid_10_steps(lib, scheme, nu_h):
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=71)
    force = dict(inner=2.0, outer=3.0, eps=0.1)
    s = make(N, nu=1e-3, dt=5e-4, force=force, scheme=scheme, hyper_nu=nu_h)
    s.set_V(V)
    s.step(10)
    ref = o.FluidSolver(N, KF, 1e-3, 5e-4, force=force, scheme=scheme, nu_h=nu_h)
    W = V
    for _ in range(10):
        W, _ = ref.step(W)
    assert rel_l2(s.get_V(), W) < 1e-12
    if nu_h:
        # the hyper term acts: without it the fields differ by far more than the tolerance
        ref0 = o.FluidSolver(N, KF, 1e-3, 5e-4, force=force, scheme=scheme)
        W0 = V
        for _ in range(10):
            W0, _ = ref0.step(W0)
        assert rel_l2(W0, W) > 1e-6


@pytest.mark.parametrize("scheme", ["EULER", "RK2"])
def test_mhd_10_steps(lib, scheme):
    N = (16, 16, 16)
    U = ic.random_phase_field(N, k0=3.0, seed=72)
    B = ic.random_phase_field(N, k0=3.0, seed=73)
    s = make(N, physics="MHD", nu=1e-3, eta=2e-3, dt=5e-4, scheme=scheme, hyper_nu=HYPER, hyper_eta=3e-6)
    s.set_V(U)
    s.set_W(B)
    s.step(10)
    ref = o.MHDSolver(N, KF, 1e-3, 2e-3, 5e-4, scheme=scheme, nu_h=HYPER, eta_h=3e-6)
    u, b = U, B
    for _ in range(10):
        u, b, _ = ref.step2(u, b)
    assert rel_l2(s.get_V() + s.get_W(), u + b) < 1e-12


@pytest.mark.parametrize("scheme", ["EULER", "RK2"])
def test_passive_scalar_10_steps(lib, scheme):
    N = (32, 32, 32)
    U = ic.random_phase_field(N, seed=74)
    T = ic.random_phase_field(N, k0=3.0, seed=75)[0]
    s = make(N, physics="SCALAR", nu=2e-3, kappa=5e-3, dt=5e-4, scheme=scheme, hyper_kappa=4e-6)
    s.set_V(U)
    s.set_T(T)
    s.step(10)
    ref = o.ScalarSolver(N, KF, 2e-3, 5e-3, 5e-4, scheme=scheme, kappa_h=4e-6)
    u, t = U, T
    for _ in range(10):
        u, t, _ = ref.step(u, t)
    assert rel_l2(s.get_V() + [s.get_T()], u + [t]) < 1e-12


@pytest.mark.parametrize("scheme", ["EULER", "RK2"])
def test_convection_10_steps(lib, scheme):
    N = (17, 16, 32)
    T = ic.rb_perturbation(N, seed=76)
    V = [np.zeros_like(T) for _ in range(3)]
    s = make(N, physics="RB", basis="SCFT", Ra=1e5, Pr=1.0, kfactor=KF_RB, dt=1e-4, scheme=scheme,
             hyper_nu=1e-7, hyper_kappa=2e-7)
    s.set_V(V)
    s.set_T(T)
    s.step(10)
    ref = o.RBSolver(N, KF_RB, 1e5, 1.0, 1e-4, scheme=scheme, nu_h=1e-7, kappa_h=2e-7)
    v, t = V, T
    for _ in range(10):
        v, t, _ = ref.step(v, t)
    assert rel_l2([s.get_T()], [t]) < 1e-12
    assert rel_l2(s.get_V(), v) < 1e-11


@pytest.mark.parametrize("scheme", ["EULER", "RK2"])
def test_fp32_mixed_against_fp64(lib, scheme):
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=77)
    out = []
    for prec in ("FP64", "FP32"):
        s = make(N, nu=1e-3, dt=5e-4, scheme=scheme, hyper_nu=HYPER, precision=prec)
        s.set_V(V)
        s.step(10)
        out.append(s.get_V())
    assert rel_l2(out[1], out[0]) < 1e-6


@pytest.mark.parametrize("scheme", ["EULER", "RK2"])
def test_fine_grained_calls_match_fused_step(lib, scheme):
    """The loop body of Ifluid_main.cc:261-278 called method by method (Time_advance starting
    from the caller's nonlinear term) equals tg_step for the scheme."""
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=78)
    force = dict(inner=2.0, outer=3.0, eps=0.1)
    a = make(N, nu=1e-3, dt=5e-4, force=force, scheme=scheme, hyper_nu=HYPER)
    b = make(N, nu=1e-3, dt=5e-4, force=force, scheme=scheme, hyper_nu=HYPER)
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


def test_served_request_equals_lone(lib):
    """RK2 with hyperviscosity in the serving loop: a batch of requests (one with another
    viscosity) equals each request's lone run bit for bit."""
    from tarang_b200.serving import Server
    N = (32, 32, 32)
    cfgs = [dict(N=N, nu=1e-3 * (1 + j), dt=1e-3, scheme="RK2", hyper_nu=HYPER) for j in range(3)]
    fields = [ic.random_phase_field(N, seed=80 + j) for j in range(3)]
    with Server(hbm_budget=8e9, max_batch=4) as srv:
        ids = [srv.submit(c, f, 6) for c, f in zip(cfgs, fields)]
        srv.drain()
        for rid, c, f in zip(ids, cfgs, fields):
            cc = dict(c)
            s = make(cc.pop("N"), **cc)
            s.set_V(f)
            s.step(6)
            want = s.get_V()
            got = srv.result(rid)
            assert all(np.array_equal(x.view(np.float64), y.view(np.float64)) for x, y in zip(got, want))


def test_slab_refuses_other_schemes(lib):
    import ctypes

    from tarang_b200 import _lib as L
    from tarang_b200.solver import make_config
    cfg = make_config((16, 16, 16), nu=1e-3, dt=1e-3, scheme="RK2")
    h = ctypes.c_void_p()
    assert L.load().tg_slab_create(ctypes.byref(cfg), 2, 0, ctypes.byref(h)) == L.TG_ERR_UNSUPPORTED
