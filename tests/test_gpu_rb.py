"""Parity of the CUDA SCFT basis and Rayleigh-Benard path with the oracle: sin/cos-Fourier
transforms (any N1, including odd 65 and 129), the scalar/RB nonlinear term with SCFT
parities, 10 RK4 steps of convection (PRLARGE + ULARGE), the Nusselt number and the
temperature shell spectrum."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic

pytestmark = pytest.mark.gpu
KF_RB = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))


def rel_l2(a, b):
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


def make(N, **kw):
    from tarang_b200.solver import IncFluid
    return IncFluid(N, basis="SCFT", **kw)


@pytest.mark.parametrize("N", [(8, 8, 8), (12, 16, 8), (65, 32, 16), (128, 16, 32), (129, 32, 32)])
@pytest.mark.parametrize("parity", [0, 1])
@pytest.mark.parametrize("precision,tol", [("FP64", 1e-13), ("FP32", 3e-6)])
def test_scft_transforms(lib, N, parity, precision, tol):
    rng = np.random.default_rng(40 + parity)
    real = rng.standard_normal(N)
    s = make(N, physics="FLUID", precision=precision)
    got = s.Forward_transform_array(o.pack_real(real), parity=parity)
    want = o.forward_scft(real, parity)
    assert np.abs(got - want).max() < tol * np.abs(want).max()
    back = o.unpack_real(s.Inverse_transform_array(want, parity=parity))
    wb = o.inverse_scft(want, parity)
    assert np.abs(back - wb).max() < tol * np.abs(wb).max()


def scft_fields(N, seed):
    """Random dealiased SCFT fields: u1 and theta sine series, u2 and u3 cosine series."""
    rng = np.random.default_rng(seed)
    par = (1, 0, 0, 1)
    out = [o.dealias(o.forward_scft(rng.standard_normal(N), p), "SCFT") for p in par]
    return out[:3], out[3]


@pytest.mark.parametrize("N", [(24, 16, 16), (33, 32, 32), (64, 32, 64)])
def test_rb_nlin(lib, N):
    V, T = scft_fields(N, 7)
    s = make(N, physics="RB", Ra=1e6, Pr=1.0, kfactor=KF_RB, dt=1e-4)
    s.set_V(V)
    s.set_T(T)
    s.Compute_nlin()
    assert rel_l2(s.get_nlin(), o.nlin_fluid(V, KF_RB, "SCFT")) < 1e-13
    assert rel_l2([s.get_Tnlin()], [o.nlin_scalar(V, T, KF_RB, "SCFT")]) < 1e-13
    s.Compute_pressure()
    nl = o.nlin_fluid(V, KF_RB, "SCFT")
    nl = [nl[0] - T, nl[1], nl[2]]  # the pressure of the reference is computed after Add_force
    s.Compute_force()
    s2 = make(N, physics="RB", Ra=1e6, Pr=1.0, kfactor=KF_RB, dt=1e-4)
    s2.set_V(V)
    s2.set_T(T)
    s2.Compute_force()
    s2.Compute_nlin()
    s2.Add_force()
    s2.Compute_pressure()
    pw = o.pressure(nl, KF_RB, "SCFT")
    assert np.abs(s2.get_pressure() - pw).max() < 1e-13 * np.abs(pw).max()


@pytest.mark.parametrize("N,precision,tol", [((33, 32, 32), "FP64", 1e-12), ((33, 32, 32), "FP32", 1e-6),
                                             ((24, 16, 32), "FP64", 1e-12)])
def test_rb_10_steps(lib, N, precision, tol):
    T = ic.rb_perturbation(N, seed=20261205)
    V = [np.zeros_like(T) for _ in range(3)]
    s = make(N, physics="RB", Ra=1e6, Pr=1.0, kfactor=KF_RB, dt=1e-4, precision=precision)
    s.set_V(V)
    s.set_T(T)
    s.step(10)
    ref = o.RBSolver(N, KF_RB, 1e6, 1.0, 1e-4)
    v, t = V, T
    for _ in range(10):
        v, t, dt = ref.step(v, t)
        assert dt == 1e-4
    assert rel_l2([s.get_T()], [t]) < tol
    assert rel_l2(s.get_V(), v) < tol * 10
    Nu = ctypes_nusselt(s)
    assert abs(Nu - ref.nusselt(v, t)) < 1e-12
    ek, _ = s.CV_Compute_shell_spectrum(group=2)
    w = o.shell_spectrum(t, 0, KF_RB, basis="SCFT")
    assert np.abs(ek[0][: len(w)] - w).max() < 1e-11 * np.abs(w).max()
    E, D = s.CV_Compute_totalenergy_diss(group=2)
    assert abs(E - o.total_energy(t, "SCFT")) < 1e-12 * abs(E)
    assert abs(D - 2 * o.total_Sn(t, 2, KF_RB, basis="SCFT")) < 1e-12 * abs(D)


def ctypes_nusselt(s):
    import ctypes
    v = ctypes.c_double()
    s._ck(s.lib.tg_nusselt(s.h, ctypes.byref(v)), "nusselt")
    return v.value


@pytest.mark.parametrize("pr_switch,u_scaling,grad", [("PRLARGE", "USMALL", 1.0), ("PRSMALL", "ULARGE", 1.0),
                                                      ("PRSMALL", "USMALL", 1.0), ("PRLARGE", "ULARGE", -1.0)])
def test_rb_scalings_10_steps(lib, pr_switch, u_scaling, grad):
    """The other nondimensionalisations of RB_slip_main.cc:222-262 (and stable stratification,
    temperature_grad = -1): diffusivities, buoyancy coefficients and Nusselt factor."""
    N = (24, 16, 32)
    Ra, Pr = 2e3, 0.7
    T = ic.rb_perturbation(N, seed=20261207)
    V = [np.zeros_like(T) for _ in range(3)]
    s = make(N, physics="RB", Ra=Ra, Pr=Pr, kfactor=KF_RB, dt=1e-4, Pr_switch=pr_switch, RB_Uscaling=u_scaling,
             temperature_grad=grad)
    s.set_V(V)
    s.set_T(T)
    s.step(10)
    ref = o.RBSolver(N, KF_RB, Ra, Pr, 1e-4, pr_switch=pr_switch, u_scaling=u_scaling, temperature_grad=grad)
    v, t = V, T
    for _ in range(10):
        v, t, dt = ref.step(v, t)
    assert rel_l2([s.get_T()], [t]) < 1e-12
    assert rel_l2(s.get_V(), v) < 1e-11
    assert abs(s.Get_Nusselt_no() - ref.nusselt(v, t)) < 1e-12 * abs(ref.nusselt(v, t))


@pytest.mark.parametrize("pr_switch,u_scaling", [("PRLARGE", "ULARGE"), ("PRLARGE", "USMALL"), ("PRSMALL", "USMALL")])
def test_rb_rotation_10_steps(lib, pr_switch, u_scaling):
    """Convection with rotation (force_field_proc 52, Compute_force_RB_rotation): the buoyancy of
    proc 51 plus the Coriolis force V x Omega scaled by the nondimensionalisation."""
    N = (24, 16, 32)
    Ra, Pr = 2e3, 0.7
    om = (0.0, 0.5, 2.0)
    rng = np.random.default_rng(3)
    V = [1e-2 * o.dealias(o.forward_scft(rng.standard_normal(N), p), "SCFT") for p in (1, 0, 0)]
    T = ic.rb_perturbation(N, seed=20261208)
    s = make(N, physics="RB", Ra=Ra, Pr=Pr, kfactor=KF_RB, dt=1e-4, Pr_switch=pr_switch, RB_Uscaling=u_scaling,
             force=dict(kind="rb_rotation", omega=om))
    s.set_V(V)
    s.set_T(T)
    s.step(10)
    ref = o.RBSolver(N, KF_RB, Ra, Pr, 1e-4, pr_switch=pr_switch, u_scaling=u_scaling, omega=om)
    v, t = V, T
    for _ in range(10):
        v, t, dt = ref.step(v, t)
    assert rel_l2(s.get_V(), v) < 1e-11
    assert rel_l2([s.get_T()], [t]) < 1e-12
    # without rotation the trajectory differs
    ref0 = o.RBSolver(N, KF_RB, Ra, Pr, 1e-4, pr_switch=pr_switch, u_scaling=u_scaling)
    v0, t0 = V, T
    for _ in range(10):
        v0, t0, _ = ref0.step(v0, t0)
    assert rel_l2(v0, v) > 1e-6
