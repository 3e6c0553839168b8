"""Energy transfer in the SCFT basis (free-slip walls along x): flux and shell-to-shell of the
velocity (Compute_flux / Compute_shell_tr with the SCFT shell products of scft_ET.cc) and of the
convection temperature (Compute_flux_RB -> Compute_flux_scalar).  The oracle restates the
reference's loops with the SCFT parities; it is pinned here by energy conservation of the
nonlinear term, shell-to-shell antisymmetry and the flux = sum of shell-to-shell identity, and
the CUDA path is checked against it."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L

KF = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
N = (33, 32, 32)
S = 8


def scft_fields(N, seed, inside=None):
    """Dealiased SCFT fields: u1 and theta sine series, u2 and u3 cosine series, the velocity made
    divergence-free (u + D p with p = div u / K^2, D = (Xderiv of the cosine series, i ky, i kz));
    optionally held to |K| <= inside."""
    rng = np.random.default_rng(seed)
    out = [o.dealias(o.forward_scft(rng.standard_normal(N), p), "SCFT") for p in (1, 0, 0, 1)]
    if inside is not None:
        K = o.kmag(N, KF, "SCFT")
        out = [np.where(K <= inside, f, 0) for f in out]
    V = out[:3]
    p = o.pressure(V, KF, "SCFT")
    V = [V[0] + o.xderiv(p, KF, "SCFT", 0), V[1] + o.yderiv(p, KF), V[2] + o.zderiv(p, KF)]
    div = o.xderiv(V[0], KF, "SCFT", 1) + o.yderiv(V[1], KF) + o.zderiv(V[2], KF)
    assert np.abs(div).max() <= 1e-12 * max(np.abs(v).max() for v in V)
    return V, out[3]


def test_oracle_scft_transfer_identities():
    kin = o.max_radius_inside(N, KF, "DEALIAS", "SCFT")
    R = o.et_radii(N, KF, S, "DEALIAS", "SCFT")
    assert np.all(np.diff(R) > 0)
    V, T = scft_fields(N, 3, inside=kin)
    z = np.zeros_like(T)
    for H, F, sign in ((V, V, -1.0), (V, [T, z, z], -1.0)):
        tr = o.compute_shell_tr_generic(H, F, F, sign, KF, S, basis="SCFT")
        fl = o.compute_flux_generic(H, F, F, sign, KF, S, basis="SCFT")
        scale = np.abs(tr).max()
        assert scale > 0
        inner = tr[1:S, 1:S]
        assert np.abs(inner + inner.T).max() <= 1e-12 * scale
        for s in range(1, S - 1):
            assert abs(fl[s] - tr[1:s + 1, s + 1:S].sum()) <= 1e-12 * scale
        # the nonlinear term conserves energy: the whole table adds up to zero
        assert abs(tr.sum()) <= 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("Nn", [(33, 32, 32), (64, 32, 64)])
def test_gpu_scft_flux_and_shell_tr(lib, Nn):
    from tarang_b200.solver import IncFluid
    V, T = scft_fields(Nn, 11)
    z = np.zeros_like(T)
    s = IncFluid(Nn, basis="SCFT", physics="RB", Ra=1e6, Pr=1.0, kfactor=KF, dt=1e-4, n_shells=S)
    s.set_V(V)
    s.set_T(T)
    assert np.allclose(s.ET_radii(), o.et_radii(Nn, KF, S, "DEALIAS", "SCFT"), rtol=0, atol=1e-13)
    for kind, F in ((L.TG_ET_UU, V), (L.TG_ET_TT, [T, z, z])):
        fw = o.compute_flux_generic(V, F, F, -1.0, KF, S, basis="SCFT")
        tw = o.compute_shell_tr_generic(V, F, F, -1.0, KF, S, basis="SCFT")
        got = s.Compute_flux(kind)
        assert np.abs(got - fw).max() <= 1e-10 * np.abs(fw).max(), kind
        got = s.Compute_shell_tr(kind)
        assert np.abs(got - tw).max() <= 1e-10 * np.abs(tw).max(), kind


@pytest.mark.gpu
@pytest.mark.parametrize("basis", ["FOUR", "SCFT"])
@pytest.mark.parametrize("pr_switch,u_scaling", [("PRLARGE", "USMALL"), ("PRLARGE", "ULARGE"),
                                                 ("PRSMALL", "USMALL"), ("PRSMALL", "ULARGE")])
def test_gpu_convection_force_feed(lib, basis, pr_switch, u_scaling):
    """Compute_force_feed_shell_RB: the buoyancy force fu theta fed into u1 and the force
    ft u1 fed into theta, per energy-transfer shell, in both bases and for every
    nondimensionalisation.  Pr != 1 and a temperature gradient of -1 keep fu, ft and the
    scalings apart (at Pr = 1 PRLARGE/USMALL has ft = 1 and a swap of fu and ft would pass)."""
    from tarang_b200.solver import IncFluid
    Ra, Pr, tg = 2.0e5, 0.7, -1.0
    if basis == "SCFT":
        Nn, kf = N, KF
        V, T = scft_fields(N, 13)
    else:
        Nn, kf = (32, 32, 32), (1.0, 1.0, 1.0)
        rng = np.random.default_rng(14)
        V = [o.dealias(o.forward_four(rng.standard_normal(Nn))) for _ in range(3)]
        T = o.dealias(o.forward_four(rng.standard_normal(Nn)))
    s = IncFluid(Nn, basis=basis, physics="RB", Ra=Ra, Pr=Pr, kfactor=kf, dt=1e-4, n_shells=S,
                 Pr_switch=pr_switch, RB_Uscaling=u_scaling, temperature_grad=tg)
    try:
        s.set_V(V)
        s.set_T(T)
        _, _, fu, ft, _ = o.rb_coefficients(Ra, Pr, pr_switch, u_scaling, tg)
        z = np.zeros_like(T)
        want_u = o.force_feed_shell([fu * T, z, z], V, kf, S, basis=basis)
        want_t = o.force_feed_shell([ft * V[0]], [T], kf, S, basis=basis)
        got_u, got_t = s.Compute_force_feed_shell(0), s.Compute_force_feed_shell(2)
    finally:
        s.close()
    assert np.abs(got_u - want_u).max() <= 1e-12 * np.abs(want_u).max()
    assert np.abs(got_t - want_t).max() <= 1e-12 * np.abs(want_t).max()
