"""Kinetic helicity flux (IncVF::Compute_kinetic_helicity_flux, FOUR).  The oracle's three-term
restatement equals, sphere by sphere, the nonlinear change of the helicity inside the sphere,
sum over 0 < |K| <= R of 2 mult Re(N . omega*) with N = D_j F(U_j U_i), and the total over all
modes vanishes (helicity is conserved by the nonlinear term); the CUDA path matches the oracle."""

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic

KF = (1.0, 1.0, 1.0)


def test_oracle_helicity_flux_is_the_helicity_leaving_the_sphere():
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=3)
    h = o.kinetic_helicity_flux(V, KF, 12)
    W = o.vorticity_four(V, KF)
    NL = o.et_nlin(V, V, KF)
    K = o.kmag(N, KF)
    mult = o.multiplicity_four(N)
    R = o.et_radii(N, KF, 12)
    val = 2 * mult * sum(np.real(a * np.conj(b)) for a, b in zip(NL, W))
    scale = np.abs(val).sum()
    assert abs(val.sum()) <= 1e-13 * scale
    for s in range(1, 12):
        assert abs(h[s] - val[(K > 0) & (K <= R[s])].sum()) <= 1e-13 * scale
    assert h[12] == 0.0   # the last sphere holds every mode


@pytest.mark.gpu
@pytest.mark.parametrize("N,S,kf", [((32, 32, 32), 12, (1.0, 1.0, 1.0)), ((64, 32, 64), 10, (1.0, 2.0, 1.0))])
def test_gpu_helicity_flux_matches_oracle(lib, N, S, kf):
    from tarang_b200.solver import IncFluid
    V = ic.random_phase_field(N, kfactor=kf, seed=17)
    s = IncFluid(N, kfactor=kf, nu=1e-3, dt=1e-3, n_shells=S)
    s.set_V(V)
    got = s.Compute_kinetic_helicity_flux()
    want = o.kinetic_helicity_flux(V, kf, S)
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
    # a second call (vorticity buffers reused) gives the same table (to the order of the
    # atomic additions)
    again = s.Compute_kinetic_helicity_flux()
    assert np.abs(again - got).max() <= 1e-13 * np.abs(want).max()


def test_oracle_magnetic_helicity_flux_scaling():
    """The magnetic helicity flux is linear in U and quadratic in B, zero without velocity,
    and zero at the last sphere (no receiver outside it); the U x B< term is checked against a
    real-space cross product of its own."""
    N = (16, 16, 16)
    U = ic.random_phase_field(N, seed=5)
    B = ic.random_phase_field(N, seed=6)
    h = o.magnetic_helicity_flux(U, B, KF, 6)
    scale = np.abs(h).max()
    assert scale > 0 and h[6] == 0.0
    assert np.abs(o.magnetic_helicity_flux([2.0 * u for u in U], B, KF, 6) - 2 * h).max() <= 1e-13 * scale
    assert np.abs(o.magnetic_helicity_flux(U, [3.0 * b for b in B], KF, 6) - 9 * h).max() <= 1e-12 * scale
    assert np.all(o.magnetic_helicity_flux([0 * u for u in U], B, KF, 6) == 0)
    ur = [np.fft.irfftn(u * np.prod(N), s=N, axes=(0, 1, 2)) for u in U]
    br = [np.fft.irfftn(b * np.prod(N), s=N, axes=(0, 1, 2)) for b in B]
    cr = [ur[1] * br[2] - ur[2] * br[1], ur[2] * br[0] - ur[0] * br[2], ur[0] * br[1] - ur[1] * br[0]]
    want = [np.fft.rfftn(c) / np.prod(N) for c in cr]
    got = o.et_nlin_cross(U, B, KF)
    assert max(np.abs(g - w).max() for g, w in zip(got, want)) <= 1e-13 * max(np.abs(w).max() for w in want)
    # curl a = B for the divergence-free B (no mean field)
    A = o.vector_potential_four(B, KF)
    assert max(np.abs(x - y).max() for x, y in zip(o.vorticity_four(A, KF), B)) <= 1e-13 * max(np.abs(b).max() for b in B)


@pytest.mark.gpu
@pytest.mark.parametrize("N,S,kf", [((32, 32, 32), 8, (1.0, 1.0, 1.0)), ((64, 32, 64), 10, (1.0, 2.0, 1.0))])
def test_gpu_magnetic_helicity_flux_matches_oracle(lib, N, S, kf):
    from tarang_b200.solver import IncFluid
    U = ic.random_phase_field(N, kfactor=kf, seed=21)
    B = ic.random_phase_field(N, kfactor=kf, seed=22)
    s = IncFluid(N, physics="MHD", kfactor=kf, nu=1e-3, eta=1e-3, dt=1e-3, n_shells=S)
    s.set_V(U)
    s.set_W(B)
    got = s.Compute_magnetic_helicity_flux()
    want = o.magnetic_helicity_flux(U, B, kf, S)
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
    # the fields are untouched, so the energy fluxes after it are those of the fields
    assert np.abs(s.get_W()[0] - B[0]).max() == 0


def _inside(V, N, r):
    K = o.kmag(N, KF)
    return [np.where(K <= r, v, 0) for v in V]


@pytest.mark.parametrize("magnetic", [False, True])
def test_oracle_helicity_shell_tr_sums_to_the_flux(magnetic):
    """With the fields held to |K| <= R_in every receiver of the flux is binned by the
    shell-to-shell table, so flux(s) = sum over giver rows n <= s and receiver columns m > s."""
    N, S = (64, 64, 64), 10   # increasing radii 2, 4, 8, 8.4, ..., 10.5, 21
    kin = o.max_radius_inside(N, KF, "DEALIAS", "FOUR")
    U = _inside(ic.random_phase_field(N, seed=8), N, kin)
    if magnetic:
        B = _inside(ic.random_phase_field(N, seed=9), N, kin)
        f, T = o.magnetic_helicity_flux(U, B, KF, S), o.magnetic_helicity_shell_tr(U, B, KF, S)
    else:
        f, T = o.kinetic_helicity_flux(U, KF, S), o.kinetic_helicity_shell_tr(U, KF, S)
    scale = np.abs(T).max()
    assert scale > 0 and np.all(T[0] == 0) and np.all(T[S] == 0)
    for s in range(1, S):
        assert abs(f[s] - T[1:s + 1, s + 1:].sum()) <= 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("magnetic", [False, True])
def test_gpu_helicity_shell_tr_matches_oracle(lib, magnetic):
    from tarang_b200.solver import IncFluid
    N, S = (32, 32, 32), 8
    U = ic.random_phase_field(N, seed=23)
    B = ic.random_phase_field(N, seed=24)
    if magnetic:
        s = IncFluid(N, physics="MHD", nu=1e-3, eta=1e-3, dt=1e-3, n_shells=S)
        s.set_V(U)
        s.set_W(B)
        got, want = s.Compute_magnetic_helicity_shell_tr(), o.magnetic_helicity_shell_tr(U, B, KF, S)
    else:
        s = IncFluid(N, nu=1e-3, dt=1e-3, n_shells=S)
        s.set_V(U)
        got, want = s.Compute_kinetic_helicity_shell_tr(), o.kinetic_helicity_shell_tr(U, KF, S)
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
