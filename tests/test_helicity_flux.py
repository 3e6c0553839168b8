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
