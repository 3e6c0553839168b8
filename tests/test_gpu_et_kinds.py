"""Energy-transfer kinds beyond U and B: the passive-scalar flux and shell-to-shell transfer
(Compute_flux_scalar / Compute_shell_tr_scalar, T< -> T> with U as helper) and the Elsasser
fluxes and shell-to-shell transfers of MHD (flux_Elsasser: Z+< -> Z+> with Z- as helper, and the
reverse), on the CUDA path against the oracle's generic restatement (1e-10 of the largest
entry, as the other transfer tests)."""

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

KF = (1.0, 1.0, 1.0)


def close(a, b, tol):
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


def test_scalar_flux_and_shell_to_shell(lib):
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    U = ic.random_phase_field(N, k0=3.0, seed=7)
    T = ic.random_phase_field(N, k0=2.0, seed=8)[0]
    s = IncFluid(N, physics="SCALAR", nu=1e-3, kappa=2e-3, dt=5e-4, n_shells=10)
    s.set_V(U)
    s.set_T(T)
    z = np.zeros_like(T)
    F = [T, z, z]
    assert close(s.Compute_flux(L.TG_ET_TT), o.compute_flux_generic(U, F, F, -1.0, KF, 10), 1e-10)
    assert close(s.Compute_shell_tr(L.TG_ET_TT), o.compute_shell_tr_generic(U, F, F, -1.0, KF, 10), 1e-10)
    # the velocity transfer of the same context is unchanged
    assert close(s.Compute_flux(L.TG_ET_UU), o.compute_flux(U, KF, 10), 1e-10)


@pytest.mark.parametrize("kind", [L.TG_ET_ZP, L.TG_ET_ZM])
def test_elsasser_flux_and_shell_to_shell(lib, kind):
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    U = ic.random_phase_field(N, k0=3.0, seed=20261203)
    B = ic.random_phase_field(N, k0=3.0, seed=20261204)
    s = IncFluid(N, physics="MHD", nu=1e-3, eta=1e-3, dt=5e-4, n_shells=8)
    s.set_V(U)
    s.set_W(B)
    Zp = [u + b for u, b in zip(U, B)]
    Zm = [u - b for u, b in zip(U, B)]
    H, F = (Zm, Zp) if kind == L.TG_ET_ZP else (Zp, Zm)
    assert close(s.Compute_flux(kind), o.compute_flux_generic(H, F, F, -1.0, KF, 8), 1e-10)
    assert close(s.Compute_shell_tr(kind), o.compute_shell_tr_generic(H, F, F, -1.0, KF, 8), 1e-10)
    # the state is untouched (the Elsasser fields are scratch)
    assert np.array_equal(s.get_V()[0], U[0]) or close(s.get_V()[0], U[0], 1e-15)


def test_kinds_rejected_for_other_physics(lib):
    from tarang_b200.solver import IncFluid
    s = IncFluid((16, 16, 16), nu=1e-3, dt=1e-3, n_shells=8)
    s.set_V(ic.random_phase_field((16, 16, 16), seed=1))
    for kind in (L.TG_ET_TT, L.TG_ET_ZP, L.TG_ET_ZM):
        with pytest.raises(L.TarangError):
            s.Compute_flux(kind)
