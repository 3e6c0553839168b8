"""Parity of the CUDA MHD path (Elsasser nonlinear term, IF-RK4 with nu and eta) with the
oracle: nonlinear terms <= 1e-13, 10-step fields <= 1e-12 relative L2 (FP64 form), FP32-mixed
<= 1e-6."""

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


def fields(N):
    U = ic.random_phase_field(N, k0=3.0, seed=20261203)
    B = ic.random_phase_field(N, k0=3.0, seed=20261204)
    return U, B


@pytest.mark.parametrize("N", [(16, 16, 16), (32, 32, 32)])
def test_mhd_nlin(lib, N):
    from tarang_b200.solver import IncFluid
    U, B = fields(N)
    s = IncFluid(N, physics="MHD", nu=1e-3, eta=1e-3, dt=5e-4)
    s.set_V(U)
    s.set_W(B)
    s.Compute_nlin()
    un, bn = o.nlin_mhd(U, B, KF)
    assert rel_l2(s.get_nlin(), un) < 1e-13
    assert rel_l2(s.get_Wnlin(), bn) < 1e-13
    # energies of both groups (Get_total_energy convention)
    E, _ = s.CV_Compute_totalenergy_diss(0)
    Eb, _ = s.CV_Compute_totalenergy_diss(1)
    assert abs(E - 0.5) < 1e-12 and abs(Eb - 0.5) < 1e-12


@pytest.mark.parametrize("precision,tol", [("FP64", 1e-12), ("FP32", 1e-6)])
def test_mhd_10_steps(lib, precision, tol):
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    U, B = fields(N)
    s = IncFluid(N, physics="MHD", nu=1e-3, eta=2e-3, dt=5e-4, precision=precision)
    s.set_V(U)
    s.set_W(B)
    s.step(10)
    ref = o.MHDSolver(N, KF, 1e-3, 2e-3, 5e-4)
    u, b = U, B
    for _ in range(10):
        u, b, dt = ref.step2(u, b)
        assert dt == 5e-4
    assert rel_l2(s.get_V(), u) < tol
    assert rel_l2(s.get_W(), b) < tol
