"""The oracle's integration schemes and hyper term (if_time_advance, exp_ksqr_hyper): RK4
through the generic driver equals the hand-written RK4; EULER and RK2 converge at first and
second order; a single shear mode, whose nonlinear term vanishes, decays exactly as
exp(-(nu K^2 + nu_h K^4) t) under every scheme."""

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic

N = (16, 16, 16)
KF = (1.0, 1.0, 1.0)


def maxdiff(a, b):
    return max(float(np.abs(x - y).max()) for x, y in zip(a, b))


def test_generic_rk4_equals_hand_written():
    V = ic.random_phase_field(N, seed=3)
    s = o.FluidSolver(N, KF, 1e-2, 1e-3)
    a, dt = s.step(V)
    b = o.if_time_advance([v.copy() for v in V], [(1e-2, 0.0)] * 3, lambda f: s.rhs(f)[0], dt, "RK4", KF)
    assert maxdiff(a, [o.dealias(x) for x in b]) == 0.0


@pytest.mark.parametrize("scheme,order", [("EULER", 1), ("RK2", 2)])
def test_convergence_order(scheme, order):
    V = ic.random_phase_field(N, seed=4)

    def run(sch, dt, n):
        s = o.FluidSolver(N, KF, 1e-2, dt, scheme=sch)
        W = [v.copy() for v in V]
        for _ in range(n):
            W, got = s.step(W)
            assert got == dt
        return W

    ref = run("RK4", 1e-3, 40)
    e1 = maxdiff(run(scheme, 4e-3, 10), ref)
    e2 = maxdiff(run(scheme, 2e-3, 20), ref)
    assert abs(e1 / e2 - 2 ** order) < 0.1 * 2 ** order


@pytest.mark.parametrize("scheme", ["EULER", "RK2", "RK4"])
def test_shear_mode_hyper_decay(scheme):
    """u_y(x) = a sin(k x): (u . grad) u = 0 and the pressure vanishes, so every scheme's
    integrating factor gives the exact decay exp(-(nu k^2 + nu_h k^4) t)."""
    k, nu, nu_h, dt, n = 3, 1e-2, 1e-4, 1e-3, 7
    real = np.zeros(N)
    x = np.arange(N[0]) * 2 * np.pi / N[0]
    real += 0.3 * np.sin(k * x)[:, None, None]
    V = [np.zeros((N[0], N[1], N[2] // 2 + 1), complex), o.forward_four(real),
         np.zeros((N[0], N[1], N[2] // 2 + 1), complex)]
    s = o.FluidSolver(N, KF, nu, dt, scheme=scheme, nu_h=nu_h)
    W = V
    for _ in range(n):
        W, got = s.step(W)
        assert got == dt
    want = [v * np.exp(-(nu * k * k + nu_h * k ** 4) * n * dt) for v in V]
    assert maxdiff(W, want) <= 1e-12 * float(np.abs(V[1]).max())
