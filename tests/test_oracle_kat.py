"""The oracle against the reference's own known answer and analytic identities (CPU).

The reference's tests hold one known answer for this path
(trunk/test/test-fftw/out1.d, printed by trunk/test/test-fftw/main_mpi.cc:93-118): an
unnormalised c2r -> r2c round trip of a unit delta at (0,0,2) on a 4^3 grid returns 64 = N^3
at (0,0,2) and zero elsewhere.  Its golden values are read from tests/golden/out1_kat.json.
"""

import json
import math
import os

import numpy as np
import pytest

from oracle import tarang_oracle as o

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_out1_delta_round_trip():
    kat = json.load(open(os.path.join(GOLD, "out1_kat.json")))
    N = tuple(kat["N"])
    A = np.zeros((N[0], N[1], N[2] // 2 + 1), complex)
    A[tuple(kat["delta_at"])] = 1.0
    r = o.inverse_four(A)
    # the c2r of the kz = N3/2 delta is (-1)^z on every (x, y)
    z = np.arange(N[2])
    assert np.allclose(r, (-1.0) ** z[None, None, :], atol=1e-15)
    # sum of squares of the 64 real values (the reference's 80 adds FFTW's padding slots)
    assert abs((r ** 2).sum() - kat["real_sum_sq_without_padding"]) < 1e-12
    B = o.forward_four(r) * np.prod(N)          # undo Norm_FOUR -> FFTW's unnormalised r2c
    want = np.array(kat["after_fft"], dtype=float).reshape(N[0], N[1], N[2] // 2 + 1)
    assert np.abs(B - want).max() < 1e-12


@pytest.mark.parametrize("N", [(8, 8, 8), (12, 12, 12), (16, 18, 20), (20, 16, 12), (64, 64, 64)])
def test_round_trip_four(N):
    rng = np.random.default_rng(1)
    real = rng.standard_normal(N)
    back = o.inverse_four(o.forward_four(real))
    assert np.abs(back - real).max() < 1e-13


@pytest.mark.parametrize("N1", [8, 12, 16, 65, 129])
@pytest.mark.parametrize("parity", [0, 1])
def test_round_trip_scft(N1, parity):
    rng = np.random.default_rng(2)
    real = rng.standard_normal((N1, 8, 8))
    spec = o.forward_scft(real, parity)
    back = o.inverse_scft(spec, parity)
    if parity == 0:
        assert np.abs(back - real).max() < 1e-12
    else:
        # the sine transform drops mode N1 (ArrayShiftRight_SCFT): project it out first
        x = (np.arange(N1) + 0.5) / N1
        s = np.sin(N1 * math.pi * x)
        real2 = real - s[:, None, None] * (np.tensordot(s, real, axes=(0, 0)) / (s @ s))[None]
        back2 = o.inverse_scft(o.forward_scft(real2, 1), 1)
        assert np.abs(back2 - real2).max() < 1e-12


def test_single_mode_four():
    N = (16, 16, 16)
    x = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    real = np.cos(2 * X + 3 * Y + 5 * Z)
    A = o.forward_four(real)
    # e^{i k.x} + e^{-i k.x}: stored half-space holds 1/2 at (2, 3, 5)
    assert abs(A[2, 3, 5] - 0.5) < 1e-14
    A[2, 3, 5] = 0
    assert np.abs(A).max() < 1e-14


def test_single_mode_scft():
    N1 = 12
    x = (np.arange(N1) + 0.5) / N1
    for m in (1, 3, 7):
        real = np.broadcast_to(np.sin(m * np.pi * x)[:, None, None], (N1, 4, 4)).copy()
        A = o.forward_scft(real, 1)
        # slot m <-> sin(m pi x): DST-II gives N1, Norm 1/(2 N1 N2 N3) -> 1/2 at (m, 0, 0)
        assert abs(A[m, 0, 0] - 0.5) < 1e-13
        A[m, 0, 0] = 0
        assert np.abs(A).max() < 1e-13
        real = np.broadcast_to(np.cos(m * np.pi * x)[:, None, None], (N1, 4, 4)).copy()
        A = o.forward_scft(real, 0)
        assert abs(A[m, 0, 0] - 0.5) < 1e-13


def _tg_fields(n):
    x = 2 * np.pi * np.arange(n) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    return X, Y, Z


def test_taylor_green_nlin_closed_form():
    n = 32
    X, Y, Z = _tg_fields(n)
    from tarang_b200 import ic
    V = ic.taylor_green((n, n, n))
    u = o.inverse_four(V[0])
    assert np.abs(u - np.sin(X) * np.cos(Y) * np.cos(Z)).max() < 1e-14
    nl = o.nlin_fluid(V, (1.0, 1.0, 1.0))
    ux, uy = np.cos(X) * np.cos(Y) * np.cos(Z), -np.sin(X) * np.sin(Y) * np.cos(Z)
    vx, vy = np.sin(X) * np.sin(Y) * np.cos(Z), -np.cos(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    assert np.abs(o.inverse_four(nl[0]) - (u * ux + v * uy)).max() < 1e-13
    assert np.abs(o.inverse_four(nl[1]) - (u * vx + v * vy)).max() < 1e-13
    assert np.abs(o.inverse_four(nl[2])).max() < 1e-13
    # total energy of TG = 1/8 and dE/dt = -2 nu Omega (Omega = enstrophy = 3/8)
    E = sum(o.total_energy_four(a) for a in V)
    assert abs(E - 0.125) < 1e-15


def test_beltrami_projected_nlin_vanishes():
    # ABC flow u = (sin z + cos y, sin x + cos z, sin y + cos x): u x omega = 0, so the
    # projected nonlinear term -P(u.grad u) = 0
    n = 16
    X, Y, Z = _tg_fields(n)
    V = [o.forward_four(np.sin(Z) + np.cos(Y)), o.forward_four(np.sin(X) + np.cos(Z)),
         o.forward_four(np.sin(Y) + np.cos(X))]
    nl = o.nlin_fluid(V, (1.0, 1.0, 1.0))
    p = o.pressure(nl, (1.0, 1.0, 1.0))
    rhs = o.rhs_from_nlin(nl, p, (1.0, 1.0, 1.0))
    assert max(np.abs(r).max() for r in rhs) < 1e-14


def test_shear_mode_exact_decay():
    # u = sin(k y) x: nlin = 0, so IF-RK4 gives the exact exp(-nu k^2 t) decay
    n, k, nu, dt = 16, 3, 0.05, 0.01
    X, Y, Z = _tg_fields(n)
    V = [o.forward_four(np.sin(k * Y)), np.zeros((n, n, n // 2 + 1), complex), np.zeros((n, n, n // 2 + 1), complex)]
    s = o.FluidSolver((n, n, n), (1.0, 1.0, 1.0), nu, dt)
    for _ in range(5):
        V, _ = s.step(V)
    want = o.forward_four(np.sin(k * Y) * math.exp(-nu * k * k * 5 * dt))
    assert np.abs(V[0] - want).max() < 1e-15


def test_inviscid_energy_conservation_of_nlin():
    from tarang_b200 import ic
    N = (16, 16, 16)
    V = ic.random_phase_field(N, seed=7)
    nl = o.nlin_fluid(V, (1.0, 1.0, 1.0))
    p = o.pressure(nl, (1.0, 1.0, 1.0))
    rhs = o.rhs_from_nlin(nl, p, (1.0, 1.0, 1.0))
    dEdt = sum(o.total_energy_four(V[i], rhs[i]) for i in range(3))
    scale = sum(o.total_energy_four(r) for r in rhs) ** 0.5
    assert abs(dEdt) < 1e-13 * scale


def test_shell_to_shell_antisymmetry_and_flux():
    from tarang_b200 import ic
    N = (64, 64, 64)
    V = ic.random_phase_field(N, seed=3)
    T = o.compute_shell_tr(V, (1.0, 1.0, 1.0), 12)
    # interior shells n, m < S: T(n, m) = -T(m, n)
    S = 12
    A = T[1:S, 1:S]
    assert np.abs(A + A.T).max() < 1e-12 * np.abs(A).max()
    # flux through sphere s = transfer from giver shells n <= s to every receiver |K| > R_s
    # (receivers beyond R_in included): the linear decomposition the CUDA path uses
    flux = o.compute_flux(V, (1.0, 1.0, 1.0), 12)
    R = o.et_radii(N, (1.0, 1.0, 1.0), S)
    K = o.kmag(N, (1.0, 1.0, 1.0))
    mult = o.multiplicity_four(N)
    bins = o.shell_index(K, R)
    Tfull = np.zeros((S + 1, S + 1))
    for n_ in range(1, S):
        G = [o.fill_array_shell(v, R[n_ - 1], R[n_], (1.0, 1.0, 1.0)) for v in V]
        nl = o.et_nlin(V, G, (1.0, 1.0, 1.0))
        val = 2 * mult * sum(np.real(nl[i] * np.conj(V[i])) for i in range(3))
        Tfull[n_] = np.bincount(bins.ravel(), weights=val.ravel(), minlength=S + 1)[: S + 1]
    assert np.allclose(-Tfull[1:S, :S], T[1:S, :S], rtol=0, atol=1e-13 * np.abs(T).max())
    for s in range(1, S):
        want = -Tfull[1: s + 1, s + 1:].sum()
        assert abs(flux[s] - want) < 1e-11 * max(1e-30, np.abs(flux).max())


def test_et_radii_scheme0():
    R = o.et_radii((64, 64, 64), (1.0, 1.0, 1.0), 12)
    s = math.log2(21 / 16) / 7
    want = [0, 2, 4, 8] + [8 * 2 ** (s * (i - 3)) for i in range(4, 10)] + [10.5, 21, 1e4]
    assert np.allclose(R, want, rtol=0, atol=1e-13)
