"""The reference's initial-condition procedures on the host (tarang_b200.ic): Taylor-Green
(velocity and the MHD magnetic table), ABC, given modes, the model energy spectrum, the RB Lorenz
modes, and the para.d dispatch of field_input_proc, checked against their real-space formulas,
incompressibility and the oracle's transforms."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic


def grid(n):
    x = 2 * np.pi * np.arange(n) / n
    return np.meshgrid(x, x, x, indexing="ij")


def test_taylor_green_velocity_and_magnetic_tables():
    N = (16, 16, 16)
    k0, amp, ampW = 2, 1.3, 0.7
    f = ic.taylor_green_field(N, k0, amp, physics="MHD", ampW=ampW)
    assert len(f) == 6
    assert all(np.array_equal(a, b) for a, b in zip(f[:3], ic.taylor_green(N, k0, amp)))
    X, Y, Z = grid(16)
    u = [o.inverse_four(a, 16) for a in f[:3]]
    w = [o.inverse_four(a, 16) for a in f[3:]]
    assert np.abs(u[0] - amp * np.sin(k0 * X) * np.cos(k0 * Y) * np.cos(k0 * Z)).max() < 1e-13
    # Setup_Taylor_Green_field_mag_field: ampW (sin sin cos, cos cos cos, 0)
    assert np.abs(w[0] - ampW * np.sin(k0 * X) * np.sin(k0 * Y) * np.cos(k0 * Z)).max() < 1e-13
    assert np.abs(w[1] - ampW * np.cos(k0 * X) * np.cos(k0 * Y) * np.cos(k0 * Z)).max() < 1e-13
    assert np.abs(w[2]).max() == 0
    s = ic.taylor_green_field(N, k0, amp, physics="SCALAR")
    assert len(s) == 4 and np.all(s[3] == 0)
    sc = ic.taylor_green_field(N, k0, amp, basis="SCFT", physics="MHD", ampW=ampW)
    assert sc[3][k0, k0, k0] == ampW / 8 and sc[3][k0, 16 - k0, k0] == -ampW / 8


def test_abc_and_modes_fields():
    N = (16, 16, 16)
    f = ic.abc_field(N, 1, 0.9, 1.0, 0.7, 0.4)
    want = o.abc_force(N, 1, 0.9, 1.0, 0.7, 0.4)
    assert all(np.array_equal(a, b) for a, b in zip(f, want))
    m = ic.modes_field([(1, 2, 3, 0.3, 0.1j), (2, 1, 0, 0.5, 0.2)], N)
    K = o.kvec(N, (1.0, 1.0, 1.0))
    div = sum(1j * Ki * mi for Ki, mi in zip(K, m))
    assert np.abs(div).max() < 1e-15
    assert m[0][(-2) % 16, (-1) % 16, 0] == np.conj(m[0][2, 1, 0])


def test_energy_spectrum_field():
    N = (32, 32, 32)
    V = ic.energy_spectrum_field(N, 1.0, seed=7)
    K = o.kvec(N, (1.0, 1.0, 1.0))
    div = sum(1j * Ki * vi for Ki, vi in zip(K, V))
    assert np.abs(div).max() < 1e-14 * max(np.abs(v).max() for v in V)
    assert all(v[0, 0, 0] == 0 for v in V)
    assert all(np.array_equal(a, b) for a, b in zip(V, ic.energy_spectrum_field(N, 1.0, seed=7)))
    # every mode of shell k has |V|^2 = 2 Sk(k) / Approx_number_modes_in_shell(k) (amp =
    # sqrt(2 ek)); the oracle's shell sum adds mult |V|^2
    Sk = ic.model_shell_spectrum(12, 1.0)
    Ek = sum(o.shell_spectrum(v, 0, (1.0, 1.0, 1.0)) for v in V)
    shell = np.ceil(o.kmag(N, (1.0, 1.0, 1.0)))
    mult = o.multiplicity(N)
    for k in range(1, 10):
        want = 2 * Sk[k] / o.approx_number_modes_in_shell(N, k, (1.0, 1.0, 1.0)) * mult[shell == k].sum()
        assert abs(Ek[k] / want - 1.0) < 1e-12, (k, Ek[k], want)


def test_rb_lorenz_field():
    N = (17, 16, 16)
    kf = (math.pi, math.pi / math.sqrt(2), math.pi / math.sqrt(2))
    f = ic.rb_lorenz_field(N, 0.3, 0.2, -0.1, kf)
    assert f[0][1, 0, 1] == 0.3 and f[3][1, 0, 1] == 0.2 and f[3][2, 0, 0] == -0.1
    # SCFT incompressibility at (1, 0, 1): kx kf1 V1 + i kz kf3 V3 = 0
    assert abs(1 * kf[0] * f[0][1, 0, 1] + 1j * kf[2] * f[2][1, 0, 1]) < 1e-15


def test_read_init_cond_dispatch(tmp_path):
    from tests.test_field_io import PARA
    from tarang_b200.para import config_from_para, read_para
    from tarang_b200.solver import write_field_file

    def cfg(proc, ints=(), floats=(0.0,)):
        t = PARA.format(N1=16, N2=16, N3=16, Ra=0, Pr=0, basis="FOUR", nu=0.01, kappa=0, dt=1e-3, S=12, proc=0)
        t = t.replace("(1)in-meta	1	1	1", f"(1)in-meta	{1 + len(ints)}	{len(floats)}	1")
        t = t.replace("(2)in-int	0", "(2)in-int	" + "	".join(map(str, (proc,) + tuple(ints))))
        t = t.replace("(3)in-float	1.0", "(3)in-float	" + "	".join(map(str, floats)))
        return config_from_para(read_para(t, n_fields=1), "FLUID")

    f = ic.read_init_cond(cfg(7, floats=(2, 0.5)))
    assert all(np.array_equal(a, b) for a, b in zip(f, ic.taylor_green((16, 16, 16), 2, 0.5)))
    f = ic.read_init_cond(cfg(8, floats=(1, 1.0, 0.5, 0.25, 2.0)))
    assert all(np.array_equal(a, b) for a, b in zip(f, ic.abc_field((16, 16, 16), 1, 2.0, 1.0, 0.5, 0.25)))
    small = ic.random_phase_field((8, 8, 8), k0=2.0, seed=1)
    (tmp_path / "in").mkdir()
    write_field_file(tmp_path / "in" / "field_in.d", small)
    c = cfg(2, ints=(8, 8, 8))
    assert c["run"]["N_in_reduced"] == (8, 8, 8)
    f = ic.read_init_cond(c, data_dir=str(tmp_path))
    assert np.allclose(f[0][1, 1, :5], small[0][1, 1, :5], rtol=1e-10)
    (tmp_path / "in" / "field_in.d").write_text("1 1 1 (0.1,0) (0.2,0)\n99 0 0\n")
    f = ic.read_init_cond(cfg(3), data_dir=str(tmp_path))
    assert f[0][1, 1, 1] == 0.1
    with pytest.raises(ValueError):
        ic.read_init_cond(cfg(4))
