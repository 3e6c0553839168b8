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


def _relative_helicity(V, N):
    kf = (1.0, 1.0, 1.0)
    Kx, Ky, Kz = o.kvec(N, kf)
    vr, vi = [v.real for v in V], [v.imag for v in V]
    H = Kx * (vr[1] * vi[2] - vr[2] * vi[1]) + Ky * (vr[2] * vi[0] - vr[0] * vi[2]) + Kz * (vr[0] * vi[1] - vr[1] * vi[0])
    E = sum(np.abs(v) ** 2 for v in V) / 2
    with np.errstate(all="ignore"):
        return H / (o.kmag(N, kf) * E), E


def test_energy_helicity_spectrum_field():
    """Init_cond_energy_helicity_spectrum: every mode off the kz = 0 plane has relative helicity
    H_k/(k E_k) = sk; MHD: W's is skW and the cross helicity Re(u . b*) / (amp ampW) is h (the
    reference's h = 2 Hc/(amp ampW), Hc = Re(u . b*)/2); divergence-free, origin zero; the
    scalar variant adds T with the a_T spectrum."""
    N = (16, 16, 16)
    F = ic.energy_helicity_spectrum_field(N, 1.0, 0.6, physics="MHD", a2=0.5, skW=-0.3, h=0.4, seed=3)
    V, W = F[:3], F[3:]
    sv, Ev = _relative_helicity(V, N)
    sw, Ew = _relative_helicity(W, N)
    sel = (Ev > 1e-30) & (Ew > 1e-30) & (np.arange(N[2] // 2 + 1)[None, None, :] > 0)
    assert sel.sum() > 100
    assert np.abs(sv[sel] - 0.6).max() < 1e-12 and np.abs(sw[sel] - (-0.3)).max() < 1e-12
    hc = sum((a * np.conj(b)).real for a, b in zip(V, W))
    assert np.abs(hc[sel] / np.sqrt(4 * Ev[sel] * Ew[sel]) - 0.4).max() < 1e-12
    K = o.kvec(N, (1.0, 1.0, 1.0))
    for X in (V, W):
        assert np.abs(sum(1j * Ki * x for Ki, x in zip(K, X))).max() < 1e-14
        assert all(x[0, 0, 0] == 0 for x in X)
    S = ic.energy_helicity_spectrum_field(N, 1.0, -0.2, physics="SCALAR", a2=0.7, seed=4)
    assert len(S) == 4 and S[3][0, 0, 0] == 0 and np.abs(S[3]).max() > 0
    s4, E4 = _relative_helicity(S[:3], N)
    m = (E4 > 1e-30) & (np.arange(N[2] // 2 + 1)[None, None, :] > 0)
    assert np.abs(s4[m] + 0.2).max() < 1e-12
    # the energy-spectrum procedure for MHD and a scalar: W and T from their own spectra
    M = ic.energy_spectrum_field(N, 1.0, physics="MHD", a2=0.3, seed=5)
    T = ic.energy_spectrum_field(N, 1.0, physics="SCALAR", a2=0.3, seed=5)
    assert len(M) == 6 and len(T) == 4 and np.abs(M[4]).max() > 0 and np.abs(T[3]).max() > 0


def test_scft_spectrum_initial_conditions():
    """The SCFT variants of field_input_procs 5 and 6 (Init_cond_energy_spectrum,
    Init_cond_energy_helicity_spectrum with basis_type SCFT, and their (T) forms for a scalar or
    convection): divergence-free in the SCFT sense (Xderiv of the sine series V1 plus i ky V2 +
    i kz V3), zero outside the SCFT 2/3 rule, the SCFT reality condition on kz = 0, the relative
    helicity sk of every mode in the Fourier basis (-i V1, V2, V3), energy per shell near the
    model spectrum, and T a sine series (imaginary phase factor i)."""
    import math
    KF = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
    N = (33, 16, 32)
    F = ic.energy_helicity_spectrum_field(N, 1.0, 0.5, KF, seed=6, physics="RB", a2=0.4, basis="SCFT")
    V, T = F[:3], F[3]
    div = o.xderiv(V[0], KF, "SCFT", 1) + o.yderiv(V[1], KF) + o.zderiv(V[2], KF)
    scale = max(float(np.abs(v).max()) for v in V) * o.kmag(N, KF, "SCFT").max()
    assert np.abs(div).max() <= 1e-13 * scale
    keep = ic.keep_mask(N, "SCFT")
    for X in V + [T]:
        assert np.all(X[~keep] == 0) and X[0, 0, 0] == 0
        for ly in range(N[1] // 2 + 1, N[1]):
            assert np.array_equal(X[:, ly, 0], np.conj(X[:, N[1] - ly, 0]))
    Kx, Ky, Kz = o.kvec(N, KF, "SCFT")
    vf = [-1j * V[0], V[1], V[2]]
    vr, vi = [v.real for v in vf], [v.imag for v in vf]
    H = Kx * (vr[1] * vi[2] - vr[2] * vi[1]) + Ky * (vr[2] * vi[0] - vr[0] * vi[2]) + Kz * (vr[0] * vi[1] - vr[1] * vi[0])
    E = sum(np.abs(v) ** 2 for v in vf) / 2
    sel = (E > 1e-30) & (np.arange(N[2] // 2 + 1)[None, None, :] > 0)
    assert sel.sum() > 100
    with np.errstate(all="ignore"):
        assert np.abs(H[sel] / (o.kmag(N, KF, "SCFT")[sel] * E[sel]) - 0.5).max() < 1e-12
    # every mode of shell k has |V|^2 = 2 Sk(k) / Approx_number_modes_in_shell_SCFT(k) (pi r^2):
    # the oracle's SCFT shell sum adds Multiplicity_factor_SCFT |V|^2
    S = ic.energy_spectrum_field(N, 1.0, KF, seed=7, physics="FLUID", basis="SCFT")
    ek = sum(o.shell_spectrum(v, 0, KF, basis="SCFT") for v in S)
    Sk = ic.model_shell_spectrum(len(ek) + 2, 1.0)
    shell = np.ceil(o.kmag(N, KF, "SCFT"))
    mult = o.multiplicity(N, "SCFT")
    kin = o.max_radius_inside(N, KF, "DEALIAS", "SCFT")
    for k in range(1, kin):
        want = 2 * Sk[k] / o.approx_number_modes_in_shell(N, k, KF, "SCFT") * mult[(shell == k) & keep].sum()
        if want == 0:          # no mode in the shell (|K| >= kf2 = 2.22)
            assert ek[k] == 0
            continue
        assert abs(ek[k] / want - 1.0) < 1e-12, (k, ek[k], want)
    # the read_init_cond dispatch reaches the SCFT procedures
    cfg = dict(N=N, basis="SCFT", physics="RB", kfactor=KF, run=dict(field_input_proc=5, init_cond_double=[0.0, 1.0, 0.3]))
    assert len(ic.read_init_cond(cfg)) == 4


def test_rayleigh_taylor_field():
    """field_input_proc 511: the tanh temperature profile in x, sine-transformed as the oracle's
    forward SCFT transform of the real field (uniform in y, z), dealiased; velocity zero."""
    N = (33, 8, 8)
    f = ic.rayleigh_taylor_field(N, 20.0)
    x = np.arange(N[0]) / N[0]
    th = x - (1 + np.tanh(20 * (x - 0.5))) / 2
    want = o.dealias(o.forward_scft(np.broadcast_to(th[:, None, None], N).copy(), 1), "SCFT")
    assert np.abs(f[3] - want).max() < 1e-14 * np.abs(want).max()
    assert all(np.all(v == 0) for v in f[:3])


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
    # proc 4: the second value is the x-vorticity (Compute_VyVz)
    f = ic.read_init_cond(cfg(4), data_dir=str(tmp_path))
    assert f[0][1, 1, 1] == 0.1 and abs(1j * (f[2][1, 1, 1] - f[1][1, 1, 1]) - 0.2) < 1e-15
    with pytest.raises(ValueError):
        ic.read_init_cond(cfg(511))
