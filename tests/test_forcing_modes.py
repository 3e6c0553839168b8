"""Fixed-mode forcings and the Coriolis configuration on the host: the mode lists of
tarang_b200.forcing against the oracle's dense force fields (Taylor-Green, ABC), the given-mode
forcing's incompressibility and conjugate modes, the force-modes file reader, and the para.d
mapping of force_field_proc 3, 4, 5 and 21.  The GPU runs of these forces are in
test_gpu_forcing.py."""

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import forcing, ic


def dense(k, F, N, comp, basis="FOUR"):
    N1, N2, N3 = N
    A = np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128)
    for (kx, ky, kz), f in zip(k, F[:, comp]):
        lx = kx if (basis == "SCFT" or kx >= 0) else kx + N1
        A[lx, ky % N2, kz] = f
    return A


@pytest.mark.parametrize("basis", ["FOUR", "SCFT"])
@pytest.mark.parametrize("k0", [1, 2, 3])
def test_taylor_green_modes_match_oracle(basis, k0):
    N = (16, 16, 16)
    k, F = forcing.taylor_green_modes(N, k0, 0.7, basis)
    want = o.taylor_green_force(N, k0, 0.7, basis)
    for c in range(3):
        assert np.array_equal(dense(k, F, N, c, basis), want[c])
    assert F.shape == (len(k), 3)


def test_taylor_green_force_is_the_real_space_field():
    """The FOUR Taylor-Green force transforms to amp (sin cos cos, -cos sin cos, 0)."""
    N = (16, 16, 16)
    amp, k0 = 1.3, 2
    F = o.taylor_green_force(N, k0, amp)
    x = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    fx = o.inverse_four(F[0], 16)
    fy = o.inverse_four(F[1], 16)
    assert np.abs(fx - amp * np.sin(k0 * X) * np.cos(k0 * Y) * np.cos(k0 * Z)).max() < 1e-13
    assert np.abs(fy + amp * np.cos(k0 * X) * np.sin(k0 * Y) * np.cos(k0 * Z)).max() < 1e-13


def test_abc_modes_match_oracle_and_real_space():
    N = (16, 16, 16)
    k0, amp, A, B, C = 1, 0.9, 1.0, 0.7, 0.4
    k, F = forcing.abc_modes(N, k0, amp, A, B, C)
    want = o.abc_force(N, k0, amp, A, B, C)
    for c in range(3):
        assert np.array_equal(dense(k, F, N, c), want[c])
    x = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = [o.inverse_four(w, 16) for w in want]
    assert np.abs(f[0] - amp * (B * np.cos(k0 * Y) + C * np.sin(k0 * Z))).max() < 1e-13
    assert np.abs(f[1] - amp * (A * np.sin(k0 * X) + C * np.cos(k0 * Z))).max() < 1e-13
    assert np.abs(f[2] - amp * (A * np.cos(k0 * X) + B * np.sin(k0 * Y))).max() < 1e-13


def test_mhd_and_scalar_columns():
    N = (16, 16, 16)
    k, F = forcing.taylor_green_modes(N, 1, 1.0, physics="MHD", ampW=0.5)
    assert F.shape[1] == 6 and np.allclose(F[:, 3:6], 0.5 * F[:, 0:3])
    k, F = forcing.abc_modes(N, 1, 1.0, 1, 1, 1, physics="SCALAR")
    assert F.shape[1] == 4 and np.all(F[:, 3] == 0)
    with pytest.raises(ValueError):
        forcing.taylor_green_modes(N, 1, 1.0, physics="RB")


@pytest.mark.parametrize("basis", ["FOUR", "SCFT"])
def test_given_modes_incompressible_with_conjugates(basis):
    N = (16, 16, 16)
    kf = (1.0, 0.5, 2.0)
    entries = [(1, 2, 3, 0.3 + 0.1j, -0.2 + 0.4j), (2, 1, 0, 0.5 + 0.2j, 0.1 - 0.3j), (3, 0, 0, 0.7 + 0.5j, 0.2 + 0.6j)]
    k, F = forcing.given_modes(entries, N, kf, basis)
    kk = {tuple(x): f for x, f in zip(k.tolist(), F)}
    for (kx, ky, kz), f in kk.items():
        dx = (1j * kx * kf[0] * f[0]) if basis == "FOUR" else (kx * kf[0] * f[0])
        div = dx + 1j * ky * kf[1] * f[1] + 1j * kz * kf[2] * f[2]
        assert abs(div) < 1e-14
    # kz = 0 entries: the read values are (Fx, Fz); the conjugate mode is forced too
    f = kk[(2, 1, 0)]
    assert f[0] == 0.5 + 0.2j and f[2] == 0.1 - 0.3j
    conj = (-2, -1, 0) if basis == "FOUR" else (2, -1, 0)
    assert np.array_equal(kk[conj], np.conj(f))
    # on the kx axis the given Fx is Fy, and Fx = 0
    f = kk[(3, 0, 0)]
    if basis == "FOUR":
        assert f[0] == 0 and f[1] == 0.7 + 0.5j and np.array_equal(kk[(-3, 0, 0)], np.conj(f))
    else:
        assert f[0] == 0 and f[1] == 0.7 and f[2] == 0.2


def test_given_modes_mhd_and_scalar():
    N = (16, 16, 16)
    k, F = forcing.given_modes([(1, 1, 1, 0.1, 0.2, 0.3, 0.4)], N, physics="MHD")
    assert F.shape == (1, 6)
    assert abs(1j * F[0, 3] + 1j * F[0, 4] + 1j * F[0, 5]) < 1e-15
    k, F = forcing.given_modes([(1, 1, 0, 0.1, 0.2, 0.5j)], N, physics="SCALAR")
    assert F.shape == (2, 4) and F[0, 3] == 0.5j and F[1, 3] == -0.5j


@pytest.mark.parametrize("basis", ["FOUR", "SCFT"])
def test_given_modes_vorticity(basis):
    """Compute_force_given_modes_VORTICITY / Init_cond_modes_VORTICITY: (Vx, Omega_x) give a
    divergence-free mode whose x-vorticity i(Ky Vz - Kz Vy) is Omega_x; on the kx axis the mode
    is zero (Compute_VyVz); the conjugates on kz = 0 follow the same rule as the simple modes."""
    N = (16, 16, 16)
    kf = (1.0, 0.5, 2.0)
    entries = [(1, 2, 3, 0.3 + 0.1j, -0.2 + 0.4j), (2, 1, 0, 0.5 + 0.2j, 0.1 - 0.3j), (3, 0, 0, 0.7, 0.2)]
    k, F = forcing.given_modes(entries, N, kf, basis, rule="vorticity")
    kk = {tuple(x): f for x, f in zip(k.tolist(), F)}
    for (kx, ky, kz, vx, om) in entries[:2]:
        f = kk[(kx, ky, kz)]
        dx = (1j * kx * kf[0] * f[0]) if basis == "FOUR" else (kx * kf[0] * f[0])
        assert abs(dx + 1j * ky * kf[1] * f[1] + 1j * kz * kf[2] * f[2]) < 1e-14
        assert abs(1j * (ky * kf[1] * f[2] - kz * kf[2] * f[1]) - om) < 1e-14 and f[0] == vx
    assert np.all(kk[(3, 0, 0)] == 0)
    conj = (-2, -1, 0) if basis == "FOUR" else (2, -1, 0)
    assert np.array_equal(kk[conj], np.conj(kk[(2, 1, 0)]))
    # MHD: each vector by its own (x, Omega_x); scalar: G as given
    k, F = forcing.given_modes([(1, 1, 1, 0.1, 0.2, 0.3, 0.4)], N, physics="MHD", rule="vorticity")
    assert abs(1j * (F[0, 5] - F[0, 4]) - 0.4) < 1e-15 and abs(1j * (F[0, 2] - F[0, 1]) - 0.2) < 1e-15
    k, F = forcing.given_modes([(1, 1, 2, 0.1, 0.2, 0.5j)], N, physics="SCALAR", rule="vorticity")
    assert F[0, 3] == 0.5j
    V = ic.modes_field(entries, N, kf, basis, rule="vorticity")
    assert V[1][2, 1, 0] == kk[(2, 1, 0)][1]


def test_read_force_modes_file(tmp_path):
    p = tmp_path / "force_field_in.d"
    p.write_text("1 2 3 (0.5,0.25) (1,-1)\n2 0 0 (0.1,0) 2.0\n64 0 0\n5 5 5 (9,9) (9,9)\n")
    e = forcing.read_force_modes_file(p, 16)
    assert e == [(1, 2, 3, 0.5 + 0.25j, 1 - 1j), (2, 0, 0, 0.1 + 0j, 2.0 + 0j)]
    p.write_text("1 2 3 (0.5,0.25)\n")
    with pytest.raises(ValueError):
        forcing.read_force_modes_file(p, 16)


def test_para_force_procs(lib):
    from tests.test_field_io import PARA
    from tarang_b200.para import config_from_para, read_para
    from tarang_b200.solver import make_config
    from tarang_b200 import _lib as L

    def cfg_for(proc, floats, ints=None):
        text = PARA.format(N1=32, N2=32, N3=32, Ra=0, Pr=0, basis="FOUR", nu=0.01, kappa=0, dt=1e-3, S=12, proc=proc)
        text = text.replace("(3)force-float	2.0	3.0	0.1	0.0", "(3)force-float	" + "	".join(map(str, floats)))
        nf = len(floats)
        ni = 1 + len(ints or [])
        text = text.replace("(1)force-meta	1	4	1", f"(1)force-meta	{ni}	{nf}	1")
        if ints:
            text = text.replace(f"(2)force-int	{proc}", f"(2)force-int	{proc}	" + "	".join(map(str, ints)))
        return config_from_para(read_para(text, n_fields=1), "FLUID")

    c = cfg_for(3, [2, 0.5, 0.0])
    assert c["force"] == dict(kind="modes") and c["run"]["force_modes"]["kind"] == "taylor_green"
    assert c["run"]["force_modes"]["k0"] == 2 and c["run"]["force_modes"]["amp"] == 0.5
    c = cfg_for(4, [1, 1.0, 0.5, 0.25, 2.0])
    fm = c["run"]["force_modes"]
    assert (fm["k0"], fm["A"], fm["B"], fm["C"], fm["amp"]) == (1, 1.0, 0.5, 0.25, 2.0)
    c = cfg_for(5, [0.0])
    assert c["run"]["force_modes"]["kind"] == "given_modes"
    c = cfg_for(21, [0.5, 1.0, 2.0])
    assert c["force"] == dict(kind="coriolis", omega=(0.5, 1.0, 2.0))
    c = cfg_for(21, [3.0], ints=[1, 3])
    assert c["force"]["omega"] == (0.0, 0.0, 3.0)
    kw = dict(c)
    kw.pop("run")
    cfg = make_config(**kw)
    assert cfg.force_kind == L.TG_FORCE_CORIOLIS and list(cfg.force_para[:3]) == [0.0, 0.0, 3.0]
    c = cfg_for(6, [0.0])
    assert c["force"] == dict(kind="modes") and c["run"]["force_modes"]["rule"] == "vorticity"
    with pytest.raises(ValueError):
        cfg_for(7, [0.0])


def test_coriolis_oracle_identities():
    """Force = V x Omega: orthogonal to V mode by mode (Re F . V* = 0) and to Omega."""
    from tarang_b200 import ic
    N = (16, 16, 16)
    V = ic.random_phase_field(N, seed=4)
    om = (0.3, -0.7, 1.1)
    F = o.force_coriolis(V, om)
    dot = sum(np.real(f * np.conj(v)) for f, v in zip(F, V))
    assert np.abs(dot).max() < 1e-16
    assert np.abs(sum(w * f for w, f in zip(om, F))).max() < 1e-16


def test_force_modes_for_para(tmp_path):
    """para.force_modes_for: the mode list of a parsed para.d (proc 3 and proc 5 with its
    in/force_field_in.d)."""
    from tests.test_field_io import PARA
    from tarang_b200.para import config_from_para, force_modes_for, read_para

    def para(proc, floats):
        t = PARA.format(N1=32, N2=32, N3=32, Ra=0, Pr=0, basis="FOUR", nu=0.01, kappa=0, dt=1e-3, S=12, proc=proc)
        t = t.replace("(3)force-float	2.0	3.0	0.1	0.0", "(3)force-float	" + "	".join(map(str, floats)))
        return t.replace("(1)force-meta	1	4	1", f"(1)force-meta	1	{len(floats)}	1")

    c = config_from_para(read_para(para(3, [2, 0.5, 0.0]), n_fields=1), "FLUID")
    k, F = force_modes_for(c)
    k2, F2 = forcing.taylor_green_modes((32, 32, 32), 2, 0.5)
    assert np.array_equal(k, k2) and np.array_equal(F, F2)
    (tmp_path / "in").mkdir()
    (tmp_path / "in" / "force_field_in.d").write_text("1 1 1 (0.1,0) (0.2,0)\n99 0 0\n")
    c = config_from_para(read_para(para(5, [0.0]), n_fields=1), "FLUID")
    k, F = force_modes_for(c, data_dir=str(tmp_path))
    assert k.tolist() == [[1, 1, 1]] and abs(F[0, 0] - 0.1) < 1e-15
    c = config_from_para(read_para(para(1, [2.0, 3.0, 0.1, 0.0]), n_fields=1), "FLUID")
    assert force_modes_for(c) is None


def test_para_rb_rotation(lib):
    from tests.test_field_io import PARA
    from tarang_b200.para import config_from_para, read_para
    from tarang_b200.solver import make_config
    from tarang_b200 import _lib as L
    t = PARA.format(N1=33, N2=32, N3=32, Ra=1e6, Pr=1.0, basis="SCFT", nu=0, kappa=0, dt=1e-4, S=10, proc=52)
    t = t.replace("(3)force-float	2.0	3.0	0.1	0.0", "(3)force-float	0.0	0.0	4.0")
    t = t.replace("(1)force-meta	1	4	1", "(1)force-meta	1	3	1")
    c = config_from_para(read_para(t, n_fields=2), "RB")
    assert c["force"] == dict(kind="rb_rotation", omega=(0.0, 0.0, 4.0))
    kw = dict(c)
    kw.pop("run")
    cfg = make_config(**kw)
    assert cfg.force_kind == L.TG_FORCE_RB_ROTATION and list(cfg.force_para[:3]) == [0.0, 0.0, 4.0]


def test_six_mode_force_and_field():
    """Setup_SIX_MODE_force_field / Setup_SIX_MODE_field: eight divergence-free modes off the kz = 0
    plane; the dynamo force (proc 101, MHD) drives the velocity only; the initial condition
    (field_input_proc 101) fills V and W from their own amplitudes."""
    N = (16, 16, 16)
    t = forcing.six_mode_table(2, 0.3, 0.5, 0.7, 0.4)
    assert len(t) == 8
    for (kx, ky, kz), v in t.items():
        assert kz > 0 and abs(kx * v[0] + ky * v[1] + kz * v[2]) < 1e-15
    k, F = forcing.six_mode_modes(N, 2, 0.3, 0.5, 0.7, 0.4)
    assert F.shape == (8, 6) and np.all(F[:, 3:] == 0)
    f = ic.six_mode_field(N, 2, (0.3, 0.5, 0.7, 0.4), (0.1, 0.2, 0.3, -0.5))
    assert f[0][2, 0, 2] == t[(2, 0, 2)][0] and f[4][(-2) % 16, 2, 4] == forcing.six_mode_table(2, 0.1, 0.2, 0.3, -0.5)[(-2, 2, 4)][1]


def test_para_liquid_metal_and_six_mode(lib):
    from tests.test_field_io import PARA
    from tarang_b200.para import config_from_para, force_modes_for, read_para
    from tarang_b200.solver import make_config
    from tarang_b200 import _lib as L
    t = PARA.format(N1=32, N2=32, N3=32, Ra=0, Pr=0, basis="FOUR", nu=0.01, kappa=0, dt=1e-3, S=12, proc=101)
    t = t.replace("(3)force-float	2.0	3.0	0.1	0.0", "(3)force-float	1.0	0.0	2.0	0.5	0.25")
    t = t.replace("(1)force-meta	1	4	1", "(1)force-meta	1	5	1")
    c = config_from_para(read_para(t, n_fields=1), "FLUID")
    assert c["force"] == dict(kind="liquid_metal", B0=(1.0, 0.0, 2.0))
    kw = dict(c)
    kw.pop("run")
    cfg = make_config(**kw)
    assert cfg.force_kind == L.TG_FORCE_LIQUID_METAL and list(cfg.force_para[:3]) == [1.0, 0.0, 2.0]
    c = config_from_para(read_para(t, n_fields=2), "MHD")
    assert c["force"] == dict(kind="modes") and c["run"]["force_modes"]["kind"] == "six_mode"
    k, F = force_modes_for(c)
    k2, F2 = forcing.six_mode_modes((32, 32, 32), 1, 0.0, 2.0, 0.5, 0.25)
    assert np.array_equal(k, k2) and np.array_equal(F, F2)
