"""Field files in the reference's text format (tg_write_field_file / tg_read_field_file; host
only): the exact text of Write_data_MPI, read-back to 12 significant digits, the
output_vx_vy_switch mode with V3 (and W3) rebuilt from incompressibility, and errors on short
files."""

import numpy as np
import pytest

from tarang_b200 import _lib as L
from tarang_b200 import ic


def test_exact_text(lib, tmp_path):
    from tarang_b200.solver import write_field_file
    N = (1, 2, 2)                               # (N1, N2, N3/2+1) = (1, 2, 2)
    a = np.array([1 + 2j, -3.5, 0.1 + 1e-13j, 123456.7890123456], dtype=np.complex128).reshape(1, 2, 2)
    p = tmp_path / "f.d"
    write_field_file(p, [a], time=0.5)
    want = "%% Time = 0.5\n(1,2) (-3.5,0) (0.1,1e-13) (123456.789012,0) \n\n"
    assert p.read_text() == want


def test_round_trip_12_digits(lib, tmp_path):
    from tarang_b200.solver import read_field_file, write_field_file
    N = (8, 6, 10)
    rng = np.random.default_rng(3)
    f = [rng.standard_normal((8, 6, 6)) + 1j * rng.standard_normal((8, 6, 6)) for _ in range(4)]
    p = tmp_path / "field.d"
    write_field_file(p, f, time=1.25)
    g = read_field_file(p, N, 4)
    for x, y in zip(f, g):
        assert np.abs(x - y).max() <= 1e-11 * np.abs(x).max()
    # appended snapshots: the reader takes the first one
    write_field_file(p, [2 * x for x in f], time=2.5, append=True)
    g = read_field_file(p, N, 4)
    assert np.abs(g[0] - f[0]).max() <= 1e-11 * np.abs(f[0]).max()
    # a file without the "%%" header line (what the reference's reader expects) reads alike
    body = "\n".join(l for l in p.read_text().splitlines() if not l.startswith("%"))
    q = tmp_path / "plain.d"
    q.write_text(body)
    assert np.abs(read_field_file(q, N, 4)[3] - f[3]).max() <= 1e-11 * np.abs(f[3]).max()


@pytest.mark.parametrize("basis,kf", [("FOUR", (1.0, 1.0, 1.0)), ("FOUR", (1.0, 0.5, 2.0))])
def test_vx_vy_mode_rebuilds_last_component(lib, tmp_path, basis, kf):
    from tarang_b200.solver import read_field_file, write_field_file
    N = (16, 16, 16)
    V = ic.random_phase_field(N, kfactor=kf, seed=8)      # divergence-free
    W = ic.random_phase_field(N, kfactor=kf, seed=9)
    p = tmp_path / "vxvy.d"
    write_field_file(p, V + W, vx_vy=True)
    text = p.read_text()
    assert text.count("(") == 2 * (2 * 16 * 16 * 9 + 16 * 16)
    g = read_field_file(p, N, 6, basis, kf, vx_vy=True)
    for x, y in zip(V + W, g):
        assert np.abs(x - y).max() <= 1e-10 * np.abs(x).max()


def test_short_or_malformed_file(lib, tmp_path):
    from tarang_b200.solver import read_field_file
    p = tmp_path / "short.d"
    p.write_text("(1,2) (3,4)\n")
    with pytest.raises(L.TarangError) as e:
        read_field_file(p, (2, 2, 2), 1)
    assert e.value.code == L.TG_ERR_ARG
    p.write_text("(1,2) (3,x) (5,6) (7,8)\n")
    with pytest.raises(L.TarangError):
        read_field_file(p, (1, 2, 2), 1)
    with pytest.raises(L.TarangError):
        read_field_file(tmp_path / "missing.d", (1, 2, 2), 1)


def test_reduced_exact_text(lib, tmp_path):
    """Output_field_reduced of a 4 x 4 x 4 field to (2, 2, 2): rows kx 0, 1 (FOUR, Nr1/2 + 1 rows
    then none below), ky 0, 1, kz 0, 1, no separators."""
    from tarang_b200.solver import write_field_file
    A = np.zeros((4, 4, 3), dtype=np.complex128)
    for i in range(4):
        for j in range(4):
            for k in range(3):
                A[i, j, k] = complex(100 * i + 10 * j + k, 1)
    p = tmp_path / "r.d"
    write_field_file(p, [A], time=1.0, reduced=(2, 2, 2))
    want = "%% Time = 1\n(0,1)(1,1)(10,1)(11,1)(100,1)(101,1)(110,1)(111,1)\n\n"
    assert p.read_text() == want


@pytest.mark.parametrize("basis", ["FOUR", "SCFT"])
def test_reduced_embeds_a_smaller_run(lib, tmp_path, basis):
    """A field file of an Nr grid read with N_in_reduced = Nr into an N grid: every mode of the
    smaller grid lands at the same wavenumber; the +Nr/2 rows also fill -Nr/2; the rest is zero.
    Writing the N-grid field reduced to Nr gives back the smaller grid's text."""
    from tarang_b200.solver import read_field_file, write_field_file
    Nr, N = (8, 8, 8), (16, 12, 16)
    rng = np.random.default_rng(5)
    small = [rng.standard_normal((8, 8, 5)) + 1j * rng.standard_normal((8, 8, 5)) for _ in range(3)]
    p = tmp_path / "small.d"
    write_field_file(p, small, time=0.0)
    big = read_field_file(p, N, 3, basis, reduced=Nr)
    four = basis == "FOUR"
    for s_, b_ in zip(small, big):
        for i in range(8):
            kx = (i if i <= 4 else i - 8) if four else i
            li = kx % 16 if four else kx
            for j in range(8):
                ky = j if j <= 4 else j - 8
                assert np.allclose(b_[li, ky % 12, :5], s_[i, j, :5], rtol=1e-11, atol=0)
        # duplicated Nyquist rows and zeros elsewhere
        assert np.allclose(b_[:, 12 - 4, :5][[0, 1, 2, 3]], b_[:, 4, :5][[0, 1, 2, 3]])
        assert np.all(b_[:, :, 5:] == 0)
        if four:
            assert np.allclose(b_[16 - 4], b_[4])
            assert np.all(b_[5:12] == 0)
    q = tmp_path / "again.d"
    write_field_file(q, big, time=0.0, reduced=Nr, basis=basis)
    again = read_field_file(q, Nr, 3, basis, reduced=Nr)
    for s_, a_ in zip(small, again):
        assert np.abs(s_ - a_).max() <= 1e-11 * np.abs(s_).max()


def test_reduced_vx_vy_and_errors(lib, tmp_path):
    from tarang_b200.solver import read_field_file, write_field_file
    N, Nr = (16, 16, 16), (8, 8, 8)
    V = ic.random_phase_field(Nr, k0=2.0, seed=3)
    p = tmp_path / "vxvy.d"
    write_field_file(p, V, vx_vy=True)
    g = read_field_file(p, N, 3, vx_vy=True, reduced=Nr)
    # V3 rebuilt from incompressibility on the big grid; the stored corner equals the small field
    Kx = np.fft.fftfreq(16, 1 / 16)[:, None, None]
    Ky = np.fft.fftfreq(16, 1 / 16)[None, :, None]
    Kz = np.arange(9)[None, None, :]
    div = 1j * (Kx * g[0] + Ky * g[1] + Kz * g[2])
    assert np.abs(div[:, :, 1:]).max() <= 1e-10 * np.abs(g[0]).max()
    assert np.allclose(g[2][1, 1, :5], V[2][1, 1, :5], rtol=1e-9)
    with pytest.raises(L.TarangError):
        read_field_file(p, N, 3, reduced=(7, 8, 8))          # FOUR Nr1 odd
    with pytest.raises(L.TarangError):
        read_field_file(p, N, 3, reduced=(32, 8, 8))         # larger than N


@pytest.mark.gpu
def test_context_round_trip(lib, tmp_path):
    """Output_field of a context, read into a new context: the same stored state."""
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    s = IncFluid(N, physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3)
    s.set_V(ic.random_phase_field(N, seed=1))
    s.set_W(ic.random_phase_field(N, seed=2))
    s.step(3)
    p = tmp_path / "state.d"
    s.Output_field(p, vx_vy=True)
    t = IncFluid(N, physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3)
    t.Init_cond_from_file(p, vx_vy=True)
    for x, y in zip(s.state_fields(), t.state_fields()):
        assert np.abs(x - y).max() <= 1e-10 * np.abs(x).max()


PARA = """#run parameters (same layout as the reference's in/para.d)
#only the numbers are read; labels are single words
# grid
{N1}	{N2}	{N3}


(1)solver-meta	2	6	2
(2)solver-int		1	0
(3)solver-float		1.0	1.0	1.0	{Ra}	{Pr}	1.0
(4)solver-string	PRLARGE	ULARGE


(1)basis	{basis}
(2)alias	DEALIAS
(3)scheme	RK4
(4)in-mode	ASCII
(5)out-mode	ASCII


(1)a 0
(2)b 0
(3)c 0
(4)d 0
(5)e 0
(6)f 0
(7)g 0
(8)h 0
(9)i 0
(10)j 0
(11)k 0
(12)l 0
(13)m 0
(14)n 3
(15)o 0
(16)p 0
(17)q 0
(18)r 0
(19)outvxvy 1
(20)invxvy 0
(21)fw 1
(22)ft 1


#coefficients
{nu}	{kappa}

#hyper
0	0


T0 	0
T1 	0.25
Tdt	{dt}
Tb	0.001
Ta	0.001
Ts	10.0


(1)s1 0.1
(2)s2 0.1
(3)s3 10
(4)s4 0.1
(5)s5 10
(6)s6 0.1
(7)s7 0.1
(8)s8 1000
(9)s9 100
(10)s10 100
(11)s11 100
(12)s12 100
(13)s13 100
(14)s14 100
(15)s15 100
(16)s16 100
(17)s17 100
(18)s18 100
(19)s19 0.1


(1)m1 0
(2)m2 5
(3)m3 5
(4)m4 1
(5)m5 10
(6)reduced	8	8	8


ET:(1)e1 0
(2)e2 {S}
(3)e3 {S}
(4)e4 9
(5)e5 5
(6)e6 6
(7)e7 5
(8)e8 0
(9)e9 0
(10)e10 0
(11)e11 0
(12)e12 0


(1)nk	2
(2)nr	1

1	0	1
2	1	0

0	0	1


(1)in-meta	1	1	1
(2)in-int	0
(3)in-float	1.0
(4)in-string	X


(1)force-meta	1	4	1
(2)force-int	{proc}
(3)force-float	2.0	3.0	0.1	0.0
(4)force-string	X
"""


def test_read_para_fluid(lib):
    from tarang_b200.para import config_from_para, read_para
    text = PARA.format(N1=64, N2=32, N3=16, Ra=0, Pr=0, basis="FOUR", nu=0.003, kappa=0, dt=0.0005, S=16, proc=1)
    p = read_para(text, n_fields=1)
    assert p["N"][1:] == [64, 32, 16] and p["switches"][19] == 1 and p["ET"][3] == 16
    assert p["out_k"] == [(1, 0, 1), (2, 1, 0)] and p["out_r"] == [(0, 0, 1)]
    c = config_from_para(p, "FLUID")
    assert c["N"] == (64, 32, 16) and c["nu"] == 0.003 and c["dt"] == 0.0005 and c["n_shells"] == 16
    assert c["force"] == dict(kind="energy_supply", inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    assert c["run"]["Tfinal"] == 0.25 and c["run"]["output_vx_vy"] == 1
    from tarang_b200.solver import make_config
    kw = dict(c)
    kw.pop("run")
    cfg = make_config(**kw)
    assert cfg.force_kind == L.TG_FORCE_ENERGY_SUPPLY and list(cfg.N) == [64, 32, 16]
    # force_field_proc 2 (constant energy and helicity) with the same parameters; for MHD the
    # next two are B's energy and helicity ratio, for a passive scalar the next one its energy
    text2 = PARA.format(N1=64, N2=32, N3=16, Ra=0, Pr=0, basis="FOUR", nu=0.003, kappa=0, dt=0.0005, S=16, proc=2)
    c2 = config_from_para(read_para(text2, n_fields=1), "FLUID")
    assert c2["force"] == dict(kind="energy_helicity", inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    kw = dict(c2)
    kw.pop("run")
    assert make_config(**kw).force_kind == L.TG_FORCE_ENERGY_HELICITY
    cm = make_config((16, 16, 16), physics="MHD", force=dict(kind="energy_helicity", inner=1.0, outer=2.0, eps=0.3,
                                                                 eps_h=0.2, eps_W=0.4, eps_hW=-0.1))
    assert list(cm.force_para) == [1.0, 2.0, 0.3, 0.2, 0.4, -0.1]
    cs = make_config((16, 16, 16), physics="SCALAR", force=dict(inner=1.0, outer=2.0, eps=0.3, eps_T=0.5))
    assert cs.force_kind == L.TG_FORCE_ENERGY_SUPPLY and list(cs.force_para) == [1.0, 2.0, 0.3, 0.0, 0.5, 0.0]


def test_read_para_scheme_and_hyper(lib):
    """integ_scheme and, with hyper_dissipation_switch (switches(1)) on, the hyper coefficients of
    U and of the scalar reach the configuration."""
    from tarang_b200.para import config_from_para, read_para
    from tarang_b200.solver import make_config
    text = PARA.format(N1=16, N2=16, N3=16, Ra=0, Pr=0, basis="FOUR", nu=0.003, kappa=0.002, dt=0.0005, S=8, proc=1)
    text = text.replace("(3)scheme\tRK4", "(3)scheme\tRK2").replace("(1)a 0", "(1)a 1")
    text = text.replace("#hyper\n0\t0", "#hyper\n1e-6\t2e-6")
    c = config_from_para(read_para(text, n_fields=2), "SCALAR")
    assert c["scheme"] == "RK2" and c["hyper_nu"] == 1e-6 and c["hyper_kappa"] == 2e-6
    kw = dict(c)
    kw.pop("run")
    cfg = make_config(**kw)
    assert cfg.scheme == L.TG_RK2 and cfg.hyper_nu == 1e-6 and cfg.hyper_kappa == 2e-6
    # switch off: the coefficients are ignored, as the reference ignores them
    c0 = config_from_para(read_para(text.replace("(1)a 1", "(1)a 0"), n_fields=2), "SCALAR")
    assert c0["hyper_nu"] == 0.0 and c0["hyper_kappa"] == 0.0
    with pytest.raises(ValueError):
        config_from_para(read_para(text.replace("(3)scheme\tRK2", "(3)scheme\tAB2"), n_fields=2), "SCALAR")


def test_read_para_convection(lib):
    import math
    from tarang_b200.para import config_from_para, read_para
    text = PARA.format(N1=33, N2=32, N3=32, Ra=1e6, Pr=1.0, basis="SCFT", nu=0, kappa=0, dt=1e-4, S=10, proc=51)
    c = config_from_para(read_para(text, n_fields=2), "RB")
    k0 = math.pi / math.sqrt(2.0)
    assert c["kfactor"] == (math.pi, k0, k0) and c["Ra"] == 1e6 and c["Pr"] == 1.0
    assert c["Pr_switch"] == "PRLARGE" and c["RB_Uscaling"] == "ULARGE" and "force" not in c


def test_reference_para_files_parse(lib):
    """The reference's own example para.d files (trunk/info/new4.21/{fluid3d,mhd3d,RB}/in/para.d,
    copied into tests/golden/para by tests/golden/make_para_fixtures.py)."""
    import math
    import os
    from tarang_b200.para import config_from_para, read_para
    from tarang_b200.solver import make_config
    base = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "para")
    got = {}
    for kind, d, n in (("FLUID", "fluid3d", 1), ("MHD", "mhd3d", 2), ("RB", "RB", 2)):
        c = config_from_para(read_para(os.path.join(base, d + ".para.d"), n_fields=n), kind)
        assert c["dt"] == 1e-3 and c["n_shells"] == 10 and c["dealias"] is True
        assert c["run"]["Tfinal"] == 0.005 and c["run"]["N_out_reduced"] == (4, 4, 4)
        kw = dict(c)
        kw.pop("run")
        make_config(**kw)
        got[kind] = c
    assert got["FLUID"]["N"] == (8, 8, 8) and got["FLUID"]["basis"] == "FOUR"
    assert got["MHD"]["N"] == (16, 16, 16) and got["MHD"]["physics"] == "MHD"
    rb = got["RB"]
    assert rb["basis"] == "SCFT" and rb["Pr"] == 6.8 and rb["Pr_switch"] == "PRLARGE"
    assert rb["RB_Uscaling"] == "USMALL" and abs(rb["kfactor"][1] - math.pi / math.sqrt(2.0)) < 1e-15
