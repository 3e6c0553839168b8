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
    assert c["force"] == dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)
    assert c["run"]["Tfinal"] == 0.25 and c["run"]["output_vx_vy"] == 1
    from tarang_b200.solver import make_config
    kw = dict(c)
    kw.pop("run")
    cfg = make_config(**kw)
    assert cfg.force_kind == L.TG_FORCE_ENERGY_SUPPLY and list(cfg.N) == [64, 32, 16]


def test_read_para_convection(lib):
    import math
    from tarang_b200.para import config_from_para, read_para
    text = PARA.format(N1=33, N2=32, N3=32, Ra=1e6, Pr=1.0, basis="SCFT", nu=0, kappa=0, dt=1e-4, S=10, proc=51)
    c = config_from_para(read_para(text, n_fields=2), "RB")
    k0 = math.pi / math.sqrt(2.0)
    assert c["kfactor"] == (math.pi, k0, k0) and c["Ra"] == 1e6 and c["Pr"] == 1.0
    assert c["Pr_switch"] == "PRLARGE" and c["RB_Uscaling"] == "ULARGE" and "force" not in c


def test_reference_para_files_parse(lib):
    """The reference's own example para.d files, where the reference tree is present."""
    import os
    from tarang_b200.para import config_from_para, read_para
    base = "/root/reference/trunk/info/new4.21"
    if not os.path.isdir(base):
        pytest.skip("reference tree absent")
    for kind, d, n in (("FLUID", "fluid3d", 1), ("MHD", "mhd3d", 2), ("RB", "RB", 2)):
        path = os.path.join(base, d, "in", "para.d")
        c = config_from_para(read_para(path, n_fields=n), kind)
        assert c["basis"] in ("FOUR", "SCFT") and c["dt"] > 0 and c["n_shells"] > 0
