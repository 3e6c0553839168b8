"""Kernel variants that compute the same transform agree to rounding: fields after a few steps
with the TMA-staged axis passes equal those with the register-staged ones (TG_AXIS_TMA=0); for
the N3 = 256 z-pass, those of the eight-lane network (the default) equal those of the 32-lane
transposed network (TG_ZPASS_OCT=0), and those equal the five-stage shuffle network's
(TG_ZPASS_OCT=0 TG_ZPASS_NET=0); for N3 = 128 the eight-lane network equals the five-stage one
(TG_ZPASS_OCT=0); all to 1e-14 (FP64) / 1e-6 (FP32-mixed) relative L2, for every
precision and physics on the fast path, dealiased rows and full rows (the kernels round
differently)."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, %r)
from tarang_b200 import ic
from tarang_b200.solver import IncFluid
cases = json.loads(sys.argv[1])
out = {}
for name, N, kw in cases:
    N = tuple(N)
    s = IncFluid(N, **kw)
    s.set_V(ic.random_phase_field(N, seed=3))
    if kw.get("physics") == "MHD":
        s.set_W(ic.random_phase_field(N, k0=3.0, seed=4))
    if kw.get("physics") in ("SCALAR", "RB"):
        s.set_T(ic.random_phase_field(N, seed=5)[0])
    s.step(3)
    f = s.get_V() + (s.get_W() if kw.get("physics") == "MHD" else [])
    f += [s.get_T()] if kw.get("physics") in ("SCALAR", "RB") else []
    out[name] = [x.view(np.float64).tobytes().hex() for x in f]
print(json.dumps(out))
""" % ROOT

CASES = [
    ("fluid64_fp64", (64, 64, 64), dict(nu=2e-3, dt=1e-3)),
    ("fluid64_fp32", (64, 64, 64), dict(nu=2e-3, dt=1e-3, precision="FP32")),
    ("fluid_aniso", (32, 128, 64), dict(nu=2e-3, dt=1e-3)),
    ("mhd32_fp64", (32, 32, 32), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3)),
    ("mhd32_fp32", (32, 32, 32), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3, precision="FP32")),
]


def run(env_tma, cases=CASES, var="TG_AXIS_TMA", extra=None):
    env = dict(os.environ)
    env[var] = env_tma
    env.update(extra or {})
    r = subprocess.run([sys.executable, "-c", SCRIPT, json.dumps(cases)], capture_output=True, text=True,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def fields(hexes):
    return [np.frombuffer(bytes.fromhex(h), dtype=np.float64) for h in hexes]


def compare(a, b, cases):
    for name, _, kw in cases:
        x, y = fields(a[name]), fields(b[name])
        num = np.sqrt(sum(float(np.sum((p - q) ** 2)) for p, q in zip(x, y)))
        den = np.sqrt(sum(float(np.sum(q ** 2)) for q in y))
        tol = 1e-6 if kw.get("precision") == "FP32" else 1e-14
        assert num / den < tol, (name, num / den)


def test_tma_axis_passes_match_register_staged(lib):
    compare(run("1"), run("0"), CASES)


ZCASES = [
    ("fluid256z_fp64", (32, 32, 256), dict(nu=2e-3, dt=1e-3)),
    ("fluid256z_fp32", (32, 32, 256), dict(nu=2e-3, dt=1e-3, precision="FP32")),
    ("mhd256z_fp64", (16, 32, 256), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3)),
    ("scalar256z_fp32", (16, 16, 256), dict(physics="SCALAR", nu=2e-3, kappa=3e-3, dt=1e-3, precision="FP32")),
]


def test_transposed_z_network_matches_shuffle_stages(lib):
    off = {"TG_ZPASS_OCT": "0"}
    compare(run("1", ZCASES, "TG_ZPASS_NET", off), run("0", ZCASES, "TG_ZPASS_NET", off), ZCASES)


KF_RB = [3.141592653589793, 2.221441469079183, 2.221441469079183]
OCASES = ZCASES + [
    ("fluid256z_full", (16, 16, 256), dict(nu=2e-3, dt=1e-3, dealias=False)),
    ("mhd256z_fp32", (16, 32, 256), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3, precision="FP32")),
    ("mhd256z_full", (16, 16, 256), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3, dealias=False)),
    ("scalar256z_fp64", (16, 16, 256), dict(physics="SCALAR", nu=2e-3, kappa=3e-3, dt=1e-3)),
    ("rb256z_fp64", (17, 16, 256), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4)),
    ("rb256z_fp32", (17, 16, 256), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4,
                                        precision="FP32")),
]


def test_eight_lane_z_network_matches_transposed_network(lib):
    compare(run("1", OCASES, "TG_ZPASS_OCT"), run("0", OCASES, "TG_ZPASS_OCT"), OCASES)


O64CASES = [
    ("fluid128z_fp64", (32, 32, 128), dict(nu=2e-3, dt=1e-3)),
    ("fluid128z_fp32", (32, 32, 128), dict(nu=2e-3, dt=1e-3, precision="FP32")),
    ("fluid128z_full", (16, 16, 128), dict(nu=2e-3, dt=1e-3, dealias=False)),
    ("fluid128z_full32", (16, 16, 128), dict(nu=2e-3, dt=1e-3, dealias=False, precision="FP32")),
    ("mhd128z_fp64", (16, 32, 128), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3)),
    ("mhd128z_fp32", (16, 32, 128), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3, precision="FP32")),
    ("mhd128z_full", (16, 16, 128), dict(physics="MHD", nu=2e-3, eta=3e-3, dt=1e-3, dealias=False)),
    ("scalar128z_fp64", (16, 16, 128), dict(physics="SCALAR", nu=2e-3, kappa=3e-3, dt=1e-3)),
    ("scalar128z_fp32", (16, 16, 128), dict(physics="SCALAR", nu=2e-3, kappa=3e-3, dt=1e-3, precision="FP32")),
    ("rb128z_fp64", (17, 16, 128), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4)),
    ("rb128z_fp32", (17, 16, 128), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4,
                                        precision="FP32")),
]


def test_eight_lane_z_network_n3_128_matches_warp_network(lib):
    """N3 = 128 (M = 64): k_z_prod_oct64 against the 32-lane radix-2 network (TG_ZPASS_OCT=0)."""
    compare(run("1", O64CASES, "TG_ZPASS_OCT"), run("0", O64CASES, "TG_ZPASS_OCT"), O64CASES)


RCASES = [
    ("rb129_fp64", (129, 32, 32), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4)),
    ("rb129_fp32", (129, 32, 32), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4,
                                       precision="FP32")),
    ("rb65_fp64", (65, 16, 32), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4)),
    ("rb33_fp64", (33, 16, 16), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4)),
    ("scft_fluid_full", (24, 16, 32), dict(basis="SCFT", nu=2e-3, dt=1e-3, kfactor=KF_RB, dealias=False)),
]


def test_register_tiled_x_pass_matches_matrix_product(lib):
    """The SCFT x-pass as a register-tiled matrix product (default) equals the shared-memory
    matrix product (TG_R2R_GEMM=0): same sums in the same order."""
    compare(run("1", RCASES, "TG_R2R_GEMM"), run("0", RCASES, "TG_R2R_GEMM"), RCASES)


TCASES = [
    ("rb129_fp32", (129, 32, 32), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4,
                                       precision="FP32")),
    ("rb65_fp32", (65, 32, 64), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4,
                                     precision="FP32")),
    ("rb33_fp32", (33, 16, 16), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4,
                                     precision="FP32")),
    ("scft_fluid_fp32", (24, 16, 32), dict(basis="SCFT", nu=2e-3, dt=1e-3, kfactor=KF_RB, precision="FP32")),
    ("scft_fluid_full32", (24, 16, 32), dict(basis="SCFT", nu=2e-3, dt=1e-3, kfactor=KF_RB, dealias=False,
                                             precision="FP32")),
    # several tiles per block: both accumulators, the operand ring and the register ring wrap
    ("rb65x128_fp32", (65, 128, 128), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4,
                                           precision="FP32")),
]


def test_tensor_core_x_pass_matches_register_tiled(lib):
    """FP32 forms: the SCFT x-pass on the tensor cores (3xTF32 tcgen05, TG_R2R_TC=1) against the
    register-tiled FP32 matrix product (TG_R2R_TC=0), to FP32-mixed rounding."""
    compare(run("1", TCASES, "TG_R2R_TC"), run("0", TCASES, "TG_R2R_TC"), TCASES)


SERVE_SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, %r)
from tarang_b200 import ic
from tarang_b200.serving import Server
from tarang_b200.solver import IncFluid
KF = (3.141592653589793, 2.221441469079183, 2.221441469079183)
N = (33, 32, 64)
out = {}
reqs = []
for j in range(3):
    cfg = dict(N=N, basis="SCFT", physics="RB", Ra=1e4 * (1 + j), Pr=1.0, kfactor=KF, dt=1e-4, precision="FP32")
    f = np.stack(ic.random_phase_field(N, seed=40 + j) + [ic.random_phase_field(N, seed=50 + j)[0]])
    reqs.append((cfg, f, 3 + j))
same = []
with Server(hbm_budget=8e9, max_batch=4) as srv:
    ids = [srv.submit(c, f, k) for c, f, k in reqs]
    srv.drain()
    for rid, (c, f, k) in zip(ids, reqs):
        c = dict(c)
        s = IncFluid(c.pop("N"), **c)
        s.set_V(list(f[:3]))
        s.set_T(f[3])
        s.step(k)
        want = s.get_V() + [s.get_T()]
        s.close()
        got = srv.result(rid)
        same.append(all(np.array_equal(a.view(np.float64), b.view(np.float64)) for a, b in zip(got, want)))
print(json.dumps(same))
""" % ROOT


def test_tensor_core_x_pass_batched_equals_lone(lib):
    """With the tensor-core x-pass forced on (TG_R2R_TC=1), requests served in one batch equal
    their lone-context runs bit for bit (a tile's result does not depend on the launch shape)."""
    env = dict(os.environ, TG_R2R_TC="1")
    r = subprocess.run([sys.executable, "-c", SERVE_SCRIPT], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1]) == [True, True, True]
