"""The C++ host side of the boundary: a C++ driver of the reference's fluid loop
(Ifluid_main.cc:258-301), written against the mirror classes of include/tarang_b200.hpp and
built with g++ against libtarang_gpu.so, gives the same fields, energies and energy-transfer
tables as the Python mirror making the same calls, bit for bit, both method by method and with
the fused step; and it agrees with the oracle."""

import math
import os
import subprocess

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = (32, 32, 32)
NU, DT, STEPS, S = 1e-3, 5e-4, 4, 16
FORCE = dict(inner=2.0, outer=3.0, eps=0.1, eps_h=0.0)


def build_driver(tmp):
    exe = os.path.join(tmp, "ifluid_driver")
    lib_dir = os.path.dirname(L.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "ifluid_driver.cc"), "-L" + lib_dir, "-ltarang_gpu",
           "-Wl,-rpath," + lib_dir, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run_driver(exe, tmp, V, mode):
    fin, fout = os.path.join(tmp, f"in{mode}.bin"), os.path.join(tmp, f"out{mode}.bin")
    np.concatenate([v.view(np.float64).ravel() for v in V]).tofile(fin)
    r = subprocess.run([exe, fin, fout, *map(str, N), repr(NU), repr(DT), str(STEPS), str(mode)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = np.fromfile(fout, dtype=np.float64)
    nf = 2 * N[0] * N[1] * (N[2] // 2 + 1)
    shape = (N[0], N[1], N[2] // 2 + 1)
    fields = [raw[i * nf:(i + 1) * nf].view(np.complex128).reshape(shape) for i in range(3)]
    rest = raw[3 * nf:]
    return fields, rest[:STEPS], rest[STEPS:STEPS + S + 1], rest[STEPS + S + 1:].reshape(S + 1, S + 1)


def python_run(V, mode):
    from tarang_b200.solver import IncFluid
    s = IncFluid(N, nu=NU, dt=DT, force=FORCE, n_shells=S)
    try:
        s.set_V(V)
        if mode == 0:
            E = []
            for _ in range(STEPS):
                s.Compute_force()
                s.Compute_nlin()
                s.Add_force()
                s.Compute_pressure()
                s.Get_dt()
                s.Time_advance()
                E.append(s.CV_Compute_totalenergy_diss()[0])
            E = np.array(E)
        else:
            E = np.asarray(s.step(STEPS))
        return s.get_V(), E, s.Compute_flux(), s.Compute_shell_tr()
    finally:
        s.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_cpp_driver_equals_python_mirror(lib, tmp_path, mode):
    exe = build_driver(str(tmp_path))
    V = ic.random_phase_field(N, seed=77)
    fc, Ec, flc, trc = run_driver(exe, str(tmp_path), V, mode)
    fp, Ep, flp, trp = python_run(V, mode)
    for a, b in zip(fc, fp):
        assert np.array_equal(a, b)
    assert np.array_equal(Ec, Ep)
    assert np.array_equal(flc, flp) and np.array_equal(trc, trp)
    # and the trajectory is the oracle's
    ref = o.FluidSolver(N, (1.0, 1.0, 1.0), NU, DT, force=FORCE)
    W = V
    for _ in range(STEPS):
        W, _ = ref.step(W)
    num = math.sqrt(sum(float(np.sum(np.abs(a - b) ** 2)) for a, b in zip(fc, W)))
    den = math.sqrt(sum(float(np.sum(np.abs(b) ** 2)) for b in W))
    assert num / den <= 1e-12
