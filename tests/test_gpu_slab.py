"""The slab-sharded solve on one GPU (tarang_b200.slab.SlabEmulation): W slab contexts in one
process, the all-to-alls as device copies and the reductions summed in rank order, all on one
stream.  Three RK4 steps against a whole-grid context: fields to 1e-13 relative L2 in FP64
(1e-6 in FP32-mixed; the slab pipeline runs the y-inverse before the x-inverse, so the rounding
differs), energies to 1e-13; and the fields of every W equal bit for bit (each row and column
transform is the same kernel whatever the partition, and dt is the fixed ceiling here)."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

KF_RB = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))


def rel_l2(a, b):
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den


CASES = [
    ("fluid32_fp64", (32, 32, 32), dict(nu=2e-3, dt=1e-3), (1, 2, 3)),
    ("fluid_aniso_fp64", (48, 40, 64), dict(nu=2e-3, dt=1e-3), (2, 5)),
    ("fluid64_fp32", (64, 64, 64), dict(nu=2e-3, dt=1e-3, precision="FP32"), (1, 4)),
    ("fluid128z_fp64", (16, 16, 128), dict(nu=2e-3, dt=1e-3), (1, 3)),
    ("scalar32_fp64", (32, 32, 32), dict(physics="SCALAR", nu=2e-3, kappa=3e-3, dt=1e-3), (1, 2)),
    ("rb_fp64", (17, 32, 32), dict(basis="SCFT", physics="RB", Ra=1e4, Pr=1.0, kfactor=KF_RB, dt=1e-4), (1, 3)),
]


@pytest.mark.parametrize("name,N,kw,worlds", CASES, ids=[c[0] for c in CASES])
def test_gpu_slab_emulation_matches_whole_grid(lib, name, N, kw, worlds):
    from tarang_b200.slab import SlabEmulation
    from tarang_b200.solver import IncFluid
    phys = kw.get("physics", "FLUID")
    V = ic.random_phase_field(N, seed=5, kfactor=kw.get("kfactor", (1.0, 1.0, 1.0)))
    if kw.get("basis") == "SCFT":
        V = [o.dealias(o.forward_scft(np.random.default_rng(9 + i).standard_normal(N), p), "SCFT")
             for i, p in enumerate((1, 0, 0))]
    T = ic.random_phase_field(N, seed=6)[0] if phys == "SCALAR" else None
    if phys == "RB":
        T = ic.rb_perturbation(N, seed=7)
    ref = IncFluid(N, **kw)
    ref.set_V(V)
    if T is not None:
        ref.set_T(T)
    E_ref = ref.step(3)
    want = ref.get_V() + ([ref.get_T()] if T is not None else [])
    ref.close()
    tol = 1e-6 if kw.get("precision") == "FP32" else 1e-13
    first = None
    for W in worlds:
        em = SlabEmulation(N, W, **kw)
        try:
            em.set_V(V)
            if T is not None:
                em.set_T(T)
            E = em.step(3)
            got = em.get_V() + ([em.get_T()] if T is not None else [])
            t, steps, dt = em.time()
        finally:
            em.close()
        assert rel_l2(got, want) <= tol, (name, W, rel_l2(got, want))
        assert np.allclose(E, E_ref, rtol=tol, atol=0), (name, W)
        assert steps == 3 and abs(t - 3 * kw["dt"]) <= 1e-15 and dt == kw["dt"]
        if first is None:
            first = got
        else:
            assert all(np.array_equal(a, b) for a, b in zip(got, first)), (name, W)


def test_gpu_slab_refusals(lib):
    import ctypes as C

    from tarang_b200.slab import SlabEmulation
    from tarang_b200.solver import make_config
    em = SlabEmulation((16, 16, 16), 2, nu=1e-2, dt=1e-3)
    try:
        h = em.ranks[0].h
        assert em.ranks[0].lib.tg_step(h, 1, None) == L.TG_ERR_STATE   # whole-grid calls refused
        assert em.ranks[0].lib.tg_energy(h, 0, None, None) == L.TG_ERR_STATE
    finally:
        em.close()
    lib_ = L.load()
    out = C.c_void_p()
    cfg = make_config((16, 16, 16), physics="MHD", nu=1e-2, eta=1e-2, dt=1e-3)
    assert lib_.tg_slab_create(C.byref(cfg), 2, 0, C.byref(out)) == L.TG_ERR_UNSUPPORTED
    cfg = make_config((16, 16, 16), nu=1e-2, dt=1e-3)
    assert lib_.tg_slab_create(C.byref(cfg), 2, 2, C.byref(out)) == L.TG_ERR_ARG
    assert lib_.tg_slab_create(C.byref(cfg), 17, 0, C.byref(out)) == L.TG_ERR_ARG  # more ranks than y planes
