"""Field transfers of the stored modes only: tg_field_upload of a state field moves the 2/3
support as strided copies straight into the solver's rows (the state equals what the previous
gather path produced: downloads, energies and a step match the oracle), and
tg_field_download_stored writes exactly the stored entries of the caller's array, leaving the
others untouched."""

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

KF = (1.0, 1.0, 1.0)


@pytest.mark.parametrize("N,physics", [((32, 32, 32), "FLUID"), ((48, 32, 64), "FLUID"), ((32, 32, 32), "MHD"),
                                       ((16, 16, 32), "SCALAR")])
def test_upload_and_stored_download(lib, N, physics):
    from tarang_b200 import _lib as L
    from tarang_b200.solver import IncFluid
    s = IncFluid(N, physics=physics, nu=1e-3, dt=1e-3)
    rng = np.random.default_rng(5)
    shape = (N[0], N[1], N[2] // 2 + 1)
    fields = [L.TG_V1, L.TG_V2, L.TG_V3] + ([L.TG_W1, L.TG_W2, L.TG_W3] if physics == "MHD" else []) + \
        ([L.TG_T] if physics == "SCALAR" else [])
    keep = ic.keep_mask(N)
    for f in fields:
        A = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)   # garbage outside the support too
        s.upload(f, A)
        full = s.download(f)
        assert np.array_equal(full, np.where(keep, A, 0))
        sentinel = np.full(shape, 7.0 + 3.0j)
        got = s.download_stored(f, sentinel.copy())
        assert np.array_equal(got[keep], A[keep])
        assert np.all(got[~keep] == 7.0 + 3.0j)


def test_step_after_stored_upload_matches_oracle(lib):
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=12)
    s = IncFluid(N, nu=1e-2, dt=1e-3)
    s.set_V(V)
    s.step(2)
    ref = o.FluidSolver(N, KF, 1e-2, 1e-3)
    Vw = V
    for _ in range(2):
        Vw, _ = ref.step(Vw)
    out = [np.zeros_like(v) for v in V]
    got = [s.download_stored(i, out[i]) for i in range(3)]
    num = np.sqrt(sum(np.sum(np.abs(a - b) ** 2) for a, b in zip(got, Vw)))
    den = np.sqrt(sum(np.sum(np.abs(b) ** 2) for b in Vw))
    assert num / den < 1e-12
