"""tg_energy_noalloc: the energy reduction for callers that cannot allocate device memory.

Such a caller (an in-situ diagnostic inside another code's time loop, whose host application
owns all device memory and forbids cudaMalloc) keeps its spectral fields in its own device
buffers.  These tests stand in for it: the fields and the output live in device buffers the
test owns and the entry point is called through the C ABI.  Two calls in a row on different
grids share the fixed scratch array; the second launches fewer blocks than the first, and its
result must not depend on what the first call left there.  Every result must equal what
tg_energy returns for the same fields and what the oracle computes, to the 1e-13 relative
tolerance of the other energy tests: dealiased and full grids, anisotropic box factors and the
8-field maximum.  The file is collected last so a failure here stops a run only after every
other test has run.
"""

import ctypes

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _noalloc_energy(lib, torch, V, N, kfactor=(1.0, 1.0, 1.0), dealias=1):
    dev = torch.from_numpy(np.concatenate([v.view(np.float64).ravel() for v in V])).cuda()
    out = torch.full((2 * len(V),), float("nan"), dtype=torch.float64, device="cuda")
    n3 = (ctypes.c_int * 3)(*N)
    kf = (ctypes.c_double * 3)(*kfactor)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.tg_energy_noalloc(ctypes.c_void_p(dev.data_ptr()), len(V), n3, kf, int(dealias),
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert rc == L.TG_OK
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _check_against_oracle(got, V, kfactor, dealias):
    alias = "DEALIAS" if dealias else "ALIAS"
    for f, v in enumerate(V):
        Ef = o.total_energy_four(v)
        Df = 2.0 * o.total_Sn(v, 2, kfactor, alias)
        assert abs(got[2 * f] - Ef) <= TOL * abs(Ef)
        assert abs(got[2 * f + 1] - Df) <= TOL * abs(Df)


def _context_energy(V, N, kfactor, dealias):
    from tarang_b200.solver import IncFluid
    s = IncFluid(N, kfactor=kfactor, dealias=bool(dealias))
    try:
        s.set_V(V)
        return s.CV_Compute_totalenergy_diss()
    finally:
        s.close()


def test_energy_noalloc_matches_tg_energy_twice(lib):
    import torch
    for N, seed in (((32, 32, 32), 101), ((16, 16, 16), 202)):
        V = ic.random_phase_field(N, seed=seed)
        E, D = _context_energy(V, N, (1.0, 1.0, 1.0), 1)
        got = _noalloc_energy(lib, torch, V, N)
        assert abs(got[0::2].sum() - E) <= TOL * abs(E)
        assert abs(got[1::2].sum() - D) <= TOL * abs(D)
        _check_against_oracle(got, V, (1.0, 1.0, 1.0), 1)


@pytest.mark.parametrize("N,kfactor,dealias", [
    ((24, 16, 32), (1.0, 1.0, 1.0), 0),        # full grid: Min_radius_outside_aliased
    ((32, 16, 24), (1.0, 2.0, 0.5), 1),        # anisotropic box
    ((20, 24, 16), (0.5, 1.5, 2.0), 0),        # both
])
def test_energy_noalloc_grids_and_boxes(lib, N, kfactor, dealias):
    import torch
    V = ic.random_phase_field(N, seed=303)
    if not dealias:
        # a field with energy in the 1/3 band as well: the full-grid radius must count it
        rng = np.random.default_rng(304)
        shape = V[0].shape
        V = [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(3)]
        V = [o.satisfy_reality(v) for v in V]
    E, D = _context_energy(V, N, kfactor, dealias)
    got = _noalloc_energy(lib, torch, V, N, kfactor, dealias)
    assert abs(got[0::2].sum() - E) <= TOL * abs(E)
    assert abs(got[1::2].sum() - D) <= TOL * abs(D)
    _check_against_oracle(got, V, kfactor, dealias)


def test_energy_noalloc_eight_fields(lib):
    import torch
    N = (16, 16, 16)
    V = []
    for seed in (11, 12, 13):
        V.extend(ic.random_phase_field(N, seed=seed))
    V = V[:8]
    got = _noalloc_energy(lib, torch, V, N)
    _check_against_oracle(got, V, (1.0, 1.0, 1.0), 1)
    # and again with the maximum after a smaller call: the same numbers
    _noalloc_energy(lib, torch, V[:2], N)
    again = _noalloc_energy(lib, torch, V, N)
    assert np.array_equal(got, again)


def test_energy_noalloc_rejects_more_fields_than_its_scratch(lib):
    n3 = (ctypes.c_int * 3)(16, 16, 16)
    kf = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    dummy = ctypes.c_void_p(16)   # never dereferenced: the call is rejected before any launch
    rc = lib.tg_energy_noalloc(dummy, 9, n3, kf, 1, dummy, None)
    assert rc == L.TG_ERR_ARG
