"""tg_energy_noalloc: the energy reduction for callers that cannot allocate device memory.

Such a caller (an in-situ diagnostic inside another code's time loop, whose host application
owns all device memory and forbids cudaMalloc) keeps its spectral fields in its own device
buffers.  This test stands in for it: the fields and the output live in device buffers the
test owns, the entry point is called through the C ABI twice in a row (different grids, so
the second call would expose partial sums left over from the first), and both results must
equal what tg_energy returns for the same fields, to the 1e-13 relative tolerance of the
other energy tests.  The file is collected last so a failure here stops a run only after
every other test has run.
"""

import ctypes

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu


def _noalloc_energy(lib, torch, V, N):
    dev = torch.from_numpy(np.concatenate([v.view(np.float64).ravel() for v in V])).cuda()
    out = torch.full((2 * len(V),), float("nan"), dtype=torch.float64, device="cuda")
    n3 = (ctypes.c_int * 3)(*N)
    kf = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.tg_energy_noalloc(ctypes.c_void_p(dev.data_ptr()), len(V), n3, kf, 1,
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert rc == L.TG_OK
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_energy_noalloc_matches_tg_energy_twice(lib):
    import torch
    from tarang_b200.solver import IncFluid
    for N, seed in (((32, 32, 32), 101), ((16, 16, 16), 202)):
        V = ic.random_phase_field(N, seed=seed)
        s = IncFluid(N)
        s.set_V(V)
        E, D = s.CV_Compute_totalenergy_diss()
        s.close()
        got = _noalloc_energy(lib, torch, V, N)
        assert abs(got[0::2].sum() - E) <= 1e-13 * abs(E)
        assert abs(got[1::2].sum() - D) <= 1e-13 * abs(D)
        for f in range(3):
            Ef = o.total_energy_four(V[f])
            assert abs(got[2 * f] - Ef) <= 1e-13 * abs(Ef)


def test_energy_noalloc_rejects_more_fields_than_its_scratch(lib):
    n3 = (ctypes.c_int * 3)(16, 16, 16)
    kf = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    dummy = ctypes.c_void_p(16)   # never dereferenced: the call is rejected before any launch
    rc = lib.tg_energy_noalloc(dummy, 9, n3, kf, 1, dummy, None)
    assert rc == L.TG_ERR_ARG
