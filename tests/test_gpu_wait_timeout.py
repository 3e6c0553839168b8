"""A TMA-staged transform pass whose bounded wait runs out reports TG_ERR_TIMEOUT to the caller.

The failure is made without a GPU fault: the test hook TG_DEBUG_SHORT_TMA_WAIT gives the first
wait for each tile no polls, so every TMA-staged block skips its tile and sets the context's
status word, while the second wait (full limit) lets the copy land before the block leaves.
The step must then fail with TG_ERR_TIMEOUT instead of returning TG_OK over fields the passes
never wrote, and the same context must run normally once the hook is off."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import _lib as L
from tarang_b200 import ic

pytestmark = pytest.mark.gpu

N = (32, 32, 32)


def _rel(got, want):
    num = math.sqrt(sum(float(np.sum(np.abs(a - b) ** 2)) for a, b in zip(got, want)))
    return num / math.sqrt(sum(float(np.sum(np.abs(b) ** 2)) for b in want))


def test_step_reports_timeout_then_recovers(lib):
    from tarang_b200.solver import IncFluid
    V = ic.random_phase_field(N, seed=7)
    s = IncFluid(N, nu=1e-2, dt=1e-3)
    try:
        s.set_V(V)
        s.step(1)                       # a normal step first: the step graph is captured later
        assert lib.tg_debug_set(s.h, L.TG_DEBUG_SHORT_TMA_WAIT, 1) == L.TG_OK
        with pytest.raises(L.TarangError) as ei:
            s.step(2)
        assert ei.value.code == L.TG_ERR_TIMEOUT
        assert b"waiting for its tile" in lib.tg_last_error(s.h)
        # the word was cleared: the context synchronises cleanly
        assert lib.tg_synchronize(s.h) == L.TG_OK
        assert lib.tg_debug_set(s.h, L.TG_DEBUG_SHORT_TMA_WAIT, 0) == L.TG_OK
        s.set_V(V)
        s.step(1)
        want, _ = o.FluidSolver(N, (1.0, 1.0, 1.0), 1e-2, 1e-3).step(V)
        assert _rel(s.get_V(), want) <= 1e-12
    finally:
        s.close()


def test_transform_reports_timeout_at_the_next_synchronising_call(lib):
    from tarang_b200.solver import IncFluid
    rng = np.random.default_rng(8)
    real = o.pack_real(rng.standard_normal(N))
    s = IncFluid(N, dealias=False)
    try:
        assert lib.tg_debug_set(s.h, L.TG_DEBUG_SHORT_TMA_WAIT, 1) == L.TG_OK
        with pytest.raises(L.TarangError) as ei:
            s.Forward_transform_array(real)
        assert ei.value.code == L.TG_ERR_TIMEOUT
        assert lib.tg_debug_set(s.h, L.TG_DEBUG_SHORT_TMA_WAIT, 0) == L.TG_OK
        got = s.Forward_transform_array(real)
        want = o.forward_four(o.unpack_real(real))
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    finally:
        s.close()


def test_debug_hook_rejects_unknown_settings(lib):
    from tarang_b200.solver import IncFluid
    s = IncFluid((16, 16, 16))
    try:
        assert lib.tg_debug_set(s.h, 99, 1) == L.TG_ERR_ARG
        assert lib.tg_debug_set(s.h, L.TG_DEBUG_SHORT_TMA_WAIT, 2) == L.TG_ERR_ARG
    finally:
        s.close()
