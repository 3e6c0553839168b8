"""Parity of the CUDA 3-D FOUR transforms (Forward/Inverse_transform_array through the C ABI)
with the oracle.  FP64 form: max error <= 1e-13 relative to the field's max; the FP32-mixed
form computes in FP32 with FP64 twiddles rounded: <= 2e-6."""

import json
import os

import numpy as np
import pytest

from oracle import tarang_oracle as o

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _solver(N, precision="FP64"):
    from tarang_b200.solver import IncFluid
    return IncFluid(N, precision=precision)


def test_out1_kat_on_gpu(lib):
    kat = json.load(open(os.path.join(GOLD, "out1_kat.json")))
    N = tuple(kat["N"])
    s = _solver(N)
    A = np.zeros((N[0], N[1], N[2] // 2 + 1), complex)
    A[tuple(kat["delta_at"])] = 1.0
    r = o.unpack_real(s.Inverse_transform_array(A))
    assert np.abs(r - (-1.0) ** np.arange(N[2])[None, None, :]).max() < 1e-15
    assert abs((r ** 2).sum() - kat["real_sum_sq_without_padding"]) < 1e-12
    B = s.Forward_transform_array(o.pack_real(r)) * np.prod(N)
    want = np.array(kat["after_fft"], dtype=float).reshape(A.shape)
    assert np.abs(B - want).max() < 1e-12


SHAPES = [(8, 8, 8), (16, 16, 16), (32, 32, 32), (64, 64, 64), (128, 64, 32), (16, 32, 64),
          (12, 18, 20), (20, 12, 24), (256, 256, 256)]


@pytest.mark.parametrize("N", SHAPES)
@pytest.mark.parametrize("precision,tol", [("FP64", 1e-13), ("FP32", 2e-6)])
def test_forward_matches_oracle(lib, N, precision, tol):
    rng = np.random.default_rng(11)
    real = rng.standard_normal(N)
    s = _solver(N, precision)
    got = s.Forward_transform_array(o.pack_real(real))
    want = o.forward_four(real)
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < tol, err


@pytest.mark.parametrize("N", SHAPES)
@pytest.mark.parametrize("precision,tol", [("FP64", 1e-13), ("FP32", 2e-6)])
def test_inverse_matches_oracle(lib, N, precision, tol):
    rng = np.random.default_rng(12)
    spec = o.forward_four(rng.standard_normal(N))
    # non-Hermitian imaginary parts on the kz = 0 / N3/2 planes are ignored by c2r
    spec[:, :, 0] += 1j * rng.standard_normal(spec.shape[:2]) * 0.1
    s = _solver(N, precision)
    got = o.unpack_real(s.Inverse_transform_array(spec))
    want = o.inverse_four(spec)
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < tol, err
    # padding slot of each row is zero (Zero_pad_last_plane_FOUR four_tr.cc:299-302)
    packed = s.Inverse_transform_array(spec)
    assert np.all(packed[:, :, -1] == 0)


def test_round_trip_identity_256(lib):
    N = (256, 256, 256)
    rng = np.random.default_rng(5)
    real = rng.standard_normal(N)
    s = _solver(N)
    spec = s.Forward_transform_array(o.pack_real(real))
    back = o.unpack_real(s.Inverse_transform_array(spec))
    assert np.abs(back - real).max() < 1e-13


def test_field_alloc_free(lib):
    """tg_field_alloc reserves distinct zeroed work fields usable by the transforms; the ninth
    reservation is TG_ERR_BUSY; tg_field_free returns the slot and its memory."""
    from tarang_b200 import _lib as L
    from tarang_b200.solver import IncFluid
    N = (16, 16, 16)
    s = IncFluid(N)
    base = s.device_bytes()
    ids = [s.alloc_field() for _ in range(L.TG_NWORK)]
    assert sorted(ids) == list(range(L.TG_WORK0, L.TG_WORK0 + L.TG_NWORK))
    assert s.device_bytes() == base + L.TG_NWORK * 16 * N[0] * N[1] * (N[2] // 2 + 1)
    with pytest.raises(L.TarangError) as e:
        s.alloc_field()
    assert e.value.code == L.TG_ERR_BUSY
    assert np.all(s.download(ids[3]) == 0)
    rng = np.random.default_rng(2)
    real = rng.standard_normal(N)
    s.upload(ids[3], o.pack_real(real))
    s._ck(s.lib.tg_forward_transform(s.h, ids[3], 0), "forward")
    want = o.forward_four(real)
    assert np.abs(s.download(ids[3]) - want).max() < 1e-13 * np.abs(want).max()
    for f in ids:
        s.free_field(f)
    assert s.device_bytes() == base
    with pytest.raises(L.TarangError):
        s.free_field(ids[0])
    again = s.alloc_field()
    assert again == L.TG_WORK0 and np.all(s.download(again) == 0)
