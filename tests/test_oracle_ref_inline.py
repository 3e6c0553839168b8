"""The oracle's wavenumber conventions against the reference's own code: the fixture
tests/golden/ref_inline.json holds the output of the reference's inline functions
(trunk/lib/four/four_inline.h, trunk/lib/scft/scft_inline.h), compiled from the reference tree
by oracle/ref_pin and run by tests/golden/make_ref_inline_fixtures.py, on FOUR and SCFT grids
(the configs' 256^3 and 129x256x256 / 65x128x128 among them) with unit and anisotropic kfactor.
Per mode: grid wavenumbers, |K| (Kmagnitude), the multiplicity factor and, per anisotropy axis,
K_parallel, K_perp and the polar angle; per grid: the aliased and dealiased radii
(Min_radius_outside, Max_radius_inside), Approx_number_modes_in_shell and the cylindrical
extents (Anis_max_Kpll, Anis_max_Krho_radius_inside; Anis_min_Kpll, which returns 0, is the
lower slab bound the oracle uses).  Integers and integer-valued factors match exactly, floating
point values to the last bit or 1 ulp."""

import json
import os

import numpy as np
import pytest

from oracle import tarang_oracle as o

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_inline.json")
CASES = json.load(open(FIX))["cases"]


def case_id(c):
    return f"{c['basis']}-{'x'.join(map(str, c['N']))}-kf{'_'.join(f'{k:.3g}' for k in c['kfactor'])}"


@pytest.mark.parametrize("c", CASES, ids=case_id)
def test_radii_and_extents(c):
    b, N, kf = c["basis"], tuple(c["N"]), tuple(c["kfactor"])
    for al in ("ALIAS", "DEALIAS"):
        assert o.min_radius_outside(N, kf, al, b) == c[f"min_radius_outside_{al}"], al
        assert o.max_radius_inside(N, kf, al, b) == c[f"max_radius_inside_{al}"], al
    got = [o.approx_number_modes_in_shell(N, r, kf, b) for r in range(1, 7)]
    np.testing.assert_allclose(got, c["approx_number_modes_in_shell_r1_6"], rtol=2e-16, atol=0)
    for a in c["anis"]:
        ax = a["axis"]
        for al in ("ALIAS", "DEALIAS"):
            assert o.kpll_max(N, kf, ax, al, b) == a[f"max_kpll_{al}"], (ax, al)
            assert o.krho_inside(N, kf, ax, al, b) == a[f"max_krho_inside_{al}"], (ax, al)
            assert a[f"min_kpll_{al}"] == 0.0


@pytest.mark.parametrize("c", [c for c in CASES if "kmag" in c], ids=case_id)
def test_modes(c):
    b, N, kf = c["basis"], tuple(c["N"]), tuple(c["kfactor"])
    kx = o.kx_four(N[0]) if b == "FOUR" else o.kx_scft(N[0])
    assert np.array_equal(kx, np.array(c["kx"]))
    assert np.array_equal(o.ky_four(N[1]), np.array(c["ky"]))
    assert np.array_equal(o.kmag(N, kf, b).ravel(), np.array(c["kmag"]))
    assert np.array_equal(o.multiplicity(N, b).ravel(), np.array(c["multiplicity"]))


@pytest.mark.parametrize("c", [c for c in CASES if any("kpll" in a for a in c["anis"])], ids=case_id)
def test_anisotropic_modes(c):
    b, N, kf = c["basis"], tuple(c["N"]), tuple(c["kfactor"])
    shape = (N[0], N[1], N[2] // 2 + 1)
    K = [np.broadcast_to(k, shape) for k in o.kvec(N, kf, b)]
    for a in c["anis"]:
        ax = a["axis"] - 1
        kpll = K[ax].ravel()
        kperp = np.sqrt(K[(ax + 1) % 3] ** 2 + K[(ax + 2) % 3] ** 2).ravel()
        assert np.array_equal(kpll, np.array(a["kpll"]))
        np.testing.assert_allclose(kperp, a["kperp"], rtol=2.3e-16, atol=0)
        theta = np.array([o._polar_angle(p, q) for p, q in zip(kperp, kpll)])
        np.testing.assert_allclose(theta, a["polar_angle"], rtol=0, atol=4.5e-16)
