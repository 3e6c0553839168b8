"""Ring and cylinder-ring spectra, their helicity forms, ring-to-ring transfers and the ring force
feed in the SCFT basis (free-slip walls along x): Compute_local_ring_spectrum_SCFT and the
cylinder / helicity variants (scft_energy.cc:814-940, 1334-1370, 1423-1480, 1794-1830),
Local_ring_mult_all_SCFT / Local_cyl_ring_mult_all_SCFT (scft_ET.cc:273-478) with kx >= 0,
Multiplicity_factor_SCFT and the Fourier-basis vector (-i V1, V2, V3).  The oracle is pinned by a
mode worked out by hand (including the reference's off-axis branch, which adds no multiplicity
factor), by sums over sectors and slabs that give shell sums, and by ring-to-ring antisymmetry;
the CUDA path is checked against it."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o

KF = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))


def scft_fields(N, seed, inside=None, kf=KF):
    """Dealiased SCFT fields: u1 and theta sine series, u2 and u3 cosine series, the velocity made
    divergence-free; optionally held to |K| <= inside."""
    rng = np.random.default_rng(seed)
    out = [o.dealias(o.forward_scft(rng.standard_normal(N), p), "SCFT") for p in (1, 0, 0, 1)]
    if inside is not None:
        K = o.kmag(N, kf, "SCFT")
        out = [np.where(K <= inside, f, 0) for f in out]
    V = out[:3]
    p = o.pressure(V, kf, "SCFT")
    V = [V[0] + o.xderiv(p, kf, "SCFT", 0), V[1] + o.yderiv(p, kf), V[2] + o.zderiv(p, kf)]
    return V, out[3]


def fourier_v(V):
    return [-1j * V[0], V[1], V[2]]


def test_scft_single_modes_by_hand():
    N = (16, 16, 16)
    kf = (1.0, 1.0, 1.0)
    V = [np.zeros((16, 16, 9), dtype=np.complex128) for _ in range(3)]
    # V1 = 2 at (m, ky, kz) = (1, 0, 1): K = (1, 0, 1), theta = pi/4 about z; -i V1 = -2i.
    # (V x K)_z = V_x K_y - V_y K_x = 0, so |V|^2 = 4 goes to S2, with no multiplicity factor
    # (the reference's off-axis branch), although Multiplicity_factor_SCFT is 2 here
    V[0][1, 0, 1] = 2.0
    e1, e2, d = o.ring_spectrum(V, kf, 3, 3, basis="SCFT")
    assert e1.sum() == 0.0 and e2[2, 2] == 4.0 and e2.sum() == 4.0
    assert d[2, 2] == pytest.approx(2 * 2.0 * 4.0)
    # on the y axis (m = 0, ky = 1, kz = 0, multiplicity 0.5): S1 = |V3|^2, S2 = |-i V1|^2
    V = [np.zeros((16, 16, 9), dtype=np.complex128) for _ in range(3)]
    V[0][0, 1, 0], V[1][0, 1, 0], V[2][0, 1, 0] = 3.0, 5.0, 1.0j
    e1, e2, _ = o.ring_spectrum(V, kf, 2, 2, basis="SCFT")
    assert e1[1, 1] == 0.5 * 1.0 and e2[1, 1] == 0.5 * 9.0 and e1.sum() + e2.sum() == 5.0
    # the same mode in the FOUR reading records (V3, V2) there (four_energy.cc:890-894)
    e1, e2, _ = o.ring_spectrum(V, kf, 2, 2)
    assert e1[1, 1] == 0.5 * 1.0 and e2[1, 1] == 0.5 * 25.0
    # cylinder about x: K_perp = 1, K_par = 0 (slab 1), S1 = |-i V1|^2 = 9 with the factor
    c1, c2, _ = o.ring_spectrum(V, kf, 1, 4, cylinder=True, basis="SCFT")
    assert c1[1, 1] == 0.5 * 9.0 and c2[1, 1] == 0.5 * 26.0


@pytest.mark.parametrize("axis", [1, 2, 3])
def test_scft_ring_sums_give_shell_sums(axis):
    """Cylinder rings: summed over slabs, cylinder shell ceil(K_perp) holds sum mult |V|^2 and the
    K^2-weighted sum; spherical rings with the axis modes removed: summed over sectors, shell
    ceil|K| holds sum |V|^2 with no multiplicity factor (the off-axis branch); helicity rings:
    summed over sectors, 2 mult K . (Vr x Vi) of the shell."""
    N = (24, 16, 32)
    kin = o.max_radius_inside(N, KF, "DEALIAS", "SCFT")
    V, _ = scft_fields(N, 20 + axis)
    Vf = fourier_v(V)
    Kv = [np.broadcast_to(k, V[0].shape) for k in o.kvec(N, KF, "SCFT")]
    K = np.sqrt(sum(k * k for k in Kv))
    ax = axis - 1
    kperp = np.sqrt(Kv[(ax + 1) % 3] ** 2 + Kv[(ax + 2) % 3] ** 2)
    mult = o.multiplicity_scft(N)
    e = sum(np.abs(v) ** 2 for v in Vf)
    # cylinders
    c1, c2, cd = o.ring_spectrum(V, KF, axis, 3, cylinder=True, basis="SCFT")
    kr = o.krho_inside(N, KF, axis, "DEALIAS", "SCFT")
    assert c1.shape[0] == kr + 1
    row = np.ceil(kperp).astype(int)
    ok = row <= kr
    want = np.bincount(row[ok], weights=(mult * e)[ok], minlength=kr + 1)
    assert np.allclose((c1 + c2).sum(axis=1), want, rtol=1e-12, atol=1e-14 * want.max())
    wd = 2 * np.bincount(row[ok], weights=(mult * K * K * e)[ok], minlength=kr + 1)
    assert np.allclose(cd.sum(axis=1), wd, rtol=1e-12, atol=1e-14 * wd.max())
    # spherical, off the axis
    Va = [np.where(kperp < o.MYEPS, 0, v) for v in V]
    e1, e2, _ = o.ring_spectrum(Va, KF, axis, 4, basis="SCFT")
    ea = sum(np.abs(v) ** 2 for v in fourier_v(Va))
    row = np.ceil(K).astype(int)
    ok = (row <= kin) & (K > o.MYEPS)
    want = np.bincount(row[ok], weights=ea[ok], minlength=kin + 1)
    assert np.allclose((e1 + e2).sum(axis=1), want, rtol=1e-12, atol=1e-14 * want.max())
    # helicity
    h = o.ring_spectrum(V, KF, axis, 4, helicity=True, basis="SCFT")[0]
    vr = np.stack([v.real for v in Vf])
    vi = np.stack([v.imag for v in Vf])
    hk = 2 * mult * sum(Kv[i] * np.cross(vr, vi, axis=0)[i] for i in range(3))
    want = np.bincount(row[ok], weights=hk[ok], minlength=kin + 1)
    assert np.allclose(h.sum(axis=1), want, rtol=1e-10, atol=1e-12 * np.abs(want).max())


def test_scft_ring_transfer_oracle_identities():
    """SCFT ring-to-ring (oracle): about x (kx >= 0) and z (kz >= 0) every stored mode has
    theta <= pi/2, so a giver ring row summed over sectors is the SCFT shell-to-shell row of its
    shell, and the transfer between two rings is antisymmetric (fields inside R_in, so the
    products are alias-free)."""
    N = (33, 32, 32)
    kin = o.max_radius_inside(N, KF, "DEALIAS", "SCFT")
    V, _ = scft_fields(N, 5, inside=kin)
    n, ns = 6, 2
    R = o.ring_radii(N, KF, n, basis="SCFT")
    assert np.all(np.diff(R) > 0)
    for axis in (1, 3):
        T = o.compute_ring_tr_generic(V, V, V, -1.0, KF, axis, n, ns, basis="SCFT")
        scale = np.abs(T).max()
        assert scale > 0
        for i in range(1, n):
            G = [o.fill_array_shell(v, R[i - 1], R[i], KF, "SCFT") for v in V]
            want = -o.shell_mult_all(o.et_nlin(V, G, KF, "SCFT"), V, R, KF, basis="SCFT")
            assert np.allclose(T[i].sum(axis=(0, 2)), want, rtol=1e-10, atol=1e-12 * scale)
        inner = T[1:n, 1:, 1:n, 1:]
        assert np.abs(inner + inner.transpose(2, 3, 0, 1)).max() <= 1e-12 * scale
    Tc = o.compute_cylinder_ring_tr_generic(V, V, V, -1.0, KF, 1, 5, 2, basis="SCFT")
    inner = Tc[1:5, 1:, 1:5, 1:]
    assert np.abs(inner + inner.transpose(2, 3, 0, 1)).max() <= 1e-12 * np.abs(Tc).max()


def _solver(N, **kw):
    from tarang_b200.solver import IncFluid
    kw.setdefault("nu", 1e-3)
    kw.setdefault("dt", 1e-4)
    return IncFluid(N, basis="SCFT", kfactor=kw.pop("kfactor", KF), **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("axis", [1, 2, 3])
@pytest.mark.parametrize("n", [1, 4])
def test_gpu_scft_ring_spectra_match_oracle(lib, axis, n):
    N = (24, 16, 32)
    V, _ = scft_fields(N, 40 + 3 * axis + n)
    s = _solver(N)
    try:
        s.set_V(V)
        for cyl in (False, True):
            got = s.CV_Compute_cylinder_ring_spectrum(n, axis) if cyl else s.CV_Compute_ring_spectrum(n, axis)
            want = o.ring_spectrum(V, KF, axis, n, cylinder=cyl, basis="SCFT")
            for g, w in zip(got, want):
                assert g.shape == w.shape
                assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max(), (cyl, axis, n)
        g = s.CV_Compute_ring_spectrum_helicity(n, axis)
        w = o.ring_spectrum(V, KF, axis, n, helicity=True, basis="SCFT")[0]
        assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
        g = s.CV_Compute_cylinder_ring_spectrum_helicity(n, axis)
        w = o.ring_spectrum(V, KF, axis, n, cylinder=True, helicity=True, basis="SCFT")[0]
        assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
    finally:
        s.close()


@pytest.mark.gpu
def test_gpu_scft_ring_spectra_aliased_grid(lib):
    """ALIAS: the SCFT box extends to kx = N1 - 1 (Anis_max_Krho_radius_inside_SCFT,
    Max_radius_inside_aliased_SCFT)."""
    N = (16, 16, 16)
    kf = (1.0, 1.0, 1.0)
    rng = np.random.default_rng(77)
    V = [o.forward_scft(rng.standard_normal(N), p) for p in (1, 0, 0)]
    s = _solver(N, kfactor=kf, dealias=False)
    try:
        s.set_V(V)
        got = s.CV_Compute_cylinder_ring_spectrum(3, 2)
        want = o.ring_spectrum(V, kf, 2, 3, cylinder=True, alias="ALIAS", basis="SCFT")
        assert got[0].shape == want[0].shape
        for g, w in zip(got, want):
            assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
        got = s.CV_Compute_ring_spectrum(3, 1)
        want = o.ring_spectrum(V, kf, 1, 3, alias="ALIAS", basis="SCFT")
        assert got[0].shape == want[0].shape
        for g, w in zip(got, want):
            assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("axis,n,ns", [(1, 6, 2), (3, 5, 3), (2, 6, 2)])
def test_gpu_scft_ring_to_ring_matches_oracle(lib, axis, n, ns):
    from tarang_b200 import _lib as L
    N = (33, 32, 32)
    V, T = scft_fields(N, 60 + axis)
    z = np.zeros_like(T)
    s = _solver(N, physics="RB", Ra=1e6, Pr=1.0)
    try:
        s.set_V(V)
        s.set_T(T)
        got, r = s.Compute_ring_tr(n, ns, axis)
        assert np.allclose(r, o.ring_radii(N, KF, n, basis="SCFT"), rtol=0, atol=0)
        want = o.compute_ring_tr_generic(V, V, V, -1.0, KF, axis, n, ns, basis="SCFT")
        assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
        got, _ = s.Compute_ring_tr(n, ns, axis, L.TG_ET_TT)
        want = o.compute_ring_tr_generic(V, [T, z, z], [T, z, z], -1.0, KF, axis, n, ns, basis="SCFT")
        assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
        got, rc = s.Compute_cylinder_ring_tr(5, ns, axis)
        kr = o.krho_inside(N, KF, axis, "DEALIAS", "SCFT")
        assert np.allclose(rc, o.ring_radii(N, KF, 5, basis="SCFT", Rin=float(kr)), rtol=0, atol=0)
        want = o.compute_cylinder_ring_tr_generic(V, V, V, -1.0, KF, axis, 5, ns, basis="SCFT")
        assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    finally:
        s.close()


@pytest.mark.gpu
def test_gpu_scft_ring_force_feed(lib):
    """Compute_force_feed_ring / _cylinder_ring with an SCFT band forcing (Ring_mult_all_SCFT)."""
    N = (24, 16, 32)
    V, _ = scft_fields(N, 90)
    s = _solver(N, nu=2e-3, dt=5e-4, force=dict(kind="energy_helicity", inner=2.0, outer=6.0, eps=0.1, eps_h=0.2))
    try:
        s.set_V(V)
        s.Compute_force()
        F = s.get_force()
        for cyl, axis, n, ns in ((False, 3, 6, 3), (True, 1, 5, 4), (False, 1, 5, 2)):
            got = s.Compute_force_feed_ring(n, ns, axis, 0, cyl)
            want = o.ring_mult_all(F, V, KF, axis, n, ns, cylinder=cyl, basis="SCFT")
            assert np.count_nonzero(want) >= 1
            assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), (cyl, axis)
    finally:
        s.close()
