"""Ring and cylindrical-ring spectra (CV_Compute_ring_spectrum / CV_Compute_cylinder_ring_spectrum,
FOUR): the oracle against a hand-computed single mode and against the isotropic shell spectrum
(summing the sectors of a shell gives the shell), and the CUDA path against the oracle on random
fields for every anisotropy axis, the magnetic field of MHD and anisotropic grids."""

import math

import numpy as np
import pytest

from oracle import tarang_oracle as o
from tarang_b200 import ic

KF = (1.0, 1.0, 1.0)


def test_single_mode_by_hand():
    N = (16, 16, 16)
    V = [np.zeros((16, 16, 9), dtype=np.complex128) for _ in range(3)]
    V[0][0, 1, 1] = 1.0          # V = (1, 0, 0) at K = (0, 1, 1)
    e1, e2, d = o.ring_spectrum(V, KF, 3, 3)
    # theta = atan(1 / 1) = pi/4 <= pi/3: sector 2; shell ceil(sqrt 2) = 2;
    # (V x K)_z / K_perp = (1 * 1 - 0) / 1 = 1, so all of |V|^2 is in S1
    assert e1[2, 2] == 1.0 and e1.sum() == 1.0 and e2.sum() == 0.0
    assert d[2, 2] == pytest.approx(2 * 2.0)
    c1, c2, _ = o.ring_spectrum(V, KF, 3, 4, cylinder=True)
    # cylinder about z: K_perp = 1 (shell 1), |K_par| = 1 in slab ceil(1 / (5 / 4)) = 1
    assert c1.sum() == 0.0 and c2[1, 1] == 1.0


@pytest.mark.parametrize("axis", [1, 2, 3])
def test_sectors_sum_to_the_shell_spectrum(axis):
    """Summed over sectors a shell holds the shell spectrum, except that for the y axis the
    reference records (V_z, V_y) on the axis itself (four_energy.cc:870-874), so |V_x|^2 of the
    modes on the y axis is missing from its ring spectrum; there the identity holds off the axis."""
    N = (16, 16, 16)
    V = ic.random_phase_field(N, seed=11 + axis)
    if axis == 2:
        for v in V:
            v[0, :, 0] = 0          # no modes on the y axis
    e1, e2, d = o.ring_spectrum(V, KF, axis, 5)
    shell = sum(o.shell_spectrum(v, 0, KF) for v in V)
    kin = o.max_radius_inside(N, KF)
    tot = (e1 + e2).sum(axis=1)
    assert np.allclose(tot[1:kin + 1], shell[1:kin + 1], rtol=1e-12, atol=1e-18)
    dshell = 2 * sum(o.shell_spectrum(v, 2, KF) for v in V)
    assert np.allclose(d.sum(axis=1)[1:kin + 1], dshell[1:kin + 1], rtol=1e-12, atol=1e-18)


@pytest.mark.gpu
@pytest.mark.parametrize("axis", [1, 2, 3])
@pytest.mark.parametrize("n", [1, 4, 5])
def test_gpu_ring_spectra_match_oracle(lib, axis, n):
    from tarang_b200.solver import IncFluid
    N = (32, 16, 24)
    kf = (1.0, 2.0, 0.5)
    V = ic.random_phase_field(N, kfactor=kf, seed=40 + 3 * axis + n)
    s = IncFluid(N, kfactor=kf, nu=1e-3, dt=1e-3)
    s.set_V(V)
    for cyl in (False, True):
        got = s.CV_Compute_cylinder_ring_spectrum(n, axis) if cyl else s.CV_Compute_ring_spectrum(n, axis)
        want = o.ring_spectrum(V, kf, axis, n, cylinder=cyl)
        for g, w in zip(got, want):
            assert g.shape == w.shape
            assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max(), (cyl, axis, n)


@pytest.mark.gpu
def test_gpu_ring_spectra_mhd_magnetic_field(lib):
    from tarang_b200 import _lib as L
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=61)
    W = ic.random_phase_field(N, k0=3.0, seed=62)
    s = IncFluid(N, physics="MHD", nu=1e-3, eta=1e-3, dt=1e-3)
    s.set_V(V)
    s.set_W(W)
    for group, F in ((0, V), (1, W)):
        got = s.CV_Compute_ring_spectrum(6, 3, group)
        want = o.ring_spectrum(F, KF, 3, 6)
        for g, w in zip(got, want):
            assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
    f = IncFluid(N, nu=1e-3, dt=1e-3)
    with pytest.raises(L.TarangError):
        f.CV_Compute_ring_spectrum(6, 3, 1)          # no magnetic field
    with pytest.raises(L.TarangError):
        f.CV_Compute_ring_spectrum(65, 1)             # more sectors than the maximum


def test_ring_transfer_oracle_identities():
    """Ring-to-ring transfer (oracle): with the z axis every mode has theta <= pi/2, so summed
    over sectors a giver ring row is the shell-to-shell transfer of its shell; and the transfer
    between two rings is antisymmetric (the helper is the whole solenoidal field; 64^3, where the
    scheme-0 radii increase, so giver and receiver rings are the same sets)."""
    N = (64, 64, 64)
    V = ic.random_phase_field(N, seed=71)
    n, ns = 6, 3
    T = o.compute_ring_tr_generic(V, V, V, -1.0, KF, 3, n, ns)
    R = o.ring_radii(N, KF, n)
    for i in range(1, n):
        G = [o.fill_array_shell(v, R[i - 1], R[i], KF) for v in V]
        want = -o.shell_mult_all(o.et_nlin(V, G, KF), V, R, KF)
        assert np.allclose(T[i].sum(axis=(0, 2)), want, rtol=1e-10, atol=1e-14 * np.abs(want).max())
    scale = np.abs(T).max()
    for i in range(1, n):
        for j in range(1, ns + 1):
            for m in range(1, n):
                for s in range(1, ns + 1):
                    assert abs(T[i, j, m, s] + T[m, s, i, j]) <= 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("N,axis,n,ns", [((32, 32, 32), 3, 6, 3), ((64, 64, 64), 1, 7, 4), ((64, 32, 32), 2, 5, 2)])
def test_gpu_ring_to_ring_matches_oracle(lib, N, axis, n, ns):
    from tarang_b200.solver import IncFluid
    V = ic.random_phase_field(N, seed=80 + axis)
    s = IncFluid(N, nu=1e-3, dt=1e-3)
    s.set_V(V)
    T, r = s.Compute_ring_tr(n, ns, axis)
    assert np.allclose(r, o.ring_radii(N, KF, n), rtol=0, atol=0)
    want = o.compute_ring_tr_generic(V, V, V, -1.0, KF, axis, n, ns)
    assert np.abs(T - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
def test_gpu_ring_to_ring_mhd_kinds(lib):
    from tarang_b200 import _lib as L
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    U = ic.random_phase_field(N, seed=91)
    B = ic.random_phase_field(N, k0=3.0, seed=92)
    s = IncFluid(N, physics="MHD", nu=1e-3, eta=1e-3, dt=1e-3)
    s.set_V(U)
    s.set_W(B)
    Zp = [u + b for u, b in zip(U, B)]
    Zm = [u - b for u, b in zip(U, B)]
    for kind, (H, F, Rf, sign) in ((L.TG_ET_UU, (U, U, U, -1.0)), (L.TG_ET_BB, (U, B, B, -1.0)),
                                   (L.TG_ET_UB, (B, U, B, 1.0)), (L.TG_ET_ZP, (Zm, Zp, Zp, -1.0)),
                                   (L.TG_ET_ZM, (Zp, Zm, Zm, -1.0))):
        T, _ = s.Compute_ring_tr(6, 2, 1, kind)
        want = o.compute_ring_tr_generic(H, F, Rf, sign, KF, 1, 6, 2)
        assert np.abs(T - want).max() <= 1e-12 * np.abs(want).max(), kind
        if kind in (L.TG_ET_ZP, L.TG_ET_ZM):
            Tc, _ = s.Compute_cylinder_ring_tr(5, 3, 2, kind)
            want = o.compute_cylinder_ring_tr_generic(H, F, Rf, sign, KF, 2, 5, 3)
            assert np.abs(Tc - want).max() <= 1e-12 * np.abs(want).max(), kind
    with pytest.raises(L.TarangError):
        s.Compute_ring_tr(6, 2, 1, L.TG_ET_BU)       # not a ring transfer of the reference
    # the Elsasser tables leave U and B as they were (Elsasser_to_UB_field)
    assert np.abs(s.get_W()[1] - B[1]).max() == 0


@pytest.mark.gpu
def test_gpu_ring_to_ring_scalar(lib):
    """ring_to_ring_SF (Compute_ring_tr_scalar compute_ring_tr.cc:104-131) and the cylinder form:
    giver T on the ring, N = U.grad T<, against T; U->U of the same run."""
    from tarang_b200 import _lib as L
    from tarang_b200.solver import IncFluid
    N = (32, 32, 32)
    U = ic.random_phase_field(N, seed=93)
    T = ic.random_phase_field(N, k0=3.0, seed=94)[0]
    z = np.zeros_like(T)
    s = IncFluid(N, physics="SCALAR", nu=1e-3, kappa=2e-3, dt=1e-3)
    s.set_V(U)
    s.set_T(T)
    got, _ = s.Compute_ring_tr(6, 3, 3, L.TG_ET_TT)
    want = o.compute_ring_tr_generic(U, [T, z, z], [T, z, z], -1.0, KF, 3, 6, 3)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    got, _ = s.Compute_cylinder_ring_tr(5, 2, 1, L.TG_ET_TT)
    want = o.compute_cylinder_ring_tr_generic(U, [T, z, z], [T, z, z], -1.0, KF, 1, 5, 2)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    got, _ = s.Compute_ring_tr(6, 3, 3, L.TG_ET_UU)
    want = o.compute_ring_tr_generic(U, U, U, -1.0, KF, 3, 6, 3)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_cylinder_ring_transfer_oracle_identity():
    """Cylinder-ring-to-ring transfer (oracle, z axis: every stored mode has K_par >= 0, so the
    givers cover the field): the transfer between two cylinder rings is antisymmetric."""
    N = (64, 64, 64)
    V = ic.random_phase_field(N, seed=72)
    n, ns = 6, 3
    T = o.compute_cylinder_ring_tr_generic(V, V, V, -1.0, KF, 3, n, ns)
    scale = np.abs(T).max()
    assert scale > 0
    for i in range(1, n):
        for j in range(1, ns + 1):
            for m in range(1, n):
                for s in range(1, ns + 1):
                    assert abs(T[i, j, m, s] + T[m, s, i, j]) <= 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("N,axis,n,ns", [((64, 64, 64), 3, 6, 3), ((64, 64, 32), 1, 5, 4), ((32, 64, 64), 2, 7, 2)])
def test_gpu_cylinder_ring_to_ring_matches_oracle(lib, N, axis, n, ns):
    from tarang_b200.solver import IncFluid
    V = ic.random_phase_field(N, seed=90 + axis)
    s = IncFluid(N, nu=1e-3, dt=1e-3)
    s.set_V(V)
    T, r = s.Compute_cylinder_ring_tr(n, ns, axis)
    assert np.allclose(r, o.ring_radii(N, KF, n, Rin=float(o.krho_inside(N, KF, axis))), rtol=0, atol=0)
    want = o.compute_cylinder_ring_tr_generic(V, V, V, -1.0, KF, axis, n, ns)
    assert np.abs(T - want).max() <= 1e-12 * np.abs(want).max()


def test_helicity_spectra_oracle_identities():
    """The shell helicity spectrum sums to the total helicity sum 2 mult K . (Vr x Vi) within
    Max_radius_inside, and the ring helicity spectrum summed over sectors gives its shells; a
    Beltrami (ABC) field has helicity spectrum k0 times twice its energy spectrum."""
    N = (32, 32, 32)
    V = ic.random_phase_field(N, seed=21)
    h = o.shell_spectrum_helicity(V, KF)
    ring = o.ring_spectrum(V, KF, 3, 4, helicity=True)[0]
    kin = o.max_radius_inside(N, KF)
    tot = sum(h)
    assert np.allclose(ring.sum(axis=1)[1:kin + 1], tot[1:kin + 1], rtol=1e-12, atol=1e-16)
    A = o.abc_force(N, 2, 1.0, 1.0, 0.7, 0.4)          # curl A = k0 A
    H = sum(o.shell_spectrum_helicity(A, KF))
    E = sum(o.shell_spectrum(a, 0, KF) for a in A)
    assert abs(H[2] - 2 * E[2]) <= 1e-12 * abs(E[2]) and abs(H).sum() == pytest.approx(abs(H[2]), rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("N,kf", [((32, 32, 32), (1.0, 1.0, 1.0)), ((64, 32, 32), (1.0, 2.0, 0.5))])
def test_gpu_helicity_spectra_match_oracle(lib, N, kf):
    from tarang_b200.solver import IncFluid
    V = ic.random_phase_field(N, kfactor=kf, seed=33)
    s = IncFluid(N, kfactor=kf, nu=1e-3, dt=1e-3)
    s.set_V(V)
    for g, w in zip(s.CV_Compute_shell_spectrum_helicity(), o.shell_spectrum_helicity(V, kf)):
        assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
    for axis in (1, 3):
        g = s.CV_Compute_ring_spectrum_helicity(4, axis)
        w = o.ring_spectrum(V, kf, axis, 4, helicity=True)[0]
        assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
        g = s.CV_Compute_cylinder_ring_spectrum_helicity(3, axis)
        w = o.ring_spectrum(V, kf, axis, 3, cylinder=True, helicity=True)[0]
        assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
