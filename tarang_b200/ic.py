"""Initial conditions of the benchmark configurations (host side, numpy; outside the hot path).

* Taylor-Green: the spectral placement of IncVF::Setup_Taylor_Green_field
  (lib/IncFlow/misc/ic_model.cc:58-89): u = amp sin(k0 x) cos(k0 y) cos(k0 z),
  v = -amp cos(k0 x) sin(k0 y) cos(k0 z), w = 0.
* Random-phase isotropic field: the construction of IncFluid::Init_cond_energy_spectrum
  (lib/IncFluid/input/init_cond_energy.cc:63-121) with Put_vector_amp_phase_comp_conj
  (lib/IncFlow/misc/ic_amp_phase.cc:54-157, anisotropy axis x): per mode
  amp = sqrt(2 E(ceil|K|) / Approx_number_modes_in_shell), three uniform phases, a vector
  perpendicular to K built from (uperp1, uperp2) and the polar/azimuthal angles of K; origin
  zeroed, dealiased, reality condition on the kz = 0 plane, then rescaled to the target energy.
  The reference seeds its RNG from time(0); here numpy's PCG64 with a fixed seed is used.
"""

from __future__ import annotations

import math

import numpy as np


def _k_grids(N, kfactor):
    N1, N2, N3 = N
    l1 = np.arange(N1)
    l2 = np.arange(N2)
    kx = np.where(l1 <= N1 // 2, l1, l1 - N1).astype(np.float64) * kfactor[0]
    ky = np.where(l2 <= N2 // 2, l2, l2 - N2).astype(np.float64) * kfactor[1]
    kz = np.arange(N3 // 2 + 1).astype(np.float64) * kfactor[2]
    return kx[:, None, None], ky[None, :, None], kz[None, None, :]


def keep_mask(N):
    """Modes kept by the 2/3 rule (universal_misc.cc:118-159, FOUR)."""
    N1, N2, N3 = N
    keep = np.ones((N1, N2, N3 // 2 + 1), dtype=bool)
    l1 = np.arange(N1)
    kx = np.where(l1 <= N1 // 2, l1, l1 - N1)
    if N1 >= 3:
        keep[np.abs(kx) >= N1 // 3] = False
    if N2 >= 3:
        keep[:, N2 // 3: 2 * N2 // 3 + 2] = False
    if N3 >= 3:
        keep[:, :, N3 // 3: N3 // 2 + 1] = False
    return keep


def energy_four(A):
    """Get_local_energy_FOUR (four_energy.cc:48-86) on one rank."""
    N1, N2 = A.shape[0], A.shape[1]
    P = np.abs(A) ** 2
    t = P.sum() + P[:, N2 // 2, :].sum() + P[N1 // 2].sum()
    t -= P[:, :, 0].sum() / 2 + P[:, N2 // 2, 0].sum() / 2 + P[N1 // 2, :, 0].sum() / 2
    t -= P[0, 0, 0] / 2
    return float(t)


def reality_kz0(A):
    """Satisfy_reality_array on the kz = 0 plane (universal_misc.cc:51-109, FOUR)."""
    A = A.copy()
    N1, N2 = A.shape[0], A.shape[1]
    plane = A[:, :, 0].copy()
    l1 = np.arange(N1)
    kx = np.where(l1 <= N1 // 2, l1, l1 - N1)
    conj_nx = np.where(-kx >= 0, -kx, -kx + N1)
    for ly in range(N2 // 2 + 1, N2):
        A[:, ly, 0] = np.conj(plane[conj_nx, N2 - ly])
    for lx in range(N1):
        if kx[lx] < 0:
            A[lx, 0, 0] = np.conj(plane[-kx[lx], 0])
    return A


def taylor_green(N, k0=1, amp=1.0):
    """IncVF::Setup_Taylor_Green_field (ic_model.cc:58-89), FOUR basis."""
    N1, N2, N3 = N
    shape = (N1, N2, N3 // 2 + 1)
    V = [np.zeros(shape, dtype=np.complex128) for _ in range(3)]
    lxp, lxm = k0, N1 - k0
    lyp, lym = k0, N2 - k0
    V[0][lxp, lyp, k0] = -1j * amp / 8
    V[0][lxp, lym, k0] = -1j * amp / 8
    V[1][lxp, lyp, k0] = 1j * amp / 8
    V[1][lxp, lym, k0] = -1j * amp / 8
    V[0][lxm, lyp, k0] = 1j * amp / 8
    V[0][lxm, lym, k0] = 1j * amp / 8
    V[1][lxm, lyp, k0] = 1j * amp / 8
    V[1][lxm, lym, k0] = -1j * amp / 8
    return V


def rb_perturbation(N, nmodes=8, amp=1e-3, seed=20261205):
    """Rayleigh-Benard initial temperature deviation in the SCFT basis: modes 1 <= m <= nmodes,
    |ky| <= nmodes, kz <= nmodes get real and imaginary parts uniform in (-amp, amp) (seeded),
    then the SCFT reality condition on the kz = 0 plane (universal_misc.cc:93-104); the velocity
    starts at zero.  Returns theta, shape (N1, N2, N3/2+1)."""
    N1, N2, N3 = N
    rng = np.random.Generator(np.random.PCG64(seed))
    T = np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128)
    kys = list(range(0, nmodes + 1)) + list(range(-nmodes, 0))
    for m in range(1, min(nmodes, N1 - 1) + 1):
        for ky in kys:
            ly = ky if ky >= 0 else ky + N2
            for kz in range(0, min(nmodes, N3 // 2) + 1):
                re, im = rng.uniform(-amp, amp, size=2)
                T[m, ly, kz] = re + 1j * im
    for ly in range(N2 // 2 + 1, N2):
        T[:, ly, 0] = np.conj(T[:, N2 - ly, 0])
    T[:, 0, 0] = T[:, 0, 0].real
    # the reference dealiases every initial condition (SCFT 2/3 rule, universal_misc.cc:142-158)
    keep = np.ones(T.shape, dtype=bool)
    if N1 >= 3:
        keep[2 * N1 // 3:] = False
    if N2 >= 3:
        keep[:, N2 // 3: 2 * N2 // 3 + 2] = False
    if N3 >= 3:
        keep[:, :, N3 // 3: N3 // 2 + 1] = False
    return np.where(keep, T, 0)


def random_phase_field(N, kfactor=(1.0, 1.0, 1.0), k0=4.0, energy=0.5, seed=20261202, dealias=True):
    """Seeded random-phase divergence-free field with E(k) ~ k^4 exp(-2 (k/k0)^2), total
    energy `energy` in the Get_total_energy convention.  Returns [V1, V2, V3]."""
    N1, N2, N3 = N
    rng = np.random.Generator(np.random.PCG64(seed))
    Kx, Ky, Kz = _k_grids(N, kfactor)
    shape = (N1, N2, N3 // 2 + 1)
    Kx = np.broadcast_to(Kx, shape)
    Ky = np.broadcast_to(Ky, shape)
    Kz = np.broadcast_to(Kz, shape)
    K = np.sqrt(Kx * Kx + Ky * Ky + Kz * Kz)
    idx = np.ceil(K)
    Ek = idx ** 4 * np.exp(-2.0 * (idx / k0) ** 2)
    approx = 2 * math.pi * np.maximum(idx, 1) ** 2 / (kfactor[0] * kfactor[1] * kfactor[2])
    amp = np.sqrt(2 * Ek / approx)
    ph = rng.random((3,) + shape) * 2 * math.pi
    u1 = amp * np.exp(1j * ph[0]) * np.cos(ph[2])
    u2 = amp * np.exp(1j * ph[1]) * np.sin(ph[2])
    # polar angle from the x axis, azimuth in the (y, z) plane (anisotropy switch 1)
    kperp = np.sqrt(Ky * Ky + Kz * Kz)
    with np.errstate(invalid="ignore", divide="ignore"):
        theta = np.arctan2(kperp, Kx)
        phi = np.arctan2(Kz, Ky)
    vpll = -u2 * np.sin(theta)
    vh1 = u2 * np.cos(theta) * np.cos(phi) + u1 * np.sin(phi)
    vh2 = u2 * np.cos(theta) * np.sin(phi) - u1 * np.cos(phi)
    on_axis = kperp <= 1e-15
    vpll = np.where(on_axis, 0, vpll)
    vh1 = np.where(on_axis, u1, vh1)
    vh2 = np.where(on_axis, u2, vh2)
    V = [vpll, vh1, vh2]
    for v in V:
        v[K <= 1e-15] = 0
    if dealias:
        keep = keep_mask(N)
        V = [np.where(keep, v, 0) for v in V]
    V = [reality_kz0(v) for v in V]
    E = sum(energy_four(v) for v in V)
    s = math.sqrt(energy / E) if E > 0 else 0.0
    return [np.ascontiguousarray(v * s) for v in V]
