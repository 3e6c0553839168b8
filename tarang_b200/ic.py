"""Initial conditions (host side, numpy; outside the hot path): the benchmark configurations and
the reference's initial-condition procedures (IncFluid::Read_init_cond init_cond_main.cc:52-206,
field_input_proc 1 field file, 2 reduced field file, 3 and 4 given modes, 5 energy spectrum, 6
energy-helicity spectrum, 7 Taylor-Green, 8 ABC, 51 RB Lorenz modes, 101 six-mode dynamo, 511
Rayleigh-Taylor), returned as the state
fields in the reference layout.

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


def _k_grids(N, kfactor, basis="FOUR"):
    N1, N2, N3 = N
    l1 = np.arange(N1)
    l2 = np.arange(N2)
    if basis == "SCFT":
        kx = l1.astype(np.float64) * kfactor[0]      # Get_kx_SCFT: the sine/cosine index m >= 0
    else:
        kx = np.where(l1 <= N1 // 2, l1, l1 - N1).astype(np.float64) * kfactor[0]
    ky = np.where(l2 <= N2 // 2, l2, l2 - N2).astype(np.float64) * kfactor[1]
    kz = np.arange(N3 // 2 + 1).astype(np.float64) * kfactor[2]
    return kx[:, None, None], ky[None, :, None], kz[None, None, :]


def keep_mask(N, basis="FOUR"):
    """Modes kept by the 2/3 rule (universal_misc.cc:118-159: FOUR |kx| < N1/3; SCFT m < 2 N1/3)."""
    N1, N2, N3 = N
    keep = np.ones((N1, N2, N3 // 2 + 1), dtype=bool)
    l1 = np.arange(N1)
    kx = np.where(l1 <= N1 // 2, l1, l1 - N1)
    if N1 >= 3 and basis == "SCFT":
        keep[2 * N1 // 3:] = False
    elif N1 >= 3:
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


def reality_kz0(A, basis="FOUR"):
    """Satisfy_reality_array on the kz = 0 plane (universal_misc.cc:51-109): FOUR
    A(kx, ky<0) = conj A(-kx, -ky), A(kx<0, 0) = conj A(-kx, 0); SCFT A(m, ky<0) = conj A(m, -ky)."""
    A = A.copy()
    N1, N2 = A.shape[0], A.shape[1]
    plane = A[:, :, 0].copy()
    if basis == "SCFT":
        for ly in range(N2 // 2 + 1, N2):
            A[:, ly, 0] = np.conj(plane[:, N2 - ly])
        return A
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
    V = _random_phase(N, kfactor, lambda idx: idx ** 4 * np.exp(-2.0 * (idx / k0) ** 2), seed, dealias)
    E = sum(energy_four(v) for v in V)
    s = math.sqrt(energy / E) if E > 0 else 0.0
    return [np.ascontiguousarray(v * s) for v in V]


def _shell_amp(N, kfactor, shell_energy, basis="FOUR"):
    """(amp, |K|): amp = sqrt(2 E(ceil|K|) / Approx_number_modes_in_shell) per stored mode
    (Approx_number_modes_in_shell: FOUR 2 pi r^2, SCFT pi r^2 over kf1 kf2 kf3, four_inline.h:
    276-306, scft_inline.h:242-260)."""
    N1, N2, N3 = N
    Kx, Ky, Kz = _k_grids(N, kfactor, basis)
    shape = (N1, N2, N3 // 2 + 1)
    Kx = np.broadcast_to(Kx, shape)
    Ky = np.broadcast_to(Ky, shape)
    Kz = np.broadcast_to(Kz, shape)
    K = np.sqrt(Kx * Kx + Ky * Ky + Kz * Kz)
    idx = np.ceil(K)
    Ek = shell_energy(idx)
    approx = (2 if basis == "FOUR" else 1) * math.pi * np.maximum(idx, 1) ** 2 / (kfactor[0] * kfactor[1] * kfactor[2])
    return np.sqrt(2 * Ek / approx), K


def _put_vector(N, kfactor, amp, ph1, ph2, ph3, dealias, basis="FOUR"):
    """Put_vector_amp_phase_comp_conj (ic_amp_phase.cc:54-157, anisotropy axis x) on every mode:
    uperp1 = amp e^{i ph1} cos(ph3), uperp2 = amp e^{i ph2} sin(ph3) turned into (Vx, Vy, Vz) by
    the polar and azimuthal angles of K; origin zeroed, dealiased, reality condition.  SCFT: the
    SCFT wavenumbers, and V1 -> i V1 (V1 is a sine series along x, ic_amp_phase.cc:151-153)."""
    N1, N2, N3 = N
    Kx, Ky, Kz = _k_grids(N, kfactor, basis)
    shape = (N1, N2, N3 // 2 + 1)
    Kx = np.broadcast_to(Kx, shape)
    Ky = np.broadcast_to(Ky, shape)
    Kz = np.broadcast_to(Kz, shape)
    K = np.sqrt(Kx * Kx + Ky * Ky + Kz * Kz)
    u1 = amp * np.exp(1j * ph1) * np.cos(ph3)
    u2 = amp * np.exp(1j * ph2) * np.sin(ph3)
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
    if basis == "SCFT":
        V[0] = 1j * V[0]
    if dealias:
        keep = keep_mask(N, basis)
        V = [np.where(keep, v, 0) for v in V]
    return [np.ascontiguousarray(reality_kz0(v, basis)) for v in V]


def _put_scalar(N, kfactor, amp, ph, dealias, basis="FOUR"):
    """Put_scalar_amp_phase_comp_conj (ic_amp_phase.cc:167-190): F = amp e^{i ph} (SCFT: i amp
    e^{i ph}, a sine series); origin zeroed, dealiased, reality condition."""
    _, K = _shell_amp(N, kfactor, lambda idx: idx, basis)
    F = np.where(K <= 1e-15, 0, amp * np.exp(1j * ph))
    if basis == "SCFT":
        F = 1j * F
    if dealias:
        F = np.where(keep_mask(N, basis), F, 0)
    return np.ascontiguousarray(reality_kz0(F, basis))


def _random_phase(N, kfactor, shell_energy, seed, dealias):
    """Random phases with the energy shell_energy(ceil|K|) spread over the shell's
    Approx_number_modes_in_shell (see the module docstring)."""
    amp, _ = _shell_amp(N, kfactor, shell_energy)
    rng = np.random.Generator(np.random.PCG64(seed))
    ph = rng.random((3,) + amp.shape) * 2 * math.pi
    return _put_vector(N, kfactor, amp, ph[0], ph[1], ph[2], dealias)


# --------------------------------------------------------------------------------------------
# The reference's initial-condition procedures
# --------------------------------------------------------------------------------------------

def _state_count(physics):
    return {"FLUID": 3, "MHD": 6, "SCALAR": 4, "RB": 4}[physics.upper()]


def modes_to_fields(k, F, N, basis="FOUR"):
    """Dense fields (N1, N2, N3/2+1) from a mode list (k (n, 3), F (n, m)): F[:, c] at (kx, ky,
    kz) of field c, zero elsewhere."""
    N1, N2, N3 = N
    out = [np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128) for _ in range(np.shape(F)[1])]
    for (kx, ky, kz), f in zip(np.asarray(k).tolist(), np.asarray(F)):
        lx = kx if (basis == "SCFT" or kx >= 0) else kx + N1
        for c, v in enumerate(f):
            out[c][lx, ky % N2, kz] = v
    return out


def taylor_green_field(N, k0=1, amp=1.0, basis="FOUR", physics="FLUID", ampW=0.0):
    """Init_cond_Taylor_Green (init_cond_TG.cc:47-120): V by Setup_Taylor_Green_field
    (ic_model.cc:58-104, the same modes and values as the Taylor-Green force), W of MHD by
    Setup_Taylor_Green_field_mag_field (ic_model.cc:122-183: real amp/8 values,
    -+ on V1, + on V2), T of a scalar zero.  Returns the state fields."""
    from . import forcing
    ns = _state_count(physics)
    k, F = forcing.taylor_green_modes(N, k0, amp, basis)
    out = modes_to_fields(k, F, N, basis)
    if ns == 6:
        a = ampW / 8
        table = ([((k0, k0, k0), -a, a), ((k0, -k0, k0), a, a), ((-k0, k0, k0), a, a), ((-k0, -k0, k0), -a, a)]
                 if basis == "FOUR" else [((k0, k0, k0), a, a), ((k0, -k0, k0), -a, a)])
        W = [np.zeros_like(out[0]) for _ in range(3)]
        for (kx, ky, kz), w1, w2 in table:
            lx = kx if (basis == "SCFT" or kx >= 0) else kx + N[0]
            W[0][lx, ky % N[1], kz] = w1
            W[1][lx, ky % N[1], kz] = w2
        out += W
    elif ns == 4:
        out.append(np.zeros_like(out[0]))
    return out


def abc_field(N, k0, amp, A, B, C, physics="FLUID", ampW=0.0):
    """Init_cond_ABC (init_cond_ABC.cc:52-151, FOUR only): Setup_ABC_field (ic_model.cc:187-236)
    for V (and W of MHD with ampW); a scalar's T is zero."""
    from . import forcing
    ns = _state_count(physics)
    if ns == 6:
        k, F = forcing.abc_modes(N, k0, amp, A, B, C, "MHD", ampW)
        return modes_to_fields(k, F, N)
    k, F = forcing.abc_modes(N, k0, amp, A, B, C)
    out = modes_to_fields(k, F, N)
    if ns == 4:
        out.append(np.zeros_like(out[0]))
    return out


def modes_field(entries, N, kfactor=(1.0, 1.0, 1.0), basis="FOUR", physics="FLUID", rule="simple"):
    """Init_cond_modes_SIMPLE (init_cond_modes.cc:107-480): entries (kx, ky, kz, Vx, Vy[, Wx, Wy
    | G]) as in_field_in.d lists them; Last_component gives each vector's third component and
    Add_complex_conj the conjugate mode on the kz = 0 and kz = N3/2 planes (the same rules as the
    given-mode force, forcing.given_modes).  rule "vorticity": Init_cond_modes_VORTICITY
    (:520-760), entries (kx, ky, kz, Vx, Omega_x[, Wx, OmegaW_x | G]) through Compute_VyVz."""
    from . import forcing
    k, F = forcing.given_modes(entries, N, kfactor, basis, physics, rule)
    return modes_to_fields(k, F, N, basis)


def model_shell_spectrum(n, a):
    """Model_initial_shell_spectrum (array_basic.cc:1400-1425): Sk(k) = a k^4 exp(-b k^1.1) /
    (k^4 + q^4)^(1 + 2.8/12), q = 1.5, b = 0.02, for k = 0 .. n-1."""
    kk = np.arange(n, dtype=np.float64)
    return a * kk ** 4 * np.exp(-0.02 * kk ** 1.1) / (kk ** 4 + 1.5 ** 4) ** (1.0 + 2.8 / 12.0)


def _model_spectrum(N, kfactor, a):
    # shells up to the largest |K| of the grid (the SCFT x index runs to N1 - 1)
    kmax = int(math.ceil(math.sqrt((N[0] * kfactor[0]) ** 2 + sum((N[i] // 2 * kfactor[i]) ** 2 for i in (1, 2))))) + 2
    Sk = model_shell_spectrum(kmax + 1, a)
    return lambda idx: Sk[np.minimum(idx.astype(int), kmax)]


def energy_spectrum_field(N, a, kfactor=(1.0, 1.0, 1.0), seed=20261202, dealias=True, physics="FLUID", a2=0.0,
                          basis="FOUR"):
    """Init_cond_energy_spectrum (init_cond_energy.cc:65-138): the energy of shell ceil|K| of the
    model spectrum, divided equally among the shell's modes (Approx_number_modes_in_shell of the
    basis), with random phases (Put_vector_amp_phase_comp_conj), the mean mode zero, dealiased,
    reality condition.  MHD (:318-413): W the same with the model spectrum of
    a2 = init_cond_double_para(2); passive scalar and convection (Init_cond_energy_spectrum(T)
    :152-223): T = ampT e^{i phaseT} with the spectrum of a2.  SCFT: the SCFT wavenumbers, mode
    count, 2/3 rule and reality condition, and V1, T multiplied by i (sine series along x).
    The reference seeds from time(0); numpy's PCG64 with `seed` stands in.  Returns the state
    fields [V1, V2, V3(, W1, W2, W3 | , T)]."""
    amp, _ = _shell_amp(N, kfactor, _model_spectrum(N, kfactor, a), basis)
    ns = _state_count(physics)
    rng = np.random.Generator(np.random.PCG64(seed))
    ph = rng.random(({3: 3, 6: 6, 4: 4}[ns],) + amp.shape) * 2 * math.pi
    out = _put_vector(N, kfactor, amp, ph[0], ph[1], ph[2], dealias, basis)
    if ns == 6:
        ampW, _ = _shell_amp(N, kfactor, _model_spectrum(N, kfactor, a2), basis)
        out += _put_vector(N, kfactor, ampW, ph[3], ph[4], ph[5], dealias, basis)
    elif ns == 4:
        ampT, _ = _shell_amp(N, kfactor, _model_spectrum(N, kfactor, a2), basis)
        out.append(_put_scalar(N, kfactor, ampT, ph[3], dealias, basis))
    return out


def energy_helicity_spectrum_field(N, a, sk, kfactor=(1.0, 1.0, 1.0), seed=20261202, dealias=True, physics="FLUID",
                                   a2=0.0, skW=0.0, h=0.0, basis="FOUR"):
    """Init_cond_energy_helicity_spectrum (init_cond_energy.cc:519-590, FOUR): as
    energy_spectrum_field with phase2 = phase1 + pi/2 and phase3 = asin(sk)/2, so every mode
    carries the relative helicity sk.  MHD (:721-824): W from the spectrum of a2 with
    zeta_b = asin(skW)/2, phase1W = phase1 - acos(h / cos(zeta - zeta_b)), phase2W = phase1W + pi/2
    (h = 2 Hc/(amp ampW)); passive scalar and convection (:604-681): T with the spectrum of a2
    and a random phase.  SCFT as in energy_spectrum_field (the relative helicity sk holds for the
    Fourier-basis vector (-i V1, V2, V3)).  Returns the state fields."""
    amp, _ = _shell_amp(N, kfactor, _model_spectrum(N, kfactor, a), basis)
    ns = _state_count(physics)
    rng = np.random.Generator(np.random.PCG64(seed))
    ph1 = rng.random(amp.shape) * 2 * math.pi
    zeta = math.asin(sk) / 2.0
    out = _put_vector(N, kfactor, amp, ph1, ph1 + math.pi / 2, np.full(amp.shape, zeta), dealias, basis)
    if ns == 6:
        ampW, _ = _shell_amp(N, kfactor, _model_spectrum(N, kfactor, a2), basis)
        zb = math.asin(skW) / 2.0
        p1w = ph1 - math.acos(h / math.cos(zeta - zb))
        out += _put_vector(N, kfactor, ampW, p1w, p1w + math.pi / 2, np.full(amp.shape, zb), dealias, basis)
    elif ns == 4:
        ampT, _ = _shell_amp(N, kfactor, _model_spectrum(N, kfactor, a2), basis)
        out.append(_put_scalar(N, kfactor, ampT, rng.random(amp.shape) * 2 * math.pi, dealias, basis))
    return out


def six_mode_field(N, k0, amp, ampW=None):
    """Init_cond_DYNAMO_SIX_MODE (init_cond_dynamo_6mode.cc:45-70, FOUR): V and W from
    Setup_SIX_MODE_field with amp = (amp101, amp011, amp112, h) and ampW likewise (W zero when
    ampW is None).  Returns [V1, V2, V3, W1, W2, W3]."""
    from . import forcing
    N1, N2, N3 = N
    out = [np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128) for _ in range(6)]
    for g, a in ((0, amp), (3, ampW)):
        if a is None:
            continue
        for (kx, ky, kz), vals in forcing.six_mode_table(int(k0), *a).items():
            for c, v in enumerate(vals):
                out[g + c][kx % N1, ky % N2, kz] = v
    return out


def rayleigh_taylor_field(N, slope):
    """Init_cond_Rayleigh_Taylor (init_cond_RayleighTaylor.cc:50-90, SCFT convection): u = 0 and
    theta(x) = x - (1 + tanh(slope (x - 1/2)))/2, uniform in y and z, sine-transformed along x.
    The reference computes x = lx / (local_N1_start + lx), which is 0/0 on the first plane and 1
    on every other; x = lx / N1 is used here.  The transform is the reference's forward SCFT of a
    field constant in y, z: theta(m, 0, 0) = (1/N1) sum_j theta_j sin(pi m (j + 1/2)/N1) for
    m = 1 .. N1 - 1 (slot 0 empty), then the 2/3 rule along x.  Returns [V1, V2, V3, theta]."""
    N1, N2, N3 = N
    out = [np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128) for _ in range(4)]
    x = np.arange(N1, dtype=np.float64) / N1
    th = x - (1.0 + np.tanh(slope * (x - 0.5))) / 2.0
    j = np.arange(N1, dtype=np.float64) + 0.5
    m = np.arange(1, N1, dtype=np.float64)
    S = np.sin(np.pi * np.outer(m, j) / N1) @ th / N1
    keep = np.arange(1, N1) < (2 * N1) // 3 if N1 >= 3 else np.ones(N1 - 1, dtype=bool)
    out[3][1:, 0, 0] = np.where(keep, S, 0.0)
    return out


def rb_lorenz_field(N, W101, T101, T200, kfactor=(1.0, 1.0, 1.0)):
    """Init_cond_RB_Lorenz (init_cond_RB_misc.cc:55-85, SCFT): V1(1,0,1) = W101, V2(1,0,1) = 0, V3
    from Last_component, theta(1,0,1) = T101, theta(2,0,0) = T200.  Returns [V1, V2, V3, theta]."""
    from . import forcing
    N1, N2, N3 = N
    out = [np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128) for _ in range(4)]
    vx, vy, vz = forcing.last_component(1, 0, 1, complex(W101), 0j, kfactor, "SCFT")
    out[0][1, 0, 1], out[1][1, 0, 1], out[2][1, 0, 1] = vx, vy, vz
    out[3][1, 0, 1] = T101
    out[3][2, 0, 0] = T200
    return out


def read_init_cond(cfg, data_dir=".", seed=20261202):
    """IncFluid::Read_init_cond (init_cond_main.cc:52-206) for a configuration from
    para.config_from_para: the initial state fields of its field_input_proc, read from
    data_dir/in/field_in.d where the procedure reads a file."""
    import os

    run = cfg.get("run", {})
    proc = run.get("field_input_proc", 0)
    N, basis, physics = tuple(cfg["N"]), cfg.get("basis", "FOUR"), cfg.get("physics", "FLUID")
    kf = tuple(cfg.get("kfactor", (1.0, 1.0, 1.0)))
    dp = list(run.get("init_cond_double", [])) + [0.0] * 10
    path = os.path.join(data_dir, "in", "field_in.d")
    ns = _state_count(physics)
    if proc in (1, 2):
        from .solver import read_field_file
        red = run.get("N_in_reduced") if proc == 2 else None
        return read_field_file(path, N, ns, basis, kf, bool(run.get("input_vx_vy", 0)), red)
    if proc in (3, 4):
        from . import forcing
        nv = {3: 2, 6: 4, 4: 3}[ns]
        return modes_field(forcing.read_force_modes_file(path, N[0], nv), N, kf, basis, physics,
                           "simple" if proc == 3 else "vorticity")
    if proc == 5:
        return energy_spectrum_field(N, dp[1], kf, seed, physics=physics, a2=dp[2], basis=basis)
    if proc == 6:
        # fluid: a, sk; scalar and convection: a, sk, a_T; MHD: a, sk, a_W, skW, h
        return energy_helicity_spectrum_field(N, dp[1], dp[2], kf, seed, physics=physics, a2=dp[3], skW=dp[4], h=dp[5],
                                              basis=basis)
    if proc == 7 and physics.upper() != "RB":
        # (convection: Init_cond_Taylor_Green_RB recurses into itself in the reference)
        return taylor_green_field(N, int(dp[1]), dp[2], basis, physics, dp[3])
    if proc == 8 and basis == "FOUR":
        return abc_field(N, int(dp[1]), dp[5], dp[2], dp[3], dp[4], physics, dp[6])
    if proc == 101 and physics.upper() == "MHD" and basis == "FOUR":
        return six_mode_field(N, int(dp[1]), tuple(dp[2:6]), tuple(dp[6:10]))
    if proc == 511 and physics.upper() == "RB" and basis == "SCFT":
        return rayleigh_taylor_field(N, dp[1])
    if proc == 51 and physics.upper() == "RB":
        return rb_lorenz_field(N, dp[1], dp[2], dp[3], kf)
    raise ValueError(f"field_input_proc {proc} ({physics}, {basis}) is not built")
