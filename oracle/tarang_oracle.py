"""CPU oracle: an FP64 restatement of Tarang-4.0's pseudo-spectral time-step path.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA path: only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl
reference`` legs of ``bench.py`` may import it.  The product (the C-ABI library
``tarang_b200/libtarang_gpu.so`` and its Python mirror) never calls it.

Parity status.  The reference (C++, blitz++, FFTW3-MPI, MPI) cannot be built on
this image, so the oracle restates its algorithms and is pinned by
  * the one known answer in the reference's own tests
    (``trunk/test/test-fftw/out1.d``: an unnormalised C2R->R2C round trip of a
    unit delta at (0,0,2) on a 4^3 grid returns 64 = N^3,
    produced by ``trunk/test/test-fftw/main_mpi.cc:93-118``), and
  * the reference's own inline wavenumber code (``lib/four/four_inline.h``,
    ``lib/scft/scft_inline.h``) compiled from the reference tree with
    declaration-only stand-ins for the MPI, FFTW and blitz++ headers
    (``oracle/ref_pin``): wavenumbers, |K|, multiplicity factors, radii and
    anisotropic extents, stored as ``tests/golden/ref_inline.json``, and
  * analytic known answers (single modes, Taylor-Green, Beltrami flow,
    exact viscous decay, energy conservation of the inviscid nonlinear term,
    antisymmetry of the shell-to-shell transfer),
  all checked in ``tests/test_oracle_*.py``.  Every other value is "parity
  unpinned by the reference's own tests" and is pinned by those identities.

Transforms use ``scipy.fft`` (pocketfft), whose unnormalised r2c/c2r and
DCT/DST-II/III definitions are the published definitions FFTW uses for
``fftw_plan_dft_r2c``/``c2r`` and REDFT10/RODFT10/REDFT01/RODFT01.

Array layout (the reference's): spectral fields are complex128 arrays of shape
(N1, N2, N3//2+1) indexed (l1, l2, l3); real-space fields are float64 arrays of
shape (N1, N2, N3) indexed (x, y, z).  Wavenumbers follow
``lib/four/four_inline.h:88-129`` (index <= N/2 counts as positive).

File:line citations are relative to the reference project root (``trunk/``).
"""

from __future__ import annotations

import math
import os

import numpy as np
import scipy.fft as sfft

_WORKERS = int(os.environ.get("TARANG_ORACLE_WORKERS", os.cpu_count() or 1))

MYEPS = 1e-15      # lib/basis_basicfn/extern_def_vars.h:81
MYEPS2 = 1e-5      # lib/basis_basicfn/extern_def_vars.h:82
INF_RADIUS = 1e4   # lib/basis_basicfn/extern_def_vars.h (INF_RADIUS used as the last sphere)


# --------------------------------------------------------------------------------------
# Wavenumber helpers  (lib/four/four_inline.h, lib/scft/scft_inline.h)
# --------------------------------------------------------------------------------------

def kx_four(N1):
    """Get_kx_FOUR  lib/four/four_inline.h:88-92 (single rank: local_N1_start = 0)."""
    l = np.arange(N1)
    return np.where(l <= N1 // 2, l, l - N1)


def ky_four(N2):
    """Get_ky3D_FOUR  lib/four/four_inline.h:129."""
    l = np.arange(N2)
    return np.where(l <= N2 // 2, l, l - N2)


def kz_four(N3):
    return np.arange(N3 // 2 + 1)


def kx_scft(N1):
    """Get_kx_SCFT  lib/scft/scft_inline.h:86 (kx = m >= 0)."""
    return np.arange(N1)


def kvec(N, kfactor, basis="FOUR"):
    """Broadcastable (Kx, Ky, Kz) grids of actual wavenumbers (globalvar_waveno_switch = 0)."""
    N1, N2, N3 = N
    kx = (kx_four(N1) if basis == "FOUR" else kx_scft(N1)).astype(np.float64) * kfactor[0]
    ky = ky_four(N2).astype(np.float64) * kfactor[1]
    kz = kz_four(N3).astype(np.float64) * kfactor[2]
    return kx[:, None, None], ky[None, :, None], kz[None, None, :]


def kmag(N, kfactor, basis="FOUR"):
    """Kmagnitude_FOUR  lib/four/four_inline.h:155-166; Kmagnitude_SCFT scft_inline.h:128-139."""
    Kx, Ky, Kz = kvec(N, kfactor, basis)
    return np.sqrt(Kx * Kx + Ky * Ky + Kz * Kz)


def ksqr(N, kfactor, basis="FOUR"):
    Kx, Ky, Kz = kvec(N, kfactor, basis)
    return Kx * Kx + Ky * Ky + Kz * Kz


def max_radius_inside(N, kfactor, alias="DEALIAS", basis="FOUR"):
    """Max_radius_inside_(de)aliased_FOUR  lib/four/four_inline.h:190-257 (SCFT: scft_inline.h)."""
    N1, N2, N3 = N
    if basis == "FOUR":
        d = 3 if alias == "DEALIAS" else 2
        kmag_ = min((N1 // d) * kfactor[0], (N2 // d) * kfactor[1])
        if N3 > 2:
            kmag_ = min(kmag_, (N3 // d) * kfactor[2])
        return int(kmag_)
    # SCFT: x extent is N1 - 1 (dealiased 2N1/3), y/z as FOUR (scft_inline.h:144-220)
    if alias == "DEALIAS":
        kmag_ = min((2 * N1 // 3) * kfactor[0], (N2 // 3) * kfactor[1])
        if N3 > 2:
            kmag_ = min(kmag_, (N3 // 3) * kfactor[2])
    else:
        kmag_ = min((N1 - 1) * kfactor[0], (N2 // 2) * kfactor[1])
        if N3 > 2:
            kmag_ = min(kmag_, (N3 // 2) * kfactor[2])
    return int(kmag_)


def min_radius_outside(N, kfactor, alias="DEALIAS", basis="FOUR"):
    """Min_radius_outside_(de)aliased_FOUR  lib/four/four_inline.h:172-228."""
    N1, N2, N3 = N
    if basis == "FOUR":
        d = 3 if alias == "DEALIAS" else 2
        return int(math.ceil(math.sqrt(((N1 // d) * kfactor[0]) ** 2 + ((N2 // d) * kfactor[1]) ** 2
                                       + ((N3 // d) * kfactor[2]) ** 2)))
    if alias == "DEALIAS":
        return int(math.ceil(math.sqrt(((2 * N1 // 3) * kfactor[0]) ** 2 + ((N2 // 3) * kfactor[1]) ** 2
                                       + ((N3 // 3) * kfactor[2]) ** 2)))
    return int(math.ceil(math.sqrt(((N1 - 1) * kfactor[0]) ** 2 + ((N2 // 2) * kfactor[1]) ** 2
                                   + ((N3 // 2) * kfactor[2]) ** 2)))


def approx_number_modes_in_shell(N, radius, kfactor, basis="FOUR"):
    """Approx_number_modes_in_shell_FOUR  four_inline.h:276-306 (3-D: hemisphere, 2 pi r^2);
    Approx_number_modes_in_shell_SCFT  scft_inline.h:242-260 (3-D: quarter sphere, pi r^2)."""
    if basis == "FOUR":
        return (2 * math.pi * radius * radius) / (kfactor[0] * kfactor[1] * kfactor[2])
    return (math.pi * radius * radius) / (kfactor[0] * kfactor[1] * kfactor[2])


def multiplicity_four(N):
    """Multiplicity_factor_FOUR  lib/four/four_inline.h:347-365 as a (N1,N2,N3/2+1) array."""
    N1, N2, N3 = N
    kx = kx_four(N1)[:, None, None]
    ky = ky_four(N2)[None, :, None]
    l3 = kz_four(N3)[None, None, :]
    f = np.where(l3 > 0, 1.0, 0.5)
    dbl = (kx == N1 // 2) | ((ky == N2 // 2) & (N2 > 1))
    return np.broadcast_to(np.where(dbl, 2 * f, f), (N1, N2, N3 // 2 + 1)).copy()


def multiplicity_scft(N):
    """Multiplicity_factor_SCFT  lib/scft/scft_inline.h:313-335."""
    N1, N2, N3 = N
    m = kx_scft(N1)[:, None, None]
    ky = ky_four(N2)[None, :, None]
    l3 = kz_four(N3)[None, None, :]
    f = np.where(l3 > 0, np.where(m > 0, 2.0, 1.0), np.where(m > 0, 1.0, 0.5))
    dbl = (ky == N2 // 2) & (N2 > 1)
    return np.broadcast_to(np.where(dbl, 2 * f, f), (N1, N2, N3 // 2 + 1)).copy()


def multiplicity(N, basis="FOUR"):
    return multiplicity_four(N) if basis == "FOUR" else multiplicity_scft(N)


# --------------------------------------------------------------------------------------
# Dealiasing and reality condition  (lib/fields/universal/universal_misc.cc)
# --------------------------------------------------------------------------------------

def dealias_keep_mask(N, basis="FOUR"):
    """Boolean mask of modes that Dealias_array keeps  (universal_misc.cc:118-159)."""
    N1, N2, N3 = N
    keep = np.ones((N1, N2, N3 // 2 + 1), dtype=bool)
    if N1 >= 3:
        if basis == "FOUR":
            kx = kx_four(N1)
            keep[np.abs(kx) >= N1 // 3, :, :] = False
        else:
            kx = kx_scft(N1)
            keep[np.abs(kx) >= 2 * N1 // 3, :, :] = False
    if N2 >= 3:
        keep[:, N2 // 3: 2 * N2 // 3 + 2, :] = False   # Range(N2/3, 2N2/3+1) inclusive
    if N3 >= 3:
        keep[:, :, N3 // 3: N3 // 2 + 1] = False       # Range(N3/3, N3/2) inclusive
    return keep


def dealias(A, basis="FOUR"):
    """Dealias_array  universal_misc.cc:118-159 (returns a new array)."""
    return np.where(dealias_keep_mask(A.shape[:2] + ((A.shape[2] - 1) * 2,), basis), A, 0)


def satisfy_reality(A, basis="FOUR"):
    """Satisfy_reality_array  universal_misc.cc:51-109: for kz = 0 and kz = N3/2 planes set
    A(kx, ky<0) = conj(A(-kx, -ky)) and A(kx<0, 0) = conj(A(-kx, 0)), from a snapshot."""
    A = A.copy()
    N1, N2 = A.shape[0], A.shape[1]
    N3h = A.shape[2] - 1
    for l3 in (0, N3h):
        plane = A[:, :, l3].copy()
        if basis == "FOUR":
            kx = kx_four(N1)
            conj_nx = np.where(-kx >= 0, -kx, -kx + N1)
            for ly in range(N2 // 2 + 1, N2):
                pos_iy = -(ly - N2)
                A[:, ly, l3] = np.conj(plane[conj_nx, pos_iy])
            for lx in range(N1):
                if kx[lx] < 0:
                    A[lx, 0, l3] = np.conj(plane[-kx[lx], 0])
        else:
            for ly in range(N2 // 2 + 1, N2):
                pos_iy = -(ly - N2)
                A[:, ly, l3] = np.conj(A[:, pos_iy, l3])
    return A


# --------------------------------------------------------------------------------------
# FOUR transforms  (lib/four/four_tr.cc)
# --------------------------------------------------------------------------------------

def forward_four(real):
    """ArrayFFT_FOUR  four_tr.cc:199-209: zero-pad, r2c (sign -1), then Norm_FOUR 1/(N1N2N3)
    (four_tr.cc:306-309).  Input real (N1,N2,N3) -> spectrum (N1,N2,N3/2+1)."""
    N1, N2, N3 = real.shape
    return sfft.rfftn(real, axes=(0, 1, 2), workers=_WORKERS) / (N1 * N2 * N3)


def inverse_four(spec, N3=None):
    """ArrayIFFT_FOUR  four_tr.cc:229-295: unnormalised c2c(y), c2c(x), c2r(z).  The c2r along
    z uses only the real parts of the kz = 0 and kz = N3/2 entries (FFTW/pocketfft c2r rule)."""
    N1, N2, M1 = spec.shape
    if N3 is None:
        N3 = 2 * (M1 - 1)
    return sfft.irfftn(spec, s=(N1, N2, N3), axes=(0, 1, 2), workers=_WORKERS) * (N1 * N2 * N3)


def xderiv_four(A, kfactor):
    """Xderiv_FOUR  four_tr.cc:314-323: B = i kx A."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    Kx, _, _ = kvec(N, kfactor)
    return 1j * Kx * A


def yderiv_four(A, kfactor):
    """Yderiv_FOUR  four_tr.cc:329-343."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    _, Ky, _ = kvec(N, kfactor)
    return 1j * Ky * A


def zderiv_four(A, kfactor):
    """Zderiv_FOUR  four_tr.cc:348-353."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    _, _, Kz = kvec(N, kfactor)
    return 1j * Kz * A


# --------------------------------------------------------------------------------------
# SCFT transforms  (lib/scft/scft_tr.cc): axis 0 (x) is sin/cos on the half-sample grid
# --------------------------------------------------------------------------------------

def forward_scft(real, parity):
    """ArraySFT_SCFT (parity 1) / ArrayCFT_SCFT (parity 0)  scft_tr.cc:230-431.
    RODFT10 / REDFT10 along x, r2c over (y, z), Norm_SCFT 1/(2 N1 N2 N3) (scft_tr.cc:89-92);
    the sine coefficients are shifted one slot right (ArrayShiftRight_SCFT scft_tr.cc:153-184):
    slot m <-> sin(m pi x), slot 0 = 0, the last DST-II coefficient is dropped."""
    N1, N2, N3 = real.shape
    if parity == 1:
        t = sfft.dst(real, type=2, axis=0, norm=None, workers=_WORKERS)
    else:
        t = sfft.dct(real, type=2, axis=0, norm=None, workers=_WORKERS)
    s = sfft.rfftn(t, axes=(1, 2), workers=_WORKERS) / (2.0 * N1 * N2 * N3)
    if parity == 1:
        out = np.zeros_like(s)
        out[1:] = s[:-1]
        return out
    return s


def inverse_scft(spec, parity, N3=None):
    """ArrayISFT_SCFT (parity 1) / ArrayICFT_SCFT (parity 0)  scft_tr.cc:440-639: shift left
    (sine), unnormalised c2r over (y, z), then RODFT01 / REDFT01 along x."""
    N1, N2, M1 = spec.shape
    if N3 is None:
        N3 = 2 * (M1 - 1)
    if parity == 1:
        s = np.zeros_like(spec)
        s[:-1] = spec[1:]
    else:
        s = spec
    r = sfft.irfftn(s, s=(N2, N3), axes=(1, 2), workers=_WORKERS) * (N2 * N3)
    if parity == 1:
        return sfft.dst(r, type=3, axis=0, norm=None, workers=_WORKERS)
    return sfft.dct(r, type=3, axis=0, norm=None, workers=_WORKERS)


def xderiv_scft(A, kfactor, parity):
    """Xderiv_Sin_SCFT (+kx, sin -> cos) / Xderiv_Cos_SCFT (-kx, cos -> sin)  scft_tr.cc:649-672.
    parity follows universal_tr.cc:186-210: parity 1 = the input is a sine series."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    Kx, _, _ = kvec(N, kfactor, "SCFT")
    return (Kx * A) if parity == 1 else (-Kx * A)


def forward(real, basis="FOUR", parity=0):
    """Forward_transform_array  universal_tr.cc:66-86."""
    return forward_four(real) if basis == "FOUR" else forward_scft(real, parity)


def inverse(spec, basis="FOUR", parity=0, N3=None):
    """Inverse_transform_array  universal_tr.cc:126-146."""
    return inverse_four(spec, N3) if basis == "FOUR" else inverse_scft(spec, parity, N3)


def xderiv(A, kfactor, basis="FOUR", parity=0):
    return xderiv_four(A, kfactor) if basis == "FOUR" else xderiv_scft(A, kfactor, parity)


yderiv = lambda A, kfactor, basis="FOUR", parity=0: yderiv_four(A, kfactor)   # noqa: E731  Fourier in y
zderiv = lambda A, kfactor, basis="FOUR", parity=0: zderiv_four(A, kfactor)   # noqa: E731  Fourier in z


# --------------------------------------------------------------------------------------
# Energies and spectra  (lib/four/four_energy.cc, lib/scft/scft_energy.cc)
# --------------------------------------------------------------------------------------

def total_energy_four(A, B=None):
    """Get_local_energy_FOUR  four_energy.cc:48-86 (and the cross form :108-168), 1 rank:
    sum over stored modes + the unstored ky = -N2/2 and kx = -N1/2 planes, kz = 0 halved,
    origin excluded."""
    if B is None:
        B = A
    N1, N2 = A.shape[0], A.shape[1]
    P = np.real(A * np.conj(B))
    t = P.sum()
    if N2 > 1:
        t += P[:, N2 // 2, :].sum()
    t += P[N1 // 2, :, :].sum()
    t -= P[:, :, 0].sum() / 2
    if N2 > 1:
        t -= P[:, N2 // 2, 0].sum() / 2
    t -= P[N1 // 2, :, 0].sum() / 2
    t -= P[0, 0, 0] / 2
    return float(t)


def total_energy_scft(A, B=None):
    """Get_total_energy_SCFT  scft_energy.cc:51-104: per ky plane 2 sum|A|^2 - sum|A(m,ky,0)|^2
    - sum|A(0,ky,kz)|^2 + |A(0,ky,0)|^2/2 (weights 2/1/1/half = Multiplicity_factor_SCFT), the
    ky = N2/2 plane counted twice, minus |A(0,0,0)|^2/2 (origin excluded)."""
    if B is None:
        B = A
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    mult = multiplicity_scft(N)
    P = np.real(A * np.conj(B))
    t = (mult * P).sum() - mult[0, 0, 0] * P[0, 0, 0]
    return float(t)


def total_energy(A, basis="FOUR", B=None):
    return total_energy_four(A, B) if basis == "FOUR" else total_energy_scft(A, B)


def total_Sn(A, n, kfactor, alias="DEALIAS", basis="FOUR"):
    """Get_local_Sn_FOUR  four_energy.cc:179-211: sum mult K^n |A|^2 over K <= kmax_outside;
    for n = 0 the origin is subtracted."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    K = kmag(N, kfactor, basis)
    kkmax = min_radius_outside(N, kfactor, alias, basis)
    mult = multiplicity(N, basis)
    # Get_local_Sn_SCFT (scft_energy.cc:187) has `if (kkmag <= kkmax);` -- the empty statement
    # makes the sum run over every mode
    inside = (K <= kkmax) if basis == "FOUR" else np.ones_like(K, dtype=bool)
    w = np.where(inside, mult * (K ** n if n != 0 else 1.0), 0.0)
    s = float((w * np.abs(A) ** 2).sum())
    if n == 0:
        s -= mult[0, 0, 0] * abs(A[0, 0, 0]) ** 2
    return s


def shell_spectrum(A, n, kfactor, alias="DEALIAS", basis="FOUR", B=None):
    """Compute_shell_spectrum_FOUR  four_energy.cc:244-338 (cross form :341-436):
    Sk(ceil|K|) += mult K^n Re(A B*) for ceil|K| <= kkmax; shells (kmax_inside, kmax] rescaled
    by Approx_number_modes_in_shell / count when count >= 1.  Length kmax_outside + 1."""
    if B is None:
        B = A
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    K = kmag(N, kfactor, basis)
    kkmax = min_radius_outside(N, kfactor, alias, basis)
    kin = max_radius_inside(N, kfactor, alias, basis)
    mult = multiplicity(N, basis)
    idx = np.ceil(K).astype(np.int64)
    sel = idx <= kkmax
    val = mult * (K ** n if n != 0 else 1.0) * np.real(A * np.conj(B))
    Sk = np.bincount(idx[sel], weights=val[sel], minlength=kkmax + 1)[: kkmax + 1]
    # SCFT counts factor/2 (Compute_local_shell_spectrum_SCFT scft_energy.cc:279)
    cmult = mult if basis == "FOUR" else mult / 2
    cnt = np.bincount(idx[sel], weights=np.broadcast_to(cmult, K.shape)[sel], minlength=kkmax + 1)[: kkmax + 1]
    for i in range(kin + 1, kkmax + 1):
        if cnt[i] >= 1:
            Sk[i] = Sk[i] * approx_number_modes_in_shell(N, i, kfactor, basis) / cnt[i]
    return Sk


# --------------------------------------------------------------------------------------
# Field operations used by the solver
# --------------------------------------------------------------------------------------

def divide_ksqr(A, kfactor, basis="FOUR"):
    """Array_divide_ksqr_FOUR  four_basic.cc:220-245 (A(0,0,0) = 0)."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    K2 = ksqr(N, kfactor, basis)
    with np.errstate(divide="ignore", invalid="ignore"):
        out = A / K2
    out[0, 0, 0] = 0.0
    return out


def exp_ksqr(A, factor, kfactor, basis="FOUR"):
    """Array_exp_ksqr_FOUR  four_basic.cc:312-337: A *= exp(factor K^2)."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    return A * np.exp(factor * ksqr(N, kfactor, basis))


def exp_ksqr_hyper(A, factor, hyper_factor, kfactor, basis="FOUR"):
    """Array_exp_ksqr_FOUR with the hyper term  four_basic.cc:377-403 (Array_exp_ksqr_SCFT
    scft_basic.cc:370-395): A *= exp((factor + hyper_factor K^2) K^2)."""
    if hyper_factor == 0:
        return exp_ksqr(A, factor, kfactor, basis)
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    K2 = ksqr(N, kfactor, basis)
    return A * np.exp((factor + hyper_factor * K2) * K2)


def if_time_advance(u0, coefs, rhs, dt, scheme, kfactor, basis="FOUR"):
    """IncFluid::Time_advance  time_advance.cc:60-163 on a list of fields: EULER, RK2 or RK4 with
    Single_time_step(dt, a, b, c) = E(b)(E(a - b) u + c dt N)  single_time_step.cc:54-86 and
    E(a) = exp(-(nu + nu_h K^2) a dt K^2) per field (Mult_field_exp_ksqr_dt mult_exp_visc.cc:
    56-165); coefs[i] = (nu, nu_h); rhs(fields) -> right-hand sides (Compute_rhs)."""
    n = len(u0)

    def E(A, i, a):
        nu, nh = coefs[i]
        return exp_ksqr_hyper(A, -nu * a * dt, -nh * a * dt, kfactor, basis)

    if scheme == "EULER":                       # Single_time_step(dt, 1, 1, 1)
        r = rhs(u0)
        return [E(u0[i] + dt * r[i], i, 1.0) for i in range(n)]
    if scheme == "RK2":
        r = rhs(u0)                             # Single_time_step(dt, 1/2, 1/2, 1/2)
        um = [E(u0[i] + (dt / 2) * r[i], i, 0.5) for i in range(n)]
        r = rhs(um)                             # Single_time_step(dt, 1, 1/2, 1) from u0
        return [E(E(u0[i], i, 0.5) + dt * r[i], i, 0.5) for i in range(n)]
    if scheme != "RK4":
        raise ValueError(scheme)
    r = rhs(u0)
    u = [E(u0[i] + (dt / 2) * r[i], i, 0.5) for i in range(n)]
    tot = [(dt / 6) * E(r[i], i, 1.0) for i in range(n)]
    r = rhs(u)
    u = [E(u0[i], i, 0.5) + (dt / 2) * r[i] for i in range(n)]
    tot = [tot[i] + (dt / 3) * E(r[i], i, 0.5) for i in range(n)]
    r = rhs(u)
    u = [E(E(u0[i], i, 0.5) + dt * r[i], i, 0.5) for i in range(n)]
    tot = [tot[i] + (dt / 3) * E(r[i], i, 0.5) for i in range(n)]
    r = rhs(u)
    tot = [tot[i] + (dt / 6) * r[i] for i in range(n)]
    return [E(u0[i], i, 1.0) + tot[i] for i in range(n)]


# --------------------------------------------------------------------------------------
# Nonlinear terms  (lib/IncFlow/nlin_calc)
# --------------------------------------------------------------------------------------

def nlin_fluid(V, kfactor, basis="FOUR", alias="DEALIAS"):
    """IncVF::Compute_nlin()  compute_nlin.cc:58-108 (normal order):
    nlin_i = D_j F(u_i u_j) with the diagonal products first (RSprod.cc:52-57, Nlin.cc:85-94),
    then the off-diagonal products u1u2, u2u3, u3u1 (RSprod.cc:70-77) and their derivatives
    (Derivative_RSprod_VV RSprod.cc:94-105); then Dealias_nlin (dealias.cc:113-119)."""
    N1, N2 = V[0].shape[0], V[0].shape[1]
    N3 = 2 * (V[0].shape[2] - 1)
    par_inv = (1, 0, 0)
    ur = [inverse(V[i], basis, par_inv[i], N3) for i in range(3)]
    nl = [forward(ur[i] * ur[i], basis, 0) for i in range(3)]
    nl[0] = xderiv(nl[0], kfactor, basis, 0)
    nl[1] = yderiv(nl[1], kfactor)
    nl[2] = zderiv(nl[2], kfactor)
    p12 = forward(ur[0] * ur[1], basis, 1)   # RV_Forward_transform_RSprod Rvf.cc:179-186: SFT, CFT, SFT
    p23 = forward(ur[1] * ur[2], basis, 0)
    p31 = forward(ur[2] * ur[0], basis, 1)
    nl[0] = nl[0] + yderiv(p12, kfactor) + zderiv(p31, kfactor)
    nl[1] = nl[1] + xderiv(p12, kfactor, basis, 1) + zderiv(p23, kfactor)
    nl[2] = nl[2] + xderiv(p31, kfactor, basis, 1) + yderiv(p23, kfactor)
    if alias == "DEALIAS":
        nl = [dealias(a, basis) for a in nl]
    return nl


def nlin_mhd(V, W, kfactor, basis="FOUR", alias="DEALIAS"):
    """IncVF::Compute_nlin(IncVF& W)  compute_nlin_VF_MHD.cc:72-164 with Elsasser variables
    (elsasser.cc:53-130): Zp = U + B, Zm = U - B;  Zp.nlin_i = D_j F(Zm_j Zp_i),
    Zm.nlin_i = D_j F(Zp_j Zm_i) (RSprod.cc:117-194); U.nlin = (Zp.nlin + Zm.nlin)/2,
    B.nlin = (Zp.nlin - Zm.nlin)/2; Dealias_nlin(W).  Returns (U.nlin, B.nlin)."""
    N3 = 2 * (V[0].shape[2] - 1)
    Zp = [V[i] + W[i] for i in range(3)]
    Zm = [V[i] - W[i] for i in range(3)]
    par_inv = (1, 0, 0)
    zp = [inverse(Zp[i], basis, par_inv[i], N3) for i in range(3)]
    zm = [inverse(Zm[i], basis, par_inv[i], N3) for i in range(3)]
    d = [forward(zp[i] * zm[i], basis, 0) for i in range(3)]
    d[0] = xderiv(d[0], kfactor, basis, 0)
    d[1] = yderiv(d[1], kfactor)
    d[2] = zderiv(d[2], kfactor)
    n = list(d)
    nw = list(d)
    v1 = forward(zp[0] * zm[1], basis, 1)
    w1 = forward(zm[0] * zp[1], basis, 1)
    v2 = forward(zp[1] * zm[2], basis, 0)
    w2 = forward(zm[1] * zp[2], basis, 0)
    v3 = forward(zp[2] * zm[0], basis, 1)
    w3 = forward(zm[2] * zp[0], basis, 1)
    # Derivative_RSprod_VV(W) RSprod.cc:170-193
    n[0] = n[0] + yderiv(v1, kfactor) + zderiv(w3, kfactor)
    n[1] = n[1] + xderiv(w1, kfactor, basis, 1) + zderiv(v2, kfactor)
    n[2] = n[2] + xderiv(v3, kfactor, basis, 1) + yderiv(w2, kfactor)
    nw[0] = nw[0] + yderiv(w1, kfactor) + zderiv(v3, kfactor)
    nw[1] = nw[1] + xderiv(v1, kfactor, basis, 1) + zderiv(w2, kfactor)
    nw[2] = nw[2] + xderiv(w3, kfactor, basis, 1) + yderiv(v2, kfactor)
    un = [0.5 * (n[i] + nw[i]) for i in range(3)]
    bn = [0.5 * (n[i] - nw[i]) for i in range(3)]
    if alias == "DEALIAS":
        un = [dealias(a, basis) for a in un]
        bn = [dealias(a, basis) for a in bn]
    return un, bn


def nlin_scalar(V, F, kfactor, basis="FOUR", alias="DEALIAS", dealias_T=True):
    """Scalar part of IncVF::Compute_nlin(IncSF& T)  compute_nlin_SF.cc:65-263:
    T.nlin = D_j F(u_j theta) with SCFT parities (x: sin*sin -> cos; y, z: sin*cos -> sin)."""
    N3 = 2 * (V[0].shape[2] - 1)
    par_inv = (1, 0, 0)
    ur = [inverse(V[i], basis, par_inv[i], N3) for i in range(3)]
    tr = inverse(F, basis, 1, N3)
    a = forward(ur[0] * tr, basis, 0)
    b = forward(ur[1] * tr, basis, 1)
    c = forward(ur[2] * tr, basis, 1)
    tn = xderiv(a, kfactor, basis, 0) + yderiv(b, kfactor) + zderiv(c, kfactor)
    if alias == "DEALIAS" and dealias_T:
        tn = dealias(tn, basis)
    return tn


# --------------------------------------------------------------------------------------
# Pressure projection and right-hand side
# --------------------------------------------------------------------------------------

def pressure(nl, kfactor, basis="FOUR", alias="DEALIAS"):
    """Compute_pressure  compute_pressure.cc:54-62: F = Xderiv(nlin1, parity 1) + Yderiv(nlin2)
    + Zderiv(nlin3) (compute_divergence.cc:55-65), F /= K^2 (F(0) = 0), dealias F."""
    p = xderiv(nl[0], kfactor, basis, 1) + yderiv(nl[1], kfactor) + zderiv(nl[2], kfactor)
    p = divide_ksqr(p, kfactor, basis)
    if alias == "DEALIAS":
        p = dealias(p, basis)
    return p


def rhs_from_nlin(nl, p, kfactor, basis="FOUR"):
    """Compute_rhs  compute_rhs.cc:52-60 with Add_pressure_gradient add_pressure_grad.cc:48-61:
    nlin_i += D_i p (parity 0), then nlin = -nlin."""
    g = [xderiv(p, kfactor, basis, 0), yderiv(p, kfactor), zderiv(p, kfactor)]
    return [-(nl[i] + g[i]) for i in range(3)]


# --------------------------------------------------------------------------------------
# Anisotropic spectra  (lib/four/four_energy.cc ring parts, lib/fields/Cvf.cc:84-190, 484-560)
# --------------------------------------------------------------------------------------

def _polar_angle(kperp, kpll):
    """Get_polar_angle  basis_basicfn_inline.h:89-113: atan(k_perp/k_par) in [0, pi)."""
    if abs(kperp) > MYEPS:
        t = math.atan(kperp / kpll) if abs(kpll) > MYEPS else math.pi / 2
    else:
        t = 0.0 if kpll >= 0 else math.pi
    return t if t >= 0 else t + math.pi


def _sector_index(theta, bounds):
    """Get_sector_index  basis_basicfn.cc:304-320."""
    if theta > math.pi / 2:
        theta = math.pi - theta
    if abs(theta) < MYEPS:
        return 1
    for i, b in enumerate(bounds):
        if theta <= b:
            return i
    return len(bounds)


def _slab_index(kpll, bounds):
    """Get_slab_index  basis_basicfn.cc:373-390."""
    kpll = abs(kpll)
    if kpll < MYEPS:
        return 1
    for i in range(1, len(bounds)):
        if kpll <= bounds[i]:
            return i
    return len(bounds)


def min_radius_outside_four(N, kfactor, alias="DEALIAS"):
    """Min_radius_outside_FOUR  four_inline.h:172-228."""
    d = 3 if alias == "DEALIAS" else 2
    return int(math.ceil(math.sqrt(sum(((N[i] // d) * kfactor[i]) ** 2 for i in range(3)))))


def shell_spectrum_helicity(V, kfactor, alias="DEALIAS"):
    """Compute_shell_spectrum_helicity_FOUR  four_energy.cc:551-651: H_i(k) = sum over shell
    ceil|K| = k of 2 mult K_i (Vr x Vi)_i, k <= Min_radius_outside; shells beyond
    Max_radius_inside rescaled by Approx_number_modes_in_shell / sum(2 mult) over the shell."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    kmax = min_radius_outside_four(N, kfactor, alias)
    kin = max_radius_inside(N, kfactor, alias)
    Kx, Ky, Kz = kvec(N, kfactor)
    shape = V[0].shape
    K = [np.broadcast_to(k, shape) for k in (Kx, Ky, Kz)]
    idx = np.ceil(np.sqrt(K[0] ** 2 + K[1] ** 2 + K[2] ** 2)).astype(np.int64)
    f = 2 * multiplicity_four(N)
    Vr = [v.real for v in V]
    Vi = [v.imag for v in V]
    cr = [Vr[1] * Vi[2] - Vr[2] * Vi[1], Vr[2] * Vi[0] - Vr[0] * Vi[2], Vr[0] * Vi[1] - Vr[1] * Vi[0]]
    sel = idx <= kmax
    cnt = np.bincount(idx[sel], weights=f[sel], minlength=kmax + 1)
    out = []
    for i in range(3):
        h = np.bincount(idx[sel], weights=(f * K[i] * cr[i])[sel], minlength=kmax + 1)
        for k in range(kin + 1, kmax + 1):
            if cnt[k] >= 1:
                h[k] *= approx_number_modes_in_shell(N, k, kfactor) / cnt[k]
        out.append(h)
    return tuple(out)


def ring_spectrum(V, kfactor, axis, n_sectors, alias="DEALIAS", cylinder=False, helicity=False, basis="FOUR"):
    """CVF::CV_Compute_ring_spectrum (Cvf.cc:484-504; Compute_local_ring_spectrum_FOUR
    four_energy.cc:828-955) or, with cylinder=True, CV_Compute_cylinder_ring_spectrum
    (Cvf.cc:537-559; Compute_local_cylinder_ring_spectrum_FOUR four_energy.cc:1450-1516),
    anisotropy axis 1..3.  Returns (ek1, ek2, dissk), each [shells][n + 1]; dissk = 2 (S1 + S2)
    with weight K^2.  Pure-Python loop over the modes: small grids only.

    basis="SCFT": Compute_local_ring_spectrum_SCFT (scft_energy.cc:814-940), the helicity and
    cylinder variants (:1334-1370, :1423-1480, :1794-1830): kx = l1 kfactor >= 0,
    Multiplicity_factor_SCFT, V = (-i V1, V2, V3), on-axis components (V2, V3), (V3, -i V1),
    (-i V1, V2) for axes 1, 2, 3, the SCFT box radii (scft_inline.h:455-520), and, as written
    there, no multiplicity factor in the off-axis branch of the spherical (V, V) spectrum."""
    N1, N2 = V[0].shape[0], V[0].shape[1]
    N3 = 2 * (V[0].shape[2] - 1)
    N = (N1, N2, N3)
    scft = basis != "FOUR"
    ax = axis - 1
    p1, p2 = (ax + 1) % 3, (ax + 2) % 3
    n = n_sectors
    if not cylinder:
        rows = max_radius_inside(N, kfactor, alias, basis) + 1
        dth = (math.pi / 2) / n
        bounds = [i * dth for i in range(n)] + [math.pi / 2]
    else:
        rows = krho_inside(N, kfactor, axis, alias, basis) + 1
        kmax = kpll_max(N, kfactor, axis, alias, basis)
        dk = kmax / n
        bounds = [0.0] + [i * dk for i in range(1, n)] + [kmax]
    out = np.zeros((4, rows, n + 1))
    mult = multiplicity(N, basis)
    kx_, ky_, kz_ = (kx_scft(N1) if scft else kx_four(N1)), ky_four(N2), kz_four(N3)
    A = [np.asarray(v) for v in V]
    on_axis = {0: (1, 2), 1: (2, 0 if scft else 1), 2: (0, 1)}[ax]
    for l1 in range(N1):
        for l2 in range(N2):
            for l3 in range(N3 // 2 + 1):
                vals = [A[c][l1, l2, l3] for c in range(3)]
                if scft:
                    vals[0] = -1j * vals[0]
                vv = sum(abs(x) ** 2 for x in vals)
                if vv == 0.0:
                    continue
                k = (kx_[l1] * kfactor[0], ky_[l2] * kfactor[1], kz_[l3] * kfactor[2])
                kpll = k[ax]
                kperp = math.sqrt(k[p1] ** 2 + k[p2] ** 2)
                K2 = k[0] ** 2 + k[1] ** 2 + k[2] ** 2
                K = math.sqrt(K2)
                f = mult[l1, l2, l3]
                if not cylinder:
                    row = math.ceil(K)
                    if not (K > MYEPS) or row >= rows:
                        continue
                    col = _sector_index(_polar_angle(kperp, kpll), bounds)
                    if kperp < MYEPS:
                        c1, c2 = on_axis
                        e1, e2 = abs(vals[c1]) ** 2, abs(vals[c2]) ** 2
                    else:
                        # cross(V, K)_axis / k_perp
                        c = vals[p1] * k[p2] - vals[p2] * k[p1]
                        e1 = abs(c) ** 2 / kperp ** 2
                        e2 = vv - e1
                        if scft and not helicity:
                            f = 1.0
                else:
                    row = math.ceil(kperp)
                    if row >= rows:
                        continue
                    col = _slab_index(kpll, bounds)
                    e1 = abs(vals[ax]) ** 2
                    e2 = vv - e1
                if helicity:
                    # Compute_local_(cylinder_)ring_spectrum_helicity_FOUR / _SCFT: 2 mult K . (Vr x Vi)
                    vr = np.array([x.real for x in vals])
                    vi = np.array([x.imag for x in vals])
                    e1 = 2.0 * float(np.dot(k, np.cross(vr, vi)))
                    e2 = 0.0
                    f = mult[l1, l2, l3]
                if col >= n + 1:
                    continue
                out[0, row, col] += f * e1
                out[1, row, col] += f * e2
                out[2, row, col] += f * K2 * e1
                out[3, row, col] += f * K2 * e2
    return out[0], out[1], 2.0 * (out[2] + out[3])


# --------------------------------------------------------------------------------------
# Forcing  (lib/IncFluid/force)
# --------------------------------------------------------------------------------------

def number_modes_in_shell(N, inner, outer, kfactor, basis="FOUR"):
    """Get_local_number_modes_in_shell_FOUR  four_basic.cc:48-90: modes with
    inner <= |K| < outer (note: half-open the other way to the forcing loop), kz = 0 counted
    once, kz > 0 twice."""
    kxm = int(math.ceil(outer / kfactor[0]))
    kym = int(math.ceil(outer / kfactor[1]))
    kzm = int(math.ceil(outer / kfactor[2]))
    cnt = 0
    kxr = range(-kxm, kxm + 1) if basis == "FOUR" else range(0, kxm + 1)
    for kx in kxr:
        for ky in range(-kym, kym + 1):
            for kz in range(0, kzm + 1):
                km = math.sqrt((kx * kfactor[0]) ** 2 + (ky * kfactor[1]) ** 2 + (kz * kfactor[2]) ** 2)
                if inner <= km < outer:
                    cnt += 1 if kz == 0 else 2
    return cnt


def _band_modes(N, kfactor, outer, basis="FOUR"):
    """The (kx, ky, kz) loop of the band forcings: kx in [-ceil(outer/kf1), +..] (FOUR) or
    [0, ceil(outer/kf1)] (SCFT, kx_min = 0, compute_force_ek_hk_supply.cc:91-95), ky in
    [-ceil(outer/kf2), +..], kz in [0, ceil(outer/kf3)], with the stored index (lx, ly, lz)."""
    N1, N2, N3 = N
    kxm = int(math.ceil(outer / kfactor[0]))
    kym = int(math.ceil(outer / kfactor[1]))
    kzm = int(math.ceil(outer / kfactor[2]))
    for kx in range(-kxm if basis == "FOUR" else 0, kxm + 1):
        for ky in range(-kym, kym + 1):
            for kz in range(0, kzm + 1):
                yield kx, ky, kz, (kx if kx >= 0 else kx + N1), (ky if ky >= 0 else ky + N2), kz


def _modal_energy(v, kx, basis):
    """CV_Modal_energy (Cvf.cc:595-600): sum of Modal_energy_FOUR |A|^2/2 (four_inline.h:370) or
    Modal_energy_SCFT |A|^2 for kx > 0, |A|^2/2 for kx = 0 (scft_inline.h:347-354)."""
    w = 0.5 if (basis == "FOUR" or kx == 0) else 1.0
    return w * float(np.sum(np.abs(v) ** 2))


def _fourier_x(v, basis):
    """The SCFT sine component along x taken to the Fourier basis, (-i V1, V2, V3)
    (Get_Modal_helicity_SCFT, Compute_Modal_vorticity_SCFT scft_basic.cc:137-186)."""
    if basis == "FOUR":
        return v
    return np.array([-1j * v[0], v[1], v[2]])


def _alpha_beta(mode, v, kk, km, e_mode, h, Ek=None):
    """alpha_k, beta_k of one mode with modal energy E_k = |v|^2/2 (CV_Modal_energy Cvf.cc:595-600)
    and helicity H_k = K . (Vr x Vi) (Get_Modal_helicity_FOUR four_basic.cc:136-155), s = H_k/(k E_k):
      mode 1 (supply, compute_force_ek_hk_supply.cc:120-138): temp = e/(2 E_k),
        alpha = temp (1 - s h)/(1 - s^2), beta = temp (h - s)/(1 - s^2); |s^2 - 1| <= MYEPS2:
        alpha = temp/2, beta = alpha/(s k);
      mode 2 (constant energy and helicity, compute_force_const_ek_hk.cc:124-147): t1 = sqrt(e/E_k),
        t2 = sqrt((1 + h)/(1 + s)), t3 = sqrt((1 - h)/(1 - s)), alpha = t1 (t2 + t3)/2,
        beta = t1 (t2 - t3)/(2 k); |s^2 - 1| <= MYEPS2: alpha = t1, beta = 0.
    None when E_k <= MYEPS.  Ek: the modal energy when it is not |v|^2/2 (SCFT); v is then the
    vector in the Fourier basis for the helicity."""
    if Ek is None:
        Ek = float(np.sum(np.abs(v) ** 2)) / 2.0
    if Ek <= MYEPS:
        return None
    Hk = float(np.dot(kk, np.cross(v.real, v.imag)))
    sk = Hk / (km * Ek)
    if mode == 1:
        temp = e_mode / (2 * Ek)
        if abs(sk * sk - 1) > MYEPS2:
            return temp * (1 - sk * h) / (1 - sk * sk), temp * (h - sk) / (1 - sk * sk)
        alpha = temp / 2
        return alpha, alpha / (sk * km)
    t1 = math.sqrt(e_mode / Ek)
    if abs(sk * sk - 1) > MYEPS2:
        t2 = math.sqrt((1 + h) / (1 + sk))
        t3 = math.sqrt((1 - h) / (1 - sk))
        return t1 / 2 * (t2 + t3), t1 / (2 * km) * (t2 - t3)
    return t1, 0.0


def force_band(V, N, kfactor, inner, outer, eps, eps_h=0.0, mode=1, gate=False, basis="FOUR"):
    """The vector force of force_field_proc 1 (Compute_force_const_energy_helicity_supply
    compute_force_ek_hk_supply.cc:51-157) or 2 (Compute_force_const_energy_helicity
    compute_force_const_ek_hk.cc:53-165), FOUR: on inner < |K| <= outer, F = alpha V + beta omega
    (Force_alpha_beta force_alpha_beta.cc:60-88: the vorticity i K x V only when beta > MYEPS),
    with e = eps / nf per mode (nf = Get_number_modes_in_shell); then Satisfy_reality_array.
    gate: the mode is skipped unless e > MYEPS (the MHD and scalar variants of proc 1 and every
    variant of proc 2).
    SCFT (the basis_type == "SCFT" branches): kx >= 0, the SCFT modal energy and multiplicity of
    the mode count, the helicity and vorticity of (-i V1, V2, V3), and Force_alpha_beta's SCFT
    form F1 = I (alpha (-I) V1 + beta omega_1), F2, F3 = alpha V + beta omega
    (force_alpha_beta.cc:90-110); the SCFT reality condition."""
    nf = number_modes_in_shell(N, inner, outer, kfactor, basis)
    e_mode = eps / nf
    F = [np.zeros_like(V[0]) for _ in range(3)]
    if gate and not e_mode > MYEPS:
        return F
    for kx, ky, kz, lx, ly, lz in _band_modes(N, kfactor, outer, basis):
        km = math.sqrt((kx * kfactor[0]) ** 2 + (ky * kfactor[1]) ** 2 + (kz * kfactor[2]) ** 2)
        if not (inner < km <= outer):
            continue
        v = np.array([V[0][lx, ly, lz], V[1][lx, ly, lz], V[2][lx, ly, lz]])
        kk = np.array([kx * kfactor[0], ky * kfactor[1], kz * kfactor[2]])
        vf = _fourier_x(v, basis)
        ab = _alpha_beta(mode, vf, kk, km, e_mode, eps_h, _modal_energy(v, kx, basis))
        if ab is None:
            continue
        alpha, beta = ab
        vort = np.zeros(3, dtype=np.complex128)
        if beta > MYEPS:      # Compute_Modal_vorticity_FOUR / _SCFT (four_basic.cc:166-186, scft_basic.cc:167-186)
            vort = 1j * np.array([kk[1] * vf[2] - kk[2] * vf[1], kk[2] * vf[0] - kk[0] * vf[2],
                                  kk[0] * vf[1] - kk[1] * vf[0]])
        for c in range(3):
            F[c][lx, ly, lz] = alpha * v[c] + beta * vort[c]
        if basis != "FOUR":
            F[0][lx, ly, lz] = alpha * v[0] + 1j * beta * vort[0]
    return [satisfy_reality(f, basis) for f in F]


def force_band_scalar(T, N, kfactor, inner, outer, eps_T, mode=1, basis="FOUR"):
    """The scalar force of procs 1 and 2 with a passive scalar (compute_force_ek_hk_supply.cc:
    270-277, compute_force_const_ek_hk.cc:262-269; Force_scalar_alpha force_alpha_beta.cc:183-198):
    F_T = alpha T with alpha = e_T / E_T(k) (proc 1) or sqrt(e_T / E_T(k)) (proc 2),
    E_T(k) = CS_Modal_energy (FOUR |T|^2/2; SCFT |T|^2, at kx = 0 |T|^2/2), when
    e_T = eps_T / nf > MYEPS and E_T(k) > MYEPS."""
    nf = number_modes_in_shell(N, inner, outer, kfactor, basis)
    e_mode = eps_T / nf
    F = np.zeros_like(T)
    if not e_mode > MYEPS:
        return F
    for kx, ky, kz, lx, ly, lz in _band_modes(N, kfactor, outer, basis):
        km = math.sqrt((kx * kfactor[0]) ** 2 + (ky * kfactor[1]) ** 2 + (kz * kfactor[2]) ** 2)
        if not (inner < km <= outer):
            continue
        Et = _modal_energy(np.array([T[lx, ly, lz]]), kx, basis)
        if Et > MYEPS:
            alpha = e_mode / Et if mode == 1 else math.sqrt(e_mode / Et)
            F[lx, ly, lz] = alpha * T[lx, ly, lz]
    return satisfy_reality(F, basis)


def force_const_energy_supply(V, N, kfactor, inner, outer, eps, eps_h=0.0, basis="FOUR"):
    """Compute_force_const_energy_helicity_supply  compute_force_ek_hk_supply.cc:51-157 (fluid):
    force_band with mode 1 and no gate on the energy per mode."""
    return force_band(V, N, kfactor, inner, outer, eps, eps_h, mode=1, gate=False, basis=basis)


def force_coriolis(V, omega):
    """Compute_force_Coriolis  compute_force_Coriolis.cc:47-80 (three-component form):
    Force1 = w2 V3 - w3 V2, Force2 = w3 V1 - w1 V3, Force3 = w1 V2 - w2 V1."""
    w1, w2, w3 = omega
    return [w2 * V[2] - w3 * V[1], w3 * V[0] - w1 * V[2], w1 * V[1] - w2 * V[0]]


def force_liquid_metal(V, kfactor, B0):
    """Compute_force_Liquid_metal  compute_force_LM.cc:46-70 with Array_mult_V0_khat_sqr_FOUR
    four_basic.cc:413-439: Force = -(B0 . K)^2 / K^2 V (0 at K = 0), dealiased."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    Kx, Ky, Kz = kvec(N, kfactor)
    K2 = Kx * Kx + Ky * Ky + Kz * Kz
    bk = B0[0] * Kx + B0[1] * Ky + B0[2] * Kz
    with np.errstate(divide="ignore", invalid="ignore"):
        f = np.where(K2 > 0, bk * bk / K2, 0.0)
    return [dealias(-f * v) for v in V]


def _lx(k, N1, basis):
    return k if (basis == "SCFT" or k >= 0) else k + N1


def taylor_green_force(N, k0, amp, basis="FOUR"):
    """IncVF::Setup_Taylor_Green_force_field  lib/IncFlow/misc/force_model.cc:57-104 as dense
    arrays (Force1, Force2, Force3): amp (sin k0x cos k0y cos k0z, -cos k0x sin k0y cos k0z, 0)
    on the modes (+-k0, +-k0, k0) (SCFT: kx = k0 only)."""
    N1, N2, N3 = N
    F = [np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128) for _ in range(3)]
    a = amp / 8
    yp, ym = k0 % N2, (-k0) % N2
    if basis == "FOUR":
        xp, xm = _lx(k0, N1, basis), _lx(-k0, N1, basis)
        F[0][xp, yp, k0] = -1j * a
        F[0][xp, ym, k0] = -1j * a
        F[1][xp, yp, k0] = 1j * a
        F[1][xp, ym, k0] = -1j * a
        F[0][xm, yp, k0] = 1j * a
        F[0][xm, ym, k0] = 1j * a
        F[1][xm, yp, k0] = 1j * a
        F[1][xm, ym, k0] = -1j * a
    else:
        F[0][k0, yp, k0] = a
        F[0][k0, ym, k0] = a
        F[1][k0, yp, k0] = 1j * a
        F[1][k0, ym, k0] = -1j * a
    return F


def abc_force(N, k0, amp, A, B, C):
    """IncVF::Setup_ABC_force_field  lib/IncFlow/misc/force_model.cc:122-170 (FOUR) as dense
    arrays: amp (B cos k0y + C sin k0z, A sin k0x + C cos k0z, A cos k0x + B sin k0y)."""
    N1, N2, N3 = N
    F = [np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128) for _ in range(3)]
    yp, ym, xp, xm = k0 % N2, (-k0) % N2, k0 % N1, (-k0) % N1
    F[0][0, yp, 0] = B * amp / 2
    F[0][0, ym, 0] = B * amp / 2
    F[0][0, 0, k0] = -1j * (C * amp / 2)
    F[1][0, 0, k0] = C * amp / 2
    F[2][0, yp, 0] = -1j * (B * amp / 2)
    F[2][0, ym, 0] = 1j * (B * amp / 2)
    F[1][xp, 0, 0] = -1j * (A * amp / 2)
    F[2][xp, 0, 0] = A * amp / 2
    F[1][xm, 0, 0] = 1j * (A * amp / 2)
    F[2][xm, 0, 0] = A * amp / 2
    return F


def fluid_force(force, V, N, kfactor, basis="FOUR"):
    """The velocity force of a run: None (decay), energy supply dict(inner, outer, eps, eps_h)
    (proc 1), dict(kind="energy_helicity", inner, outer, eps, eps_h) (proc 2),
    dict(kind="static", F=[F1, F2, F3, ...]) (a fixed force field) or
    dict(kind="coriolis", omega=(w1, w2, w3))."""
    if force is None:
        return None
    kind = force.get("kind", "energy_supply")
    if kind == "energy_supply":
        return force_const_energy_supply(V, N, kfactor, force["inner"], force["outer"], force["eps"],
                                         force.get("eps_h", 0.0), basis)
    if kind == "energy_helicity":
        return force_band(V, N, kfactor, force["inner"], force["outer"], force["eps"], force.get("eps_h", 0.0),
                          mode=2, gate=True, basis=basis)
    if kind == "static":
        return list(force["F"][:3])
    if kind == "coriolis":
        return force_coriolis(V, force["omega"])
    if kind == "liquid_metal":
        return force_liquid_metal(V, kfactor, force["B0"])
    raise ValueError(kind)


# --------------------------------------------------------------------------------------
# Integrating-factor RK4  (lib/IncFluid/time_advance)
# --------------------------------------------------------------------------------------

def get_dt(E, N, kfactor, Tdt, alias="DEALIAS", basis="FOUR"):
    """IncFluid::Get_dt  compute_dt.cc:47-59: min(dx / (sqrt(E) 20), Tdt), dx = 2 pi / kmax_inside."""
    kmax = max_radius_inside(N, kfactor, alias, basis)
    dx = 2 * math.pi / kmax
    dt = dx / (math.sqrt(E) * 20) if E > 0 else float("inf")
    return min(dt, Tdt)


class FluidSolver:
    """The fluid loop iteration of Ifluid_main.cc:258-301 with IncFluid::Time_advance (RK4)
    time_advance.cc:100-155, Single_time_step single_time_step.cc:54-86 and Compute_RK4_parts
    single_time_step.cc:440-444, Compute_force_TO_rhs single_time_step.cc:351-365."""

    def __init__(self, N, kfactor, nu, Tdt, basis="FOUR", alias="DEALIAS", force=None, scheme="RK4", nu_h=0.0):
        self.N = tuple(N)
        self.kfactor = tuple(kfactor)
        self.nu = nu
        self.Tdt = Tdt
        self.basis = basis
        self.alias = alias
        self.force = force   # see fluid_force
        self.scheme = scheme  # integ_scheme EULER / RK2 / RK4
        self.nu_h = nu_h      # hyper_dissipation_coefficient (0: hyper_dissipation_switch off)

    # Compute_force(); Compute_nlin(); Add_force(); Compute_pressure(); Compute_rhs()
    def rhs(self, V):
        F = fluid_force(self.force, V, self.N, self.kfactor, self.basis)
        nl = nlin_fluid(V, self.kfactor, self.basis, self.alias)
        if F is not None:
            nl = [nl[i] - F[i] for i in range(3)]
        p = pressure(nl, self.kfactor, self.basis, self.alias)
        return rhs_from_nlin(nl, p, self.kfactor, self.basis), F

    def E(self, V, a, dt):
        return [exp_ksqr(v, -self.nu * a * dt, self.kfactor, self.basis) for v in V]

    def step(self, V):
        """One loop iteration; returns (V_new, dt)."""
        E0 = sum(total_energy(v, self.basis) for v in V)
        dt = get_dt(E0, self.N, self.kfactor, self.Tdt, self.alias, self.basis)
        u0 = [v.copy() for v in V]
        if self.scheme != "RK4" or self.nu_h != 0:
            u = if_time_advance(u0, [(self.nu, self.nu_h)] * 3, lambda f: self.rhs(f)[0], dt, self.scheme,
                                self.kfactor, self.basis)
            if self.alias == "DEALIAS":
                u = [dealias(a, self.basis) for a in u]
            return u, dt
        # stage 1: Single_time_step(dt, 1/2, 1/2, 1/2): V += dt/2 N; V *= E(1/2)
        r, _ = self.rhs(u0)
        u = [u0[i] + (dt / 2) * r[i] for i in range(3)]
        u = self.E(u, 0.5, dt)
        r = self.E(r, 1.0, dt)
        tot = [(dt / 6) * r[i] for i in range(3)]
        # stage 2: Single_time_step(dt, 1/2, 0, 1/2): V = E(1/2) u0 + dt/2 N
        r, _ = self.rhs(u)
        u = self.E(u0, 0.5, dt)
        u = [u[i] + (dt / 2) * r[i] for i in range(3)]
        r = self.E(r, 0.5, dt)
        tot = [tot[i] + (dt / 3) * r[i] for i in range(3)]
        # stage 3: Single_time_step(dt, 1, 1/2, 1): V = E(1/2)(E(1/2) u0 + dt N)
        r, _ = self.rhs(u)
        u = self.E(u0, 0.5, dt)
        u = [u[i] + dt * r[i] for i in range(3)]
        u = self.E(u, 0.5, dt)
        r = self.E(r, 0.5, dt)
        tot = [tot[i] + (dt / 3) * r[i] for i in range(3)]
        # stage 4
        r, _ = self.rhs(u)
        tot = [tot[i] + (dt / 6) * r[i] for i in range(3)]
        u = self.E(u0, 1.0, dt)
        u = [u[i] + tot[i] for i in range(3)]
        if self.alias == "DEALIAS":
            u = [dealias(a, self.basis) for a in u]
        return u, dt


class MHDSolver(FluidSolver):
    """The MHD loop of src/IMHD/IMHD_main.cc with Time_advance(IncVF& W)
    time_advance_VF_MHD.cc:59-182: the same IF-RK4 with nu for U and eta for B; only U.nlin is
    projected (Compute_pressure uses U's nlin), W.nlin -> -W.nlin (compute_rhs.cc:111-119)."""

    def __init__(self, N, kfactor, nu, eta, Tdt, basis="FOUR", alias="DEALIAS", force=None, scheme="RK4", nu_h=0.0,
                 eta_h=0.0):
        super().__init__(N, kfactor, nu, Tdt, basis, alias, force, scheme, nu_h)
        self.eta = eta
        self.eta_h = eta_h

    def rhs2(self, V, W):
        """Compute_force(W), Compute_nlin(W), Add_force(W) (add_force.cc:58-66): U.nlin -= F,
        W.nlin -= W.Force (a static force's components 3..5; zero otherwise)."""
        un, bn = nlin_mhd(V, W, self.kfactor, self.basis, self.alias)
        kind = self.force.get("kind", "energy_supply") if self.force is not None else None
        if kind in ("energy_supply", "energy_helicity"):
            # Compute_force_const_energy_helicity_supply(W) compute_force_ek_hk_supply.cc:292-437,
            # Compute_force_const_energy_helicity(W) compute_force_const_ek_hk.cc:296-446
            f, mode = self.force, (1 if kind == "energy_supply" else 2)
            F = force_band(V, self.N, self.kfactor, f["inner"], f["outer"], f["eps"], f.get("eps_h", 0.0), mode, True)
            FW = force_band(W, self.N, self.kfactor, f["inner"], f["outer"], f.get("eps_W", 0.0), f.get("eps_hW", 0.0),
                            mode, True)
            un = [un[i] - F[i] for i in range(3)]
            bn = [bn[i] - FW[i] for i in range(3)]
        else:
            F = fluid_force(self.force, V, self.N, self.kfactor)
            if F is not None:
                un = [un[i] - F[i] for i in range(3)]
                if self.force.get("kind") == "static" and len(self.force["F"]) > 3:
                    bn = [bn[i] - self.force["F"][3 + i] for i in range(3)]
        p = pressure(un, self.kfactor, self.basis, self.alias)
        ru = rhs_from_nlin(un, p, self.kfactor, self.basis)
        rb = [-b for b in bn]
        return ru, rb

    def Eb(self, V, a, dt):
        return [exp_ksqr(v, -self.eta * a * dt, self.kfactor, self.basis) for v in V]

    def step2(self, V, W):
        E0 = sum(total_energy(v, self.basis) for v in V) + sum(total_energy(w, self.basis) for w in W)
        kmax = max_radius_inside(self.N, self.kfactor, self.alias, self.basis)
        dx = 2 * math.pi / kmax
        dt = dx / (math.sqrt(E0) * 20)
        B0sqr = sum(float(np.real(w[0, 0, 0])) ** 2 for w in W)
        if B0sqr > MYEPS:
            dt = min(dt, dx / (math.sqrt(B0sqr) * 20))
        dt = min(dt, self.Tdt)
        u0 = [v.copy() for v in V]
        b0 = [w.copy() for w in W]
        if self.scheme != "RK4" or self.nu_h != 0 or self.eta_h != 0:
            f = if_time_advance(u0 + b0, [(self.nu, self.nu_h)] * 3 + [(self.eta, self.eta_h)] * 3,
                                lambda x: list(sum(self.rhs2(x[:3], x[3:]), [])), dt, self.scheme, self.kfactor,
                                self.basis)
            u, b = f[:3], f[3:]
            if self.alias == "DEALIAS":
                u = [dealias(a, self.basis) for a in u]
                b = [dealias(a, self.basis) for a in b]
            return u, b, dt
        ru, rb = self.rhs2(u0, b0)
        u = self.E([u0[i] + (dt / 2) * ru[i] for i in range(3)], 0.5, dt)
        b = self.Eb([b0[i] + (dt / 2) * rb[i] for i in range(3)], 0.5, dt)
        totu = [(dt / 6) * x for x in self.E(ru, 1.0, dt)]
        totb = [(dt / 6) * x for x in self.Eb(rb, 1.0, dt)]
        ru, rb = self.rhs2(u, b)
        u = [x + (dt / 2) * y for x, y in zip(self.E(u0, 0.5, dt), ru)]
        b = [x + (dt / 2) * y for x, y in zip(self.Eb(b0, 0.5, dt), rb)]
        totu = [t + (dt / 3) * x for t, x in zip(totu, self.E(ru, 0.5, dt))]
        totb = [t + (dt / 3) * x for t, x in zip(totb, self.Eb(rb, 0.5, dt))]
        ru, rb = self.rhs2(u, b)
        u = self.E([x + dt * y for x, y in zip(self.E(u0, 0.5, dt), ru)], 0.5, dt)
        b = self.Eb([x + dt * y for x, y in zip(self.Eb(b0, 0.5, dt), rb)], 0.5, dt)
        totu = [t + (dt / 3) * x for t, x in zip(totu, self.E(ru, 0.5, dt))]
        totb = [t + (dt / 3) * x for t, x in zip(totb, self.Eb(rb, 0.5, dt))]
        ru, rb = self.rhs2(u, b)
        totu = [t + (dt / 6) * x for t, x in zip(totu, ru)]
        totb = [t + (dt / 6) * x for t, x in zip(totb, rb)]
        u = [x + t for x, t in zip(self.E(u0, 1.0, dt), totu)]
        b = [x + t for x, t in zip(self.Eb(b0, 1.0, dt), totb)]
        if self.alias == "DEALIAS":
            u = [dealias(a, self.basis) for a in u]
            b = [dealias(a, self.basis) for a in b]
        return u, b, dt


def rb_coefficients(Ra, Pr, pr_switch="PRLARGE", u_scaling="ULARGE", temperature_grad=1.0):
    """(nu, kappa, fu, ft, nuf) of a Rayleigh-Benard nondimensionalisation:
    RB_slip_main.cc:222-262 (nu = coefficient of grad^2 u, kappa of grad^2 theta),
    compute_force_RB.cc:50-105 (Force1 = fu theta, T.Force = ft u1) and nusselt.cc:53-89
    (Nu = 1 + nuf <u1, theta>)."""
    small = u_scaling == "USMALL"
    if pr_switch == "PRSMALL":
        return ((1.0 if small else math.sqrt(Pr / Ra)), (1.0 / Pr if small else 1.0 / math.sqrt(Pr * Ra)),
                (Ra if small else Pr), temperature_grad / Pr,
                (2 * Pr * Pr if small else 2 * Pr * math.sqrt(Ra * Pr)))
    if pr_switch == "PRLARGE":
        return ((Pr if small else math.sqrt(Pr / Ra)), (1.0 if small else 1.0 / math.sqrt(Pr * Ra)),
                (Ra * Pr if small else 1.0), temperature_grad,
                (2.0 if small else 2 * math.sqrt(Ra * Pr)))
    raise ValueError(pr_switch)


class RBSolver:
    """Rayleigh-Benard convection (RB_SLIP; Pr_switch PRLARGE or PRSMALL, RB_Uscaling ULARGE or
    USMALL, rb_coefficients) and the loop src/RBslip/RB_slip_main.cc:365-400; Compute_force_RB
    compute_force_RB.cc:51-105 (Force1 = fu theta, T.Force = ft u1); Compute_nlin(T) ->
    Compute_nlin_scalar compute_nlin_SF.cc:80-177 with Dealias_nlin(T); IF-RK4 of
    time_advance_SF.cc for u (nu) and theta (kappa); Get_dt(T) = Get_dt().
    Fields: V = [u1 (sin), u2 (cos), u3 (cos)], T = theta (sin) in the SCFT basis."""

    def __init__(self, N, kfactor, Ra, Pr, Tdt, basis="SCFT", alias="DEALIAS", temperature_grad=1.0,
                 pr_switch="PRLARGE", u_scaling="ULARGE", omega=None, scheme="RK4", nu_h=0.0, kappa_h=0.0):
        self.scheme, self.nu_h, self.kappa_h = scheme, nu_h, kappa_h
        self.N = tuple(N)
        self.kfactor = tuple(kfactor)
        self.nu, self.kappa, self.fu, self.ft, self.nuf = rb_coefficients(Ra, Pr, pr_switch, u_scaling,
                                                                         temperature_grad)
        self.Ra, self.Pr = Ra, Pr
        self.Tdt = Tdt
        self.basis = basis
        self.alias = alias
        self.tg = temperature_grad
        # Compute_force_RB_rotation (compute_force_RB.cc:132-165): the Coriolis force V x omega
        # scaled by Pr (PRLARGE, USMALL), 1 (PRSMALL, USMALL) or sqrt(Pr/Ra) (ULARGE)
        self.omega = omega
        if u_scaling == "ULARGE":
            self.cor = math.sqrt(Pr / Ra)
        else:
            self.cor = Pr if pr_switch == "PRLARGE" else 1.0

    def rhs(self, V, T):
        nl = nlin_fluid(V, self.kfactor, self.basis, self.alias)
        tn = nlin_scalar(V, T, self.kfactor, self.basis, self.alias, dealias_T=True)
        F1 = self.fu * T
        TF = self.ft * V[0]
        if self.alias == "DEALIAS":     # Dealias_force(T)
            F1 = dealias(F1, self.basis)
            TF = dealias(TF, self.basis)
        if self.omega is not None:
            C = force_coriolis(V, self.omega)
            nl = [nl[0] - self.cor * C[0], nl[1] - self.cor * C[1], nl[2] - self.cor * C[2]]
        nl = [nl[0] - F1, nl[1], nl[2]]
        tn = tn - TF
        p = pressure(nl, self.kfactor, self.basis, self.alias)
        return rhs_from_nlin(nl, p, self.kfactor, self.basis), -tn

    def E(self, V, coef, a, dt):
        return [exp_ksqr(v, -coef * a * dt, self.kfactor, self.basis) for v in V]

    def step(self, V, T):
        E0 = sum(total_energy(v, self.basis) for v in V)
        dt = get_dt(E0, self.N, self.kfactor, self.Tdt, self.alias, self.basis)
        u0 = [v.copy() for v in V]
        t0 = T.copy()
        nu, ka = self.nu, self.kappa
        if self.scheme != "RK4" or self.nu_h != 0 or self.kappa_h != 0:
            def rhs(f):
                ru, rt = self.rhs(f[:3], f[3])
                return ru + [rt]
            f = if_time_advance(u0 + [t0], [(nu, self.nu_h)] * 3 + [(ka, self.kappa_h)], rhs, dt, self.scheme,
                                self.kfactor, self.basis)
            u, t = f[:3], f[3]
            if self.alias == "DEALIAS":
                u = [dealias(a, self.basis) for a in u]
                t = dealias(t, self.basis)
            return u, t, dt
        ru, rt = self.rhs(u0, t0)
        u = self.E([u0[i] + (dt / 2) * ru[i] for i in range(3)], nu, 0.5, dt)
        t = self.E([t0 + (dt / 2) * rt], ka, 0.5, dt)[0]
        totu = [(dt / 6) * x for x in self.E(ru, nu, 1.0, dt)]
        tott = (dt / 6) * self.E([rt], ka, 1.0, dt)[0]
        ru, rt = self.rhs(u, t)
        u = [x + (dt / 2) * y for x, y in zip(self.E(u0, nu, 0.5, dt), ru)]
        t = self.E([t0], ka, 0.5, dt)[0] + (dt / 2) * rt
        totu = [a + (dt / 3) * x for a, x in zip(totu, self.E(ru, nu, 0.5, dt))]
        tott = tott + (dt / 3) * self.E([rt], ka, 0.5, dt)[0]
        ru, rt = self.rhs(u, t)
        u = self.E([x + dt * y for x, y in zip(self.E(u0, nu, 0.5, dt), ru)], nu, 0.5, dt)
        t = self.E([self.E([t0], ka, 0.5, dt)[0] + dt * rt], ka, 0.5, dt)[0]
        totu = [a + (dt / 3) * x for a, x in zip(totu, self.E(ru, nu, 0.5, dt))]
        tott = tott + (dt / 3) * self.E([rt], ka, 0.5, dt)[0]
        ru, rt = self.rhs(u, t)
        totu = [a + (dt / 6) * x for a, x in zip(totu, ru)]
        tott = tott + (dt / 6) * rt
        u = [x + a for x, a in zip(self.E(u0, nu, 1.0, dt), totu)]
        t = self.E([t0], ka, 1.0, dt)[0] + tott
        if self.alias == "DEALIAS":
            u = [dealias(a, self.basis) for a in u]
            t = dealias(t, self.basis)
        return u, t, dt

    def nusselt(self, V, T):
        """Get_Nusselt_no  nusselt.cc:53-89: 1 + nuf <u1, theta> (PRLARGE + ULARGE: nuf =
        2 sqrt(Ra Pr))."""
        return 1 + self.nuf * total_energy(V[0], self.basis, T)


class ScalarSolver(RBSolver):
    """The passive-scalar loop src/IScalar/Iscalar_main.cc:272-300: Compute_force(T),
    Compute_nlin(T) (Compute_nlin_scalar compute_nlin_SF.cc:80-177 with Dealias_nlin(T)),
    Add_force(T) (add_force.cc:57-63), Compute_pressure, Get_dt(T) = Get_dt() (compute_dt.cc:66-69)
    and the IF-RK4 of time_advance_SF.cc with nu for u and kappa for T: the convection loop
    without buoyancy.  force: None, or dict(kind="energy_supply" | "energy_helicity", inner, outer,
    eps, eps_h, eps_T) (procs 1, 2 with the scalar variants compute_force_ek_hk_supply.cc:164-289,
    compute_force_const_ek_hk.cc:167-293)."""

    def __init__(self, N, kfactor, nu, kappa, Tdt, basis="FOUR", alias="DEALIAS", force=None, scheme="RK4",
                 nu_h=0.0, kappa_h=0.0):
        self.scheme, self.nu_h, self.kappa_h = scheme, nu_h, kappa_h
        self.N = tuple(N)
        self.kfactor = tuple(kfactor)
        self.nu, self.kappa = nu, kappa
        self.fu = self.ft = 0.0
        self.Tdt = Tdt
        self.basis = basis
        self.alias = alias
        self.omega = None
        self.force = force

    def rhs(self, V, T):
        nl = nlin_fluid(V, self.kfactor, self.basis, self.alias)
        tn = nlin_scalar(V, T, self.kfactor, self.basis, self.alias, dealias_T=True)
        if self.force is not None:
            f = self.force
            mode = 1 if f.get("kind", "energy_supply") == "energy_supply" else 2
            F = force_band(V, self.N, self.kfactor, f["inner"], f["outer"], f["eps"], f.get("eps_h", 0.0), mode, True,
                           self.basis)
            FT = force_band_scalar(T, self.N, self.kfactor, f["inner"], f["outer"], f.get("eps_T", 0.0), mode,
                                   self.basis)
            nl = [nl[i] - F[i] for i in range(3)]
            tn = tn - FT
        p = pressure(nl, self.kfactor, self.basis, self.alias)
        return rhs_from_nlin(nl, p, self.kfactor, self.basis), -tn


# --------------------------------------------------------------------------------------
# Energy transfer: flux and shell-to-shell  (lib/IncFlow/EnergyTrdir, lib/four/four_ET.cc)
# --------------------------------------------------------------------------------------

def et_radii(N, kfactor, no_shells, alias="DEALIAS", basis="FOUR"):
    """EnergyTr::EnergyTr shell radii, scheme 0  EnergyTr.cc:136-160:
    R = {0, 2, 4, 8, 8 * 2^(s (i - 3)) for i = 4..S-3, R_in/2, R_in, INF}, s = log2(R_in/16)/(S-5)."""
    S = no_shells
    R_in = 1.0 * max_radius_inside(N, kfactor, alias, basis)
    R = np.zeros(S + 1)
    R[0], R[1], R[2], R[3] = 0.0, 2.0, 4.0, 8.0
    R[S - 2] = R_in / 2
    R[S - 1] = R_in
    R[S] = INF_RADIUS
    if S > 6:
        s = math.log2(R_in / 16.0) / (S - 5)
        for i in range(4, S - 2):
            R[i] = 8 * 2.0 ** (s * (i - 3))
    return R


def fill_array_shell(A, inner, outer, kfactor, basis="FOUR"):
    """Fill_array_shell  universal_ET.cc:45-65: B = A on inner < |K| <= outer, else 0."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    K = kmag(N, kfactor, basis)
    return np.where((K > inner) & (K <= outer), A, 0)


def et_nlin(V, G, kfactor, basis="FOUR"):
    """IncVF::EnergyTr_Compute_nlin()  ET_compute_nlin.cc:85-120 with the ET products
    (ET_RSprod.cc:49-169): N_i = D_j F(V_j G_i); not projected, not dealiased."""
    N3 = 2 * (V[0].shape[2] - 1)
    par_inv = (1, 0, 0)
    vr = [inverse(V[i], basis, par_inv[i], N3) for i in range(3)]
    gr = [inverse(G[i], basis, par_inv[i], N3) for i in range(3)]
    n = [forward(vr[i] * gr[i], basis, 0) for i in range(3)]
    n[0] = xderiv(n[0], kfactor, basis, 0)
    n[1] = yderiv(n[1], kfactor)
    n[2] = zderiv(n[2], kfactor)
    v1 = forward(vr[0] * gr[1], basis, 1)   # V1r = V1 G2
    g1 = forward(gr[0] * vr[1], basis, 1)   # G1  = G1 V2
    v2 = forward(vr[1] * gr[2], basis, 0)   # V2r = V2 G3
    g2 = forward(gr[1] * vr[2], basis, 0)   # G2  = G2 V3
    v3 = forward(vr[2] * gr[0], basis, 1)   # V3r = V3 G1
    g3 = forward(gr[2] * vr[0], basis, 1)   # G3  = G3 V1
    # Derivative_RSprod_VV_ET  ET_RSprod.cc:155-168
    n[0] = n[0] + yderiv(g1, kfactor) + zderiv(v3, kfactor)
    n[1] = n[1] + xderiv(v1, kfactor, basis, 1) + zderiv(g2, kfactor)
    n[2] = n[2] + xderiv(g3, kfactor, basis, 1) + yderiv(v2, kfactor)
    return n


def shell_mult_single(A, B, inner, outer, kfactor, basis="FOUR"):
    """Shell_mult_single_FOUR  four_ET.cc:49-106: sum_{inner<|K|<=outer} 2 mult Re(A B*)."""
    N = (A.shape[0], A.shape[1], 2 * (A.shape[2] - 1))
    K = kmag(N, kfactor, basis)
    mult = multiplicity(N, basis)
    sel = (K > inner) & (K <= outer)
    return float((2 * mult * np.real(A * np.conj(B)))[sel].sum())


def shell_index(K, R):
    """Get_shell_index  basis_basicfn.cc:288-299: the first index (linear scan) with
    K <= R[index].  The radii need not be sorted (scheme 0 with R_in <= 16)."""
    K = np.asarray(K)
    out = np.full(K.shape, len(R), dtype=np.int64)
    for i in range(len(R) - 1, -1, -1):
        out = np.where(K <= R[i], i, out)
    return out


def shell_mult_all(As, Bs, R, kfactor, alias="DEALIAS", basis="FOUR"):
    """Shell_mult_all_FOUR (vector form)  four_ET.cc:181-256: for |K| <= kmax_inside,
    result[shell_index(|K|)] += 2 mult Re(sum_i A_i B_i*).  Length S+1."""
    A0 = As[0]
    N = (A0.shape[0], A0.shape[1], 2 * (A0.shape[2] - 1))
    K = kmag(N, kfactor, basis)
    kin = max_radius_inside(N, kfactor, alias, basis)
    mult = multiplicity(N, basis)
    val = 2 * mult * sum(np.real(a * np.conj(b)) for a, b in zip(As, Bs))
    sel = K <= kin
    idx = shell_index(K[sel], R)
    return np.bincount(idx, weights=val[sel], minlength=len(R))[: len(R)]


def force_feed_shell(F, V, kfactor, no_shells, alias="DEALIAS", basis="FOUR"):
    """IncVF::Compute_force_feed_shell  compute_force_feed.cc:70-76: Shell_mult_all(Force, V)
    on the energy-transfer shells (forceV_shell, length S+1)."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias, basis)
    return shell_mult_all(F, V, R, kfactor, alias, basis)


def compute_flux(V, kfactor, no_shells, alias="DEALIAS", basis="FOUR"):
    """IncVF::Compute_flux()  compute_flux.cc:52-69: for sphere s = 1..S, G = u on
    0 < |K| <= R_s, flux(s) = -sum_{|K| > R_s} 2 mult Re(N(G) . u*).  Length S+1, [0] = 0."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias, basis)
    flux = np.zeros(no_shells + 1)
    for s in range(1, no_shells + 1):
        G = [fill_array_shell(v, 0.0, R[s], kfactor, basis) for v in V]
        n = et_nlin(V, G, kfactor, basis)
        flux[s] = -sum(shell_mult_single(n[i], V[i], R[s], INF_RADIUS, kfactor, basis) for i in range(3))
    return flux


def compute_shell_tr(V, kfactor, no_shells, alias="DEALIAS", basis="FOUR"):
    """IncVF::Compute_shell_tr()  compute_shell_tr.cc:59-79: row n (1..S-1) = -Shell_mult_all of
    N(u^(n)) against u, giver shell n = (R_{n-1}, R_n].  Shape (S+1, S+1)."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias, basis)
    T = np.zeros((no_shells + 1, no_shells + 1))
    for n_ in range(1, no_shells):
        G = [fill_array_shell(v, R[n_ - 1], R[n_], kfactor, basis) for v in V]
        n = et_nlin(V, G, kfactor, basis)
        T[n_, :] = -shell_mult_all(n, V, R, kfactor, alias, basis)
    return T


def compute_flux_generic(H, F, Rf, sign, kfactor, no_shells, alias="DEALIAS", basis="FOUR"):
    """The flux loops of IncVF::Compute_flux(IncVF& W)  compute_flux.cc:140-215 in one form:
    for sphere s, G = F on 0 < |K| <= R_s, N = D_j F(H_j G_i) (EnergyTr_Compute_nlin with helper
    H), flux(s) = sign * sum_{|K| > R_s} 2 mult Re(N . Rf*).
      U->U: (H, F, Rf, sign) = (U, U, U, -1)   flux_self            (:52-69)
      B->B: (U, B, B, -1)                      W.flux_self          (:168-181)
      U->B: (B, U, B, +1)                      flux_VF_in_out       (:150-163)
      B->U: (U, B, U, +1)                      W.flux_VF_in_out     (:187-201)"""
    N = (H[0].shape[0], H[0].shape[1], 2 * (H[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias, basis)
    flux = np.zeros(no_shells + 1)
    for s in range(1, no_shells + 1):
        G = [fill_array_shell(f, 0.0, R[s], kfactor, basis) for f in F]
        n = et_nlin(H, G, kfactor, basis)
        flux[s] = sign * sum(shell_mult_single(n[i], Rf[i], R[s], INF_RADIUS, kfactor, basis) for i in range(3))
    return flux


def compute_shell_tr_generic(H, F, Rf, sign, kfactor, no_shells, alias="DEALIAS", basis="FOUR"):
    """The shell-to-shell loops of IncVF::Compute_shell_tr(IncVF& W)  compute_shell_tr.cc:156-200:
    row n = sign * Shell_mult_all(D_j F(H_j F^(n)_i), Rf).
      U->U: (U, U, U, -1); B->B: (U, B, B, -1) (:163-175); U->B: (B, U, B, +1) (:182-197)."""
    N = (H[0].shape[0], H[0].shape[1], 2 * (H[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias, basis)
    T = np.zeros((no_shells + 1, no_shells + 1))
    for n_ in range(1, no_shells):
        G = [fill_array_shell(f, R[n_ - 1], R[n_], kfactor, basis) for f in F]
        n = et_nlin(H, G, kfactor, basis)
        T[n_, :] = sign * shell_mult_all(n, Rf, R, kfactor, alias, basis)
    return T


def vorticity_four(V, kfactor):
    """Compute_Modal_vorticity_FOUR  four_basic.cc:166-186 on every mode: omega = i K x V."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    kx, ky, kz = kvec(N, kfactor)
    return [1j * (ky * V[2] - kz * V[1]), 1j * (kz * V[0] - kx * V[2]), 1j * (kx * V[1] - ky * V[0])]


def kinetic_helicity_flux(V, kfactor, no_shells, alias="DEALIAS"):
    """IncVF::Compute_kinetic_helicity_flux  compute_helicity_flux.cc:47-75 (FOUR): for sphere s
    (radius R_s of the energy-transfer radii), with X< = X on 0 < |K| <= R_s and
    P(N, R) = sum_{|K| > R_s} 2 mult Re(N . R*) (Shell_mult_single / Shell_mult_vorticity
    four_ET.cc:811-890): flux(s) = -P(N(U, U<), omega)/2 - P(N(U, omega<), U)/2
    + P(N(omega, U<), U)/2, N(H, G) = D_j F(H_j G_i)."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias)
    K = kmag(N, kfactor)
    mult = multiplicity_four(N)
    W = vorticity_four(V, kfactor)
    out = np.zeros(no_shells + 1)

    def P(nl, Rf, r):
        sel = K > r
        return float(np.sum((2 * mult * sum(np.real(a * np.conj(b)) for a, b in zip(nl, Rf)))[sel]))

    for s_ in range(1, no_shells + 1):
        r = R[s_]
        inside = (K > 0) & (K <= r)
        U_in = [np.where(inside, v, 0) for v in V]
        W_in = [np.where(inside, w, 0) for w in W]
        out[s_] = (-P(et_nlin(V, U_in, kfactor), W, r) / 2 - P(et_nlin(V, W_in, kfactor), V, r) / 2
                   + P(et_nlin(W, U_in, kfactor), V, r) / 2)
    return out


def _axis_extent(N, kfactor, i, alias="DEALIAS", basis="FOUR"):
    """Largest |k_i| of the (de)aliased box along axis i = 0, 1, 2; SCFT x: 2 N1/3 dealiased,
    N1 - 1 aliased (scft_inline.h:489-520)."""
    d = 3 if alias == "DEALIAS" else 2
    if basis != "FOUR" and i == 0:
        return ((2 * N[0] // 3) if alias == "DEALIAS" else (N[0] - 1)) * kfactor[0]
    return (N[i] // d) * kfactor[i]


def krho_inside(N, kfactor, axis, alias="DEALIAS", basis="FOUR"):
    """Anis_max_Krho_radius_inside_FOUR  four_inline.h:517-546 (_SCFT scft_inline.h:489-520)."""
    p1, p2 = axis % 3, (axis + 1) % 3
    return int(min(_axis_extent(N, kfactor, p1, alias, basis), _axis_extent(N, kfactor, p2, alias, basis)))


def kpll_max(N, kfactor, axis, alias="DEALIAS", basis="FOUR"):
    """Anis_max_Kpll_FOUR / _SCFT (scft_inline.h:455-485; dealiased SCFT axis 2 is (N2/2) kf as
    written there)."""
    if basis != "FOUR" and alias == "DEALIAS" and axis == 2:
        return (N[1] // 2) * kfactor[1]
    return _axis_extent(N, kfactor, axis - 1, alias, basis)


def vector_potential_four(B, kfactor):
    """a = i K x B / K^2 (the potential Shell_mult_vector_potential four_ET.cc:905-965 pairs
    with: 2 mult / K^2 Re(N . conj(i K x B))), zero at K = 0."""
    N = (B[0].shape[0], B[0].shape[1], 2 * (B[0].shape[2] - 1))
    K2 = ksqr(N, kfactor)
    W = vorticity_four(B, kfactor)
    with np.errstate(divide="ignore", invalid="ignore"):
        return [np.where(K2 > 0, w / K2, 0) for w in W]


def et_nlin_cross(V, G, kfactor, basis="FOUR"):
    """IncVF::EnergyTr_Compute_nlin_UcrossB  ET_compute_nlin.cc:317-337: F(V x G)."""
    N3 = 2 * (V[0].shape[2] - 1)
    vr = [inverse(V[i], basis, 0, N3) for i in range(3)]
    gr = [inverse(G[i], basis, 0, N3) for i in range(3)]
    return [forward(vr[1] * gr[2] - vr[2] * gr[1], basis, 0), forward(vr[2] * gr[0] - vr[0] * gr[2], basis, 0),
            forward(vr[0] * gr[1] - vr[1] * gr[0], basis, 0)]


def magnetic_helicity_flux(U, B, kfactor, no_shells, alias="DEALIAS"):
    """IncVF::Compute_magnetic_helicity_flux  compute_helicity_flux.cc:94-135 (FOUR): for
    sphere s, flux(s) = P(N(B, U<), a)/2 - P(N(U, B<), a)/2 + P(F(U x B<), B)/2, with
    a = i K x B / K^2, X< = X on 0 < |K| <= R_s, P(N, R) = sum_{|K| > R_s} 2 mult Re(N . R*)."""
    N = (U[0].shape[0], U[0].shape[1], 2 * (U[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias)
    K = kmag(N, kfactor)
    mult = multiplicity_four(N)
    A = vector_potential_four(B, kfactor)
    out = np.zeros(no_shells + 1)

    def P(nl, Rf, r):
        return float(np.sum((2 * mult * sum(np.real(x * np.conj(y)) for x, y in zip(nl, Rf)))[K > r]))

    for s_ in range(1, no_shells + 1):
        r = R[s_]
        inside = (K > 0) & (K <= r)
        U_in = [np.where(inside, v, 0) for v in U]
        B_in = [np.where(inside, b, 0) for b in B]
        out[s_] = (P(et_nlin(B, U_in, kfactor), A, r) / 2 - P(et_nlin(U, B_in, kfactor), A, r) / 2
                   + P(et_nlin_cross(U, B_in, kfactor), B, r) / 2)
    return out


def kinetic_helicity_shell_tr(V, kfactor, no_shells, alias="DEALIAS"):
    """IncVF::Compute_kinetic_helicity_shell_tr  compute_helicity_shell_tr.cc:56-109 (FOUR): row n
    (giver shell R_{n-1} < |K| <= R_n, n = 1 .. no_shells-1) = -Sv(N(U, U^(n)), U)/2
    - Sa(N(U, omega^(n)), U)/2 + Sa(N(omega, U^(n)), U)/2, where Sa(N, R) bins
    2 mult Re(N . R*) by Get_shell_index over |K| <= R_in (Shell_mult_all_FOUR four_ET.cc:181-256)
    and Sv(N, U) = Sa(N, i K x U) (Shell_mult_vorticity_all_FOUR four_ET.cc:999-1090)."""
    N = (V[0].shape[0], V[0].shape[1], 2 * (V[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias)
    W = vorticity_four(V, kfactor)
    T = np.zeros((no_shells + 1, no_shells + 1))
    for n_ in range(1, no_shells):
        G = [fill_array_shell(f, R[n_ - 1], R[n_], kfactor) for f in V]
        Gw = [fill_array_shell(f, R[n_ - 1], R[n_], kfactor) for f in W]
        T[n_, :] = (-shell_mult_all(et_nlin(V, G, kfactor), W, R, kfactor, alias) / 2
                    - shell_mult_all(et_nlin(V, Gw, kfactor), V, R, kfactor, alias) / 2
                    + shell_mult_all(et_nlin(W, G, kfactor), V, R, kfactor, alias) / 2)
    return T


def magnetic_helicity_shell_tr(U, B, kfactor, no_shells, alias="DEALIAS"):
    """IncVF::Compute_magnetic_helicity_shell_tr  compute_helicity_shell_tr.cc:114-172 (FOUR): row n
    = Sp(N(B, U^(n)), B)/2 - Sp(N(U, B^(n)), B)/2 + Sa(F(U x B^(n)), B)/2 with
    Sp(N, B) = Sa(N, a), a = i K x B / K^2 (Shell_mult_vector_potential_all_FOUR
    four_ET.cc:1094-1190).  At K = 0 the reference divides 0 by |K|^2 = 0; the oracle takes a = 0
    there, so column 0 holds the U x B< term alone."""
    N = (U[0].shape[0], U[0].shape[1], 2 * (U[0].shape[2] - 1))
    R = et_radii(N, kfactor, no_shells, alias)
    A = vector_potential_four(B, kfactor)
    T = np.zeros((no_shells + 1, no_shells + 1))
    for n_ in range(1, no_shells):
        Gu = [fill_array_shell(f, R[n_ - 1], R[n_], kfactor) for f in U]
        Gb = [fill_array_shell(f, R[n_ - 1], R[n_], kfactor) for f in B]
        T[n_, :] = (shell_mult_all(et_nlin(B, Gu, kfactor), A, R, kfactor, alias) / 2
                    - shell_mult_all(et_nlin(U, Gb, kfactor), A, R, kfactor, alias) / 2
                    + shell_mult_all(et_nlin_cross(U, Gb, kfactor), B, R, kfactor, alias) / 2)
    return T


def ring_radii(N, kfactor, n_ring_shells, alias="DEALIAS", basis="FOUR", Rin=None):
    """EnergyTr::EnergyTr ring shell radii, scheme 0  EnergyTr.cc:190-210 (cylinder shells
    :300-320 with Rin = Anis_max_Krho_radius_inside)."""
    if Rin is None:
        Rin = float(max_radius_inside(N, kfactor, alias, basis))
    n = n_ring_shells
    r = [0.0] * (n + 1)
    r[1], r[2] = 4.0, 8.0
    r[n - 2], r[n - 1], r[n] = Rin / 2, Rin, INF_RADIUS
    if n > 5:
        s = math.log2(Rin / 16.0) / (n - 4)
        for i in range(3, n - 2):
            r[i] = 8 * 2.0 ** (s * (i - 2))
    return r


def _theta_grid(N, kfactor, axis, basis="FOUR"):
    """AnisKvect_polar_angle_FOUR (_SCFT) on the dense grid: unfolded, in [0, pi)."""
    K = kvec(N, kfactor, basis)
    shape = (N[0], N[1], N[2] // 2 + 1)
    K = [np.broadcast_to(k, shape) for k in K]
    ax = axis - 1
    kpll = K[ax]
    kperp = np.sqrt(K[(ax + 1) % 3] ** 2 + K[(ax + 2) % 3] ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.where(np.abs(kperp) > MYEPS,
                     np.where(np.abs(kpll) > MYEPS, np.arctan(kperp / kpll), math.pi / 2),
                     np.where(kpll >= 0, 0.0, math.pi))
    return np.where(t >= 0, t, t + math.pi)


def compute_cylinder_ring_tr_generic(H, F, Rf, sign, kfactor, axis, n_shells, n_slabs, alias="DEALIAS",
                                     basis="FOUR"):
    """IncVF::Compute_cylinder_ring_tr  compute_cylin_ring_tr.cc:53-80: giver (i, j) = F on
    r[i-1] < K_perp <= r[i], h_{j-1} < K_par <= h_j (signed; K_par = 0 in slab 1;
    Fill_array_cylinder_ring universal_ET.cc:100-125); T[i, j, m, s] = sign * sum over receiver
    (m, s) with K_perp <= Krho_max of 2 mult Re(N . Rf*) (Local_cyl_ring_mult_all_FOUR
    four_ET.cc:492-530, Compute_cylinder_ring_index basis_basicfn.cc:412-445; SCFT
    Local_cyl_ring_mult_all_SCFT scft_ET.cc:436-478)."""
    N = (H[0].shape[0], H[0].shape[1], 2 * (H[0].shape[2] - 1))
    kr = krho_inside(N, kfactor, axis, alias, basis)
    R = ring_radii(N, kfactor, n_shells, alias, basis, Rin=float(kr))
    ax = axis - 1
    kmax = kpll_max(N, kfactor, axis, alias, basis)
    dk = kmax / n_slabs
    hb = [0.0] + [i * dk for i in range(1, n_slabs)] + [kmax]
    Kv = [np.broadcast_to(k, (N[0], N[1], N[2] // 2 + 1)) for k in kvec(N, kfactor, basis)]
    kpll = Kv[ax]
    kperp = np.sqrt(Kv[(ax + 1) % 3] ** 2 + Kv[(ax + 2) % 3] ** 2)
    mult = multiplicity(N, basis)
    shell = shell_index(kperp, R)
    akp = np.abs(kpll)
    slab = np.full(kperp.shape, len(hb), dtype=np.int64)
    for i in range(len(hb) - 1, 0, -1):
        slab = np.where(akp <= hb[i], i, slab)
    slab = np.where(akp < MYEPS, 1, slab)
    n1, n2 = n_shells + 1, n_slabs + 1
    ok = (kperp <= kr) & (shell <= n_shells) & (slab <= n_slabs)
    flat = (shell * n2 + slab)[ok]
    T = np.zeros((n1, n2, n1, n2))
    for i in range(1, n_shells):
        for j in range(1, n_slabs + 1):
            lo, hi, hl, hh = R[i - 1], R[i], hb[j - 1], hb[j]
            inr = (kperp > lo) & (kperp <= hi) & (((kpll > hl) & (kpll <= hh)) | ((np.abs(kpll) < MYEPS) & (hl < MYEPS)))
            G = [np.where(inr, f, 0) for f in F]
            nl = et_nlin(H, G, kfactor, basis)
            val = 2 * mult * sum(np.real(a * np.conj(b)) for a, b in zip(nl, Rf))
            T[i, j] = sign * np.bincount(flat, weights=val[ok], minlength=n1 * n2).reshape(n1, n2)
    return T


def ring_mult_all(A, B, kfactor, axis, n_ring_shells, n_sectors, alias="DEALIAS", cylinder=False, basis="FOUR"):
    """Ring_mult_all / Local_ring_mult_all_FOUR (four_ET.cc:335-386) and Cyl_ring_mult_all /
    Local_cyl_ring_mult_all_FOUR (:492-530): sum of 2 mult Re(A . B*) binned by receiver ring
    (scheme-0 ring radii, equal sectors of the folded polar angle up to pi/2, |K| <= R_in,
    |K| > MYEPS) or cylinder ring (radii up to Anis_max_Krho_radius_inside, slabs of |K_par|).
    [shell][sector] of shape (n+1, ns+1).  It gives Compute_force_feed_ring and
    Compute_force_feed_cylinder_ring (compute_force_feed.cc:162-300) with A the force.  SCFT:
    Local_ring_mult_all_SCFT / Local_cyl_ring_mult_all_SCFT (scft_ET.cc:273-478)."""
    N = (A[0].shape[0], A[0].shape[1], 2 * (A[0].shape[2] - 1))
    mult = multiplicity(N, basis)
    val = 2 * mult * sum(np.real(a * np.conj(b)) for a, b in zip(A, B))
    n1, n2 = n_ring_shells + 1, n_sectors + 1
    if not cylinder:
        R = ring_radii(N, kfactor, n_ring_shells, alias, basis)
        dth = (math.pi / 2) / n_sectors
        sec = [i * dth for i in range(n_sectors)] + [math.pi / 2]
        K = kmag(N, kfactor, basis)
        th = _theta_grid(N, kfactor, axis, basis)
        kin = max_radius_inside(N, kfactor, alias, basis)
        shell = shell_index(K, R)
        thf = np.where(th > math.pi / 2, math.pi - th, th)
        sector = np.full(K.shape, len(sec), dtype=np.int64)
        for i in range(len(sec) - 1, -1, -1):
            sector = np.where(thf <= sec[i], i, sector)
        sector = np.where(np.abs(thf) < MYEPS, 1, sector)
        ok = (K <= kin) & (K > MYEPS) & (shell <= n_ring_shells) & (sector <= n_sectors)
    else:
        kr = krho_inside(N, kfactor, axis, alias, basis)
        R = ring_radii(N, kfactor, n_ring_shells, alias, basis, Rin=float(kr))
        ax = axis - 1
        kmax = kpll_max(N, kfactor, axis, alias, basis)
        dk = kmax / n_sectors
        hb = [0.0] + [i * dk for i in range(1, n_sectors)] + [kmax]
        Kv = [np.broadcast_to(k, (N[0], N[1], N[2] // 2 + 1)) for k in kvec(N, kfactor, basis)]
        kperp = np.sqrt(Kv[(ax + 1) % 3] ** 2 + Kv[(ax + 2) % 3] ** 2)
        shell = shell_index(kperp, R)
        akp = np.abs(Kv[ax])
        sector = np.full(kperp.shape, len(hb), dtype=np.int64)
        for i in range(len(hb) - 1, 0, -1):
            sector = np.where(akp <= hb[i], i, sector)
        sector = np.where(akp < MYEPS, 1, sector)
        ok = (kperp <= kr) & (shell <= n_ring_shells) & (sector <= n_sectors)
    flat = (shell * n2 + sector)[ok]
    return np.bincount(flat, weights=val[ok], minlength=n1 * n2).reshape(n1, n2)


def compute_ring_tr_generic(H, F, Rf, sign, kfactor, axis, n_ring_shells, n_sectors, alias="DEALIAS", basis="FOUR"):
    """IncVF::Compute_ring_tr  compute_ring_tr.cc:60-90 (MHD kinds :174-215) in one form:
    giver ring (i, j): G = F on r[i-1] < |K| <= r[i], sector_{j-1} < theta <= sector_j
    (Fill_array_ring universal_ET.cc:70-100), N = D_j F(H_j G_i); T[i, j, m, s] = sign *
    sum over receiver ring (m, s) of 2 mult Re(N . Rf*) (Local_ring_mult_all_FOUR
    four_ET.cc:330-386 with Compute_ring_index basis_basicfn.cc:324-352; SCFT
    Local_ring_mult_all_SCFT scft_ET.cc:273-346)."""
    N = (H[0].shape[0], H[0].shape[1], 2 * (H[0].shape[2] - 1))
    R = ring_radii(N, kfactor, n_ring_shells, alias, basis)
    dth = (math.pi / 2) / n_sectors
    sec = [i * dth for i in range(n_sectors)] + [math.pi / 2]
    K = kmag(N, kfactor, basis)
    th = _theta_grid(N, kfactor, axis, basis)
    kin = max_radius_inside(N, kfactor, alias, basis)
    mult = multiplicity(N, basis)
    sel = (K <= kin) & (K > MYEPS)
    shell = shell_index(K, R)
    thf = np.where(th > math.pi / 2, math.pi - th, th)
    sector = np.full(K.shape, len(sec), dtype=np.int64)
    for i in range(len(sec) - 1, -1, -1):
        sector = np.where(thf <= sec[i], i, sector)
    sector = np.where(np.abs(thf) < MYEPS, 1, sector)
    n1, n2 = n_ring_shells + 1, n_sectors + 1
    ok = sel & (shell <= n_ring_shells) & (sector <= n_sectors)
    flat = (shell * n2 + sector)[ok]
    T = np.zeros((n1, n2, n1, n2))
    for i in range(1, n_ring_shells):
        for j in range(1, n_sectors + 1):
            lo, hi, left, right = R[i - 1], R[i], sec[j - 1], sec[j]
            inr = (K > lo) & (K <= hi) & (((th > left) & (th <= right)) | ((np.abs(th) < MYEPS) & (left < MYEPS)))
            G = [np.where(inr, f, 0) for f in F]
            nl = et_nlin(H, G, kfactor, basis)
            val = 2 * mult * sum(np.real(a * np.conj(b)) for a, b in zip(nl, Rf))
            T[i, j] = sign * np.bincount(flat, weights=val[ok], minlength=n1 * n2).reshape(n1, n2)
    return T


# --------------------------------------------------------------------------------------
# Convenience: the reference's packed real layout (N1, N2, N3/2+1) complex <-> (N1, N2, N3)
# --------------------------------------------------------------------------------------

def pack_real(real):
    """Real (N1,N2,N3) -> the reference's in-place layout: complex (N1,N2,N3/2+1) whose slot l3
    holds (x[2 l3], x[2 l3 + 1]); the last slot is the zeroed padding (four_tr.cc:299-302)."""
    N1, N2, N3 = real.shape
    out = np.zeros((N1, N2, N3 // 2 + 1), dtype=np.complex128)
    out[:, :, : N3 // 2] = real[:, :, 0::2] + 1j * real[:, :, 1::2]
    return out


def unpack_real(packed):
    N1, N2, M1 = packed.shape
    N3 = 2 * (M1 - 1)
    out = np.empty((N1, N2, N3))
    out[:, :, 0::2] = packed[:, :, : N3 // 2].real
    out[:, :, 1::2] = packed[:, :, : N3 // 2].imag
    return out


# --------------------------------------------------------------------------------------
# Test infrastructure: a random-projection sketch of a set of spectral fields, so that golden
# fixtures of large grids can hold a few numbers per field instead of the fields themselves.
# --------------------------------------------------------------------------------------

def sketch(fields, n_proj=64, seed=7919):
    """Projections p_j = sum over every entry of Re(F) Re(w_j) + Im(F) Im(w_j), j < n_proj, of
    the fields (concatenated), with weights w_j uniform in [-1, 1] per real component from the
    seeded PCG64 stream (seed, j).  For a difference d of two field sets, the projections of
    d have variance |d|^2 / 3, so rel_from_sketch estimates |d| / |F| (within ~20 % for 64
    projections).  Returns (p, |F|)."""
    flat = [np.ascontiguousarray(f).view(np.float64).ravel() for f in fields]
    n = sum(x.size for x in flat)
    p = np.zeros(n_proj)
    for j in range(n_proj):
        rng = np.random.Generator(np.random.PCG64([seed, j]))
        w = rng.random(n) * 2.0 - 1.0
        o = 0
        for x in flat:
            p[j] += float(np.dot(x, w[o:o + x.size]))
            o += x.size
    norm = math.sqrt(sum(float(np.dot(x, x)) for x in flat))
    return p, norm


def rel_from_sketch(p_got, p_want, norm_want):
    """Estimate of |F_got - F_want| / |F_want| from two sketches with the same weights."""
    d = np.asarray(p_got) - np.asarray(p_want)
    return math.sqrt(3.0 * float(np.dot(d, d)) / len(d)) / norm_want
