"""Fixed forces on a few modes (force_field_proc 3, 4, 5) as the mode lists that
``tg_set_force_modes`` takes, and the Coriolis force (proc 21) as a config.

Each builder returns ``(k, F)``: ``k`` an int array of shape (n, 3) with the (kx, ky, kz)
wavenumber indices of the forced modes and ``F`` a complex array of shape (n, nstate) with the
force on every state field there (V1, V2, V3, then W1..W3 of MHD or T of a scalar)::

    U = IncFluid(N, force=dict(kind="modes"), nu=1e-2, dt=1e-3)
    U.set_force_modes(*taylor_green_modes(N, k0=1, amp=1.0))

    R = IncFluid(N, force=dict(kind="coriolis", omega=(0.0, 0.0, 2.0)), nu=1e-2, dt=1e-3)

The values follow lib/IncFlow/misc/force_model.cc (Setup_Taylor_Green_force_field 57-104,
Setup_ABC_force_field 122-170) and lib/IncFluid/force/compute_force_modes.cc:97-440
(Compute_force_given_modes_SIMPLE with IncVF::Last_component field_k_fns.cc:52-114).
"""

from __future__ import annotations

import math

import numpy as np

_NSTATE = {"FLUID": 3, "MHD": 6, "SCALAR": 4}


def _nstate(physics: str) -> int:
    try:
        return _NSTATE[physics.upper()]
    except KeyError:
        raise ValueError(f"fixed forces are defined for FLUID, MHD and SCALAR, not {physics}")


def _pack(modes: dict, ns: int):
    """{(kx, ky, kz): [F per state field]} -> (k, F), in insertion order."""
    k = np.array(list(modes.keys()), dtype=np.int32).reshape(-1, 3)
    F = np.zeros((len(modes), ns), dtype=np.complex128)
    for i, v in enumerate(modes.values()):
        F[i, :len(v)] = v
    return k, F


def _set(modes: dict, key, comp: int, value, ns: int):
    v = modes.setdefault(tuple(int(x) for x in key), [0j] * ns)
    v[comp] = complex(value)


def taylor_green_modes(N, k0: int, amp: float, basis: str = "FOUR", physics: str = "FLUID",
                       ampW: float = 0.0):
    """Setup_Taylor_Green_force_field(k0, amp) (force_model.cc:57-104): the force
    amp (sin k0x cos k0y cos k0z, -cos k0x sin k0y cos k0z, 0) on (+-k0, +-k0, k0) (SCFT: kx = k0
    only).  MHD forces W alike with ampW (compute_force_TG.cc:79-92); a scalar's force is 0."""
    ns = _nstate(physics)
    k0 = int(k0)
    modes: dict = {}

    def put(amplitude, c0):
        a = amplitude / 8
        if basis == "FOUR":
            _set(modes, (k0, k0, k0), c0, -1j * a, ns)
            _set(modes, (k0, -k0, k0), c0, -1j * a, ns)
            _set(modes, (k0, k0, k0), c0 + 1, 1j * a, ns)
            _set(modes, (k0, -k0, k0), c0 + 1, -1j * a, ns)
            _set(modes, (-k0, k0, k0), c0, 1j * a, ns)
            _set(modes, (-k0, -k0, k0), c0, 1j * a, ns)
            _set(modes, (-k0, k0, k0), c0 + 1, 1j * a, ns)
            _set(modes, (-k0, -k0, k0), c0 + 1, -1j * a, ns)
        elif basis == "SCFT":
            _set(modes, (k0, k0, k0), c0, a, ns)
            _set(modes, (k0, -k0, k0), c0, a, ns)
            _set(modes, (k0, k0, k0), c0 + 1, 1j * a, ns)
            _set(modes, (k0, -k0, k0), c0 + 1, -1j * a, ns)
        else:
            raise ValueError(basis)

    put(amp, 0)
    if ns == 6:
        put(ampW, 3)
    return _pack(modes, ns)


def abc_modes(N, k0: int, amp: float, A: float, B: float, C: float, physics: str = "FLUID",
              ampW: float = 0.0):
    """Setup_ABC_force_field(k0, amp, A, B, C) (force_model.cc:122-170, FOUR only): the force
    amp (B cos k0y + C sin k0z, A sin k0x + C cos k0z, A cos k0x + B sin k0y).  MHD forces W
    alike with ampW (compute_force_ABC.cc:116-131)."""
    ns = _nstate(physics)
    k0 = int(k0)
    modes: dict = {}

    def put(a, c0):
        _set(modes, (0, k0, 0), c0, B * a / 2, ns)
        _set(modes, (0, -k0, 0), c0, B * a / 2, ns)
        _set(modes, (0, 0, k0), c0, -1j * (C * a / 2), ns)
        _set(modes, (0, 0, k0), c0 + 1, C * a / 2, ns)
        _set(modes, (0, k0, 0), c0 + 2, -1j * (B * a / 2), ns)
        _set(modes, (0, -k0, 0), c0 + 2, 1j * (B * a / 2), ns)
        _set(modes, (k0, 0, 0), c0 + 1, -1j * (A * a / 2), ns)
        _set(modes, (k0, 0, 0), c0 + 2, A * a / 2, ns)
        _set(modes, (-k0, 0, 0), c0 + 1, 1j * (A * a / 2), ns)
        _set(modes, (-k0, 0, 0), c0 + 2, A * a / 2, ns)

    put(amp, 0)
    if ns == 6:
        put(ampW, 3)
    return _pack(modes, ns)


def six_mode_table(k0: int, amp101: float, amp011: float, amp112: float, h: float) -> dict:
    """The six modes of IncVF::Setup_SIX_MODE_force_field (force_model.cc:172-236) and
    Setup_SIX_MODE_field (ic_model.cc:238-301), FOUR: {(kx, ky, kz): (V1, V2, V3)} at
    (0, +-k0, k0), (+-k0, 0, k0) and (+-k0, +-k0, 2 k0) with f1 = 2 amp101/sqrt(2 + h^2),
    f2 = 2 amp011/sqrt(2 + h^2), f3 = 4 amp112/sqrt(6 + 10 h^2).  The values are the reference's
    table as written."""
    f1 = 2.0 / math.sqrt(2 + h * h) * amp101
    f2 = 2.0 / math.sqrt(2 + h * h) * amp011
    f3 = 4.0 / math.sqrt(6 + 10 * h * h) * amp112
    I = 1j
    t = {
        (0, k0, k0): (-h * f2 / 4 + 0j, I * f2 / 4, -I * f2 / 4),
        (0, -k0, k0): (h * f2 / 4 + 0j, -I * f2 / 4, -I * f2 / 4),
        (k0, 0, k0): (I * f1 / 4, -h * f1 / 4 + 0j, -I * f1 / 4),
        (k0, k0, 2 * k0): (I * f3 / 8, I * f3 / 8 + h * f3 / 4, -I * f3 / 8 - h * f3 / 8),
        (k0, -k0, 2 * k0): (I * f3 / 8, -I * f3 / 8 + h * f3 / 4, -I * f3 / 8 + h * f3 / 8),
        (-k0, 0, k0): (-I * f1 / 4, h * f1 / 4 + 0j, -I * f1 / 4),
        (-k0, k0, 2 * k0): (-I * f3 / 8, I * f3 / 8 - h * f3 / 4, -I * f3 / 8 + h * f3 / 8),
        (-k0, -k0, 2 * k0): (-I * f3 / 8, -I * f3 / 8 - h * f3 / 4, -I * f3 / 8 - h * f3 / 8),
    }
    return t


def six_mode_modes(N, k0: int, amp101: float, amp011: float, amp112: float, h: float, physics: str = "MHD"):
    """Compute_force_DYNAMO_SIX_MODE (compute_force_dynamo_6mode.cc:45-80): the six-mode force on
    the velocity only (B's force zero), as (k, F) for IncFluid.set_force_modes."""
    ns = _nstate(physics)
    modes: dict = {}
    for key, vals in six_mode_table(k0, amp101, amp011, amp112, h).items():
        for c, v in enumerate(vals):
            _set(modes, key, c, v, ns)
    return _pack(modes, ns)


def _dx(basis, kfactor, kx, v):
    """DxVx (universal_inline.h): FOUR i kx kf1 v, SCFT kx kf1 v."""
    return (1j * kx * kfactor[0] * v) if basis == "FOUR" else (kx * kfactor[0] * v)


def last_component(kx, ky, kz, Fx, Fy, kfactor, basis="FOUR"):
    """IncVF::Last_component (field_k_fns.cc:52-114, 3D grid): kz != 0: Fz from K . F = 0;
    kz = 0: the given values are (Fx, Fz), Fy from Fx (ky != 0) or (0, Fx) on the kx axis."""
    if kz != 0:
        temp = _dx(basis, kfactor, kx, Fx) + 1j * ky * kfactor[1] * Fy
        return Fx, Fy, temp / (-1j * kz * kfactor[2])
    Fz = Fy
    if ky == 0:
        return 0j, Fx, Fz
    return Fx, _dx(basis, kfactor, kx, Fx) / (-1j * ky * kfactor[1]), Fz


def compute_vyvz(kx, ky, kz, Vx, Omega, kfactor, basis="FOUR"):
    """IncVF::Compute_VyVz (field_k_fns.cc:126-157): the (Vx, Vy, Vz) of a divergence-free mode
    with the given Vx and x-vorticity Omega, K_perp^2 = Ky^2 + Kz^2:
    Vy = (i Ky DxVx + i Kz Omega)/K_perp^2, Vz = (i Kz DxVx - i Ky Omega)/K_perp^2; on the kx axis
    (ky = kz = 0) all three are 0."""
    Ky, Kz = ky * kfactor[1], kz * kfactor[2]
    kp2 = Ky * Ky + Kz * Kz
    if ky == 0 and kz == 0:
        return 0j, 0j, 0j
    d = _dx(basis, kfactor, kx, Vx)
    return Vx, (1j * Ky * d + 1j * Kz * Omega) / kp2, (1j * Kz * d - 1j * Ky * Omega) / kp2


def given_modes(entries, N, kfactor=(1.0, 1.0, 1.0), basis: str = "FOUR", physics: str = "FLUID",
                rule: str = "simple"):
    """Compute_force_given_modes_SIMPLE (compute_force_modes.cc:97-440): entries are
    (kx, ky, kz, Fx, Fy) for a fluid, (kx, ky, kz, Fx, Fy, FxW, FyW) for MHD and
    (kx, ky, kz, Fx, Fy, G) for a scalar.  Each vector's third component comes from
    Last_component.  rule "vorticity": Compute_force_given_modes_VORTICITY (:470-700), the second
    value of each vector is its x-vorticity and Compute_VyVz gives (Fx, Fy, Fz).  On the kz = 0
    and kz = N3/2 planes the conjugate mode is added to the force
    (FOUR: F(-kx, -ky, kz) = F*; SCFT: F(kx, -ky, kz) = F*, or on ky = 0 F1 = 0 and the
    imaginary parts of F2, F3 and G dropped), which is what Assign_force_and_comp_conj
    (field_k_fns.cc:462-500) states as its purpose."""
    ns = _nstate(physics)
    N3 = int(N[2])
    modes: dict = {}
    for e in entries:
        kx, ky, kz = (int(x) for x in e[:3])
        third = compute_vyvz if rule == "vorticity" else last_component
        vals = list(third(kx, ky, kz, complex(e[3]), complex(e[4]), kfactor, basis))
        if ns == 6:
            vals += list(third(kx, ky, kz, complex(e[5]), complex(e[6]), kfactor, basis))
        elif ns == 4:
            vals.append(complex(e[5]))
        for c, v in enumerate(vals):
            _set(modes, (kx, ky, kz), c, v, ns)
        if kz == 0 or kz == N3 // 2:
            if basis == "FOUR" or ky != 0:
                kc = (-kx, -ky, kz) if basis == "FOUR" else (kx, -ky, kz)
                for c, v in enumerate(vals):
                    _set(modes, kc, c, np.conj(v), ns)
            else:
                v = modes[(kx, ky, kz)]
                for c0 in range(0, ns - ns % 3, 3):     # each vector: F1 = 0, F2 and F3 real
                    v[c0] = 0j
                    v[c0 + 1] = complex(v[c0 + 1].real, 0.0)
                    v[c0 + 2] = complex(v[c0 + 2].real, 0.0)
                if ns == 4:
                    v[3] = complex(v[3].real, 0.0)
    return _pack(modes, ns)


def read_force_modes_file(path, N1: int, n_values: int = 2):
    """in/force_field_in.d as IncFluid::Read_waveno_force_field reads it
    (compute_force_modes.cc:47-85): repeated "kx ky kz" integers followed by n_values complex
    numbers "(re,im)"; a kx >= N1 (or the end of the file) ends the list.  Returns the entries
    for given_modes."""
    toks = open(path).read().split()
    out, p = [], 0
    while p < len(toks):
        kx = int(toks[p])
        if kx >= N1:
            break
        if p + 3 + n_values > len(toks):
            raise ValueError(f"{path}: truncated mode entry")
        ky, kz = int(toks[p + 1]), int(toks[p + 2])
        vals = []
        for t in toks[p + 3:p + 3 + n_values]:
            t = t.strip()
            if t.startswith("(") and t.endswith(")"):
                re_, im_ = t[1:-1].split(",")
                vals.append(complex(float(re_), float(im_)))
            else:
                vals.append(complex(float(t), 0.0))
        out.append((kx, ky, kz, *vals))
        p += 3 + n_values
    return out
