"""Python mirror of Tarang's field/solver class API over the C ABI (include/tarang_gpu.h).

Method names follow the reference (lib/IncFluid/IncFluid.h, lib/IncFlow/IncVF.h,
lib/fields/Cvf.h) so that a driver written against the reference reads the same:

    U = IncFluid(N=(64, 64, 64), nu=0.01, dt=1e-3)
    U.set_V([v1, v2, v3])                     # spectral fields, (N1, N2, N3/2+1) complex128
    for it in range(100):                     # Ifluid_main.cc:258-301
        U.Compute_force(); U.Compute_nlin(); U.Add_force(); U.Compute_pressure()
        U.Tdt = U.Get_dt(); U.Time_advance()
        E, D = U.CV_Compute_totalenergy_diss()

``IncFluid.step(n)`` runs the same loop body n times in one call (one CUDA graph per step).
Every call goes to the CUDA library; there is no CPU path.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

_BASIS = {"FOUR": L.TG_FOUR, "SCFT": L.TG_SCFT}
_PHYS = {"FLUID": L.TG_FLUID, "INC_FLUID": L.TG_FLUID, "MHD": L.TG_MHD, "INC_MHD": L.TG_MHD,
         "SCALAR": L.TG_SCALAR, "INC_SCALAR": L.TG_SCALAR, "RB": L.TG_RB, "RB_SLIP": L.TG_RB}
_PREC = {"FP64": L.TG_FP64, "FP32": L.TG_FP32_MIXED, "FP32_MIXED": L.TG_FP32_MIXED}
_SCHEME = {"EULER": L.TG_EULER, "RK2": L.TG_RK2, "RK4": L.TG_RK4}


_DP_T = C.POINTER(C.c_double)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_config(N, basis="FOUR", physics="FLUID", precision="FP64", dealias=True,
                kfactor=(1.0, 1.0, 1.0), nu=0.01, eta=None, kappa=None, dt=1e-3,
                force=None, n_shells=12, device=0, Ra=0.0, Pr=0.0, stream=None,
                Pr_switch="PRLARGE", RB_Uscaling="ULARGE", temperature_grad=1.0, scheme="RK4",
                hyper_nu=0.0, hyper_eta=None, hyper_kappa=None) -> L.tg_config:
    lib = L.load()
    cfg = L.tg_config()
    lib.tg_config_default(C.byref(cfg))
    cfg.N[:] = [int(n) for n in N]
    cfg.basis = _BASIS[basis] if isinstance(basis, str) else int(basis)
    cfg.physics = _PHYS[physics] if isinstance(physics, str) else int(physics)
    cfg.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
    cfg.dealias = 1 if dealias else 0
    cfg.scheme = _SCHEME[scheme] if isinstance(scheme, str) else int(scheme)
    cfg.hyper_nu = float(hyper_nu)
    cfg.hyper_eta = float(hyper_nu if hyper_eta is None else hyper_eta)
    cfg.hyper_kappa = float(hyper_nu if hyper_kappa is None else hyper_kappa)
    cfg.kfactor[:] = [float(k) for k in kfactor]
    cfg.nu = float(nu)
    cfg.eta = float(nu if eta is None else eta)
    cfg.kappa = float(nu if kappa is None else kappa)
    cfg.dt = float(dt)
    if force is None and cfg.physics == L.TG_RB:
        cfg.force_kind = L.TG_FORCE_RB          # Compute_force_RB (force_field_proc 51)
    elif force is None or force == "decay":
        cfg.force_kind = L.TG_FORCE_DECAY
    elif force.get("kind") == "modes":
        cfg.force_kind = L.TG_FORCE_MODES          # fixed modes, IncFluid.set_force_modes
    elif force.get("kind") == "coriolis":
        cfg.force_kind = L.TG_FORCE_CORIOLIS       # Force = V x omega (force_field_proc 21)
        cfg.force_para[:3] = [float(x) for x in force["omega"]]
    elif force.get("kind") == "liquid_metal":
        cfg.force_kind = L.TG_FORCE_LIQUID_METAL   # -(B0 . K)^2/K^2 V (force_field_proc 101)
        cfg.force_para[:3] = [float(x) for x in force["B0"]]
    elif force.get("kind") == "rb_rotation":
        cfg.force_kind = L.TG_FORCE_RB_ROTATION    # buoyancy + scaled V x omega (proc 52)
        cfg.force_para[:3] = [float(x) for x in force["omega"]]
    elif force.get("kind", "energy_supply") not in ("energy_supply", "energy_helicity"):
        raise ValueError(f"force kind {force.get('kind')}")
    else:
        # force_field_proc 1 (energy supply) or 2 (constant energy and helicity): U's parameters,
        # then B's (MHD) or the scalar's energy (passive scalar)
        supply = force.get("kind", "energy_supply") == "energy_supply"
        cfg.force_kind = L.TG_FORCE_ENERGY_SUPPLY if supply else L.TG_FORCE_ENERGY_HELICITY
        p = [force.get("inner"), force.get("outer"), force.get("eps"), force.get("eps_h", 0.0),
             force.get("eps_W", force.get("eps_T", 0.0)), force.get("eps_hW", 0.0)]
        cfg.force_para[:] = [float(x) for x in p]
    cfg.n_shells = int(n_shells)
    cfg.rb_ra = float(Ra)
    cfg.rb_pr = float(Pr)
    cfg.rb_pr_switch = {"PRLARGE": L.TG_RB_PRLARGE, "PRSMALL": L.TG_RB_PRSMALL}[Pr_switch]
    cfg.rb_u_scaling = {"ULARGE": L.TG_RB_ULARGE, "USMALL": L.TG_RB_USMALL}[RB_Uscaling]
    cfg.rb_temp_grad = float(temperature_grad)
    cfg.device = int(device)
    cfg.stream = C.c_void_p(int(stream)) if stream else None
    return cfg


def write_field_file(path, fields, time=0.0, vx_vy=False, append=False, reduced=None, basis="FOUR"):
    """Write state fields (each (N1, N2, N3/2+1) complex128, reference order) in the reference's
    field-file text format (tg_write_field_file); with reduced = (Nr1, Nr2, Nr3) only the
    low-wavenumber corner, as Output_field_reduced writes it (tg_write_field_file_reduced)."""
    lib = L.load()
    arrs = [np.ascontiguousarray(f, dtype=np.complex128) for f in fields]
    N1, N2, M3 = arrs[0].shape
    Nc = (C.c_int * 3)(N1, N2, 2 * (M3 - 1))
    ptrs = (_DP_T * len(arrs))(*[_dptr(a.view(np.float64)) for a in arrs])
    if reduced is None:
        rc = lib.tg_write_field_file(str(path).encode(), float(time), Nc, len(arrs), ptrs, 1 if vx_vy else 0,
                                     1 if append else 0)
    else:
        Nr = (C.c_int * 3)(*[int(n) for n in reduced])
        b = _BASIS[basis] if isinstance(basis, str) else int(basis)
        rc = lib.tg_write_field_file_reduced(str(path).encode(), float(time), Nc, Nr, b, len(arrs), ptrs,
                                             1 if vx_vy else 0, 1 if append else 0)
    if rc != L.TG_OK:
        raise L.TarangError(rc, f"write_field_file {path}")


def read_field_file(path, N, n_fields, basis="FOUR", kfactor=(1.0, 1.0, 1.0), vx_vy=False, reduced=None):
    """Read n_fields state fields of grid N from a reference field file (tg_read_field_file);
    with reduced = (Nr1, Nr2, Nr3) the file holds the low-wavenumber corner only (a smaller run's
    field file or Output_field_reduced; tg_read_field_file_reduced, as Init_cond_reduced)."""
    lib = L.load()
    shape = (N[0], N[1], N[2] // 2 + 1)
    arrs = [np.zeros(shape, dtype=np.complex128) for _ in range(n_fields)]
    Nc = (C.c_int * 3)(*[int(n) for n in N])
    kf = (C.c_double * 3)(*[float(k) for k in kfactor])
    ptrs = (_DP_T * n_fields)(*[_dptr(a.view(np.float64)) for a in arrs])
    b = _BASIS[basis] if isinstance(basis, str) else int(basis)
    if reduced is None:
        rc = lib.tg_read_field_file(str(path).encode(), Nc, b, kf, n_fields, ptrs, 1 if vx_vy else 0)
    else:
        Nr = (C.c_int * 3)(*[int(n) for n in reduced])
        rc = lib.tg_read_field_file_reduced(str(path).encode(), Nc, Nr, b, kf, n_fields, ptrs, 1 if vx_vy else 0)
    if rc != L.TG_OK:
        raise L.TarangError(rc, f"read_field_file {path}")
    return arrs


class IncFluid:
    """Solver context: the reference's IncFluid U (with IncVF W for MHD, IncSF T for scalars)."""

    def __init__(self, N, **kw):
        self.lib = L.load()
        self.N = tuple(int(n) for n in N)
        self.cfg = make_config(self.N, **kw)
        self.kw = kw
        h = C.c_void_p()
        rc = self.lib.tg_ctx_create(C.byref(self.cfg), C.byref(h))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_ctx_create failed")
        self.h = h
        self.shape = (self.N[0], self.N[1], self.N[2] // 2 + 1)
        self.ndoubles = 2 * self.shape[0] * self.shape[1] * self.shape[2]
        self.Tdt = self.cfg.dt

    # ------------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "h", None):
            self.lib.tg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        if rc != L.TG_OK:
            msg = self.lib.tg_last_error(self.h)
            raise L.TarangError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    # ------------------------------------------------------------------ fields
    def upload(self, field: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        if a.shape != self.shape:
            raise ValueError(f"field shape {a.shape} != {self.shape}")
        self._ck(self.lib.tg_field_upload(self.h, field, _dptr(a.view(np.float64)), self.ndoubles), "upload")

    def download(self, field: int) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.complex128)
        self._ck(self.lib.tg_field_download(self.h, field, _dptr(out.view(np.float64)), self.ndoubles), "download")
        return out

    def download_stored(self, field: int, out: np.ndarray):
        """The stored (dealiased) modes of a state field into `out` (complex128, reference
        layout), leaving its other entries as they are (tg_field_download_stored)."""
        if out.shape != self.shape or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous complex128 array of the field's shape")
        self._ck(self.lib.tg_field_download_stored(self.h, field, _dptr(out.view(np.float64)), self.ndoubles),
                 "download_stored")
        return out

    def alloc_field(self) -> int:
        """A reserved work field id (tg_field_alloc); release it with free_field."""
        f = C.c_int()
        self._ck(self.lib.tg_field_alloc(self.h, C.byref(f)), "field alloc")
        return f.value

    def free_field(self, field: int):
        self._ck(self.lib.tg_field_free(self.h, int(field)), "field free")

    def set_V(self, V):
        for i, v in enumerate(V):
            self.upload(L.TG_V1 + i, v)

    def get_V(self):
        return [self.download(L.TG_V1 + i) for i in range(3)]

    def set_W(self, W):
        for i, w in enumerate(W):
            self.upload(L.TG_W1 + i, w)

    def get_W(self):
        return [self.download(L.TG_W1 + i) for i in range(3)]

    def set_T(self, T):
        self.upload(L.TG_T, T)

    def get_T(self):
        return self.download(L.TG_T)

    def get_nlin(self):
        return [self.download(L.TG_NLIN1 + i) for i in range(3)]

    def get_Wnlin(self):
        return [self.download(L.TG_WNLIN1 + i) for i in range(3)]

    def get_Tnlin(self):
        return self.download(L.TG_TNLIN)

    def get_pressure(self):
        return self.download(L.TG_PRESSURE)

    def get_force(self):
        return [self.download(L.TG_FORCE1 + i) for i in range(3)]

    # ------------------------------------------------------------------ transforms
    def Forward_transform_array(self, real_packed: np.ndarray, parity: int = 0, slot: int = 0) -> np.ndarray:
        """universal_tr.cc:66-86 on a work field: real data in the reference's in-place layout."""
        f = L.TG_WORK0 + slot
        self.upload(f, real_packed)
        self._ck(self.lib.tg_forward_transform(self.h, f, parity), "forward")
        return self.download(f)

    def Inverse_transform_array(self, spec: np.ndarray, parity: int = 0, slot: int = 0) -> np.ndarray:
        """universal_tr.cc:126-146 on a work field; returns the packed real layout."""
        f = L.TG_WORK0 + slot
        self.upload(f, spec)
        self._ck(self.lib.tg_inverse_transform(self.h, f, parity), "inverse")
        return self.download(f)

    # ------------------------------------------------------------------ solver calls
    def Compute_force(self):
        self._ck(self.lib.tg_compute_force(self.h), "Compute_force")

    def set_force_modes(self, k, F):
        """The fixed force of force=dict(kind="modes") (tg_set_force_modes): k (n, 3) wavenumber
        indices, F (n, nstate) complex force on each state field there (tarang_b200.forcing
        builds both for the Taylor-Green, ABC and given-mode forcings)."""
        k = np.ascontiguousarray(k, dtype=np.int32).reshape(-1, 3)
        F = np.ascontiguousarray(F, dtype=np.complex128)
        ns = {L.TG_FLUID: 3, L.TG_MHD: 6}.get(self.cfg.physics, 4)
        if F.ndim != 2 or F.shape != (k.shape[0], ns):
            raise ValueError(f"F must have one row of {ns} values per mode")
        self._ck(self.lib.tg_set_force_modes(self.h, k.shape[0], k.ctypes.data_as(C.POINTER(C.c_int)),
                                             _dptr(F.view(np.float64))), "set_force_modes")

    def Compute_nlin(self):
        self._ck(self.lib.tg_compute_nlin(self.h), "Compute_nlin")

    def Add_force(self):
        self._ck(self.lib.tg_add_force(self.h), "Add_force")

    def Compute_pressure(self):
        self._ck(self.lib.tg_compute_pressure(self.h), "Compute_pressure")

    def Compute_rhs(self):
        self._ck(self.lib.tg_compute_rhs(self.h), "Compute_rhs")

    def Get_dt(self) -> float:
        dt = C.c_double()
        self._ck(self.lib.tg_get_dt(self.h, C.byref(dt)), "Get_dt")
        self.Tdt = dt.value
        return dt.value

    def Time_advance(self):
        self._ck(self.lib.tg_time_advance(self.h), "Time_advance")

    def step(self, n: int = 1, energies: bool = True):
        """n iterations of the loop body Ifluid_main.cc:261-286; returns E after each step."""
        e = np.empty(max(n, 1), dtype=np.float64)
        rc = self.lib.tg_step(self.h, int(n), _dptr(e) if energies else None)
        self._ck(rc, "step")
        return e[:n]

    def synchronize(self):
        self._ck(self.lib.tg_synchronize(self.h), "synchronize")

    def time(self):
        t = C.c_double()
        s = C.c_longlong()
        self._ck(self.lib.tg_time(self.h, C.byref(t), C.byref(s)), "time")
        return t.value, s.value

    def device_bytes(self) -> int:
        b = C.c_size_t()
        self._ck(self.lib.tg_device_bytes(self.h, C.byref(b)), "device_bytes")
        return b.value

    # ------------------------------------------------------------------ diagnostics
    def CV_Compute_totalenergy_diss(self, group: int = 0):
        E = C.c_double()
        D = C.c_double()
        self._ck(self.lib.tg_energy(self.h, group, C.byref(E), C.byref(D)), "energy")
        return E.value, D.value

    def kmax_outside(self) -> int:
        import math
        d = 3 if self.cfg.dealias else 2
        kf = self.cfg.kfactor
        N = self.N
        if self.cfg.basis == L.TG_SCFT:   # Min_radius_outside_SCFT: kx extent 2N1/3 (N1 aliased)
            nx = (2 * N[0] // 3) if self.cfg.dealias else N[0]
        else:
            nx = N[0] // d
        return int(math.ceil(math.sqrt((nx * kf[0]) ** 2 + ((N[1] // d) * kf[1]) ** 2
                                       + ((N[2] // d) * kf[2]) ** 2)))

    def CV_Compute_shell_spectrum(self, group: int = 0):
        n = self.kmax_outside() + 1
        nc = 1 if group == 2 else 3
        ek = np.zeros(nc * n)
        dk = np.zeros(n)
        self._ck(self.lib.tg_shell_spectrum(self.h, group, _dptr(ek), _dptr(dk), n), "shell spectrum")
        return ek.reshape(nc, n), dk

    def ET_radii(self):
        S = self.cfg.n_shells
        r = np.zeros(S + 1)
        self._ck(self.lib.tg_et_radii(self.h, _dptr(r), S + 1), "et radii")
        return r

    def Compute_flux(self, kind: int = L.TG_ET_UU):
        S = self.cfg.n_shells
        f = np.zeros(S + 1)
        self._ck(self.lib.tg_flux(self.h, kind, _dptr(f), S + 1), "flux")
        return f

    def Compute_shell_tr(self, kind: int = L.TG_ET_UU):
        S = self.cfg.n_shells
        t = np.zeros((S + 1) * (S + 1))
        self._ck(self.lib.tg_shell_to_shell(self.h, kind, _dptr(t), S + 1), "shell_tr")
        return t.reshape(S + 1, S + 1)

    def _ring(self, fn, cyl, n, axis, group):
        rs, cs = C.c_int(), C.c_int()
        self._ck(self.lib.tg_ring_sizes(self.h, axis, C.byref(rs), C.byref(cs)), "ring sizes")
        rows = cs.value if cyl else rs.value
        out = [np.zeros((rows, n + 1)) for _ in range(3)]
        self._ck(fn(self.h, group, axis, n, *[_dptr(a) for a in out], rows * (n + 1)), "ring spectrum")
        return tuple(out)

    def CV_Compute_ring_spectrum(self, n_sectors, axis=1, group=0):
        """CVF::CV_Compute_ring_spectrum (tg_ring_spectrum): (ek1, ek2, dissk), each
        [shell][sector] over shells 0..Max_radius_inside and sectors 0..n_sectors about `axis`
        (1 x, 2 y, 3 z); group 0 velocity, 1 magnetic field."""
        return self._ring(self.lib.tg_ring_spectrum, False, n_sectors, axis, group)

    def CV_Compute_cylinder_ring_spectrum(self, n_slabs, axis=1, group=0):
        """CVF::CV_Compute_cylinder_ring_spectrum (tg_cylinder_ring_spectrum): (ek1, ek2,
        dissk), each [cylindrical shell][slab] along `axis`."""
        return self._ring(self.lib.tg_cylinder_ring_spectrum, True, n_slabs, axis, group)

    def CV_Compute_shell_spectrum_helicity(self, group=0):
        """CVF::CV_Compute_shell_spectrum_helicity (tg_shell_spectrum_helicity): (h1, h2, h3)."""
        n = self.kmax_outside() + 1
        out = [np.zeros(n) for _ in range(3)]
        self._ck(self.lib.tg_shell_spectrum_helicity(self.h, group, *[_dptr(a) for a in out], n),
                 "helicity spectrum")
        return tuple(out)

    def CV_Compute_ring_spectrum_helicity(self, n_sectors, axis=1, group=0):
        """CV_Compute_ring_spectrum_helicity (tg_ring_spectrum_helicity): [shell][sector]."""
        rs = C.c_int()
        self._ck(self.lib.tg_ring_sizes(self.h, axis, C.byref(rs), None), "ring sizes")
        h = np.zeros((rs.value, n_sectors + 1))
        self._ck(self.lib.tg_ring_spectrum_helicity(self.h, group, axis, n_sectors, _dptr(h), h.size),
                 "ring helicity")
        return h

    def CV_Compute_cylinder_ring_spectrum_helicity(self, n_slabs, axis=1, group=0):
        """CV_Compute_cylinder_ring_spectrum_helicity (tg_cylinder_ring_spectrum_helicity)."""
        cs = C.c_int()
        self._ck(self.lib.tg_ring_sizes(self.h, axis, None, C.byref(cs)), "ring sizes")
        h = np.zeros((cs.value, n_slabs + 1))
        self._ck(self.lib.tg_cylinder_ring_spectrum_helicity(self.h, group, axis, n_slabs, _dptr(h), h.size),
                 "cylinder helicity")
        return h

    def Compute_kinetic_helicity_flux(self):
        """IncVF::Compute_kinetic_helicity_flux (tg_helicity_flux): flux_hk, n_shells + 1 entries."""
        S = self.cfg.n_shells
        out = np.zeros(S + 1)
        self._ck(self.lib.tg_helicity_flux(self.h, _dptr(out), out.size), "helicity flux")
        return out

    def Compute_magnetic_helicity_flux(self):
        """IncVF::Compute_magnetic_helicity_flux (tg_magnetic_helicity_flux), MHD: W.flux_hk,
        n_shells + 1 entries."""
        S = self.cfg.n_shells
        out = np.zeros(S + 1)
        self._ck(self.lib.tg_magnetic_helicity_flux(self.h, _dptr(out), out.size), "magnetic helicity flux")
        return out

    def Compute_kinetic_helicity_shell_tr(self):
        """IncVF::Compute_kinetic_helicity_shell_tr (tg_helicity_shell_to_shell): shelltoshell_hk,
        (n_shells + 1) x (n_shells + 1)."""
        S = self.cfg.n_shells
        t = np.zeros((S + 1) * (S + 1))
        self._ck(self.lib.tg_helicity_shell_to_shell(self.h, _dptr(t), S + 1), "helicity shell_tr")
        return t.reshape(S + 1, S + 1)

    def Compute_magnetic_helicity_shell_tr(self):
        """IncVF::Compute_magnetic_helicity_shell_tr (tg_magnetic_helicity_shell_to_shell), MHD:
        W.shelltoshell_hk, (n_shells + 1) x (n_shells + 1)."""
        S = self.cfg.n_shells
        t = np.zeros((S + 1) * (S + 1))
        self._ck(self.lib.tg_magnetic_helicity_shell_to_shell(self.h, _dptr(t), S + 1), "magnetic helicity shell_tr")
        return t.reshape(S + 1, S + 1)

    def Compute_ring_tr(self, n_ring_shells, n_sectors, axis=1, kind=L.TG_ET_UU):
        """IncVF::Compute_ring_tr (tg_ring_to_ring): T[i, j, m, s], the transfer from giver
        ring (shell i, sector j) to receiver ring (m, s); kind TG_ET_UU, or for MHD TG_ET_BB,
        TG_ET_UB.  Also returns the ring radii."""
        r = np.zeros(n_ring_shells + 1)
        self._ck(self.lib.tg_ring_radii(self.h, n_ring_shells, _dptr(r), r.size), "ring radii")
        n1, n2 = n_ring_shells + 1, n_sectors + 1
        T = np.zeros((n1, n2, n1, n2))
        self._ck(self.lib.tg_ring_to_ring(self.h, kind, axis, n_ring_shells, n_sectors, _dptr(T), T.size),
                 "ring transfer")
        return T, r

    def Compute_cylinder_ring_tr(self, n_cylinder_shells, n_slabs, axis=1, kind=L.TG_ET_UU):
        """IncVF::Compute_cylinder_ring_tr (tg_cylinder_ring_to_ring): T[i, j, m, s] from giver
        cylinder ring (shell i, slab j) to receiver (m, s), and the cylinder radii."""
        r = np.zeros(n_cylinder_shells + 1)
        self._ck(self.lib.tg_cylinder_radii(self.h, axis, n_cylinder_shells, _dptr(r), r.size), "cylinder radii")
        n1, n2 = n_cylinder_shells + 1, n_slabs + 1
        T = np.zeros((n1, n2, n1, n2))
        self._ck(self.lib.tg_cylinder_ring_to_ring(self.h, kind, axis, n_cylinder_shells, n_slabs, _dptr(T),
                                                   T.size), "cylinder ring transfer")
        return T, r

    def Compute_force_feed_shell(self, group: int = 0):
        """IncVF::Compute_force_feed_shell (compute_force_feed.cc:70-155): forceV_shell (group 0),
        W.forceV_shell (group 1, MHD) or forceSF_shell (group 2, passive scalar), S+1 entries."""
        S = self.cfg.n_shells
        f = np.zeros(S + 1)
        self._ck(self.lib.tg_force_feed_group(self.h, int(group), _dptr(f), S + 1), "force feed")
        return f

    def Compute_force_feed_ring(self, n_ring_shells, n_sectors, axis=1, group=0, cylinder=False):
        """IncVF::Compute_force_feed_ring / Compute_force_feed_cylinder_ring (tg_force_feed_ring):
        forceV_ring (group 0), W.forceV_ring (1) or forceSF_ring (2) as [shell][sector]."""
        out = np.zeros((n_ring_shells + 1) * (n_sectors + 1))
        self._ck(self.lib.tg_force_feed_ring(self.h, int(group), 1 if cylinder else 0, int(axis), int(n_ring_shells),
                                             int(n_sectors), _dptr(out), out.size), "ring force feed")
        return out.reshape(n_ring_shells + 1, n_sectors + 1)

    def Get_Nusselt_no(self) -> float:
        """IncVF::Get_Nusselt_no (nusselt.cc:53-89): Nu = 1 + 2 sqrt(Ra Pr) <u1, theta>."""
        v = C.c_double()
        self._ck(self.lib.tg_nusselt(self.h, C.byref(v)), "nusselt")
        return v.value

    # ------------------------------------------------------------------ field files
    def state_fields(self):
        """V, then W (MHD) or T (scalar, convection): the reference's field-file order."""
        out = self.get_V()
        if self.cfg.physics == L.TG_MHD:
            out += self.get_W()
        elif self.cfg.physics in (L.TG_SCALAR, L.TG_RB):
            out.append(self.get_T())
        return out

    def Output_field(self, path, vx_vy=False, append=False, reduced=None):
        """IncFluid::Output_field (output_field.cc:43-108): the state at the current time; with
        reduced = N_out_reduced, Output_field_reduced (output_field.cc:505-600)."""
        basis = "SCFT" if self.cfg.basis == L.TG_SCFT else "FOUR"
        write_field_file(path, self.state_fields(), self.time()[0], vx_vy, append, reduced, basis)

    def Init_cond_from_file(self, path, vx_vy=False, reduced=None):
        """IncFluid::Init_cond (init_cond_field.cc:47-223): the state read from a field file;
        with reduced = N_in_reduced, Init_cond_reduced (init_cond_field.cc:294-400)."""
        n = {L.TG_MHD: 6, L.TG_SCALAR: 4, L.TG_RB: 4}.get(self.cfg.physics, 3)
        basis = "SCFT" if self.cfg.basis == L.TG_SCFT else "FOUR"
        f = read_field_file(path, self.N, n, basis, tuple(self.cfg.kfactor), vx_vy, reduced)
        self.set_V(f[:3])
        if n == 6:
            self.set_W(f[3:])
        elif n == 4:
            self.set_T(f[3])
