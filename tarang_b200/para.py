"""The reference's run parameters file ``in/para.d``, read the way src/read_para.cc:190-670 reads
it, and mapped to a solver configuration the way the drivers do (src/IFluid/Ifluid_main.cc:
132-227, src/IMHD/IMHD_main.cc, src/RBslip/RB_slip_main.cc:150-240, IncFluid::IncFluid
lib/IncFluid/IncFluid.cc:175-217).

The file is positional: read_para.cc takes tokens with ``>>`` (labels are read into a dummy
string) and skips fixed numbers of lines with ``getline``.  ``_Stream`` reproduces those two
operations exactly, so a file the reference reads is read the same way here::

    p = read_para("in/para.d", n_fields=1)
    cfg = config_from_para(p, "FLUID")     # keyword arguments of solver.make_config
    U = IncFluid(**cfg)
"""

from __future__ import annotations

import math

_N_FIELDS = {"FLUID": 1, "MHD": 2, "SCALAR": 2, "RB": 2}


class _Stream:
    """istream >> token (skips leading whitespace, newlines included) and getline (the rest of
    the current line, newline consumed)."""

    def __init__(self, text: str):
        self.t = text
        self.p = 0

    def token(self) -> str:
        n = len(self.t)
        while self.p < n and self.t[self.p].isspace():
            self.p += 1
        if self.p >= n:
            raise ValueError("para.d ends early")
        q = self.p
        while q < n and not self.t[q].isspace():
            q += 1
        tok, self.p = self.t[self.p:q], q
        return tok

    def getline(self, k: int = 1):
        for _ in range(k):
            q = self.t.find("\n", self.p)
            self.p = len(self.t) if q < 0 else q + 1

    def int(self) -> int:
        return int(self.token())

    def float(self) -> float:
        return float(self.token())


def read_para(source, n_fields: int = 1, dim: int = 3) -> dict:
    """Parameters of a para.d file (path or text); n_fields = number_of_fields of the program
    (fluid 1, MHD 2, scalar and convection 2).  Indices follow the reference's 1-based arrays
    (entry 0 unused) so p["switches"][19] is output_vx_vy_switch."""
    text = source
    if "\n" not in str(source):
        with open(source) as fh:
            text = fh.read()
    s = _Stream(text)
    p = {}
    s.getline(3)
    p["N"] = [0] + [s.int() for _ in range(dim)]
    s.getline(3)
    # solver parameters
    s.token()
    p["solver_meta"] = [0] + [s.int() for _ in range(3)]
    s.token()
    p["solver_int"] = [0] + [s.int() for _ in range(p["solver_meta"][1])]
    s.token()
    p["solver_double"] = [0.0] + [s.float() for _ in range(p["solver_meta"][2])]
    s.getline()
    s.token()
    p["solver_string"] = [""] + [s.token() for _ in range(p["solver_meta"][3])]
    s.getline(3)
    # string switches: basis, alias, integration scheme, input and output number modes
    sw = [""]
    for _ in range(5):
        s.token()
        sw.append(s.token())
    p["string_switches"] = sw
    s.getline(3)
    sw = [0]
    for _ in range(22):
        s.token()
        sw.append(s.int())
    p["switches"] = sw
    s.getline(4)
    p["diss"] = [s.float() for _ in range(n_fields)]
    s.getline(3)
    p["hyper_diss"] = [s.float() for _ in range(n_fields)]
    s.getline(3)
    tp = [0.0]
    for _ in range(5):
        s.token()
        tp.append(s.float())
    p["time_para"] = tp            # Tinit, Tfinal, Tdt, Tdiag_basic_init, Tdiag_advanced_init
    s.getline(3)
    ts = [0.0]
    for _ in range(19):
        s.token()
        ts.append(s.float())
    p["time_save"] = ts
    s.getline(3)
    mo = [0]
    for _ in range(5):
        s.token()
        mo.append(s.int())
    s.token()
    mo += [s.int() for _ in range(dim)]  # N_out_reduced
    p["misc_output"] = mo
    s.getline(3)
    et = [0]
    for _ in range(11):
        s.token()
        et.append(s.int())
    p["ET"] = et                   # (2) no-spheres, (3) no-shells, ...
    s.getline(3)
    s.token()
    nk = s.int()
    s.token()
    nr = s.int()
    p["no_output_k_r"] = [0, nk, nr]
    s.getline(2)
    p["out_k"] = [(s.int(), s.int(), s.int()) for _ in range(nk)]
    s.getline(2)
    p["out_r"] = [(s.int(), s.int(), s.int()) for _ in range(nr)]
    s.getline(3)
    for part in ("init_cond", "force"):
        s.token()
        meta = [0] + [s.int() for _ in range(3)]
        s.token()
        ints = [0] + [s.int() for _ in range(meta[1])]
        s.token()
        dbls = [0.0] + [s.float() for _ in range(meta[2])]
        s.getline()
        s.token()
        strs = [""] + [s.token() for _ in range(meta[3])]
        s.getline(3)
        p[part + "_meta"], p[part + "_int"], p[part + "_double"], p[part + "_string"] = meta, ints, dbls, strs
    return p


def config_from_para(p: dict, kind: str = "FLUID") -> dict:
    """Keyword arguments of solver.make_config (N, basis, physics, dealias, kfactor,
    coefficients, dt, forcing, shells) for a parsed para.d, plus 'run' with the time span, the
    field I/O switches and the initial-condition procedure.  Raises ValueError for what the GPU
    solver does not run (other schemes, other forcings).  The integration scheme (EULER, RK2,
    RK4) and, with hyper_dissipation_switch (switches(1)) on, the hyper coefficients of U and of
    W or T (IncVF.cc:70-83, IncSF.cc:62-65) carry over."""
    kind = kind.upper()
    if kind not in _N_FIELDS:
        raise ValueError(f"kind {kind}")
    basis, alias, scheme = p["string_switches"][1], p["string_switches"][2], p["string_switches"][3]
    if scheme not in ("EULER", "RK2", "RK4"):
        raise ValueError(f"integration scheme {scheme}: EULER, RK2 and RK4 run on the GPU")
    hyper = p["switches"][1] != 0
    sd, si = p["solver_double"], p["solver_int"]
    if kind == "RB":
        # RB_slip_main.cc:150-240: kfactor given or scaled by (pi, pi/sqrt 2, pi/sqrt 2); Ra
        # given or in units of the critical 27 pi^4 / 4; Pr
        if len(si) > 1 and si[1] == 1:
            k0 = math.pi / math.sqrt(2.0)
            kf = (math.pi * sd[1], k0 * sd[2], k0 * sd[3])
        else:
            kf = (sd[1], sd[2], sd[3])
        ra = sd[4] if not (len(si) > 2 and si[2] == 1) else (27.0 * math.pi ** 4 / 4.0) * sd[4]
        pr = sd[5]
        pr_switch = p["solver_string"][1] if len(p["solver_string"]) > 1 else "PRLARGE"
        u_scaling = p["solver_string"][2] if len(p["solver_string"]) > 2 else "ULARGE"
        if pr_switch not in ("PRLARGE", "PRSMALL"):
            raise ValueError(f"Pr_switch {pr_switch}: PRLARGE and PRSMALL run on the GPU")
        if u_scaling not in ("ULARGE", "USMALL"):
            raise ValueError(f"RB_Uscaling {u_scaling}")
        temp_grad = sd[6] if len(sd) > 6 else 1.0
    else:
        kf = (sd[1], sd[2], sd[3])
    cfg = dict(N=tuple(p["N"][1:4]), basis=basis, physics=kind, dealias=(alias == "DEALIAS"),
               kfactor=kf, nu=p["diss"][0], dt=p["time_para"][3], n_shells=p["ET"][3], scheme=scheme,
               hyper_nu=p["hyper_diss"][0] if hyper else 0.0)
    if kind == "MHD":
        cfg["eta"] = p["diss"][1]
        cfg["hyper_eta"] = p["hyper_diss"][1] if hyper else 0.0
    elif kind == "SCALAR":
        cfg["kappa"] = p["diss"][1]
    elif kind == "RB":
        cfg.update(Ra=ra, Pr=pr, Pr_switch=pr_switch, RB_Uscaling=u_scaling, temperature_grad=temp_grad)
    if kind in ("SCALAR", "RB"):
        cfg["hyper_kappa"] = p["hyper_diss"][1] if hyper else 0.0
    proc = p["force_int"][1] if len(p["force_int"]) > 1 else 0
    fd = p["force_double"] + [0.0] * 7
    run_force = None
    if proc in (1, 2) and kind != "RB":
        # compute_force_ek_hk_supply.cc / compute_force_const_ek_hk.cc: force_double(1..4) for U,
        # (5, 6) the energy and helicity ratio of W (MHD) or (5) the scalar's energy (scalar)
        f = dict(kind="energy_supply" if proc == 1 else "energy_helicity", inner=fd[1], outer=fd[2], eps=fd[3],
                 eps_h=fd[4])
        if kind == "MHD":
            f.update(eps_W=fd[5], eps_hW=fd[6])
        elif kind == "SCALAR":
            f.update(eps_T=fd[5])
        cfg["force"] = f
    elif proc in (3, 4) and kind != "RB":
        # compute_force_TG.cc:47-92, compute_force_ABC.cc:50-131: k0, amplitudes (W: the next)
        cfg["force"] = dict(kind="modes")
        if proc == 3:
            run_force = dict(kind="taylor_green", k0=int(fd[1]), amp=fd[2], ampW=fd[3])
        else:
            run_force = dict(kind="abc", k0=int(fd[1]), A=fd[2], B=fd[3], C=fd[4], amp=fd[5], ampW=fd[6])
    elif proc in (5, 6) and kind != "RB":
        # the modes come from in/force_field_in.d (forcing.read_force_modes_file); proc 6 gives
        # each vector's x-vorticity in place of its y component (Compute_VyVz)
        cfg["force"] = dict(kind="modes")
        run_force = dict(kind="given_modes", file="in/force_field_in.d", rule="simple" if proc == 5 else "vorticity")
    elif proc == 101 and kind == "FLUID":
        # Compute_force_Liquid_metal (compute_force_LM.cc:46-70): B0 = force_double(1..3)
        cfg["force"] = dict(kind="liquid_metal", B0=(fd[1], fd[2], fd[3]))
    elif proc == 101 and kind == "MHD":
        # Compute_force_DYNAMO_SIX_MODE (compute_force_dynamo_6mode.cc:45-80): k0, amp101,
        # amp011, amp112, h
        cfg["force"] = dict(kind="modes")
        run_force = dict(kind="six_mode", k0=int(fd[1]), amp=(fd[2], fd[3], fd[4], fd[5]))
    elif proc == 21 and kind != "RB":
        # compute_force_Coriolis.cc:47-80 takes the number of components from force_int(1),
        # which is also force_field_proc (21), so as written it sets neither branch; the
        # evident meaning is kept: force_int(2) = 1 with omega along axis force_int(3) given by
        # force_double(1), else omega = force_double(1..3)
        fi = p["force_int"] + [0] * 3
        if fi[2] == 1 and fi[3] in (1, 2, 3):
            om = [0.0, 0.0, 0.0]
            om[fi[3] - 1] = fd[1]
        else:
            om = [fd[1], fd[2], fd[3]]
        cfg["force"] = dict(kind="coriolis", omega=tuple(om))
    elif proc == 52 and kind == "RB":
        # Compute_force_RB_rotation (compute_force_RB.cc:132-195): buoyancy plus the Coriolis
        # force, Omega read as for proc 21
        fi = p["force_int"] + [0] * 3
        if fi[2] == 1 and fi[3] in (1, 2, 3):
            om = [0.0, 0.0, 0.0]
            om[fi[3] - 1] = fd[1]
        else:
            om = [fd[1], fd[2], fd[3]]
        cfg["force"] = dict(kind="rb_rotation", omega=tuple(om))
    elif proc != 0 and kind != "RB":
        raise ValueError(f"force_field_proc {proc} is not supported")
    cfg["run"] = dict(Tinit=p["time_para"][1], Tfinal=p["time_para"][2],
                      output_vx_vy=p["switches"][19], input_vx_vy=p["switches"][20],
                      field_input_proc=p["init_cond_int"][1] if len(p["init_cond_int"]) > 1 else 0,
                      init_cond_double=list(p["init_cond_double"]),
                      N_in_reduced=tuple(p["init_cond_int"][2:5]) if (len(p["init_cond_int"]) > 4 and
                                                                       p["init_cond_int"][1] == 2) else None,
                      N_out_reduced=tuple(p["misc_output"][6:9]),
                      force_modes=run_force)
    return cfg


def force_modes_for(cfg: dict, data_dir: str = "."):
    """(k, F) for IncFluid.set_force_modes when config_from_para mapped a fixed-mode forcing
    (cfg["run"]["force_modes"]), else None.  A given-modes forcing reads
    data_dir/in/force_field_in.d (IncFluid::Open_force_waveno_input_files)."""
    import os

    from . import forcing
    fm = cfg.get("run", {}).get("force_modes")
    if not fm:
        return None
    N, basis, physics = cfg["N"], cfg.get("basis", "FOUR"), cfg.get("physics", "FLUID")
    if fm["kind"] == "taylor_green":
        return forcing.taylor_green_modes(N, fm["k0"], fm["amp"], basis, physics, fm["ampW"])
    if fm["kind"] == "six_mode":
        if basis != "FOUR":
            raise ValueError("the six-mode force is FOUR only (force_model.cc:238-243)")
        return forcing.six_mode_modes(N, fm["k0"], *fm["amp"], physics=physics)
    if fm["kind"] == "abc":
        if basis != "FOUR":
            raise ValueError("ABC forcing is FOUR only (force_model.cc:164-168)")
        return forcing.abc_modes(N, fm["k0"], fm["amp"], fm["A"], fm["B"], fm["C"], physics, fm["ampW"])
    n_values = {"FLUID": 2, "MHD": 4, "SCALAR": 3}[physics]
    entries = forcing.read_force_modes_file(os.path.join(data_dir, fm["file"]), N[0], n_values)
    return forcing.given_modes(entries, N, cfg.get("kfactor", (1.0, 1.0, 1.0)), basis, physics,
                               fm.get("rule", "simple"))
