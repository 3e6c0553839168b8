"""Serving loop over the C ABI (``tg_server_*`` in include/tarang_gpu.h).

Independent solves (each one a reference program run: a configuration, initial fields and a
step count) are submitted to one server per GPU.  The server admits them by an HBM budget,
keeps their spectral state resident and advances requests of the same shape together, one
CUDA graph per batch step::

    srv = Server(hbm_budget=150e9, max_batch=64)
    rid = srv.submit(dict(N=(64, 64, 64), nu=3e-3, dt=1e-3, precision="FP32"), fields, 200)
    srv.drain()
    st = srv.poll(rid)            # state, steps_done, submit/start/finish times, energy
    out = srv.result(rid)         # final fields, reference layout

A request's result does not depend on what else the server holds; it equals
``IncFluid.step(n)`` on the same configuration and fields, bit for bit.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .solver import make_config

_NSTATE = {L.TG_FLUID: 3, L.TG_MHD: 6, L.TG_SCALAR: 4, L.TG_RB: 4}
STATES = {L.TG_REQ_QUEUED: "queued", L.TG_REQ_RUNNING: "running", L.TG_REQ_DONE: "done",
          L.TG_REQ_FAILED: "failed"}


def request_bytes(config: dict, batch: int = 1) -> int:
    """Device bytes that a batch of ``batch`` requests of this configuration holds."""
    lib = L.load()
    cfg = make_config(**config)
    b = C.c_size_t()
    rc = lib.tg_request_bytes(C.byref(cfg), int(batch), C.byref(b))
    if rc != L.TG_OK:
        raise L.TarangError(rc, "tg_request_bytes")
    return b.value


class Server:
    def __init__(self, hbm_budget: float = 150e9, max_batch: int = 64, device: int = 0,
                 use_graphs: bool = True, keep_results: bool = True, borrow_inputs: bool = False):
        """borrow_inputs: submit keeps a reference to the fields array instead of copying it;
        the array must not change until the request has left the queue."""
        self.lib = L.load()
        sc = L.tg_server_config()
        sc.hbm_budget_bytes = int(hbm_budget)
        sc.max_batch = int(max_batch)
        sc.device = int(device)
        sc.use_graphs = 1 if use_graphs else 0
        sc.keep_results = 1 if keep_results else 0
        sc.borrow_inputs = 1 if borrow_inputs else 0
        self.borrow = bool(borrow_inputs)
        self._held: dict[int, np.ndarray] = {}   # borrowed fields, kept alive until admission
        h = C.c_void_p()
        rc = self.lib.tg_server_create(C.byref(sc), C.byref(h))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_create")
        self.h = h
        self.shapes: dict[int, tuple] = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.tg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, config: dict, fields, n_steps: int) -> int:
        """config: keyword arguments of ``make_config`` (N, physics, nu, dt, precision, ...);
        fields: the state fields (V, then W or T), each (N1, N2, N3/2+1) complex128, or one
        C-contiguous complex128 array of shape (n_fields, N1, N2, N3/2+1) (used without a copy)."""
        cfg = make_config(**config)
        N = tuple(cfg.N)
        shape = (N[0], N[1], N[2] // 2 + 1)
        ns = _NSTATE[cfg.physics]
        if (isinstance(fields, np.ndarray) and fields.dtype == np.complex128 and fields.shape == (ns,) + shape
                and fields.flags.c_contiguous):
            init = fields
        else:
            if len(fields) != ns:
                raise ValueError(f"{ns} state fields expected, got {len(fields)}")
            init = np.empty((ns,) + shape, dtype=np.complex128)
            for i, f in enumerate(fields):
                if np.shape(f) != shape:
                    raise ValueError(f"field shape {np.shape(f)} != {shape}")
                init[i] = f
        flat = init.view(np.float64).reshape(-1)
        rq = L.tg_request()
        rq.cfg = cfg
        rq.n_steps = int(n_steps)
        rq.init = flat.ctypes.data_as(C.POINTER(C.c_double))
        rq.n_doubles = flat.size
        rid = C.c_longlong()
        rc = self.lib.tg_server_submit(self.h, C.byref(rq), C.byref(rid))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_submit")
        self.shapes[rid.value] = (ns,) + shape
        if self.borrow:
            self._held[rid.value] = flat
        return rid.value

    def pump(self) -> int:
        n = C.c_int()
        rc = self.lib.tg_server_pump(self.h, C.byref(n))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_pump")
        self._drop_admitted()
        return n.value

    def pump_begin(self):
        """Launch one round's steps and return at once; submissions made before pump_end
        overlap the round on the device."""
        rc = self.lib.tg_server_pump_begin(self.h)
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_pump_begin")

    def pump_end(self) -> int:
        """Admit, wait for the round opened by pump_begin, retire; requests running or queued."""
        n = C.c_int()
        rc = self.lib.tg_server_pump_end(self.h, C.byref(n))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_pump_end")
        self._drop_admitted()
        return n.value

    def _drop_admitted(self):
        # borrowed fields of requests that have left the queue are no longer read
        if self._held:
            for rid in [r for r in self._held if self.poll(r)["state"] != "queued"]:
                del self._held[rid]

    def drain(self, max_rounds: int = 0):
        rc = self.lib.tg_server_drain(self.h, int(max_rounds))
        self._drop_admitted()
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_drain")

    def poll(self, rid: int) -> dict:
        st = L.tg_request_status()
        rc = self.lib.tg_server_poll(self.h, int(rid), C.byref(st))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_poll")
        return dict(state=STATES[st.state], error=st.error, steps_done=st.steps_done,
                    submit_s=st.submit_s, start_s=st.start_s, finish_s=st.finish_s,
                    final_energy=st.final_energy, t_final=st.t_final)

    def result(self, rid: int):
        shp = self.shapes[rid]
        out = np.empty(shp, dtype=np.complex128)
        flat = out.view(np.float64).reshape(-1)
        rc = self.lib.tg_server_result(self.h, int(rid), flat.ctypes.data_as(C.POINTER(C.c_double)), flat.size)
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_result")
        return [out[i] for i in range(shp[0])]

    def release(self, rid: int):
        self.lib.tg_server_release(self.h, int(rid))

    def take_finished(self, max_ids: int = 4096) -> list[int]:
        """Ids of requests finished (done or failed) since the last call."""
        buf = (C.c_longlong * max_ids)()
        out: list[int] = []
        while True:
            n = C.c_int()
            rc = self.lib.tg_server_take_finished(self.h, buf, max_ids, C.byref(n))
            if rc != L.TG_OK:
                raise L.TarangError(rc, "tg_server_take_finished")
            out += buf[: n.value]
            if n.value < max_ids:
                return out

    def stats(self) -> dict:
        st = L.tg_server_stats()
        rc = self.lib.tg_server_stats_get(self.h, C.byref(st))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_stats_get")
        return {k: getattr(st, k) for k, _ in L.tg_server_stats._fields_}

    def batch_stats(self) -> list:
        """Per resident batch: shape N, physics, precision, capacity, n_active and step_ms, the
        device time of one step of the whole batch at step_ms_n_active running requests; device_ms
        and steps, the device time and number of all its batch steps so far."""
        buf = (L.tg_batch_stat * 64)()
        n = C.c_int()
        rc = self.lib.tg_server_batch_stats(self.h, buf, 64, C.byref(n))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_server_batch_stats")
        out = []
        for b in buf[: n.value]:
            d = {k: getattr(b, k) for k, _ in L.tg_batch_stat._fields_}
            d["N"] = tuple(b.N)
            out.append(d)
        return out

    def clock(self) -> float:
        return self.lib.tg_server_clock(self.h)
