"""Slab-sharded single solve over several GPUs (``tg_slab_*`` in include/tarang_gpu.h).

The reference splits one solve over MPI ranks in slabs (basis_basicfn.cc:49-281): each rank
holds ``local_N1`` kx planes of the spectral fields and ``local_N2`` y planes of the real ones,
and every 3-D transform does an all-to-all transpose between the two.  Here each rank (one
process per GPU) holds a slab of the stored kx rows in a context of its own; an RHS evaluation
is three local phases with two all-to-alls between them, issued through ``torch.distributed``
(NCCL) on the stream the context queues on, and the energy sums of a step are all-reduced
before Get_dt::

    solver = SlabSolver((512, 512, 512), nu=1e-3, dt=5e-4)      # inside torchrun, NCCL group
    solver.set_V(V)                                              # every rank: the full fields
    solver.step(10)
    V = solver.get_V()                                           # this rank's rows filled in

``SlabEmulation`` runs the same phases for W ranks inside one process on one GPU, the exchanges
as device copies and the sums in rank order, all on one stream (nothing waits on another
kernel); it is how a single GPU checks the sharded solve against a whole-grid context.
``plan``, ``pack_chunks`` and ``unpack_chunks`` restate the partition and the chunk layouts of
the exchanges in numpy (the layout tg_slab.cu packs).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .solver import make_config

_NSTATE = {L.TG_FLUID: 3, L.TG_SCALAR: 4, L.TG_RB: 4}


# ------------------------------------------------------------------------------ partition
def split(n: int, W: int, i: int) -> tuple[int, int]:
    """start and count of part i of n items over W parts, the first n % W parts one larger."""
    b, rem = divmod(n, W)
    count = b + (1 if i < rem else 0)
    return i * b + min(i, rem), count


def plan(nkx: int, N2: int, W: int) -> dict:
    """kx rows (xs, xn) and y planes (ys, yn) of every rank."""
    xs, xn = zip(*(split(nkx, W, r) for r in range(W)))
    ys, yn = zip(*(split(N2, W, r) for r in range(W)))
    return {"xs": list(xs), "xn": list(xn), "ys": list(ys), "yn": list(yn)}


def pack_chunks(a: np.ndarray, p: dict) -> np.ndarray:
    """[nx][N2][kzp] -> the inverse send buffer: W chunks [nx][yn[d]][kzp], flattened."""
    return np.concatenate([a[:, y0:y0 + n, :].ravel() for y0, n in zip(p["ys"], p["yn"])])


def unpack_chunks(buf: np.ndarray, nx: int, kzp: int, p: dict) -> np.ndarray:
    """the forward receive buffer (W chunks [nx][yn[s]][kzp]) -> [nx][N2][kzp]."""
    N2 = sum(p["yn"])
    out = np.empty((nx, N2, kzp), dtype=buf.dtype)
    off = 0
    for y0, n in zip(p["ys"], p["yn"]):
        out[:, y0:y0 + n, :] = buf[off:off + nx * n * kzp].reshape(nx, n, kzp)
        off += nx * n * kzp
    return out


def inverse_splits(p: dict, rank: int, kzp: int) -> tuple[list, list]:
    """element counts of the inverse all-to-all: (input splits, output splits) of `rank`."""
    nx, ny = p["xn"][rank], p["yn"][rank]
    return [nx * n * kzp for n in p["yn"]], [n * ny * kzp for n in p["xn"]]


def forward_splits(p: dict, rank: int, kzp: int) -> tuple[list, list]:
    """element counts of the forward all-to-all: (input splits, output splits) of `rank`."""
    nx, ny = p["xn"][rank], p["yn"][rank]
    return [n * ny * kzp for n in p["xn"]], [nx * n * kzp for n in p["yn"]]


# ------------------------------------------------------------------------------ device views
class _DeviceBuffer:
    """A device pointer seen as a 1-D real array (``__cuda_array_interface__``)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _tensor(ptr: int, n_complex: int, elem_bytes: int):
    import torch
    typestr = "<f8" if elem_bytes == 16 else "<f4"
    return torch.as_tensor(_DeviceBuffer(ptr, 2 * n_complex, typestr), device="cuda")


class _Rank:
    """One slab context and the device views of its exchange buffers."""

    def __init__(self, N, world, rank, stream_ptr, **kw):
        self.lib = L.load()
        cfg = make_config(N, stream=stream_ptr, **kw)
        h = C.c_void_p()
        rc = self.lib.tg_slab_create(C.byref(cfg), int(world), int(rank), C.byref(h))
        if rc != L.TG_OK:
            raise L.TarangError(rc, "tg_slab_create")
        self.h = h
        self.N = tuple(N)
        info = L.tg_slab_info()
        self._ck(self.lib.tg_slab_info_get(self.h, C.byref(info)), "tg_slab_info_get")
        self.info = info
        W = info.world
        self.plan = {"xs": list(info.xs[:W]), "xn": list(info.xn[:W]), "ys": list(info.ys[:W]),
                     "yn": list(info.yn[:W])}
        self.nstate = _NSTATE[cfg.physics]
        kzp, eb = info.kzp, int(info.elem_bytes)
        nx, ny = info.nx, info.ny
        n_inv_send = nx * N[1] * kzp
        n_inv_recv = info.nkx * ny * kzp

        def buf(which, f, n):
            p = C.c_void_p()
            self._ck(self.lib.tg_slab_buffer(self.h, which, f, C.byref(p)), "tg_slab_buffer")
            return _tensor(p.value, n, eb)

        self.inv_send = [buf(L.TG_SLAB_INV_SEND, f, n_inv_send) for f in range(info.nin)]
        self.inv_recv = [buf(L.TG_SLAB_INV_RECV, f, n_inv_recv) for f in range(info.nin)]
        self.fwd_send = [buf(L.TG_SLAB_FWD_SEND, q, n_inv_recv) for q in range(info.nprod)]
        self.fwd_recv = [buf(L.TG_SLAB_FWD_RECV, q, n_inv_send) for q in range(info.nprod)]
        import torch
        for which, name in ((L.TG_SLAB_SUMS, "sums"), (L.TG_SLAB_GLOBAL_SUMS, "global_sums")):
            p = C.c_void_p()
            self._ck(self.lib.tg_slab_buffer(self.h, which, 0, C.byref(p)), "tg_slab_buffer")
            setattr(self, name, torch.as_tensor(_DeviceBuffer(p.value, 8, "<f8"), device="cuda"))
        # real-element splits (two reals per complex value)
        a, b = inverse_splits(self.plan, info.rank, kzp)
        self.inv_splits = ([2 * x for x in a], [2 * x for x in b])
        a, b = forward_splits(self.plan, info.rank, kzp)
        self.fwd_splits = ([2 * x for x in a], [2 * x for x in b])

    def _ck(self, rc, what):
        if rc != L.TG_OK:
            msg = self.lib.tg_last_error(self.h)
            raise L.TarangError(rc, f"{what}: {msg.decode() if msg else ''}")

    def phase(self, phase, stage=0):
        self._ck(self.lib.tg_slab_phase(self.h, int(phase), int(stage)), f"tg_slab_phase {phase}")

    def upload(self, f, arr):
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        self._ck(self.lib.tg_slab_upload(self.h, int(f), a.ctypes.data_as(C.POINTER(C.c_double))), "tg_slab_upload")

    def download(self, f, out):
        self._ck(self.lib.tg_slab_download(self.h, int(f), out.ctypes.data_as(C.POINTER(C.c_double))),
                 "tg_slab_download")

    def scalars(self):
        s = np.zeros(8)
        t = np.zeros(8)
        self._ck(self.lib.tg_slab_scalars(self.h, s.ctypes.data_as(C.POINTER(C.c_double)),
                                          t.ctypes.data_as(C.POINTER(C.c_double))), "tg_slab_scalars")
        return s, t

    def close(self):
        if getattr(self, "h", None):
            self.lib.tg_ctx_destroy(self.h)
            self.h = None


class _SlabBase:
    ranks: list

    def _set(self, f, arr):
        for r in self.ranks:
            r.upload(f, arr)
        self.dt_ready = False

    def set_V(self, V):
        for i, v in enumerate(V):
            self._set(i, v)

    def set_T(self, T):
        self._set(3, T)

    def _get(self, f):
        N = self.ranks[0].N
        out = np.zeros((N[0], N[1], N[2] // 2 + 1), dtype=np.complex128)
        for r in self.ranks:
            r.download(f, out)
        return out

    def get_V(self):
        return [self._get(i) for i in range(3)]

    def get_T(self):
        return self._get(3)

    def _rhs(self, stage):
        for r in self.ranks:
            r.phase(0, stage)
        self._exchange_inverse()
        for r in self.ranks:
            r.phase(1, stage)
        self._exchange_forward()
        for r in self.ranks:
            r.phase(2, stage)

    def _dt(self):
        for r in self.ranks:
            r.phase(4)
        self._sum_reductions()
        for r in self.ranks:
            r.phase(5)
        self.dt_ready = True

    def step(self, n: int = 1):
        """n RK4 steps (Ifluid_main.cc:261-286); returns the energy of U after each step."""
        if not self.dt_ready:
            self._dt()
        out = []
        for _ in range(n):
            for stage in (1, 2, 3, 4):
                self._rhs(stage)
            self._sum_reductions()
            for r in self.ranks:
                r.phase(3)
            out.append(self.energy())
        return out

    def energy(self) -> float:
        """CV_total_energy of U summed over the ranks (after a step or before the first)."""
        s, _ = self.ranks[0].scalars()
        return float(s[0])

    def time(self):
        _, t = self.ranks[0].scalars()
        return float(t[1]), int(t[2]), float(t[0])

    def close(self):
        for r in self.ranks:
            r.close()


class SlabEmulation(_SlabBase):
    """W slab contexts in one process on one GPU, all on one stream: the exchanges are device
    copies chunk by chunk and the reductions are summed in rank order."""

    def __init__(self, N, world: int, **kw):
        import torch
        kw.setdefault("device", torch.cuda.current_device())
        self.stream = torch.cuda.Stream()
        self.ranks = [_Rank(N, world, r, self.stream.cuda_stream, **kw) for r in range(world)]
        self.dt_ready = False

    def _alltoall(self, send_of, recv_of, splits_of, nf):
        import torch
        W = len(self.ranks)
        with torch.cuda.stream(self.stream):
            for f in range(nf):
                for r in range(W):
                    dst = recv_of(r, f)
                    out_splits = splits_of(r)[1]
                    off = 0
                    for s in range(W):
                        src = send_of(s, f)
                        in_splits = splits_of(s)[0]
                        so = sum(in_splits[:r])
                        n = in_splits[r]
                        assert n == out_splits[s]
                        dst[off:off + n].copy_(src[so:so + n])
                        off += n

    def _exchange_inverse(self):
        self._alltoall(lambda s, f: self.ranks[s].inv_send[f], lambda r, f: self.ranks[r].inv_recv[f],
                       lambda r: self.ranks[r].inv_splits, self.ranks[0].info.nin)

    def _exchange_forward(self):
        self._alltoall(lambda s, f: self.ranks[s].fwd_send[f], lambda r, f: self.ranks[r].fwd_recv[f],
                       lambda r: self.ranks[r].fwd_splits, self.ranks[0].info.nprod)

    def _sum_reductions(self):
        import torch
        with torch.cuda.stream(self.stream):
            tot = self.ranks[0].sums.clone()
            for r in self.ranks[1:]:
                tot += r.sums
            for r in self.ranks:
                r.global_sums.copy_(tot)


class SlabSolver(_SlabBase):
    """This process's rank of a slab-sharded solve; ``torch.distributed`` must be initialised
    (NCCL, one process per GPU).  The exchanges are ``all_to_all_single`` on the current stream."""

    def __init__(self, N, **kw):
        import torch
        import torch.distributed as dist
        self.dist = dist
        world, rank = dist.get_world_size(), dist.get_rank()
        kw.setdefault("device", torch.cuda.current_device())
        self.stream = torch.cuda.current_stream()
        self.ranks = [_Rank(N, world, rank, self.stream.cuda_stream, **kw)]
        self.dt_ready = False

    def _exchange_inverse(self):
        r = self.ranks[0]
        for f in range(r.info.nin):
            self.dist.all_to_all_single(r.inv_recv[f], r.inv_send[f], r.inv_splits[1], r.inv_splits[0])

    def _exchange_forward(self):
        r = self.ranks[0]
        for q in range(r.info.nprod):
            self.dist.all_to_all_single(r.fwd_recv[q], r.fwd_send[q], r.fwd_splits[1], r.fwd_splits[0])

    def _sum_reductions(self):
        r = self.ranks[0]
        r.global_sums.copy_(r.sums)
        self.dist.all_reduce(r.global_sums)

    def get_V(self):
        """The full fields with this rank's kx rows filled in (zeros elsewhere)."""
        return super().get_V()
