"""The slab-sharded solve's partition and exchanges on the CPU (no GPU): the split of the stored
kx rows and the y planes over the ranks, and the chunk layouts of the two all-to-alls of an RHS
evaluation (tarang_b200/slab.py restates the layout tg_slab.cu packs), run as two and three gloo
ranks with torch.distributed.all_to_all_single.  Each rank's inverse receive must be all stored
kx rows of its y planes, and its forward receive, unpacked, its kx rows of all y planes.  The
device phases around these exchanges are checked on a GPU (tests/test_gpu_slab.py); the NCCL
path across several GPUs is unmeasured on hardware (one GPU per run here)."""

import json
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from tarang_b200 import slab  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_plan_covers_rows_and_planes_once():
    for n in (1, 5, 7, 64, 171):
        for W in range(1, min(n, 9) + 1):
            starts, counts = zip(*(slab.split(n, W, r) for r in range(W)))
            assert sum(counts) == n and starts[0] == 0
            assert all(starts[r] + counts[r] == starts[r + 1] for r in range(W - 1))
            assert max(counts) - min(counts) <= 1


def _global(nkx, N2, kzp, salt):
    i = np.arange(nkx * N2 * kzp, dtype=np.float64).reshape(nkx, N2, kzp)
    return (i + salt) + 1j * (-i * 3 - salt)


def _rank_main(rank, world, port, outdir, nkx, N2, kzp):
    import datetime

    import torch
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    from tarang_b200 import slab as S
    p = S.plan(nkx, N2, world)
    x0, nx, y0, ny = p["xs"][rank], p["xn"][rank], p["ys"][rank], p["yn"][rank]
    res = {}
    # inverse: each rank holds the y-inverse outputs of its kx rows, [nx][N2][kzp]
    G = _global(nkx, N2, kzp, 1.0)
    send = S.pack_chunks(G[x0:x0 + nx], p)
    a, b = S.inverse_splits(p, rank, kzp)
    recv = torch.empty(2 * sum(b), dtype=torch.float64)
    torch.distributed.all_to_all_single(recv, torch.from_numpy(send.view(np.float64).copy()),
                                        [2 * v for v in b], [2 * v for v in a])
    got = recv.numpy().view(np.complex128).reshape(nkx, ny, kzp)
    res["inverse_ok"] = bool(np.array_equal(got, G[:, y0:y0 + ny, :]))
    # forward: each rank holds the x-forward outputs of its y planes, [nkx][ny][kzp]
    H = _global(nkx, N2, kzp, 7.0)
    send2 = np.ascontiguousarray(H[:, y0:y0 + ny, :]).ravel()
    a, b = S.forward_splits(p, rank, kzp)
    recv2 = torch.empty(2 * sum(b), dtype=torch.float64)
    torch.distributed.all_to_all_single(recv2, torch.from_numpy(send2.view(np.float64).copy()),
                                        [2 * v for v in b], [2 * v for v in a])
    back = S.unpack_chunks(recv2.numpy().view(np.complex128), nx, kzp, p)
    res["forward_ok"] = bool(np.array_equal(back, H[x0:x0 + nx]))
    # the reductions: every rank's sums add to the same global sums
    sums = torch.tensor([float(rank + 1), 2.0 * rank], dtype=torch.float64)
    torch.distributed.all_reduce(sums)
    res["sums"] = sums.tolist()
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as fh:
        json.dump(res, fh)


@pytest.mark.parametrize("world,nkx,N2,kzp", [(2, 7, 5, 8), (3, 11, 8, 16)])
def test_gloo_ranks_exchange(tmp_path, world, nkx, N2, kzp):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), nkx, N2, kzp))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    want = [sum(r + 1 for r in range(world)), sum(2.0 * r for r in range(world))]
    for r in range(world):
        assert res[r]["inverse_ok"] and res[r]["forward_ok"], r
        assert res[r]["sums"] == want
