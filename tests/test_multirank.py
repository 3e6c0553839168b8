"""The multi-rank host logic of bench.py, run as two gloo ranks on the CPU: requests are sharded
by rank with every request served exactly once, timings reduce to the maximum over ranks,
per-rank results are gathered in rank order, and the reference arm runs on rank 0 only."""

import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import datetime

    import torch
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    import bench
    res = {}
    res["shard"] = bench.shard(10, rank, world)
    res["max"] = bench.max_over_ranks([float(rank), 10.0 - rank], True, device="cpu")
    res["gather"] = bench.gather_all({"rank": rank, "vals": list(range(rank + 1))}, True)
    r, w, _ = bench.dist_info()
    res["dist_info"] = [r, w]
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as fh:
        json.dump(res, fh)


def test_two_gloo_ranks(tmp_path):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    served = sorted(i for r in res for i in r["shard"])
    assert served == list(range(10))
    assert set(res[0]["shard"]).isdisjoint(res[1]["shard"])
    for r in range(world):
        assert res[r]["max"] == [1.0, 10.0]
        assert res[r]["gather"] == [{"rank": 0, "vals": [0]}, {"rank": 1, "vals": [0, 1]}]
        assert res[r]["dist_info"] == [r, world]


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    args = bench.parse(["--impl", "reference", "--size", "8", "--steps", "1", "--warmup", "1"])
    bench.run_reference(args, 1, 2)          # rank 1 of 2: no work, no output
    assert capsys.readouterr().out == ""
    bench.run_reference(args, 0, 1)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "steps/s" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
