"""Multi-process host logic of bench.py's replica mode on CPU (gloo,
world_size 2): every rank times its own channel and rank 0 reports the max
over ranks; the reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    import bench
    w, r, _ = bench.dist_setup()
    assert (w, r) == (ws, rank)
    t = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out[rank] = float(t.item())
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ws = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(ws, port, out), nprocs=ws, join=True)
    assert out[0] == out[1] == 11.0


def test_reference_arm_only_on_rank0(capsys):
    import argparse

    import bench
    args = argparse.Namespace(steps=1, warmup=0, workload="tg_64x64x64")
    rc = bench.run_reference(args, bench.WORKLOADS["tg_64x64x64"], 2, 1)
    assert rc == 0
    assert capsys.readouterr().out == ""


def test_batch64_channel_split_covers_and_balances():
    """bench.py splits the 64 channels across ranks (no data-path
    collective): every channel on exactly one rank, shares within 5 % of
    each other at 2, 4 and 8 ranks."""
    import bench
    from chapsim1ww_b200 import batch64_configs
    cells = [c["nx"] * c["ny"] * c["nz"] for c in batch64_configs(seed=3)]
    for ws in (1, 2, 4, 8):
        parts = [bench.shard_channels(cells, ws, r) for r in range(ws)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64)), ws
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) <= 1.05 * min(loads), (ws, loads)


def _batch_split_worker(rank, ws, port, out):
    """Each gloo rank computes its own share; the shares gathered over the
    process group partition the channel list."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    import bench
    from chapsim1ww_b200 import batch64_configs
    cells = [c["nx"] * c["ny"] * c["nz"] for c in batch64_configs(seed=3)]
    w, r, _ = bench.dist_setup()
    mine = bench.shard_channels(cells, w, r)
    got = [None] * ws
    dist.all_gather_object(got, mine)
    out[rank] = got
    dist.barrier()
    dist.destroy_process_group()


def test_batch64_channel_split_gloo():
    ws = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_batch_split_worker, args=(ws, port, out), nprocs=ws, join=True)
    assert out[0] == out[1]
    assert sorted(out[0][0] + out[0][1]) == list(range(64))
    assert not set(out[0][0]) & set(out[0][1])


def test_reference_arm_reports_what_it_ran(capsys):
    """The reference arm times exactly the requested warm-up and timed steps
    (of a bounded z-slab sample) and prints the same config block as the GPU
    arm."""
    import argparse
    import json

    import bench
    args = argparse.Namespace(steps=2, warmup=1, workload="tg_64x64x64", precision="fp64", ref_budget=1.0)
    wl = bench.WORKLOADS["tg_64x64x64"]
    assert bench.run_reference(args, wl, 1, 0) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["config"] == bench.workload_config(args, wl)
    assert "1 warm-up + 2 timed" in line["cpu_baseline"]["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0
