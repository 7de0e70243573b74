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
