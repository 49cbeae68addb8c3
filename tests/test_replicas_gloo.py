"""Host logic of the multi-rank benchmark (replicas, one per GPU) on CPU ranks
over gloo: the job time is the max over ranks, the job throughput counts every
rank's DOF, and only rank 0 reports."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        mine = [10.0 + rank, 5.0 - rank, 7.0 * (rank + 1)]
        got = bench.rank_max(mine, ws, torch.device("cpu"))
        q.put((rank, got, bench.job_gdofs(1_000_000, ws, got[0] / 4)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2])
def test_rank_max_and_job_throughput(ws):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = dict((r, (g, v)) for r, g, v in (q.get(timeout=120) for _ in range(ws)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(ws):
        got, val = out[r]
        assert got == [10.0 + ws - 1, 5.0, 7.0 * ws]          # element-wise max over ranks
        assert val == pytest.approx(ws * 1e6 / ((10.0 + ws - 1) / 4 * 1e-3) / 1e9)
