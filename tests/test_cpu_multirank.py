"""World-size-2 gloo run of the multi-rank bench plumbing on CPU: each rank
works on its own field (replicas, no data-path collective); the step time is
the max over ranks and the job rate counts every rank's field."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from cortado_b200 import fields
        from oracle import oracle as O
        x = fields.sinusoid((4, 64, 64), 2 + rank).reshape(-1).numpy()  # this rank's own field
        s = O.store_encode(x, 1e-3, threads=1)
        ms = 10.0 + 5.0 * rank
        worst = bench.max_over_ranks(ms, world, torch.device("cpu"))
        q.put((rank, worst, len(s), bench.job_gbs(x.nbytes, world, worst)))
    finally:
        torch.distributed.destroy_process_group()


def test_two_rank_replicas_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(r[1] == 15.0 for r in res)          # max over ranks
    assert res[0][2] != res[1][2]                   # independent fields
    assert res[0][3] == pytest.approx(2 * 4 * 64 * 64 * 4 * 1e-9 / 15e-3)
