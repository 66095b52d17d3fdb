"""The multi-GPU path of bench.py is N independent replicas: its host logic
(per-rank seeds, max over ranks, whole-job aggregate) run as two gloo ranks
on the CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, local_ms, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(local_ms[rank], dist, "cpu")
        out.put((rank, ms, bench.replica_seed(rank),
                 bench.aggregate_solves_per_s(world, 1024, ms)))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_slowest_time():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    local_ms = [7.5, 8.25]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, local_ms, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [8.25, 8.25]
    assert res[0][2] != res[1][2]  # independent replica batches
    assert res[0][3] == pytest.approx(2 * 1024 / 8.25e-3)
