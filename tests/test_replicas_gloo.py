"""Multi-rank host logic of bench.py --gpus N, as two gloo ranks on the CPU."""

from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp

from tests.helpers import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, queue):
    import sys

    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from porerad_b200 import replicas

    replicas.init("gloo", timeout_s=60)
    replicas.barrier()
    t = replicas.max_over_ranks([10.0 * (rank + 1), 1.0 - rank])
    # per-rank results: equal lists agree on every rank; one differing entry fails on every rank
    same = replicas.all_equal([123456789012, 7, rank * 0])
    differ = replicas.all_equal([123456789012, 7 + rank, 0])
    import bench

    args = type("A", (), {"gpus": world, "steps": 1, "warmup": 0, "cpu_seconds": 0.1})()
    ref_line = bench.run_reference(args, bench.WORKLOADS["c1"]) if rank == 1 else None
    replicas.finalize()
    queue.put((rank, t, ref_line, same, differ))


def test_two_rank_max_and_rank0_only_reference():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict()
    for _ in range(world):
        rank, t, ref, same, differ = q.get(timeout=120)
        out[rank] = (t, ref, same, differ)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == [20.0, 1.0] and out[1][0] == [20.0, 1.0]
    assert out[1][1] is None  # ranks other than 0 run no reference work
    assert all(out[r][2] is True and out[r][3] is False for r in range(world))
