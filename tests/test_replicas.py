"""The multi-GPU form of the benchmark is independent replicas, one per rank
(the loop does not shard): the only collective is the max over ranks of each
rank's timed region, and the reference arm runs on rank 0 alone.  Checked
here with world size 2 on the gloo backend, on the CPU."""
import os
import sys
import types
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        w, r, loc = bench.dist_setup()
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, w, device="cpu")
        ref = bench.run_reference(types.SimpleNamespace(workload="c2", steps=1, warmup=0), w, r) if r else None
        dist.barrier()
        q.put((rank, w, r, loc, slowest, ref))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time():
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[:4] for g in got] == [(0, 2, 0, 0), (1, 2, 1, 1)]
    assert all(g[4] == 15.0 for g in got)      # both ranks report the slower replica's time
    assert got[1][5] is None                   # the reference arm does no work off rank 0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
