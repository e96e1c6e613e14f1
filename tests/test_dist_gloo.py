"""bench.py's host logic on CPU: the multi-process plumbing on gloo ranks (world size 2:
barrier, max-over-ranks timing, the whole-job value of the replicas-only path) and the
scan's algorithmic byte count behind the roofline."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        # rank r "took" 10 * (r + 1) ms: the job time is the slowest rank's
        total = bench.max_over_ranks(10.0 * (rank + 1), world, device="cpu")
        value = bench.replica_value(world, 1000, 5, total)
        bench.barrier(world)
        out.put((rank, total, value))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_timing_and_replica_value():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, total, value in res:
        assert total == 20.0
        assert value == pytest.approx(2 * 1000 * 5 / 0.020)


def test_algorithmic_scan_bytes():
    # post-filter query: M code bytes per candidate; predicate-first: 4*l label bytes per
    # candidate plus M code bytes per survivor
    sys.path.insert(0, str(ROOT))
    import bench
    got = bench.algorithmic_scan_bytes([1000, 2000, 0], [900, 10, 0], [False, True, True], M=32, l=4)
    assert got == 1000 * 32 + (2000 * 16 + 10 * 32)


def test_algorithmic_scan_bytes_with_morton_precheck():
    import bench
    # predicate-first query: 8 bytes of Morton code per candidate, labels only for the 300
    # candidates inside the cell box, codes for the 10 survivors; post-filter unchanged
    got = bench.algorithmic_scan_bytes([1000, 2000], [900, 10], [False, True], M=32, l=4, zin_q=[0, 300])
    assert got == 1000 * 32 + (2000 * 8 + 300 * 16 + 10 * 32)
