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
    # predicate inside the ADC scan: a post-filter query reads M code bytes per candidate, a
    # predicate-first one 4*l label bytes per candidate plus M code bytes per survivor
    sys.path.insert(0, str(ROOT))
    import bench
    got = bench.algorithmic_scan_bytes([1000, 2000, 0], [900, 10, 0], [False, True, True], M=32, l=4)
    assert got == (0.0, 1000 * 32 + (2000 * 16 + 10 * 32))


def test_algorithmic_scan_bytes_of_the_predicate_pass():
    import bench
    # the predicate pass reads the 4-byte packed label ranks of the 2000 checked candidates and
    # the labels of the 300 inside the rank box; the ADC scan reads the codes of the 10
    # survivors and of every candidate of the post-filter query
    got = bench.algorithmic_scan_bytes([1000, 2000], [900, 10], [False, True], M=32, l=4, read_q=[0, 300],
                                       chk_q=[0, 2000], cbytes=4)
    assert got == (2000 * 4 + 300 * 16, 1000 * 32 + 10 * 32)
    # no rank check (most candidates in the box): labels for all, no ranks
    got = bench.algorithmic_scan_bytes([2000], [10], [True], M=32, l=4, read_q=[2000], chk_q=[0], cbytes=4)
    assert got == (2000 * 16, 10 * 32)


def test_refine_algorithmic_bytes():
    import bench
    # query 0 post-filter: 5000 selected entries, each a 4-byte id lookup and 4 bytes of ranks,
    # labels (4*l) for the 40 whose ranks sat on the box's edge, 100 exact rows of 4*d; query 1
    # predicate-first: 300 entries, every one an exact row
    got = bench.refine_algorithmic_bytes([5000, 300], [False, True], [100, 300], [40, 0], l=4, d=128, rank_bytes=4)
    assert got == 5300 * 4 + 5000 * 4 + 40 * 16 + 400 * 512
    # without packed ranks the post-filter entries read no rank bytes
    got = bench.refine_algorithmic_bytes([5000], [False], [100], [5000], l=4, d=128, rank_bytes=0)
    assert got == 5000 * 4 + 5000 * 16 + 100 * 512
