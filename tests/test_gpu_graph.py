"""CUDA-graph query path (QUERY_GRAPH=1) and the scan autotuner, against the plain path.

A replay enqueues the captured kernels with the budget computed on the device, so its
results must equal the plain path's bit for bit; a batch with more candidates than the
captured distance capacity must say so through hdg_query_status.
"""
import numpy as np
import pytest

from hdgrid_b200 import datasets
from tests.helpers import build_gpu

pytestmark = pytest.mark.gpu
INV = np.uint64(0xFFFFFFFFFFFFFFFF)


def _io(ws, base, k, device):
    import torch
    import hdgrid_b200 as hg
    q = torch.from_numpy(ws["queries"]).to(device)
    ql = torch.from_numpy(ws["query_labels"]).to(device)
    dist = torch.empty((q.shape[0], k), dtype=torch.float32, device=device)
    ids = torch.empty((q.shape[0], k), dtype=torch.int64, device=device)
    return q, ql, dist, ids, hg.query_input_t(base, q, ql), hg.query_output_t(dist, ids)


def test_graph_replay_equals_plain_path(cuda):
    import torch
    ws = datasets.config2(scale=0.01, n_queries=256, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000)
    k = ws["k"]
    idx, base, _ = build_gpu(ws, cuda)
    q, ql, dist, ids, qin, qout = _io(ws, base, k, cuda)
    idx.query(qin, qout)
    torch.cuda.synchronize()
    ref_d, ref_i = dist.clone(), ids.clone()
    # a second batch in the same buffers: reversed queries and labels
    q2, ql2 = torch.flip(q, [0]).contiguous(), torch.flip(ql, [0]).contiguous()
    q.copy_(q2), ql.copy_(ql2)
    idx.query(qin, qout)
    torch.cuda.synchronize()
    ref2_d, ref2_i = dist.clone(), ids.clone()

    idx.set_param("query_graph", 1)
    for rep in range(3):  # capture (plain results), then two replays
        q.copy_(q2 if rep % 2 == 0 else torch.flip(q2, [0]))
        ql.copy_(ql2 if rep % 2 == 0 else torch.flip(ql2, [0]))
        dist.fill_(-1.0)
        idx.query(qin, qout)
        idx.status()
        torch.cuda.synchronize()
        want_d, want_i = (ref2_d, ref2_i) if rep % 2 == 0 else (ref_d, ref_i)
        assert torch.equal(ids, want_i), rep
        assert torch.equal(dist.view(torch.int32), want_d.view(torch.int32)), rep
    st = idx.last_query_stats()
    assert st["queries"] == 256 and st["launches"] >= 6


def test_graph_capacity_cut_reports_oom(cuda):
    import torch
    import hdgrid_b200 as hg
    ws = datasets.config1(scale=0.03, n_queries=64, max_grids=50_000)
    k = ws["k"]
    idx, base, _ = build_gpu(ws, cuda)
    q, ql, dist, ids, qin, qout = _io(ws, base, k, cuda)
    good = ql.clone()
    ql.fill_(5e7)  # every box clamps to the last label cell: a handful of candidates
    idx.set_param("query_graph", 1)
    idx.query(qin, qout)  # plain run + capture, distance capacity twice this batch
    torch.cuda.synchronize()
    small = idx.last_query_stats()["coarse_total"]
    ql.copy_(good)
    idx.query(qin, qout)  # replay: far more candidates than captured for
    assert small < 1000
    with pytest.raises(hg.HDGError) as e:
        idx.status()
    assert e.value.status == 4  # HDG_ERR_OOM
    torch.cuda.synchronize()
    got = ids.cpu().numpy().view(np.uint64)
    d = dist.cpu().numpy()
    assert np.all(np.isinf(d[got == INV]))
    # the plain path on the same batch still answers every query
    idx.set_param("query_graph", 0)
    idx.query(qin, qout)
    torch.cuda.synchronize()
    assert (ids.cpu().numpy().view(np.uint64)[:, 0] != INV).mean() > 0.9


def test_autotune_keeps_results_and_picks_a_variant(cuda):
    import torch
    ws = datasets.config2(scale=0.01, n_queries=256, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000)
    k = ws["k"]
    idx, base, _ = build_gpu(ws, cuda)
    q, ql, dist, ids, qin, qout = _io(ws, base, k, cuda)
    idx.query(qin, qout)
    torch.cuda.synchronize()
    ref_d, ref_i = dist.clone(), ids.clone()
    choice = idx.autotune(qin, qout)
    assert choice["scan_cpt"] in (1, 2, 4)
    assert choice["scan_chunk"] in (8192, 16384, 32768, 65536)
    assert choice["scan_ms"] > 0
    # the scan order of a candidate depends on its position only, so every variant gives
    # the same distances bit for bit
    idx.query(qin, qout)
    torch.cuda.synchronize()
    assert torch.equal(ids, ref_i)
    assert torch.equal(dist.view(torch.int32), ref_d.view(torch.int32))


def test_concurrent_queries_on_two_streams(cuda):
    """Two host threads query one index on two streams at once: each stream has its own
    workspace, so every answer equals the one the same batch gets alone."""
    import threading
    import torch
    ws = datasets.config2(scale=0.01, n_queries=256, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000)
    k = ws["k"]
    idx, base, _ = build_gpu(ws, cuda)
    a = _io(ws, base, k, cuda)
    b = _io(ws, base, k, cuda)
    b[0].copy_(torch.flip(a[0], [0]))
    b[1].copy_(torch.flip(a[1], [0]))
    refs = []
    for io in (a, b):
        idx.query(io[4], io[5])
        torch.cuda.synchronize()
        refs.append((io[2].clone(), io[3].clone()))
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    errors = []

    def worker(io, st, ref):
        try:
            for _ in range(6):
                with torch.cuda.stream(st):
                    io[2].fill_(-1.0)
                idx.query(io[4], io[5], stream=st)
                st.synchronize()
                if not (torch.equal(io[3], ref[1]) and torch.equal(io[2].view(torch.int32), ref[0].view(torch.int32))):
                    errors.append("mismatch")
        except Exception as ex:  # reported below
            errors.append(repr(ex))

    threads = [threading.Thread(target=worker, args=(io, st, ref)) for io, st, ref in zip((a, b), streams, refs)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
