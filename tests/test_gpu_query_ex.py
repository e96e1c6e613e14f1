"""hdg_query_ex: per-query k, probe count and schedule, against the oracle given the same
per-query arrays, and against hdg_query where the arrays are uniform.

Integer stages (probe lists, Morton candidate ranges) must be bit-identical per query;
results follow the parity bar of the uniform query (same id sets for >= 98 % of the
queries, distances within 1e-4 relative of FP64).
"""
import numpy as np
import pytest

from hdgrid_b200 import datasets
from tests.helpers import build_gpu, exact_l2_f64, fetch_trace, query_gpu, save_and_open_oracle

pytestmark = pytest.mark.gpu
INV = np.uint64(0xFFFFFFFFFFFFFFFF)


def _query_ex(idx, base, ws, k_max, qk=None, nprobe=None, sched=None, device="cuda:0"):
    import torch
    import hdgrid_b200 as hg
    q = torch.from_numpy(ws["queries"]).to(device)
    ql = torch.from_numpy(ws["query_labels"]).to(device)
    dist = torch.empty((q.shape[0], k_max), dtype=torch.float32, device=device)
    ids = torch.empty((q.shape[0], k_max), dtype=torch.int64, device=device)
    t = lambda a, dt: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(device, dt)
    idx.query_ex(hg.query_input_t(base, q, ql), hg.query_output_t(dist, ids), k=t(qk, torch.uint32),
                 n_probe=t(nprobe, torch.uint32), schedule=t(sched, torch.uint8))
    torch.cuda.synchronize()
    return dist.cpu().numpy(), ids.cpu().numpy().view(np.uint64)


def _compare(ws, idx, g_dist, g_ids, o_dist, o_ids, otr, qk, exps0):
    nq = ws["queries"].shape[0]
    tr = fetch_trace(idx, nq)
    for name in ("box", "cells", "zrange", "list_counts", "probe_lists", "range_start", "range_len"):
        a, b = tr[name], otr[name]
        if a.dtype == np.float32:
            a, b = a.view(np.uint32), b.view(np.uint32)
        mism = np.argwhere(a != b)
        assert mism.size == 0, f"{name} differs at {mism[:5].tolist()}"
    # slots past each query's own k are empty
    kk = np.arange(g_ids.shape[1])[None, :]
    past = kk >= qk[:, None]
    assert np.all(g_ids[past] == INV) and np.all(np.isinf(g_dist[past]))
    same = np.mean([set(a.tolist()) == set(b.tolist()) for a, b in zip(g_ids, o_ids)])
    assert same >= 0.98, same
    valid = g_ids != INV
    if exps0 > 1:
        ex = exact_l2_f64(ws["base"], ws["queries"], g_ids)
        rel = np.abs(g_dist[valid] - ex[valid]) / np.maximum(ex[valid], 1e-12)
        assert rel.max() <= 1e-4, rel.max()


def test_query_ex_uniform_arrays_equal_query(cuda):
    ws = datasets.config2(scale=0.01, n_queries=200, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000)
    k = ws["k"]
    idx, base, _ = build_gpu(ws, cuda)
    d0, i0 = query_gpu(idx, base, ws, k, cuda)
    nq = ws["queries"].shape[0]
    d1, i1 = _query_ex(idx, base, ws, k, qk=np.full(nq, k), nprobe=np.full(nq, 24), sched=np.zeros(nq),
                       device=cuda)
    assert np.array_equal(i0, i1) and np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
    d2, i2 = _query_ex(idx, base, ws, k, device=cuda)
    assert np.array_equal(i0, i2) and np.array_equal(d0.view(np.uint32), d2.view(np.uint32))


def test_query_ex_per_query_k_matches_uniform_rows(cuda):
    # the budget of a query depends on its own k only (beta is a batch sum of candidate
    # counts), so each row equals the row of a uniform query with that k
    ws = datasets.config2(scale=0.01, n_queries=240, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000)
    idx, base, _ = build_gpu(ws, cuda)
    nq = ws["queries"].shape[0]
    qk = np.where(np.random.default_rng(5).random(nq) < 0.5, 10, 100).astype(np.uint32)
    d, i = _query_ex(idx, base, ws, 100, qk=qk, device=cuda)
    d10, i10 = query_gpu(idx, base, ws, 10, cuda)
    d100, i100 = query_gpu(idx, base, ws, 100, cuda)
    for r in range(nq):
        if qk[r] == 10:
            assert np.array_equal(i[r, :10], i10[r]) and np.all(i[r, 10:] == INV), r
        else:
            assert np.array_equal(i[r], i100[r]), r


@pytest.mark.parametrize("workload", ["config2", "config4", "config1"])
def test_query_ex_matches_oracle(cuda, workload):
    if workload == "config2":
        ws = datasets.config2(scale=0.01, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                              max_grids=20_000)
    elif workload == "config4":
        ws = datasets.config4(scale=0.002, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                              max_grids=4096)
    else:
        ws = datasets.config1(scale=0.05, n_queries=200, max_grids=100_000, sub_lists=24)
    import hdgrid_b200 as hg
    idx, base, _ = build_gpu(ws, cuda)
    nq = ws["queries"].shape[0]
    rng = np.random.default_rng(11)
    k_max = 100
    qk = rng.choice([10, 37, 100], nq).astype(np.uint32)
    nprobe = rng.choice([1, 6, 24, 500], nq).astype(np.uint32)   # 500 clamps to sub_lists
    sched = (rng.random(nq) < 0.4).astype(np.uint8)
    g_dist, g_ids = _query_ex(idx, base, ws, k_max, qk=qk, nprobe=nprobe, sched=sched, device=cuda)
    ora, _ = save_and_open_oracle(idx)
    o_dist, o_ids, otr = ora.query(ws["queries"], ws["query_labels"], ws["base"], k_max, qk=qk, n_probe=nprobe,
                                   schedule=sched)
    exps0 = int(hg.parse_config(ws["hdgrid_conf"])["exps0"])
    _compare(ws, idx, g_dist, g_ids, o_dist, o_ids, otr, np.minimum(qk, k_max), exps0)
    # predicate-first queries return only points inside their label box
    spec = hg.parse_filter(ws["filter_conf"])
    fd = int(hg.parse_config(ws["hdgrid_conf"])["filter_dim"])
    import oracle
    ranges = oracle.recover_filters(spec, ws["query_labels"], filter_dim=fd)
    lab = ws["labels"]
    l = lab.shape[1]
    for r in np.nonzero(sched)[0]:
        got = g_ids[r][g_ids[r] != INV].astype(np.int64)
        box = ranges[r].reshape(l, 2)
        assert np.all((lab[got] >= box[:, 0]) & (lab[got] <= box[:, 1])), r


def test_query_ex_rejects_schedule_without_rerank(cuda):
    import torch
    import hdgrid_b200 as hg
    ws = datasets.config1(scale=0.03, n_queries=16, max_grids=50_000, exps0=1)
    idx, base, _ = build_gpu(ws, cuda)
    with pytest.raises(hg.HDGError) as e:
        _query_ex(idx, base, ws, 10, sched=np.ones(16), device=cuda)
    assert e.value.status == 1
    with pytest.raises(hg.HDGError) as e:  # wrong dtype for a per-query array
        q = torch.from_numpy(ws["queries"]).to(cuda)
        ql = torch.from_numpy(ws["query_labels"]).to(cuda)
        out = hg.query_output_t(torch.empty((16, 10), device=cuda), torch.empty((16, 10), dtype=torch.int64,
                                                                                 device=cuda))
        idx.query_ex(hg.query_input_t(base, q, ql), out, k=torch.ones(16, dtype=torch.int64, device=cuda))
    assert e.value.status == 1
