"""Parity on the full-size indexes the benchmark runs, for a 1,000-query batch.

config2 (1M x 384, shift/map/div filters, post-filter schedule), config3 (the same data with the
BF16 tensor-core coarse pruning and the FP16 LUT) and config5 (10M x 128, range filters, the
learned per-query probe counts and schedules): the GPU index is built at full size, a
1,000-query batch of the workload's query distribution runs through the C ABI, and the oracle
runs the same batch on the same index file.  Integer stages are bit-exact (filter boxes, cell
boxes, Morton codes, per-list counts, probe lists, Morton ranges), recall@k is within 0.002 of
the oracle's and every returned distance is within 1e-4 relative of FP64.  The oracle counts
per list from the index's prefix counts here (the reference's own method; the direct count,
its independent check, runs at the smaller sizes of test_gpu_parity.py).
"""
import numpy as np
import pytest

from hdgrid_b200 import datasets
from tests.helpers import exact_l2_f64, fetch_trace, save_and_open_oracle

pytestmark = pytest.mark.gpu
INV = np.uint64(0xFFFFFFFFFFFFFFFF)
N_SUB = 1000


def _run(ws, cuda, learned=False):
    import torch
    import hdgrid_b200 as hg
    import oracle
    from hdgrid_b200 import learned as L
    from pathlib import Path
    idx = hg.SuperGridIndex.from_text(ws["hdgrid_conf"], ws["filter_conf"])
    base = torch.from_numpy(ws["base"]).to(cuda)
    labels = torch.from_numpy(ws["labels"]).to(cuda)
    idx.build(hg.build_input_t(base, labels))
    k = ws["k"]
    q = torch.from_numpy(ws["queries"][:N_SUB]).to(cuda)
    ql = torch.from_numpy(ws["query_labels"][:N_SUB]).to(cuda)
    dist = torch.empty((N_SUB, k), device=cuda)
    ids = torch.empty((N_SUB, k), dtype=torch.int64, device=cuda)
    qin, qout = hg.query_input_t(base, q, ql), hg.query_output_t(dist, ids)
    ks = ws.get("ks")
    ks_sub = None if ks is None else ks[:N_SUB].astype(np.uint32)
    if learned:
        w = Path(hg.__file__).resolve().parent / "learned_weights" / "config5.npy"
        idx.set_mlp_weights(np.load(w))
        idx.set_param("learned", 1)
    if ks_sub is not None:
        idx.query_ex(qin, qout, k=torch.from_numpy(ks_sub).to(cuda))
    else:
        idx.query(qin, qout)
    torch.cuda.synchronize()
    g_dist, g_ids = dist.cpu().numpy(), ids.cpu().numpy().view(np.uint64)
    tr = fetch_trace(idx, N_SUB)
    nprobe = sched = None
    if learned:
        nprobe = np.frombuffer(idx.debug_fetch("learned_nprobe").tobytes(), np.uint32)[:N_SUB].copy()
        sched = np.frombuffer(idx.debug_fetch("learned_schedule").tobytes(), np.uint8)[:N_SUB].copy()
    ora, _ = save_and_open_oracle(idx)
    o_dist, o_ids, otr = ora.query(ws["queries"][:N_SUB], ws["query_labels"][:N_SUB], ws["base"], k,
                                   qk=ks_sub, n_probe=nprobe, schedule=sched, prefix_counts=True)
    for name in ("box", "cells", "zrange", "list_counts", "probe_lists", "range_start", "range_len"):
        a, b = tr[name], otr[name]
        if a.dtype == np.float32:
            a, b = a.view(np.uint32), b.view(np.uint32)
        mism = np.argwhere(a != b)
        assert mism.size == 0, f"{name} differs at {mism[:5].tolist()}"
    spec = hg.parse_filter(ws["filter_conf"])
    fd = int(hg.parse_config(ws["hdgrid_conf"])["filter_dim"])
    ranges = oracle.recover_filters(spec, ws["query_labels"][:N_SUB], filter_dim=fd)
    _, gt = oracle.bruteforce_f64(ws["base"], ws["labels"], ws["queries"][:N_SUB], ranges, k)
    if ks_sub is not None:
        r_g, r_o = L.micro_recall(g_ids, gt, ks_sub), L.micro_recall(o_ids, gt, ks_sub)
    else:
        r_g, r_o = datasets.recall(g_ids, gt), datasets.recall(o_ids, gt)
    assert abs(r_g - r_o) <= 0.002, (r_g, r_o)
    ex = exact_l2_f64(ws["base"], ws["queries"][:N_SUB], g_ids)
    valid = g_ids != INV
    rel = np.abs(g_dist[valid] - ex[valid]) / np.maximum(ex[valid], 1e-12)
    assert rel.max() <= 1e-4, rel.max()
    return idx, r_g


def test_full_config2_postfilter(cuda):
    ws = datasets.config2(n_queries=N_SUB)
    _, r = _run(ws, cuda)
    assert r >= 0.9, r


def test_full_config3_precision(cuda):
    ws = datasets.config3(n_queries=N_SUB)
    _run(ws, cuda)


def test_full_config5_learned(cuda):
    ws = datasets.config5(n_queries=N_SUB)
    idx, _ = _run(ws, cuda, learned=True)
    st = idx.last_query_stats()
    assert st["n_cand_ref"] == st["n_cand_used"]
