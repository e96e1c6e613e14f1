"""The learned per-query schedule: MLP kernels against the CPU oracle (forward, gradients),
training, the query path's use of the network, and what the trained network gains over
the plain schedule on held-out queries of the 10M x 128 workload's distribution."""
import json

import numpy as np
import pytest

from hdgrid_b200 import datasets
from oracle import mlp_oracle as mo
from tests.helpers import build_gpu

pytestmark = pytest.mark.gpu
PROBES = (1, 2, 4, 8, 16, 32, 64, 128, 256)  # this index probes at most 256 of its 512 lists


def _index():
    import hdgrid_b200 as hg
    ws = datasets.config1(scale=0.02, n_queries=4)
    return hg.SuperGridIndex.from_text(ws["hdgrid_conf"], ws["filter_conf"])


def _xy(n, seed):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal((n, mo.F)) * 0.7).astype(np.float32)
    y = np.stack([rng.uniform(0, 8, n), rng.integers(0, 2, n)], axis=1).astype(np.float32)
    return x, y


def test_mlp_forward_matches_oracle(cuda):
    import torch
    idx = _index()
    idx.mlp_init(5)
    w = idx.mlp_weights()
    x, _ = _xy(257, 1)
    zg = idx.mlp_forward(torch.from_numpy(x).to(cuda)).cpu().numpy()
    zo, _ = mo.forward(w, x)
    # FP32 accumulation against float64: a BF16 rounding of a hidden unit can flip, which
    # moves an output by a fraction of a percent at most
    assert np.abs(zg - zo).max() <= 1e-2 * (1.0 + np.abs(zo).max()), np.abs(zg - zo).max()


def test_mlp_gradients_match_oracle(cuda):
    import torch
    idx = _index()
    idx.mlp_init(9)
    w = idx.mlp_weights()
    x, y = _xy(300, 2)
    g, loss = idx.mlp_gradients(torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda))
    lo, go = mo.loss_and_grad(w, x, y)
    assert abs(loss - lo) <= 1e-4 * abs(lo), (loss, lo)
    gg, oo = mo.split(g.cpu().numpy().astype(np.float64)), mo.split(go)
    for name, _ in mo.SHAPES:
        rel = np.linalg.norm(gg[name] - oo[name]) / max(np.linalg.norm(oo[name]), 1e-12)
        assert rel <= 5e-3, (name, rel)


def test_mlp_training_fits_a_rule(cuda):
    import torch
    idx = _index()
    rng = np.random.default_rng(3)
    x = rng.standard_normal((4096, mo.F)).astype(np.float32)
    y = np.stack([np.clip(4 + 1.5 * x[:, 0] - x[:, 1], 0, 8), (x[:, 2] + 0.5 * x[:, 3] > 0)], axis=1).astype(np.float32)
    xt, yt = torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda)
    idx.mlp_init(1)
    _, loss0 = idx.mlp_gradients(xt, yt)
    loss = idx.mlp_train(xt, yt, epochs=60, batch=256, lr=3e-3, seed=1)
    assert loss < 0.15 * loss0, (loss0, loss)
    z = idx.mlp_forward(xt).cpu().numpy()
    acc = np.mean((z[:, 1] > 0) == (y[:, 1] > 0.5))
    assert acc > 0.93, acc
    assert np.mean(np.abs(z[:, 0] - y[:, 0])) < 0.4


@pytest.fixture(scope="module")
def learned_setup():
    """A config4-distribution index (500k points) with a network trained on 6000 queries."""
    import torch
    import hdgrid_b200 as hg
    from hdgrid_b200 import learned as L
    dev = "cuda:0"
    ws = datasets.config4(scale=0.05, n_queries=8000, clusters=64, sub_clusters=8, n_list=64, sub_lists=256,
                          exps0=16, max_grids=65536)
    idx, base, labels = build_gpu(ws, dev)
    q = torch.from_numpy(ws["queries"]).to(dev)
    ql = torch.from_numpy(ws["query_labels"]).to(dev)
    ranges = torch.empty((q.shape[0], 8), device=dev)
    hg.recover_filters(ws["filter_conf"], ql, ranges)
    gd = torch.empty((q.shape[0], 100), device=dev)
    gi = torch.empty((q.shape[0], 100), dtype=torch.int64, device=dev)
    hg.bruteforce_knn(base, labels, q, ranges, 100, gd, gi)
    gt = gi.cpu().numpy().view(np.uint64)
    ks = ws["ks"].astype(np.uint32)
    tr, te = slice(0, 6000), slice(6000, 8000)
    btr = L.Batch(base, q[tr], ql[tr], ks[tr])
    bte = L.Batch(base, q[te], ql[te], ks[te])
    y, _ = L.label_queries(idx, btr, gt[tr], probes=PROBES)
    ftr = idx.query_features(btr.q, btr.ql, 100, k=btr.k)
    fte = idx.query_features(bte.q, bte.ql, 100, k=bte.k)
    loss = L.train(idx, ftr, y, epochs=80, batch=256, lr=2e-3, seed=1)
    return dict(idx=idx, base=base, btr=btr, bte=bte, gt_te=gt[te], fte=fte, y=y, loss=loss, ws=ws)


def test_learned_query_path_uses_the_network(cuda, learned_setup):
    import torch
    from hdgrid_b200 import learned as L
    s = learned_setup
    idx, b = s["idx"], s["bte"]
    p, f = L.predicted_settings(idx, s["fte"], 256)
    ids_explicit, _ = b.run(idx, n_probe=torch.from_numpy(p).to(cuda), schedule=torch.from_numpy(f).to(cuda))
    idx.set_param("learned", 1)
    try:
        ids_learned, _ = b.run(idx)
    finally:
        idx.set_param("learned", 0)
    assert np.array_equal(ids_explicit, ids_learned)


def _timed_qps(b, idx, reps=3, **kw):
    """Queries per second of the batch through hdg_query_ex, the fastest of reps device-timed
    runs after one warm-up run; also returns that run's ids."""
    import torch
    ids, _ = b.run(idx, **kw)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        idx.query_ex(b.qin, b.qout, k=b.k, **kw)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return b.q.shape[0] / (best / 1e3), ids


def test_learned_schedule_gains_over_plain(cuda, learned_setup):
    """Held-out queries: QPS of the learned schedule against the fastest plain setting at
    equal recall.  The plain side is every uniform probe count of both of the reference's
    schedules: the post-filter budget min(exps0 * k * beta, max_row_len) with its exact
    re-rank (Super-Grid-IVF_PQ.cu:1196-1236) and the pre-filter schedule of exps0 <= 1
    (:1246).  The learned recall must reach the best plain recall (or 0.95) within 0.005, and
    its QPS must be at least 1.5x that of the fastest plain setting whose recall is at least
    the learned recall."""
    from hdgrid_b200 import learned as L
    s = learned_setup
    idx, b, gt = s["idx"], s["bte"], s["gt_te"]
    exps0 = int(idx.params["exps0"])
    plain = []
    try:
        for sched, e0v in (("post-filter", exps0), ("pre-filter", 1)):
            idx.set_param("exps0", e0v)
            for p in PROBES:
                idx.set_param("sub_lists", p)
                qps, ids = _timed_qps(b, idx)
                plain.append({"schedule": sched, "sub_lists": p, "recall": L.micro_recall(ids, gt, b.ks), "qps": qps})
    finally:
        idx.set_param("exps0", exps0)
        idx.set_param("sub_lists", 256)
    idx.set_param("learned", 1)
    try:
        lqps, ids = _timed_qps(b, idx)
    finally:
        idx.set_param("learned", 0)
    lrec = L.micro_recall(ids, gt, b.ks)
    p, f = L.predicted_settings(idx, s["fte"], 256)
    cmp = L.compare_at_equal_recall(lrec, lqps, plain, target=0.95)
    print(json.dumps({"plain": plain, "learned": {"recall": lrec, "qps": lqps, "pre_flag_share": float(f.mean()),
                                                  "median_probe": float(np.median(p))},
                      "versus": cmp, "train_loss": s["loss"]}))
    best_plain = max(r["recall"] for r in plain)
    assert lrec >= min(0.95, best_plain) - 0.005, (lrec, best_plain)
    # the comparator: the fastest plain setting whose recall reaches the learned recall
    reach = [r for r in plain if r["recall"] >= lrec]
    if reach:
        assert lqps >= 1.5 * max(r["qps"] for r in reach), (lqps, reach)
