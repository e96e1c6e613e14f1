"""Train the learned per-query schedule for the 10M x 128 workload and evaluate it.

    python -m hdgrid_b200.train_learned [--scale 1.0] [--train 200000] [--heldout 50000]
        [--out hdgrid_b200/learned_weights/config5.npy]

Builds the config5 index (config4's data: 10M x 128, 4 label dims, range filters), labels
``--train`` queries of an independent query stream (query seed 2002, filter seed 2004) by
running the plain method at every probe count under both schedules, trains the BF16 MLP
on the GPU, calibrates the probe-count output on ``--val`` further queries of that stream
(the smallest log2 offset reaching recall 0.955), and evaluates on ``--heldout`` queries of
the standard stream: recall@k against the exact filtered kNN, bytes scanned and device
time, for the plain schedule at every uniform probe count and for the learned schedule.
Writes the weights (.npy, f32) and a JSON report next to them.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np


def _gt(hg, base, labels, q, ql, filter_conf, k, step=10_000):
    import torch
    out = np.empty((q.shape[0], k), np.uint64)
    for a in range(0, q.shape[0], step):
        b = min(q.shape[0], a + step)
        rng = torch.empty((b - a, 2 * labels.shape[1]), device=base.device)
        hg.recover_filters(filter_conf, ql[a:b].contiguous(), rng)
        gd = torch.empty((b - a, k), device=base.device)
        gi = torch.empty((b - a, k), dtype=torch.int64, device=base.device)
        hg.bruteforce_knn(base, labels, q[a:b].contiguous(), rng, k, gd, gi)
        out[a:b] = gi.cpu().numpy().view(np.uint64)
    return out


def main():
    import torch
    import hdgrid_b200 as hg
    from hdgrid_b200 import datasets
    from hdgrid_b200 import learned as L
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--train", type=int, default=200_000)
    ap.add_argument("--heldout", type=int, default=50_000)
    ap.add_argument("--val", type=int, default=10_000)
    ap.add_argument("--target", type=float, default=0.98, help="per-query recall a label must reach")
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--exps0", type=int, default=0, help="refine ratio of the index (0 = config5's)")
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--step", type=int, default=10_000, help="queries per labelling / evaluation batch")
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "learned_weights" / "config5.npy"))
    args = ap.parse_args()
    dev = torch.device("cuda:0")
    t0 = time.time()
    ev = datasets.config5(scale=args.scale, n_queries=args.heldout, break_down=0,
                          **({"exps0": args.exps0} if args.exps0 else {}))
    tr = datasets.config4(scale=args.scale, n_queries=args.train + args.val, query_seed=2002, filter_seed=2004,
                          with_base=False)
    idx = hg.SuperGridIndex.from_text(ev["hdgrid_conf"], ev["filter_conf"])
    base = torch.from_numpy(ev["base"]).to(dev)
    labels = torch.from_numpy(ev["labels"]).to(dev)
    idx.build(hg.build_input_t(base, labels))
    torch.cuda.synchronize()
    log = {"build_s": round(time.time() - t0, 1)}
    print(json.dumps(log), flush=True)

    qtr = torch.from_numpy(tr["queries"]).to(dev)
    qltr = torch.from_numpy(tr["query_labels"]).to(dev)
    kstr = tr["ks"].astype(np.uint32)
    t1 = time.time()
    gt_tr = _gt(hg, base, labels, qtr, qltr, ev["filter_conf"], 100)
    log["gt_train_s"] = round(time.time() - t1, 1)
    ys, feats = [], []
    t1 = time.time()
    hits = tot = 0
    for a in range(0, args.train, args.step):
        b = min(args.train, a + args.step)
        batch = L.Batch(base, qtr[a:b], qltr[a:b], kstr[a:b])
        y, inf = L.label_queries(idx, batch, gt_tr[a:b], target=args.target)
        hits += inf["hits"]
        tot += inf["total"]
        ys.append(y)
        feats.append(idx.query_features(batch.q, batch.ql, 100, k=batch.k))
    y = np.concatenate(ys)
    f = torch.cat(feats).contiguous()
    log["label_s"] = round(time.time() - t1, 1)
    log["label_pre_share"] = float(y[:, 1].mean())
    log["label_probe_hist"] = np.bincount(y[:, 0].astype(int), minlength=len(L.PROBES)).tolist()
    log["label_recall_bound"] = hits / max(tot, 1)
    t1 = time.time()
    loss = L.train(idx, f, y, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=1)
    log["train_s"] = round(time.time() - t1, 1)
    log["train_loss"] = loss
    vb = L.Batch(base, qtr[args.train:], qltr[args.train:], kstr[args.train:])
    log["calibration"] = L.calibrate(idx, vb, gt_tr[args.train:], max_probe=max(L.PROBES))
    print(json.dumps(log), flush=True)

    # held-out evaluation: the plain schedules (no network) at every uniform probe count --
    # the post-filter budget with its exact re-rank, and the pre-filter schedule (exps0 = 1)
    # -- and the learned schedule, each device-timed
    qev = torch.from_numpy(ev["queries"]).to(dev)
    qlev = torch.from_numpy(ev["query_labels"]).to(dev)
    ksev = ev["ks"].astype(np.uint32)
    gt_ev = _gt(hg, base, labels, qev, qlev, ev["filter_conf"], 100)
    info = idx.info()
    m, l, d = info["M"], info["l"], info["d"]
    exps0 = int(idx.params["exps0"])
    scheds = (("post-filter", exps0), ("pre-filter", 1))
    plain = {(sname, p): [0, 0, 0.0, 0.0] for sname, _ in scheds for p in L.PROBES}
    learned = [0, 0, 0.0, 0.0]

    def timed(batch, **kw):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.run(idx, **kw)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    for a in range(0, qev.shape[0], args.step):
        b = min(qev.shape[0], a + args.step)
        batch = L.Batch(base, qev[a:b], qlev[a:b], ksev[a:b])
        for sname, e0v in scheds:
            idx.set_param("exps0", e0v)
            for p in L.PROBES:
                idx.set_param("sub_lists", p)
                ids, work = batch.run(idx)
                if e0v <= 1:  # no re-rank in the pre-filter schedule
                    work = dict(work, sel=np.zeros_like(work["sel"]), rows=np.zeros_like(work["rows"]))
                h, t = L._hits(ids, gt_ev[a:b], batch.ks)
                v = plain[(sname, p)]
                v[0] += int(h.sum())
                v[1] += int(t.sum())
                v[2] += float(L.query_bytes(work, 1 if e0v <= 1 else 0, m, l, d).sum())
                v[3] += timed(batch)
        idx.set_param("exps0", exps0)
        idx.set_param("sub_lists", max(L.PROBES))
        fe = idx.query_features(batch.q, batch.ql, 100, k=batch.k)
        pp, ff = L.predicted_settings(idx, fe, max(L.PROBES))
        idx.set_param("learned", 1)
        ids, work = batch.run(idx)
        learned[3] += timed(batch)
        idx.set_param("learned", 0)
        h, t = L._hits(ids, gt_ev[a:b], batch.ks)
        learned[0] += int(h.sum())
        learned[1] += int(t.sum())
        learned[2] += float(L.query_bytes(work, ff, m, l, d).sum())
    n = qev.shape[0]
    plain_rows = [{"schedule": sname, "sub_lists": p, "recall": v[0] / max(v[1], 1), "bytes": v[2],
                   "qps": n / (v[3] / 1e3)} for (sname, p), v in plain.items()]
    lrow = {"recall": learned[0] / max(learned[1], 1), "bytes": learned[2], "qps": n / (learned[3] / 1e3)}
    report = dict(log, heldout=args.heldout, train=args.train, plain=plain_rows, learned=lrow,
                  learned_vs_plain=L.compare_at_equal_recall(lrow["recall"], lrow["qps"], plain_rows))
    out = Path(args.out)
    out.parent.mkdir(parents=True, exist_ok=True)
    np.save(out, idx.mlp_weights())
    out.with_name(out.stem + "_report.json").write_text(json.dumps(report, indent=1))
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
