"""Learned per-query schedule: labels from running the plain method, GPU training, evaluation.

Labelling follows the method itself: every training query is run through the index at each
probe count of ``PROBES`` under both schedules (0 = the index's own post-filter schedule,
Super-Grid-IVF_PQ.cu:1196-1236; 1 = predicate-first scan with an exact re-rank of exps0 * k,
the schedule of the reference's batch-split branch, :1165-1171), and is labelled with the
cheapest setting -- fewest bytes read by the scan and the re-rank -- whose recall@k against
the exact filtered kNN reaches ``target``; when none does, the setting with the best recall.
The MLP (48 -> 128 -> 128 -> 2, BF16, trained by the library's own kernels) regresses
log2(probe count) and classifies the schedule.  The plain schedule stays the fallback
(LEARNED=0) and, with the brute-force kNN, the yardstick of the learned schedule's recall.
"""
from __future__ import annotations

import numpy as np

PROBES = (1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024)
# index of b3[0] (the bias of the log2 probe-count output) in the parameter vector
B3_PROBE = 128 * 48 + 128 + 128 * 128 + 128 + 2 * 128
INV = np.uint64(0xFFFFFFFFFFFFFFFF)


def _hits(found: np.ndarray, gt: np.ndarray, ks: np.ndarray):
    """Per query: |found[:k] & gt[:k]| and |valid gt[:k]| (UINT64_MAX entries ignored; the
    ids of one result row are distinct)."""
    n, w = gt.shape
    col = np.arange(w)[None, :]
    hits = np.zeros(n, np.int64)
    tot = np.zeros(n, np.int64)
    for a in range(0, n, 2048):
        b = min(n, a + 2048)
        keep = col < ks[a:b, None].astype(np.int64)
        g = np.where(keep, gt[a:b], INV)
        f = np.where(keep[:, :found.shape[1]], found[a:b, :w], INV - np.uint64(1))
        valid = g != INV
        hits[a:b] = ((f[:, :, None] == g[:, None, :]) & valid[:, None, :]).any(2).sum(1)
        tot[a:b] = valid.sum(1)
    return hits, tot


def per_query_recall(found: np.ndarray, gt: np.ndarray, ks: np.ndarray) -> np.ndarray:
    """recall@k of each query (k from ks); 1.0 when the query has no valid ground truth."""
    h, t = _hits(found, gt, ks)
    return np.where(t > 0, h / np.maximum(t, 1), 1.0)


def micro_recall(found, gt, ks) -> float:
    """sum of hits / sum of valid ground-truth ids (the reference's recall denominator)."""
    h, t = _hits(found, gt, ks)
    return float(h.sum() / t.sum()) if t.sum() else 1.0


class Batch:
    """Device-resident query batch plus the output buffers of width k_max."""

    def __init__(self, base, queries, query_labels, ks, k_max=100):
        import torch
        import hdgrid_b200 as hg
        dev = base.device
        self.q = torch.as_tensor(queries, device=dev).contiguous()
        self.ql = torch.as_tensor(query_labels, device=dev).contiguous()
        self.ks = np.asarray(ks, dtype=np.uint32)
        self.k = torch.from_numpy(self.ks).to(dev)
        self.k_max = k_max
        self.dist = torch.empty((self.q.shape[0], k_max), dtype=torch.float32, device=dev)
        self.ids = torch.empty((self.q.shape[0], k_max), dtype=torch.int64, device=dev)
        self.qin = hg.query_input_t(base, self.q, self.ql)
        self.qout = hg.query_output_t(self.dist, self.ids)

    def run(self, idx, n_probe=None, schedule=None):
        """Query through hdg_query_ex; returns (ids [q x k_max] u64, per-query work): the
        work dict holds, per query, the scanned candidates ``cand``, the candidates with a
        finite ADC distance ``nfin`` (the predicate survivors of a predicate-first query), the
        selection handed to the re-rank ``sel`` and the rows re-ranked exactly ``rows``."""
        import torch
        idx.query_ex(self.qin, self.qout, k=self.k, n_probe=n_probe, schedule=schedule)
        torch.cuda.synchronize()
        n = self.q.shape[0]

        def u32(name):
            return np.frombuffer(idx.debug_fetch(name).tobytes(), np.uint32)[:n].astype(np.int64)
        work = {"cand": np.frombuffer(idx.debug_fetch("qstat").tobytes(), np.uint32).reshape(-1, 4)[:n, 0]
                .astype(np.int64), "nfin": u32("nfin"), "sel": u32("cand_count"), "rows": u32("refine_rows")}
        return self.ids.cpu().numpy().view(np.uint64).copy(), work


def query_bytes(work: dict, schedule, m: int, l: int, d: int) -> np.ndarray:
    """Bytes a query reads per schedule (0 = post-filter, 1 = predicate-first), per query:
    the scan (M code bytes per candidate; predicate-first: 4*l label bytes per candidate and M
    per predicate survivor), the post-filter predicate on the selection (4*l per selected
    candidate) and the exact re-rank (4*d per row)."""
    sch = np.broadcast_to(np.asarray(schedule), work["cand"].shape).astype(bool)
    cand = work["cand"].astype(np.float64)
    scan = np.where(sch, cand * (4 * l) + work["nfin"] * m, cand * m)
    refine = np.where(sch, 0.0, work["sel"] * (4.0 * l)) + work["rows"] * (4.0 * d)
    return scan + refine


def scan_bytes(cand: np.ndarray, schedule: int, m: int, l: int) -> np.ndarray:
    """Bytes the ADC scan reads: M code bytes per candidate, plus 4*l label bytes when the
    predicate runs inside the scan."""
    return cand.astype(np.float64) * (m + (4 * l if schedule else 0))


def label_queries(idx, batch: Batch, gt: np.ndarray, probes=PROBES, target: float = 0.95, schedules=(0, 1)):
    """Per-query labels y [q x 2] = (log2 probe count, schedule) and the recall / cost tables."""
    import torch
    info = idx.info()
    m, l, d = info["M"], info["l"], info["d"]
    nq = batch.q.shape[0]
    dev = batch.q.device
    rec = np.zeros((len(schedules), len(probes), nq))
    cost = np.zeros((len(schedules), len(probes), nq))
    hits = np.zeros((len(schedules), len(probes), nq), np.int64)
    tot = np.zeros(nq, np.int64)
    for si, s in enumerate(schedules):
        sch = torch.full((nq,), s, dtype=torch.uint8, device=dev)
        for pi, p in enumerate(probes):
            npb = torch.full((nq,), p, dtype=torch.uint32, device=dev)
            ids, work = batch.run(idx, n_probe=npb, schedule=sch)
            h, tot = _hits(ids, gt, batch.ks)
            hits[si, pi] = h
            rec[si, pi] = np.where(tot > 0, h / np.maximum(tot, 1), 1.0)
            cost[si, pi] = query_bytes(work, s, m, l, d)
    y = np.zeros((nq, 2), np.float32)
    chosen_hits = np.zeros(nq, np.int64)
    chosen_cost = np.zeros(nq)
    for i in range(nq):
        ok = rec[:, :, i] >= target
        if ok.any():
            c = np.where(ok, cost[:, :, i], np.inf)
            si, pi = np.unravel_index(np.argmin(c), c.shape)
        else:
            best = rec[:, :, i].max()
            c = np.where(rec[:, :, i] >= best - 1e-12, cost[:, :, i], np.inf)
            si, pi = np.unravel_index(np.argmin(c), c.shape)
        y[i, 0] = np.log2(probes[pi])
        y[i, 1] = schedules[si]
        chosen_hits[i] = hits[si, pi, i]
        chosen_cost[i] = cost[si, pi, i]
    # what a network reproducing every label exactly would reach
    return y, {"recall": rec, "cost": cost, "label_recall": float(chosen_hits.sum() / max(tot.sum(), 1)),
               "label_bytes": float(chosen_cost.sum()), "hits": int(chosen_hits.sum()), "total": int(tot.sum())}


def train(idx, feats, y, epochs=60, batch=512, lr=2e-3, seed=1, init=True) -> float:
    """Trains the index's MLP on (features, labels) with the library's GPU kernels."""
    import torch
    dev = feats.device
    yt = torch.as_tensor(y, dtype=torch.float32, device=dev).contiguous()
    if init:
        idx.mlp_init(seed)
    return idx.mlp_train(feats, yt, epochs=epochs, batch=batch, lr=lr, seed=seed)


def calibrate(idx, batch: Batch, gt: np.ndarray, target: float = 0.955, max_probe: int = 1024,
              steps=(0.0, 0.25, 0.5, 0.75, 1.0, 1.25, 1.5, 2.0, 2.5, 3.0)) -> dict:
    """Shifts the probe-count output by the smallest offset (log2 units) whose micro recall on
    a validation batch reaches ``target``, written into the output bias b3[0]; when none
    does, the smallest offset within 0.0005 of the best recall seen.  Returns the offset and
    the validation recall of each offset tried."""
    import torch
    w0 = idx.mlp_weights()
    feats = idx.query_features(batch.q, batch.ql, batch.k_max, k=batch.k)
    seen = {}
    chosen = None
    for off in steps:
        w = w0.copy()
        w[B3_PROBE] += off
        idx.set_mlp_weights(w)
        p, f = predicted_settings(idx, feats, max_probe)
        ids, _ = batch.run(idx, n_probe=torch.from_numpy(p).to(batch.q.device),
                           schedule=torch.from_numpy(f).to(batch.q.device))
        seen[off] = micro_recall(ids, gt, batch.ks)
        if seen[off] >= target:
            chosen = off
            break
    if chosen is None:  # out of reach: the cheapest offset within 0.0005 of the best recall
        best = max(seen.values())
        chosen = min(o for o, r in seen.items() if r >= best - 5e-4)
    w = w0.copy()
    w[B3_PROBE] += chosen
    idx.set_mlp_weights(w)
    return {"offset": chosen, "validation_recall": seen}


def predicted_settings(idx, feats, max_probe: int):
    """Per-query (probe count, schedule) the trained network gives, as the query path
    derives them (round(2^z0) clamped to [1, max_probe], z1 > 0)."""
    z = idx.mlp_forward(feats).cpu().numpy()
    p = np.clip(np.rint(np.exp2(np.clip(z[:, 0], 0, 20))), 1, max_probe).astype(np.uint32)
    return p, (z[:, 1] > 0).astype(np.uint8)


def compare_at_equal_recall(learned_recall: float, learned_qps: float, plain: list, target: float = 0.95) -> dict:
    """The learned schedule against the plain schedules at equal recall.  ``plain`` holds one
    dict per plain setting with its ``recall`` and ``qps``.  The bar is recall@k >= target and
    >= the learned recall; the fastest plain setting over the bar is the comparator.  When no
    plain setting reaches it, the comparator is the plain setting with the highest recall,
    which the learned schedule then also beats in recall."""
    bar = max(target, learned_recall) if learned_recall >= target else learned_recall
    ok = [p for p in plain if p["recall"] >= bar]
    if ok:
        best = max(ok, key=lambda p: p["qps"])
        basis = f"fastest plain setting with recall >= {bar:.4f}"
    else:
        best = max(plain, key=lambda p: (p["recall"], p["qps"]))
        basis = f"no plain setting reaches recall {bar:.4f}: the plain setting with the highest recall"
    return {"target_recall": target, "learned_recall": learned_recall, "learned_meets_target": learned_recall >= target,
            "learned_qps": learned_qps, "plain": best, "speedup": learned_qps / best["qps"], "basis": basis}
