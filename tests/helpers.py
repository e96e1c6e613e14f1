"""Shared helpers for the GPU parity tests: build an index on the GPU from a synthetic
workload, run the product query through the C ABI and the oracle on the same index file."""
from __future__ import annotations

import tempfile
from pathlib import Path

import numpy as np

TRACE_NAMES = ["box", "cells", "zrange", "list_counts", "probe_clusters", "probe_lists", "range_start", "range_len"]
TRACE_DTYPES = {"box": np.float32, "cells": np.int32, "zrange": np.uint64, "list_counts": np.uint32,
                "probe_clusters": np.uint32, "probe_lists": np.uint32, "range_start": np.uint32,
                "range_len": np.uint32}


class Run:
    pass


def build_gpu(ws: dict, device="cuda:0"):
    import torch
    import hdgrid_b200 as hg
    idx = hg.SuperGridIndex.from_text(ws["hdgrid_conf"], ws["filter_conf"])
    base = torch.from_numpy(ws["base"]).to(device)
    labels = torch.from_numpy(ws["labels"]).to(device)
    idx.build(hg.build_input_t(base, labels))
    torch.cuda.synchronize()
    return idx, base, labels


def query_gpu(idx, base, ws: dict, k: int, device="cuda:0"):
    import torch
    import hdgrid_b200 as hg
    q = torch.from_numpy(ws["queries"]).to(device)
    ql = torch.from_numpy(ws["query_labels"]).to(device)
    dist = torch.empty((q.shape[0], k), dtype=torch.float32, device=device)
    ids = torch.empty((q.shape[0], k), dtype=torch.int64, device=device)
    idx.query(hg.query_input_t(base, q, ql), hg.query_output_t(dist, ids))
    torch.cuda.synchronize()
    return dist.cpu().numpy(), ids.cpu().numpy().view(np.uint64)


def fetch_trace(idx, nq: int) -> dict:
    out = {}
    for n in TRACE_NAMES:
        raw = idx.debug_fetch(n)
        out[n] = raw.view(TRACE_DTYPES[n]).reshape(nq, -1)
    return out


def save_and_open_oracle(idx):
    import oracle
    d = tempfile.mkdtemp(prefix="hdg_")
    path = str(Path(d) / "index.hdg")
    idx.save(path)
    return oracle.OracleIndex(path), path


def exact_l2_f64(base: np.ndarray, queries: np.ndarray, ids: np.ndarray) -> np.ndarray:
    out = np.full(ids.shape, np.inf)
    inv = np.uint64(0xFFFFFFFFFFFFFFFF)
    for i in range(ids.shape[0]):
        ok = ids[i] != inv
        rows = base[ids[i][ok].astype(np.int64)].astype(np.float64)
        out[i, ok] = ((rows - queries[i].astype(np.float64)) ** 2).sum(1)
    return out
