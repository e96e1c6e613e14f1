"""The search-engine binary: the reference's argv, dataset directory and result files.

    search-engine <algorithm> <HDGrid.conf> [filter.conf]

It reads the dataset directory named by HDGrid.conf's PATH, builds the index, answers every
test query, writes res/distances_0 (f32) and res/neighbors_0 (u64), topk per query, and
prints the recall against PATH/neighbors.
"""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from hdgrid_b200 import datasets
from tests.helpers import build_gpu, query_gpu

pytestmark = pytest.mark.gpu
BIN = Path(__file__).resolve().parents[1] / "hdgrid_b200" / "bin" / "search-engine"


def test_search_engine_cli_matches_api(cuda, tmp_path):
    import hdgrid_b200 as hg
    import oracle
    ws = datasets.config1(scale=0.05, n_queries=300, max_grids=100_000)
    spec = hg.parse_filter(ws["filter_conf"])
    ranges = oracle.recover_filters(spec, ws["query_labels"])
    _, gt = oracle.bruteforce_f64(ws["base"], ws["labels"], ws["queries"], ranges, ws["k"])
    conf = datasets.write_dataset_dir(ws, tmp_path / "data", neighbors=gt)
    run = subprocess.run([str(BIN), "Super-Grid", conf], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    assert "search finish" in run.stdout
    k = ws["k"]
    ids = np.fromfile(tmp_path / "res" / "neighbors_0", np.uint64).reshape(-1, k)
    dist = np.fromfile(tmp_path / "res" / "distances_0", np.float32).reshape(-1, k)
    assert ids.shape == (300, k) and dist.shape == (300, k)
    m = re.search(r"final recall: ([0-9.]+)", run.stdout)
    assert m, run.stdout
    printed = float(m.group(1))
    assert abs(printed - datasets.recall(ids, gt)) < 1e-5
    # the same query through the Python API on an index built from the same data
    idx, base, _ = build_gpu(ws, cuda)
    d2, i2 = query_gpu(idx, base, ws, k, cuda)
    same = np.mean([set(a.tolist()) == set(b.tolist()) for a, b in zip(ids, i2)])
    assert same >= 0.98, same
    assert abs(printed - datasets.recall(i2, gt)) <= 0.01
    # the explicit filter.conf argument and the default PATH/filter.conf agree
    run2 = subprocess.run([str(BIN), "super-grid", conf, str(tmp_path / "data" / "filter.conf")], cwd=tmp_path,
                          capture_output=True, text=True, timeout=300)
    assert run2.returncode == 0, run2.stderr


def test_search_engine_cli_rejects_other_index_types(cuda, tmp_path):
    ws = datasets.config1(scale=0.02, n_queries=8)
    conf = datasets.write_dataset_dir(ws, tmp_path / "data")
    run = subprocess.run([str(BIN), "cagra-post", conf], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert run.returncode != 0 and "search-engine:" in run.stderr


def test_merge_topk_matches_numpy(cuda):
    import torch
    import hdgrid_b200 as hg
    rng = np.random.default_rng(4)
    q, k, nb = 37, 20, 3
    dist = rng.integers(0, 50, size=(q, k * nb)).astype(np.float32)  # many ties
    ids = rng.integers(0, 1000, size=(q, k * nb)).astype(np.uint64)
    ids[:, 5] = np.uint64(0xFFFFFFFFFFFFFFFF)
    offsets = np.array([0, 1000, 2000], np.int64)
    od = torch.empty((q, k), device=cuda)
    oi = torch.empty((q, k), dtype=torch.int64, device=cuda)
    hg.merge_topk(torch.from_numpy(dist).to(cuda), torch.from_numpy(ids.view(np.int64)).to(cuda), k,
                  torch.from_numpy(offsets).to(cuda), od, oi)
    got_i = oi.cpu().numpy().view(np.uint64)
    got_d = od.cpu().numpy()
    inv = np.uint64(0xFFFFFFFFFFFFFFFF)
    for r in range(q):
        cand = []
        for j in range(k * nb):
            if ids[r, j] != inv:
                cand.append((float(dist[r, j]), int(ids[r, j]) + int(offsets[j // k])))
        cand.sort()
        want = cand[:k]
        assert [int(x) for x in got_i[r]] == [c[1] for c in want], r
        assert np.array_equal(got_d[r], np.array([c[0] for c in want], np.float32)), r


def test_search_engine_cli_data_batches(cuda, tmp_path):
    """MEM_BOUND below the base set's size: three data batches, each with its own index,
    merged on the GPU; the result equals merging the three indexes' own answers."""
    import torch
    import hdgrid_b200 as hg
    import oracle
    ws = datasets.config1(scale=0.05, n_queries=200, max_grids=100_000)
    n, d = ws["base"].shape
    per_row = d * 4 + 64
    ws3 = datasets.config1(scale=0.05, n_queries=200, max_grids=100_000, mem_bound=per_row * ((n + 2) // 3))
    spec = hg.parse_filter(ws["filter_conf"])
    ranges = oracle.recover_filters(spec, ws["query_labels"])
    _, gt = oracle.bruteforce_f64(ws["base"], ws["labels"], ws["queries"], ranges, ws["k"])
    conf = datasets.write_dataset_dir(ws3, tmp_path / "data", neighbors=gt)
    run = subprocess.run([str(BIN), "super-grid", conf], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    assert "3 data batches" in run.stdout, run.stdout
    k = ws["k"]
    ids = np.fromfile(tmp_path / "res" / "neighbors_0", np.uint64).reshape(-1, k)
    # the same three indexes through the Python API, merged on the host
    rows = (n + 2) // 3
    parts = []
    for b in range(3):
        sub = dict(ws3)
        sub["base"], sub["labels"] = ws["base"][b * rows:(b + 1) * rows], ws["labels"][b * rows:(b + 1) * rows]
        idx, base, _ = build_gpu(sub, cuda)
        dd, ii = query_gpu(idx, base, sub, k, cuda)
        ok = ii != np.uint64(0xFFFFFFFFFFFFFFFF)
        parts.append((dd, np.where(ok, ii + np.uint64(b * rows), ii)))
    same = 0
    for r in range(ids.shape[0]):
        cand = sorted((float(dd[r, j]), int(ii[r, j])) for dd, ii in parts for j in range(k)
                      if ii[r, j] != np.uint64(0xFFFFFFFFFFFFFFFF))[:k]
        same += set(c[1] for c in cand) == set(int(x) for x in ids[r] if x != np.uint64(0xFFFFFFFFFFFFFFFF))
    assert same / ids.shape[0] >= 0.98, same
    assert float(re.search(r"final recall: ([0-9.]+)", run.stdout).group(1)) > 0.5
