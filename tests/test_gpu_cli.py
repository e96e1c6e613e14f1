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
