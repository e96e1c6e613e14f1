"""Seeded synthetic workloads with the shapes of the HDGrid benchmark configurations.

The reference is evaluated on HDF5 datasets (sift10m, cc_news, app_reviews) that are not
available here; these generators stand in for them with the stated shapes, sizes and value
distributions.  Seeds: base 1001, queries 1002, labels 1003, filters 1004.

* ``config1``  100k x 128 Gaussian mixture (64 components, sigma 0.3), one int label in
  [0, 1e6) stored as f32, shift filter +-30000 (about 6 % selectivity).
* ``config2``  1M x 384 L2-normalised mixture (1024 components); labels = timestamp uniform
  over [0, 3e7) (f32-rounded) and two ints in [0, 1e4); filters shift [604800, 0] / map
  over a 10-entry interval table / div 10.  The fixed 604800-wide window over a 3e7 span
  caps any query's selectivity at 2.02 %, so per-query selectivity is log-uniform in
  [0.1 %, 2 %] (the map interval and the div threshold set it).
* ``config3``  config2 with LUT_FP16=1, the BF16 coarse GEMM pruning the list ranking, exps0 4.
* ``config4``  10M x 128 mixture, 4 int labels in [0, 1e6), type-3 range filters
  (filter_dim = 2); per-query selectivity log-uniform in [0.01 %, 90 %] split evenly over
  1-4 random dims; k drawn from {10, 100}.
Every generator takes a ``scale`` so tests can run the same distributions at small sizes.
"""
from __future__ import annotations

import numpy as np

SEED_BASE, SEED_QUERY, SEED_LABEL, SEED_FILTER = 1001, 1002, 1003, 1004


def mixture(n: int, d: int, n_comp: int, seed: int, centers_seed: int = 7, sigma: float = 0.3,
            normalise: bool = False) -> np.ndarray:
    crng = np.random.default_rng(centers_seed)
    centers = crng.standard_normal((n_comp, d), dtype=np.float32)
    rng = np.random.default_rng(seed)
    comp = rng.integers(0, n_comp, size=n)
    x = rng.standard_normal((n, d), dtype=np.float32)
    x *= np.float32(sigma)
    x += centers[comp]
    if normalise:
        x /= np.linalg.norm(x, axis=1, keepdims=True).astype(np.float32)
    return np.ascontiguousarray(x, dtype=np.float32)


def hdgrid_conf(**kv) -> str:
    base = dict(topk=100, pq_dim=32, n_clusters=256, exps0=4, clusters=8, sub_clusters=8, max_grids=1000000,
                n_list=8, sub_lists=64, filter_dim=1, label_mask=0, is_split=0, n_split=1, break_down=0,
                enable_multi_gpu=0, mem_bound=5000000000, is_calc_mem_predictor_coeff=0, lowest_query_batch=125,
                data_width=1)
    base.update(kv)
    lines = [f"{k} = {v}" for k, v in base.items()]
    lines.append('path = "dataset/synthetic/"')
    return "\n".join(lines) + "\n"


def config1(scale: float = 1.0, n_queries: int = 1000, **conf):
    n = max(2000, int(100_000 * scale))
    base = mixture(n, 128, 64, SEED_BASE)
    queries = mixture(n_queries, 128, 64, SEED_QUERY)
    lrng = np.random.default_rng(SEED_LABEL)
    labels = lrng.integers(0, 1_000_000, size=(n, 1)).astype(np.float32)
    frng = np.random.default_rng(SEED_FILTER)
    qlabels = frng.integers(0, 1_000_000, size=(n_queries, 1)).astype(np.float32)
    filt = "l = 1\nfilter0:\n\ttype = 0\n\tshift_val = [30000, 30000]\n"
    c = dict(clusters=8, sub_clusters=8, pq_dim=32, max_grids=1_000_000, n_list=8, sub_lists=64, exps0=4, topk=100)
    c.update(conf)
    return dict(name="config1", base=base, labels=labels, queries=queries, query_labels=qlabels,
                hdgrid_conf=hdgrid_conf(**c), filter_conf=filt, k=int(c["topk"]))


# map filter: 10 interval entries over [0, 1e4), nested fractions of the range
MAP_FRACTIONS = [1.0, 0.75, 0.5, 0.35, 0.25, 0.18, 0.125, 0.09, 0.0625, 0.05]


def _map_table() -> list[int]:
    t = []
    for f in MAP_FRACTIONS:
        t += [0, int(round(f * 10_000)) - 1]
    return t


def config2(scale: float = 1.0, n_queries: int = 10_000, **conf):
    n = max(4000, int(1_000_000 * scale))
    comps = max(16, int(1024 * min(1.0, scale * 4)))
    base = mixture(n, 384, comps, SEED_BASE, normalise=True)
    queries = mixture(n_queries, 384, comps, SEED_QUERY, normalise=True)
    lrng = np.random.default_rng(SEED_LABEL)
    ts = lrng.integers(0, 30_000_000, size=n).astype(np.int64).astype(np.float32)
    a = lrng.integers(0, 10_000, size=n).astype(np.float32)
    b = lrng.integers(0, 10_000, size=n).astype(np.float32)
    labels = np.stack([ts, a, b], axis=1).astype(np.float32)
    frng = np.random.default_rng(SEED_FILTER)
    window = 604_800 / 30_000_000
    sel = np.exp(frng.uniform(np.log(0.001), np.log(0.02), size=n_queries))
    r = np.minimum(1.0, sel / window)
    fr = np.array(MAP_FRACTIONS)
    q_ts = frng.integers(604_800, 30_000_000, size=n_queries).astype(np.float32)
    q_map = np.empty(n_queries, np.float32)
    q_div = np.empty(n_queries, np.float32)
    for i in range(n_queries):
        ok = np.nonzero(fr >= r[i])[0]
        j = int(frng.choice(ok))
        q_map[i] = j + 1  # the reference indexes the table with label - 1
        keep = min(1.0, r[i] / fr[j])
        lo = int(np.floor((1.0 - keep) * 10_000))
        q_div[i] = lo * 10
    qlabels = np.stack([q_ts, q_map, q_div], axis=1).astype(np.float32)
    table = ", ".join(str(v) for v in _map_table())
    filt = ("l = 3\nfilter0:\n\ttype = 0\n\tshift_val = [604800, 0]\n"
            f"filter1:\n\ttype = 1\n\tinterval_map = [{table}]\n"
            "filter2:\n\ttype = 2\n\tdiv_value = [10]\n")
    # n_list / sub_lists / exps0: the recall@100 >= 0.95 operating point of the plain schedule
    # on this workload (selectivity <= 2 % spreads the filtered neighbours over every list);
    # max_grids 3e7: the 74 x 74 x 5477 grid, whose counts the compressed prefix rows hold
    c = dict(clusters=64, sub_clusters=8, pq_dim=96, max_grids=30_000_000, n_list=64, sub_lists=512, exps0=10,
             topk=100)
    c.update(conf)
    return dict(name="config2", base=base, labels=labels, queries=queries, query_labels=qlabels,
                hdgrid_conf=hdgrid_conf(**c), filter_conf=filt, k=int(c["topk"]), selectivity=sel)


def config3(scale: float = 1.0, n_queries: int = 10_000, **conf):
    """Precision variant of config2: BF16 tensor-core coarse GEMM over all C + C*S centroids
    (sub_lists below the list count, so the ranking is pruned by it), FP16 LUT summed in
    FP32, and an exact FP32 re-rank of exps0*k*beta candidates with exps0 = 4."""
    c = dict(lut_fp16=1, coarse_bf16=1, sub_lists=448, exps0=4)
    c.update(conf)
    ws = config2(scale=scale, n_queries=n_queries, **c)
    ws["name"] = "config3"
    return ws


def config4(scale: float = 1.0, n_queries: int = 100_000, query_seed: int = SEED_QUERY,
            filter_seed: int = SEED_FILTER, with_base: bool = True, **conf):
    """query_seed / filter_seed select an independent query stream of the same distribution
    (the learned schedule trains on one and is evaluated on the standard one);
    with_base=False skips the base set and its labels (None)."""
    n = max(8000, int(10_000_000 * scale))
    base = mixture(n, 128, 1024, SEED_BASE) if with_base else None
    queries = mixture(n_queries, 128, 1024, query_seed)
    lrng = np.random.default_rng(SEED_LABEL)
    labels = lrng.integers(0, 1_000_000, size=(n, 4)).astype(np.float32) if with_base else None
    frng = np.random.default_rng(filter_seed)
    sel = np.exp(frng.uniform(np.log(0.0001), np.log(0.9), size=n_queries))
    ql = np.zeros((n_queries, 8), np.float32)
    ql[:, 1::2] = 1_000_000
    for i in range(n_queries):
        j = int(frng.integers(1, 5))
        dims = frng.choice(4, size=j, replace=False)
        w = sel[i] ** (1.0 / j)
        for dd in dims:
            width = max(1, int(round(w * 1_000_000)))
            lo = int(frng.integers(0, 1_000_000 - width + 1))
            ql[i, 2 * dd] = lo
            ql[i, 2 * dd + 1] = lo + width - 1
    ks = frng.choice([10, 100], size=n_queries)
    filt = "l = 4\n" + "".join(f"filter{i}:\n\ttype = 3\n" for i in range(4))
    # n_list / sub_lists / exps0: where the plain schedule's recall stops rising on this
    # workload (0.72 at 64 lists; more lists add cost, not recall)
    c = dict(clusters=512, sub_clusters=8, pq_dim=32, max_grids=65536, n_list=64, sub_lists=64, exps0=32, topk=100,
             filter_dim=2)
    c.update(conf)
    return dict(name="config4", base=base, labels=labels, queries=queries, query_labels=ql,
                hdgrid_conf=hdgrid_conf(**c), filter_conf=filt, k=int(c["topk"]), selectivity=sel, ks=ks)


def config5(scale: float = 1.0, n_queries: int = 50_000, **conf):
    """The learned variant: config4's data and queries with the index set up for per-query
    probe counts up to 1024 lists (n_list 128 clusters of 8 lists) and exps0 32."""
    c = dict(n_list=128, sub_lists=1024, exps0=32)
    c.update(conf)
    ws = config4(scale=scale, n_queries=n_queries, **c)
    ws["name"] = "config5"
    return ws


def write_dataset_dir(ws: dict, path, neighbors=None) -> str:
    """Writes a workload in the reference's dataset-directory format (what src/read_hfs5.py
    produces and src/utils/io_utils.cu:3-28, 201-313 reads): `keys` and `dtypes`, one line per
    key, and per key the raw row-major array plus `<key>_size` (int32 rows, cols).  Keys:
    train_vec, train_label, test_vec, test_label and, when given, neighbors (int32, -1 for
    missing).  Also writes HDGrid.conf (PATH pointing here) and filter.conf; returns the
    HDGrid.conf path."""
    import os
    d = str(path).rstrip("/") + "/"
    os.makedirs(d, exist_ok=True)
    arrays = [("train_vec", ws["base"]), ("train_label", ws["labels"]), ("test_vec", ws["queries"]),
              ("test_label", ws["query_labels"])]
    if neighbors is not None:
        nb = np.asarray(neighbors)
        if nb.dtype == np.uint64:
            nb = np.where(nb == np.uint64(0xFFFFFFFFFFFFFFFF), -1, nb.astype(np.int64))
        arrays.append(("neighbors", nb.astype(np.int32)))
    for key, a in arrays:
        a = np.ascontiguousarray(a)
        a.tofile(d + key)
        np.array([a.shape[0], a.shape[1]], np.int32).tofile(d + key + "_size")
    with open(d + "keys", "w") as f:
        f.write("".join(k + "\n" for k, _ in arrays))
    with open(d + "dtypes", "w") as f:
        f.write("".join(str(np.asarray(a).dtype) + "\n" for _, a in arrays))
    conf = "\n".join(line for line in ws["hdgrid_conf"].splitlines() if not line.lower().startswith("path"))
    with open(d + "HDGrid.conf", "w") as f:
        f.write(conf + f'\npath = "{d}"\n')
    with open(d + "filter.conf", "w") as f:
        f.write(ws["filter_conf"])
    return d + "HDGrid.conf"


def recall(found_ids: np.ndarray, gt_ids: np.ndarray) -> float:
    """|result ∩ GT| / |valid GT| with UINT64_MAX (or -1) GT entries ignored
    (src/verification/verification.cuh:97-153 without its app_reviews_points side file)."""
    found = found_ids.astype(np.uint64)
    gt = gt_ids.astype(np.uint64)
    inv = np.uint64(0xFFFFFFFFFFFFFFFF)
    hits = total = 0
    for f, g in zip(found, gt):
        gs = set(int(x) for x in g if x != inv)
        total += len(gs)
        hits += len(gs.intersection(int(x) for x in set(f.tolist()) if x != inv))
    return hits / total if total else 1.0
