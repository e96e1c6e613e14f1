"""GPU path (libhdgrid through the C ABI) against the CPU oracle on the same index.

Integer stages -- filter boxes, cell boxes, Morton codes, per-list counts, probe lists,
Morton candidate ranges, pool layout -- must be bit-identical.  Final results: distances
within 1e-4 relative of FP64, recall within 0.002 of the oracle's own search.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from hdgrid_b200 import datasets
from tests.helpers import build_gpu, exact_l2_f64, fetch_trace, query_gpu, save_and_open_oracle

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())
pytestmark = pytest.mark.gpu
INV = np.uint64(0xFFFFFFFFFFFFFFFF)


def _t(a, dev, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.to(dev) if dtype is None else t.to(dev, dtype)


# ---- the reference's known-answer vectors through the GPU kernels ------------------------

def test_gpu_pq_lut_kat(cuda):
    import torch
    import hdgrid_b200 as hg
    k = KATS["pq_lut"]
    c = _t(np.array(k["centers"], np.float32), cuda)
    q = _t(np.array(k["queries"], np.float32).reshape(k["n_queries"], -1), cuda)
    out = torch.empty(k["n_queries"] * k["pq_dim"] * k["n_codes"], device=cuda)
    hg.pq_lut(c, q, k["pq_dim"], k["pq_len"], k["n_codes"], out)
    np.testing.assert_allclose(out.cpu().numpy(), k["expected"], atol=k["tolerance"], rtol=0)


def test_gpu_pq_adc_kat(cuda):
    import torch
    import hdgrid_b200 as hg
    k = KATS["pq_adc"]
    cb = _t(np.array(k["codebook_colmajor"], np.uint8), cuda)
    lut = _t(np.array(k["lut"], np.float32), cuda)
    out = torch.empty(k["n_queries"] * k["n_data"], device=cuda)
    hg.pq_adc(cb, k["n_data"], lut, k["n_queries"], k["pq_dim"], k["n_codes"], None, k["n_data"], out)
    np.testing.assert_allclose(out.cpu().numpy(), k["expected"], atol=k["tolerance"], rtol=0)


def test_gpu_label_predicate_kat(cuda):
    import torch
    import hdgrid_b200 as hg
    k = KATS["label_predicate"]
    nq, nc, l = k["n_queries"], k["n_candi"], k["l"]
    rng = _t(np.array(k["constraints"], np.float32), cuda)
    lab = _t(np.array(k["candidate_labels"], np.float32), cuda)
    idx = _t(np.arange(nq * nc, dtype=np.int64), cuda)
    out = torch.empty(nq * nc, dtype=torch.int32, device=cuda)
    hg.label_mask(rng, lab, l, nq * nc, nq, idx, nc, out)
    assert out.cpu().tolist() == k["expected_kept"]


def test_gpu_recover_filters_bit_exact(cuda):
    import torch
    import hdgrid_b200 as hg
    import oracle
    ws = datasets.config2(scale=0.005, n_queries=300)
    ql = _t(ws["query_labels"], cuda)
    out = torch.empty((300, 6), device=cuda)
    hg.recover_filters(ws["filter_conf"], ql, out)
    spec = hg.parse_filter(ws["filter_conf"])
    ref = oracle.recover_filters(spec, ws["query_labels"])
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_gpu_bruteforce_matches_fp64_oracle(cuda):
    import torch
    import hdgrid_b200 as hg
    import oracle
    ws = datasets.config1(scale=0.05, n_queries=64)
    spec = hg.parse_filter(ws["filter_conf"])
    ranges = oracle.recover_filters(spec, ws["query_labels"])
    d64, i64 = oracle.bruteforce_f64(ws["base"], ws["labels"], ws["queries"], ranges, 50)
    dist = torch.empty((64, 50), device=cuda)
    ids = torch.empty((64, 50), dtype=torch.int64, device=cuda)
    hg.bruteforce_knn(_t(ws["base"], cuda), _t(ws["labels"], cuda), _t(ws["queries"], cuda), _t(ranges, cuda), 50,
                      dist, ids)
    gi = ids.cpu().numpy().view(np.uint64)
    assert datasets.recall(gi, i64) >= 0.999
    ok = np.isfinite(d64)
    np.testing.assert_allclose(dist.cpu().numpy()[ok], d64[ok], rtol=1e-4, atol=1e-5)


# ---- end-to-end parity on the GPU-built index --------------------------------------------

def _parity(ws, cuda, min_recall=None, exact_ids=False, adc_rotated=False, layout=True):
    import hdgrid_b200 as hg
    import oracle
    k = ws["k"]
    idx, base, labels = build_gpu(ws, cuda)
    g_dist, g_ids = query_gpu(idx, base, ws, k, cuda)
    nq = ws["queries"].shape[0]
    tr = fetch_trace(idx, nq)
    ora, path = save_and_open_oracle(idx)
    # (the layout check recounts a dense [cells x lists] prefix table: small grids only)
    if layout:
        assert ora.check_layout() == 0, "pool layout / Morton codes / prefix counts differ from the labels"
    o_dist, o_ids, otr = ora.query(ws["queries"], ws["query_labels"], ws["base"], k, adc_rotated=adc_rotated)
    for name in ("box", "cells", "zrange", "list_counts", "probe_clusters", "probe_lists", "range_start",
                 "range_len"):
        a, b = tr[name], otr[name]
        assert a.shape == b.shape, name
        if name == "probe_clusters":  # the chosen set is what the schedule defines
            a, b = np.sort(a, axis=1), np.sort(b, axis=1)
        if a.dtype == np.float32:
            a, b = a.view(np.uint32), b.view(np.uint32)
        mism = np.argwhere(a != b)
        assert mism.size == 0, f"{name} differs at {mism[:5].tolist()}"
    # ground truth: FP64 filtered brute force with the f32 predicate
    spec = hg.parse_filter(ws["filter_conf"])
    fd = int(hg.parse_config(ws["hdgrid_conf"])["filter_dim"])
    ranges = oracle.recover_filters(spec, ws["query_labels"], filter_dim=fd)
    _, gt = oracle.bruteforce_f64(ws["base"], ws["labels"], ws["queries"], ranges, k)
    r_gpu, r_ora = datasets.recall(g_ids, gt), datasets.recall(o_ids, gt)
    assert abs(r_gpu - r_ora) <= 0.002, (r_gpu, r_ora)
    if min_recall is not None:
        assert r_gpu >= min_recall, r_gpu
    same = np.mean([set(a.tolist()) == set(b.tolist()) for a, b in zip(g_ids, o_ids)])
    assert same >= (1.0 if exact_ids else 0.98), same
    # final distances within 1e-4 relative of FP64 for every returned id
    ex = exact_l2_f64(ws["base"], ws["queries"], g_ids)
    valid = g_ids != INV
    if hg.parse_config(ws["hdgrid_conf"])["exps0"] > 1:
        rel = np.abs(g_dist[valid] - ex[valid]) / np.maximum(ex[valid], 1e-12)
        assert rel.max() <= 1e-4, rel.max()
    assert np.all(np.isinf(g_dist[~valid]))
    return idx, dict(r_gpu=r_gpu, r_ora=r_ora, g_ids=g_ids, g_dist=g_dist, o_ids=o_ids, o_dist=o_dist, path=path)


def test_parity_config1_small(cuda):
    ws = datasets.config1(scale=0.05, n_queries=200, max_grids=100_000)
    _parity(ws, cuda)


def test_parity_config1_full(cuda):
    ws = datasets.config1()
    _, r = _parity(ws, cuda, min_recall=0.9)


def test_parity_config2_small_postfilter(cuda):
    ws = datasets.config2(scale=0.01, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000)
    _parity(ws, cuda)


def test_parity_config4_small_range_filters(cuda):
    import oracle
    ws = datasets.config4(scale=0.002, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=4096)
    _, r = _parity(ws, cuda)
    # the oracle's prefix-count mode (the reference's inclusion-exclusion, used by the timed CPU
    # arm) gives the same per-list counts and results as its direct count
    ora = oracle.OracleIndex(r["path"])
    _, ids_p, tp = ora.query(ws["queries"], ws["query_labels"], ws["base"], ws["k"], prefix_counts=True)
    _, ids_d, td = ora.query(ws["queries"], ws["query_labels"], ws["base"], ws["k"])
    assert np.array_equal(tp["list_counts"], td["list_counts"])
    assert np.array_equal(ids_p, ids_d)


def test_parity_prefilter_rotated_adc(cuda):
    # exps0 <= 1: predicate before ADC, ADC distances are the output.  With M a multiple of
    # 32 the scan sums each 32-subspace group in a lane-rotated order (bank-conflict-free
    # LUT); the oracle in its rotated test mode sums in the same order, so ids and
    # distances must match bit for bit.
    ws = datasets.config2(scale=0.01, n_queries=200, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000, exps0=1)
    _, r = _parity(ws, cuda, exact_ids=True, adc_rotated=True)
    valid = r["g_ids"] != INV
    assert np.array_equal(r["g_ids"], r["o_ids"])
    assert np.array_equal(r["g_dist"][valid].view(np.uint32), r["o_dist"][valid].view(np.uint32))


def test_parity_prefilter_compacted_scan(cuda):
    # M = 32 (one subspace group): the predicate pass lists each predicate-first query's
    # survivors (label-rank pre-check, then the labels) in arrival order, and the ADC scan sums
    # each survivor from the subspace of its recorded position -- so ids and ADC distances
    # still equal the oracle's bit for bit
    ws = datasets.config4(scale=0.004, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=32,
                          max_grids=4096, exps0=1)
    idx, r = _parity(ws, cuda, exact_ids=True, adc_rotated=True)
    valid = r["g_ids"] != INV
    assert valid.any()
    assert np.array_equal(r["g_ids"], r["o_ids"])
    assert np.array_equal(r["g_dist"][valid].view(np.uint32), r["o_dist"][valid].view(np.uint32))
    # every candidate's labels or label ranks were read, and the rank check skipped some labels
    nq = ws["queries"].shape[0]
    cand = np.frombuffer(idx.debug_fetch("qstat").tobytes(), np.uint32).reshape(-1, 4)[:nq, 0]
    read = np.frombuffer(idx.debug_fetch("labels_read").tobytes(), np.uint32)[:nq]
    chk = np.frombuffer(idx.debug_fetch("ranks_read").tobytes(), np.uint32)[:nq]
    assert np.all((chk == cand) | ((chk == 0) & (read == cand)))
    assert np.all(read <= cand) and read.sum() < cand.sum()


def _few_values(ws):
    # dim 1 holds 5 distinct values, dim 3 one; every third query's dim-1 box has bounds equal
    # to two of the values
    ws = dict(ws)
    lab = ws["labels"].copy()
    lab[:, 1] = (lab[:, 1] // 200_000) * 200_000
    lab[:, 3] = 500_000
    ql = ws["query_labels"].copy()
    ql[::3, 2] = 200_000
    ql[::3, 3] = 400_000
    ws["labels"], ws["query_labels"] = lab, ql
    return ws


def test_parity_prefilter_label_ranks(cuda):
    # the predicate pass tests each candidate's packed label ranks (a guarded field per label dim:
    # the number of the index's per-dim thresholds at or below the label) against the query's
    # rank box before it reads the labels.  Quantile thresholds (config2's three dims, 9 bits;
    # config4's four dims, 7 bits) and one rank per distinct value (a dim of 5 values, a
    # constant dim) with box bounds equal to label values all give the oracle's ids and
    # distances bit for bit, and the ranks spare label reads
    cases = [datasets.config2(scale=0.01, n_queries=120, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                              max_grids=20_000, exps0=1)]
    ws = datasets.config4(scale=0.004, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=32,
                          max_grids=4096, exps0=1)
    cases += [ws, _few_values(ws)]
    for ws in cases:
        idx, r = _parity(ws, cuda, exact_ids=True, adc_rotated=True)
        info = idx.info()
        l = info["l"]
        assert info["rank_pack_bytes"] == 4, info
        assert info["rank_bits"] == min(12, (32 - l) // l), info
        valid = r["g_ids"] != INV
        assert valid.any()
        assert np.array_equal(r["g_ids"], r["o_ids"])
        assert np.array_equal(r["g_dist"][valid].view(np.uint32), r["o_dist"][valid].view(np.uint32))
        nq = ws["queries"].shape[0]
        read = np.frombuffer(idx.debug_fetch("labels_read").tobytes(), np.uint32)[:nq]
        chk = np.frombuffer(idx.debug_fetch("ranks_read").tobytes(), np.uint32)[:nq]
        assert read.sum() < chk.sum(), (read.sum(), chk.sum())


def test_parity_postfilter_label_ranks(cuda):
    # post-filter: the re-rank reads an entry's labels only when its ranks sit on the rank box's
    # edge (outside the box fails, inside the inner box passes); each query's ids equal the
    # oracle's
    for ws in (datasets.config4(scale=0.004, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=32,
                                max_grids=4096, exps0=32),):
        for w in (ws, _few_values(ws)):
            idx, r = _parity(w, cuda, exact_ids=True, adc_rotated=True)  # every query's id set equal
            nq = w["queries"].shape[0]
            sel = np.frombuffer(idx.debug_fetch("cand_count").tobytes(), np.uint32)[:nq]
            lab = np.frombuffer(idx.debug_fetch("refine_labels_read").tobytes(), np.uint32)[:nq]
            assert 0 < lab.sum() < sel.sum(), (lab.sum(), sel.sum())


def test_parity_prefilter_rotated_adc_fp16_lut(cuda):
    # LUT_FP16=1: entries rounded to binary16 and widened back to f32 in shared memory; the
    # oracle rounds the same way, so ids and distances still match bit for bit
    ws = datasets.config2(scale=0.01, n_queries=200, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000, exps0=1, lut_fp16=1)
    _, r = _parity(ws, cuda, exact_ids=True, adc_rotated=True)
    valid = r["g_ids"] != INV
    assert np.array_equal(r["g_ids"], r["o_ids"])
    assert np.array_equal(r["g_dist"][valid].view(np.uint32), r["o_dist"][valid].view(np.uint32))


def test_parity_precision_variant(cuda):
    # BF16 coarse GEMM pruning + FP16 LUT + exact FP32 re-rank: integer stages bit-exact,
    # final distances within 1e-4 relative of FP64 (checked inside _parity)
    ws = datasets.config3(scale=0.01, n_queries=300, clusters=16, sub_clusters=4, n_list=12, sub_lists=20,
                          max_grids=20_000)
    _parity(ws, cuda)


def test_parity_prefilter_generic_exact(cuda):
    # M = 16 (not a multiple of 32) takes the natural-order scan: ids and ADC distances
    # equal the oracle's bit for bit
    ws = datasets.config1(scale=0.05, n_queries=200, max_grids=100_000, exps0=1, pq_dim=16)
    _, r = _parity(ws, cuda)
    valid = r["g_ids"] != INV
    assert np.array_equal(r["g_ids"], r["o_ids"])
    assert np.array_equal(r["g_dist"][valid].view(np.uint32), r["o_dist"][valid].view(np.uint32))


@pytest.mark.parametrize("n_split", [1, 8])
def test_parity_is_split_range_filters(cuda, n_split):
    # is_split = 1: each probed list's Morton interval cut into n_split parts whose starts
    # move by up to three next-in-box jumps (parts with no reachable in-box code dropped);
    # every part's (start, len) must equal the oracle's
    ws = datasets.config4(scale=0.002, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=4096, is_split=1, n_split=n_split)
    idx, r = _parity(ws, cuda)
    assert idx.last_query_stats()["coarse_total"] > 0


def test_parity_is_split_postfilter_three_dims(cuda):
    ws = datasets.config2(scale=0.01, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000, is_split=1, n_split=16)
    idx, _ = _parity(ws, cuda)
    split_total = idx.last_query_stats()["coarse_total"]
    idx.set_param("is_split", 0)
    query_gpu(idx, _base_of(ws, cuda), ws, ws["k"], cuda)
    assert split_total <= idx.last_query_stats()["coarse_total"]


def _base_of(ws, dev):
    import torch
    return torch.from_numpy(ws["base"]).to(dev)


def test_select_handles_large_budget(cuda):
    # a candidate budget far above the old shared-memory top-K limit (exps0 = 40 -> 4000+)
    ws = datasets.config2(scale=0.01, n_queries=100, clusters=16, sub_clusters=4, n_list=16, sub_lists=64,
                          max_grids=20_000, exps0=40)
    _parity(ws, cuda)


def test_parity_postfilter_budget_is_not_capped(cuda):
    # The post-filter budget is the reference's min(exps0 * k * beta, max_row_len)
    # (Super-Grid-IVF_PQ.cu:1219-1222) with no cap: exps0 = 200 and k = 100 put it at 20,000
    # or more (beta >= 1), above the 16,384 clamp an earlier version applied.  The oracle
    # takes the same uncapped budget; with its ADC summed in the scan's order the selected sets
    # agree, and the re-ranked results match.
    ws = datasets.config4(scale=0.01, n_queries=200, clusters=16, sub_clusters=4, n_list=16, sub_lists=64,
                          max_grids=4096, exps0=200)
    idx, r = _parity(ws, cuda, adc_rotated=True)
    st = idx.last_query_stats()
    assert st["schedule"] == "post-filter"
    assert st["n_cand_ref"] == st["n_cand_used"] > 16384, st
    qs = np.frombuffer(idx.debug_fetch("qstat").tobytes(), np.uint32).reshape(-1, 4)
    bud = np.frombuffer(idx.debug_fetch("budget").tobytes(), np.uint32)[:qs.shape[0]]
    sel = np.frombuffer(idx.debug_fetch("cand_count").tobytes(), np.uint32)[:qs.shape[0]]
    nfin = np.frombuffer(idx.debug_fetch("nfin").tobytes(), np.uint32)[:qs.shape[0]]
    assert (bud == st["n_cand_ref"]).all()
    # every query selects min(n_cand, its finite ADC distances) candidates
    assert np.array_equal(sel, np.minimum(bud, nfin))
    assert (sel > 16384).any()


@pytest.mark.parametrize("case", ["config2", "config4", "config1"])
def test_parity_compressed_prefix_rows(cuda, case):
    # PREFIX_ROWS=1: the per-list prefix counts kept as compressed rows (change points along the
    # grid's diff dim, the reference's compress_HOPS_data form); every stored count equals the
    # oracle's dense recount (check_layout) and the per-list counts of every query equal its
    # direct count (inside _parity)
    if case == "config2":
        ws = datasets.config2(scale=0.01, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                              max_grids=20_000, prefix_rows=1)
    elif case == "config4":
        ws = datasets.config4(scale=0.002, n_queries=300, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                              max_grids=4096, prefix_rows=1)
    else:
        ws = datasets.config1(scale=0.05, n_queries=200, max_grids=100_000, prefix_rows=1)
    idx, r = _parity(ws, cuda)
    assert idx.info()["prefix_entries"] > 0
    # the same index built dense gives the same results
    ws_dense = dict(ws, hdgrid_conf=ws["hdgrid_conf"].replace("prefix_rows = 1", "prefix_rows = 2"))
    idx2, base2, _ = build_gpu(ws_dense, cuda)
    assert idx2.info()["prefix_entries"] == 0
    d2, i2 = query_gpu(idx2, base2, ws_dense, ws["k"], cuda)
    assert np.array_equal(i2, r["g_ids"]) and np.array_equal(d2.view(np.uint32), r["g_dist"].view(np.uint32))


def test_parity_masked_label_dim(cuda):
    ws = datasets.config2(scale=0.01, n_queries=150, clusters=16, sub_clusters=4, n_list=8, sub_lists=24,
                          max_grids=20_000, label_mask=0b010)
    _parity(ws, cuda)


def test_save_load_roundtrip_identical(cuda):
    import hdgrid_b200 as hg
    ws = datasets.config1(scale=0.03, n_queries=64, max_grids=50_000)
    idx, base, _ = build_gpu(ws, cuda)
    d1, i1 = query_gpu(idx, base, ws, ws["k"], cuda)
    ora, path = save_and_open_oracle(idx)
    idx2 = hg.SuperGridIndex.load(path)
    d2, i2 = query_gpu(idx2, base, ws, ws["k"], cuda)
    assert np.array_equal(i1, i2) and np.array_equal(d1.view(np.uint32), d2.view(np.uint32))
    assert idx2.info()["tot_cells"] == idx.info()["tot_cells"]


# ---- edge cases ------------------------------------------------------------------------

def test_empty_filter_and_short_results(cuda):
    ws = datasets.config1(scale=0.03, n_queries=8, max_grids=50_000)
    # query 0: label far outside the data -> box matches nothing in the predicate
    ws["query_labels"][0, 0] = 5e7
    # query 1: a zero-width window (shift is raised to 1e-7 both sides) -> at most a few
    idx, base, _ = build_gpu(ws, cuda)
    ws2 = dict(ws)
    ws2["filter_conf"] = "l = 1\nfilter0:\n\ttype = 0\n\tshift_val = [0, 0]\n"
    idx2, base2, _ = build_gpu(ws2, cuda)
    d, i = query_gpu(idx2, base2, ws2, ws2["k"], cuda)
    assert np.all((i[:, -1] == INV)), "a point-window filter cannot return 100 results"
    assert np.all(np.isinf(d[i == INV]))


def test_query_errors_are_status_codes(cuda):
    import torch
    import hdgrid_b200 as hg
    ws = datasets.config1(scale=0.03, n_queries=4, max_grids=50_000)
    idx = hg.SuperGridIndex.from_text(ws["hdgrid_conf"], ws["filter_conf"])
    q = torch.zeros((4, 128), device=cuda)
    ql = torch.zeros((4, 1), device=cuda)
    out_d = torch.empty((4, 10), device=cuda)
    out_i = torch.empty((4, 10), dtype=torch.int64, device=cuda)
    with pytest.raises(hg.HDGError) as e:  # not built yet
        idx.query(hg.query_input_t(q, q, ql), hg.query_output_t(out_d, out_i))
    assert e.value.status == 7
    base = torch.from_numpy(ws["base"]).to(cuda)
    with pytest.raises(hg.HDGError) as e:  # labels with the wrong number of dims
        idx.build(hg.build_input_t(base, torch.zeros((base.shape[0], 2), device=cuda)))
    assert e.value.status == 1
