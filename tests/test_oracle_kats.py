"""The CPU oracle against the reference's own known-answer vectors (tests/golden/)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def test_pq_lut_kat():
    k = KATS["pq_lut"]
    lut = oracle.pq_lut(np.array(k["centers"]), np.array(k["queries"]).reshape(k["n_queries"], -1),
                        k["pq_dim"], k["pq_len"], k["n_codes"])
    np.testing.assert_allclose(lut.ravel(), k["expected"], atol=k["tolerance"], rtol=0)


def test_pq_adc_kat():
    k = KATS["pq_adc"]
    lut = np.array(k["lut"], np.float32)
    out = oracle.pq_adc(np.array(k["codebook_colmajor"]), k["n_data"], lut, k["n_queries"], k["pq_dim"],
                        k["n_codes"])
    np.testing.assert_allclose(out.ravel(), k["expected"], atol=k["tolerance"], rtol=0)


def test_pq_adc_invalid_index_gives_flt_max():
    k = KATS["pq_adc"]
    idx = np.array([[0, 99, 3, 2**64 - 1]] * 3, np.uint64)
    out = oracle.pq_adc(np.array(k["codebook_colmajor"]), k["n_data"], np.array(k["lut"], np.float32),
                        k["n_queries"], k["pq_dim"], k["n_codes"], indices=idx)
    assert out[0, 1] == np.finfo(np.float32).max and out[2, 3] == np.finfo(np.float32).max
    np.testing.assert_allclose(out[:, 0], [0.6, 0.8, 1.0], atol=1e-5)


def test_label_predicate_kat():
    k = KATS["label_predicate"]
    nq, nc, l = k["n_queries"], k["n_candi"], k["l"]
    labels = np.array(k["candidate_labels"], np.float32).reshape(nq * nc, l)
    idx = np.arange(nq * nc, dtype=np.uint64).reshape(nq, nc)
    mask = oracle.label_mask(np.array(k["constraints"]).reshape(nq, 2 * l), labels, indices=idx)
    assert mask.ravel().tolist() == k["expected_kept"]


def test_label_predicate_inclusive_bounds_and_invalid_ids():
    ranges = np.array([[1.0, 2.0]], np.float32)
    labels = np.array([[1.0], [2.0], [0.9999999], [2.0000002]], np.float32)
    idx = np.array([[0, 1, 2, 3, 4, 2**64 - 1]], np.uint64)
    assert oracle.label_mask(ranges, labels, indices=idx).ravel().tolist() == [1, 1, 0, 0, 0, 0]


def test_select_elements_kat():
    k = KATS["select_elements"]
    inp = np.array(k["input"], np.float32).reshape(k["n_row"], k["n_dim_i"])
    idx = np.array(k["indices"], np.uint64).reshape(2, 3)
    assert oracle.select_elements(inp, idx, True).ravel().tolist() == k["expected_rows"]
    assert oracle.select_elements(inp, idx, False).ravel().tolist() == k["expected_elements"]


def test_morton_encode_known_values():
    # MSB-first interleave over valid dims in dim order (src/core/zorder.cu:3-15)
    assert oracle.morton_encode([0b11, 0b00], 2, 2, 0b11) == 0b1010
    assert oracle.morton_encode([0b01, 0b10], 2, 2, 0b11) == 0b0110
    # a masked dim contributes no bits
    assert oracle.morton_encode([0b11, 0b00, 0b11], 3, 2, 0b101) == 0b1111
    # single dim: the code is the coordinate
    assert oracle.morton_encode([12345], 1, 20, 1) == 12345


def test_grid_id_float_semantics():
    # ((uint64)((x - left) * M)) / span in f32: 999999 * 1e6 is not representable in f32
    assert oracle.grid_id(5.0, 0, 1_000_000, 1_000_000) == 5
    # negative products saturate to 0 (CUDA float->uint64 conversion)
    assert oracle.grid_id(3.0, 10, 100, 100) == 0
    v = oracle.grid_id(999_999.0, 0, 999_999, 999_999)
    assert v in (999_998, 999_999)
    prod = np.float32(np.float32(999_999.0) * np.float32(999_999.0))
    assert v == int(prod) // 999_999


def test_grid_shape_three_dims():
    # 3 dims with spans 9999, 9999, 3e7 and max_grids 3e7 -> 74 x 74 x 5477, 13 Morton bits
    g = oracle.grid_shape([0, 0, 0], [2.9999e7, 9999, 9999], 30_000_000)
    assert g["dims"] == [74, 74, 5477]
    assert g["shuffle"][2] == 0 and sorted(g["shuffle"][:2]) == [1, 2]
    assert g["max_bits"] == 13 and g["valid_map"] == 0b111


def test_grid_shape_masked_dim_and_single_dim():
    g = oracle.grid_shape([0, 0], [999_999, 9999], 100_000, label_mask=0b01)
    # label dim 0 masked: it sorts last (largest span), gets one cell and no Morton bits;
    # label dim 1 is the only valid dim and takes main_grids = floor(sqrt(1e5)) = 316
    assert g["shuffle"] == [1, 0] and g["dims"] == [316, 1] and g["valid_map"] == 0b01
    g1 = oracle.grid_shape([0], [999_999], 1_000_000)
    assert g1["dims"] == [999_999] and g1["max_bits"] == 20


def test_grid_shape_span_is_an_f32_difference():
    # calc_grid_shape's `ceil(global_max[i]) - floor(global_min[i])` runs on float elements
    # (Super-Grid-IVF_PQ.cu:326): under nvcc the float overloads are chosen, so a span above
    # 2^24 whose exact difference is odd is rounded to f32 before the uint64 conversion
    g = oracle.grid_shape([13.0], [29_999_980.0], 1_000_000_000)
    want = int(np.float32(np.ceil(np.float32(29_999_980.0))) - np.float32(np.floor(np.float32(13.0))))
    assert want == 29_999_968 and g["span"] == [want]
    # below 2^24 the f32 difference is exact
    assert oracle.grid_shape([3.0], [9_999.0], 1_000_000)["span"] == [9_996]


def test_recover_filters_out_of_table_and_saturating_casts():
    # map: label - 1 indexes a 2-row table; labels past it (also 2^30 and above, where
    # 2 * v + 1 no longer fits in 32 bits, and 3e9, which the GPU's f32 -> s32 cast saturates
    # to INT_MAX) and label 0 give the empty box (FLT_MAX, -FLT_MAX)
    fmax = np.finfo(np.float32).max
    spec = {"l": 1, "type": [1], "shift_val": [0.0, 0.0], "div_value": [0], "interval_map": [1.0, 2.0, 3.0, 4.0]}
    bad = np.array([[3.0], [2.0 ** 30], [1.5e9], [3e9], [0.0], [-5.0]], np.float32)
    out = oracle.recover_filters(spec, bad)
    assert (out[:, 0] == fmax).all() and (out[:, 1] == -fmax).all(), out
    assert oracle.recover_filters(spec, np.array([[2.0]], np.float32)).ravel().tolist() == [3.0, 4.0]
    # div: (int)label saturates at INT_MAX / INT_MIN as on the GPU (an x86 cast gives INT_MIN)
    spec2 = {"l": 1, "type": [2], "shift_val": [0.0, 0.0], "div_value": [10], "interval_map": []}
    out2 = oracle.recover_filters(spec2, np.array([[3e9], [-3e9], [57.0]], np.float32))
    assert out2[:, 0].tolist() == [np.float32(2147483647 // 10), np.float32(-(2147483648 // 10)), 5.0]


def test_recover_filters_types():
    spec = {"l": 3, "type": [0, 1, 2], "shift_val": [604800.0, 0.0, 0, 0, 0, 0], "div_value": [0, 0, 10],
            "interval_map": [0.0, 9999.0, 100.0, 200.0]}
    ql = np.array([[1_000_000.0, 2.0, 57.0]], np.float32)
    out = oracle.recover_filters(spec, ql)
    assert out[0, 0] == np.float32(1_000_000 - 604_800)
    # zero shift is raised to 1e-7 in double, then rounded to f32
    assert out[0, 1] == np.float32(np.float64(1_000_000.0) + 1e-7)
    assert out[0, 2:4].tolist() == [100.0, 200.0]  # label 2 -> entry 1 (label - 1)
    assert out[0, 4] == 5.0 and out[0, 5] == np.finfo(np.float32).max
    spec3 = {"l": 2, "type": [3, 3], "shift_val": [0.0] * 4, "div_value": [0, 0], "interval_map": []}
    out3 = oracle.recover_filters(spec3, np.array([[1, 2, 3, 4]], np.float32), filter_dim=2)
    assert out3.ravel().tolist() == [1, 2, 3, 4]


def test_bruteforce_respects_filter_and_order():
    rng = np.random.default_rng(0)
    data = rng.standard_normal((500, 16)).astype(np.float32)
    labels = rng.integers(0, 100, size=(500, 1)).astype(np.float32)
    q = rng.standard_normal((4, 16)).astype(np.float32)
    ranges = np.array([[10, 30]] * 4, np.float32)
    dist, ids = oracle.bruteforce_f64(data, labels, q, ranges, 10)
    for i in range(4):
        ok = np.nonzero((labels[:, 0] >= 10) & (labels[:, 0] <= 30))[0]
        d = ((data[ok].astype(np.float64) - q[i]) ** 2).sum(1)
        order = ok[np.lexsort((ok, d))][:10]
        assert ids[i].tolist() == order.tolist()
        assert np.all(np.diff(dist[i]) >= 0)


def test_oracle_matches_reference_stage_vectors():
    # tests/golden/reference_stages.json: inputs of tests/golden/make_reference_stage_vectors.py
    # with the outputs of the reference's own device functions (compiled from its sources by
    # oracle/ref_build.py, run on a GPU); the oracle's restatements must reproduce them bit for bit
    f = Path(__file__).parent / "golden" / "reference_stages.json"
    if not f.exists():
        pytest.skip("tests/golden/reference_stages.json not generated yet")
    data = json.loads(f.read_text())
    cs, ref = data["inputs"], data["reference"]
    for name in ("recover_shift_map_div", "recover_ranges"):
        c = cs[name]
        o = oracle.recover_filters(c["spec"], np.array(c["labels"], np.float32), filter_dim=c["filter_dim"])
        assert o.view(np.uint32).tolist() == ref[name], name
    for g, r in zip(cs["grid_id"], ref["grid_id"]):
        assert [oracle.grid_id(v, g["left"], g["span"], g["M"]) for v in np.array(g["x"], np.float32)] == r
    g = cs["cell_boxes"]
    o = oracle.cell_boxes(np.array(g["boxes"], np.float32), g["dims"], g["shuffle"], g["left"], g["span"])
    assert o.tolist() == ref["cell_boxes"]
    for m, r in zip(cs["morton"], ref["morton"]):
        c = np.array(m["coords"], np.int32)
        assert [oracle.morton_encode(row, m["dims"], m["max_bits"], m["valid_map"]) for row in c] == r
    for z, r in zip(cs["next_z"], ref["next_z"]):
        nx, ok = oracle.next_in_box(np.array(z["cur"], np.uint64), np.array(z["boxes"], np.int32), z["dims"],
                                    z["max_bits"], z["valid_map"])
        assert ok.tolist() == r["ok"]
        assert [int(v) for v, f in zip(nx, ok) if f] == [v for v, f in zip(r["next"], r["ok"]) if f]
