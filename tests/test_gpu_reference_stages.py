"""The oracle's integer stages against the reference's own device code, run on the GPU.

oracle/_ref/libhdgref.so (built by oracle/ref_build.py from a reference checkout) holds the
reference's denormalize_labels_kernel (src/core/preprocessing.cu:3-32), get_grid_id_device and
get_filter_grid_ranges_kernel (src/index/2-level_index/Super-Grid-IVF_PQ.cu:24-26, 930-961),
morton_encode (src/core/zorder.cu:3-15) and getNextZValueBaseline (zorder.cu:83-244), compiled
unchanged behind a small harness.  On the seeded inputs of
tests/golden/make_reference_stage_vectors.py the oracle's restatements must agree bit for bit,
and so must the product's filter recovery (which the parity tests chain to the rest of the
product's integer stages through the oracle).
"""
import numpy as np
import pytest

import oracle
from tests.golden.make_reference_stage_vectors import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    r = oracle.reference_stages()
    if r is None:
        pytest.skip("oracle/_ref/libhdgref.so not built (python oracle/ref_build.py REFERENCE_CHECKOUT)")
    return r


@pytest.fixture(scope="module")
def cs():
    return cases()


def _filter_conf(spec):
    lines = [f"l = {spec['l']}"]
    for i in range(spec["l"]):
        t = spec["type"][i]
        lines += [f"filter{i}:", f"\ttype = {t}"]
        if t == 0:
            lines.append(f"\tshift_val = [{spec['shift_val'][2 * i]:g}, {spec['shift_val'][2 * i + 1]:g}]")
        elif t == 1:
            lines.append("\tinterval_map = [" + ", ".join(f"{v:g}" for v in spec["interval_map"]) + "]")
        elif t == 2:
            lines.append(f"\tdiv_value = [{spec['div_value'][i]}]")
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("name", ["recover_shift_map_div", "recover_ranges"])
def test_filter_recovery_matches_the_reference(cuda, ref, cs, name):
    import torch
    import hdgrid_b200 as hg
    c = cs[name]
    lab = np.array(c["labels"], np.float32)
    r = ref.denormalize(c["spec"], lab, c["filter_dim"])
    o = oracle.recover_filters(c["spec"], lab, filter_dim=c["filter_dim"])
    assert np.array_equal(o.view(np.uint32), r.view(np.uint32)), np.argwhere(o.view(np.uint32) != r.view(np.uint32))[:5]
    out = torch.empty((lab.shape[0], 2 * c["spec"]["l"]), device=cuda)
    hg.recover_filters(_filter_conf(c["spec"]), torch.from_numpy(lab).to(cuda), out)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), r.view(np.uint32))


def test_grid_ids_match_the_reference(ref, cs):
    for g in cs["grid_id"]:
        x = np.array(g["x"], np.float32)
        r = ref.grid_id(x, g["left"], g["span"], g["M"])
        o = np.array([oracle.grid_id(v, g["left"], g["span"], g["M"]) for v in x], np.int32)
        bad = np.nonzero(r != o)[0]
        assert bad.size == 0, (g["left"], g["span"], g["M"], x[bad[:5]], r[bad[:5]], o[bad[:5]])


def test_cell_boxes_match_the_reference(ref, cs):
    g = cs["cell_boxes"]
    boxes = np.array(g["boxes"], np.float32)
    r = ref.filter_grid_ranges(boxes, g["dims"], g["shuffle"], g["left"], g["span"])
    o = oracle.cell_boxes(boxes, g["dims"], g["shuffle"], g["left"], g["span"])
    assert np.array_equal(r, o), np.argwhere(r != o)[:5]


def test_morton_codes_match_the_reference(ref, cs):
    for m in cs["morton"]:
        c = np.array(m["coords"], np.int32)
        r = ref.morton_encode(c, m["dims"], m["max_bits"], m["valid_map"])
        o = np.array([oracle.morton_encode(row, m["dims"], m["max_bits"], m["valid_map"]) for row in c], np.uint64)
        assert np.array_equal(r, o), (m["dims"], m["max_bits"], m["valid_map"])


def test_next_in_box_matches_the_reference(ref, cs):
    for z in cs["next_z"]:
        cur, boxes = np.array(z["cur"], np.uint64), np.array(z["boxes"], np.int32)
        rn, rok = ref.next_z(cur, boxes, z["dims"], z["max_bits"], z["valid_map"])
        on, ook = oracle.next_in_box(cur, boxes, z["dims"], z["max_bits"], z["valid_map"])
        assert np.array_equal(rok, ook), (z["dims"], z["max_bits"], np.argwhere(rok != ook)[:5])
        assert np.array_equal(rn[rok == 1], on[ook == 1]), (z["dims"], z["max_bits"])
