"""Golden vectors of the reference's integer stages, from the reference's own device code.

    python tests/golden/make_reference_stage_vectors.py OUT.json

Runs on a GPU machine with oracle/_ref/libhdgref.so (built by oracle/ref_build.py from a
reference checkout): the reference's denormalize_labels_kernel (src/core/preprocessing.cu:3-32),
get_grid_id_device and get_filter_grid_ranges_kernel
(src/index/2-level_index/Super-Grid-IVF_PQ.cu:24-26, 930-961), morton_encode
(src/core/zorder.cu:3-15) and getNextZValueBaseline (zorder.cu:83-244) on the seeded inputs of
``cases()``, written with their outputs as JSON (tests/golden/reference_stages.json holds one
such file; tests/test_oracle_kats.py checks the oracle against it on the CPU).

Every input stays inside what the reference code indexes safely: map-filter labels inside the
interval table, boxes whose cell ids fit in an int, a non-zero valid map with max_bits * (valid
dims) <= 64.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

FMAX = float(np.finfo(np.float32).max)


def _f32(a):
    return np.asarray(a, np.float32)


def cases(seed: int = 2024) -> dict:
    """Seeded inputs of every stage."""
    rng = np.random.default_rng(seed)
    out = {}
    # filter recovery: shift (a zero shift too) / map / div over three dims, and type 3
    table = []
    for f in (1.0, 0.75, 0.5, 0.35, 0.25, 0.18, 0.125, 0.09, 0.0625, 0.05):
        table += [0.0, float(int(round(f * 10_000)) - 1)]
    n = 200
    ts = rng.integers(0, 30_000_000, size=n).astype(np.float32)
    mp = rng.integers(1, 11, size=n).astype(np.float32)  # label - 1 inside the 10-row table
    dv = rng.integers(-200_000, 2_000_000, size=n).astype(np.float32)
    dv[:7] = [3e9, -3e9, 2147483520.0, -2147483648.0, 0.0, 9.0, np.nan]  # saturating casts, zero, below the
    # divisor, NaN (the map dim keeps in-table labels: the reference indexes its table with them)
    out["recover_shift_map_div"] = {
        "spec": {"l": 3, "type": [0, 1, 2], "shift_val": [604800.0, 0.0, 0.0, 0.0, 0.0, 0.0], "div_value": [0, 0, 10],
                 "interval_map": table},
        "labels": np.stack([ts, mp, dv], axis=1).tolist(), "filter_dim": 1}
    lo = rng.integers(0, 1_000_000, size=(n, 2)).astype(np.float32)
    w = rng.integers(0, 200_000, size=(n, 2)).astype(np.float32)
    out["recover_ranges"] = {
        "spec": {"l": 2, "type": [3, 3], "shift_val": [0.0] * 4, "div_value": [0, 0], "interval_map": []},
        "labels": np.stack([lo[:, 0], lo[:, 0] + w[:, 0], lo[:, 1], lo[:, 1] + w[:, 1]], axis=1).tolist(),
        "filter_dim": 2}
    # grid cell ids of one dim: the f32 subtraction and product, the saturating u64 cast
    x = np.concatenate([rng.uniform(-1e6, 4e7, size=180), [np.nan, np.inf, -np.inf, -1.0, 0.0, 13.0, 12.5,
                                                            29_999_980.0, 29_999_981.0, 3e7, 16777217.0, 1e20,
                                                            -1e20, 29_999_968.0, 5e6, 5e6 + 1, 7.0, 8.0, 1e-30,
                                                            2.0 ** 31]]).astype(np.float32)
    out["grid_id"] = [{"x": [float(v) for v in x], "left": left, "span": span, "M": m}
                      for left, span, m in ((13, 29_999_968, 5477), (0, 9_999, 74), (0, 999_999, 16), (7, 1, 1),
                                            (0, 30_000_000, 30_000_000))]
    # cell boxes: three shuffled dims; lows may sit below the data and highs be FLT_MAX
    grid = {"dims": [74, 74, 5477], "shuffle": [1, 2, 0], "left": [0, 0, 13], "span": [9_999, 9_999, 29_999_968]}
    b = np.empty((n, 6), np.float32)
    for d, span in ((0, 29_999_968), (1, 9_999), (2, 9_999)):
        a = rng.uniform(-0.2 * span, 1.2 * span, size=n)
        c = a + rng.uniform(0, 0.7 * span, size=n)
        b[:, 2 * d], b[:, 2 * d + 1] = a, c
    b[:10, 1] = FMAX
    b[10:20, 4] = -5.0
    b[20:30, 2:4] = b[20:30, 3:1:-1]  # lo above hi: an empty box
    b[30:34, 5] = np.nan  # NaN high bound (the cast gives 2^63, clamped to the grid's end)
    out["cell_boxes"] = dict(grid, boxes=b.tolist())
    # Morton codes
    mort = []
    for dims, bits, vm in ((3, 13, 0b111), (4, 16, 0b1111), (1, 20, 0b1), (3, 8, 0b101), (8, 8, 0xFF), (2, 32, 0b11)):
        c = rng.integers(0, 2 ** bits, size=(100, dims), dtype=np.int64).astype(np.int32)
        mort.append({"dims": dims, "max_bits": bits, "valid_map": vm, "coords": c.tolist()})
    out["morton"] = mort
    # next code inside a cell box (getNextZValueBaseline)
    nz = []
    for dims, bits, vm in ((3, 5, 0b111), (4, 4, 0b1111), (2, 8, 0b11), (3, 6, 0b011), (4, 13, 0b1111)):
        act = bin(vm).count("1")
        lo_c = rng.integers(0, 2 ** bits, size=(150, dims))
        hi_c = np.minimum(2 ** bits - 1, lo_c + rng.integers(0, 2 ** (bits - 1), size=(150, dims)))
        box = np.empty((150, 2 * dims), np.int32)
        box[:, 0::2], box[:, 1::2] = lo_c, hi_c
        cur = rng.integers(0, 2 ** (bits * act) - 1, size=150, dtype=np.uint64)
        nz.append({"dims": dims, "max_bits": bits, "valid_map": vm, "cur": [int(v) for v in cur],
                   "boxes": box.tolist()})
    out["next_z"] = nz
    return out


def run_reference(ref, cs: dict) -> dict:
    """Outputs of the reference kernels (an oracle.ReferenceStages) for cases()."""
    res = {}
    for name in ("recover_shift_map_div", "recover_ranges"):
        c = cs[name]
        res[name] = ref.denormalize(c["spec"], np.array(c["labels"], np.float32), c["filter_dim"]).view(np.uint32).tolist()
    res["grid_id"] = [ref.grid_id(np.array(g["x"], np.float32), g["left"], g["span"], g["M"]).tolist()
                      for g in cs["grid_id"]]
    g = cs["cell_boxes"]
    res["cell_boxes"] = ref.filter_grid_ranges(np.array(g["boxes"], np.float32), g["dims"], g["shuffle"], g["left"],
                                               g["span"]).tolist()
    res["morton"] = [[int(v) for v in ref.morton_encode(np.array(m["coords"], np.int32), m["dims"], m["max_bits"],
                                                         m["valid_map"])] for m in cs["morton"]]
    res["next_z"] = []
    for z in cs["next_z"]:
        nx, ok = ref.next_z(np.array(z["cur"], np.uint64), np.array(z["boxes"], np.int32), z["dims"], z["max_bits"],
                            z["valid_map"])
        res["next_z"].append({"next": [int(v) for v in nx], "ok": ok.tolist()})
    return res


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_reference_stage_vectors.py OUT.json")
    root = Path(__file__).resolve().parents[2]
    sys.path.insert(0, str(root))
    import oracle
    ref = oracle.reference_stages()
    if ref is None:
        raise SystemExit("oracle/_ref/libhdgref.so is missing: python oracle/ref_build.py REFERENCE_CHECKOUT")
    cs = cases()
    Path(sys.argv[1]).write_text(json.dumps({"generator": "tests/golden/make_reference_stage_vectors.py",
                                             "seed": 2024, "inputs": cs, "reference": run_reference(ref, cs)}))


if __name__ == "__main__":
    main()
