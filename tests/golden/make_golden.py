"""Extract the known-answer vectors of the reference's kernel tests into reference_kats.json.

The reference's standalone tests (src/verification/test_*.cuh) no longer compile (they
include headers that do not exist), but their input and expected arrays still pin the
semantics of the kernels.  This script reads those files as text, parses the brace
initialisers by name and writes them as JSON.  It needs the reference checkout and only
runs where that checkout exists; the JSON it wrote is committed next to it.

    python tests/golden/make_golden.py /path/to/HDGrid
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path


def _array(text: str, name: str) -> list[float]:
    m = re.search(re.escape(name) + r"\s*(?:\[[^\]]*\])?\s*=\s*\{(.*?)\};", text, re.S)
    if not m:
        raise KeyError(name)
    body = re.sub(r"//[^\n]*", "", m.group(1))
    return [float(x.rstrip("f")) for x in re.findall(r"-?\d+(?:\.\d+)?f?", body)]


def main(ref: Path) -> None:
    v = ref / "src" / "verification"
    lut = (v / "test_lut_build.cuh").read_text()
    adc = (v / "test_compute_pq_dis.cuh").read_text()
    flt = (v / "test_filter.cuh").read_text()
    sel = (v / "test_select_element.cuh").read_text()
    out = {
        "source": "HDGrid src/verification/test_*.cuh known-answer vectors",
        "pq_lut": {
            "file": "src/verification/test_lut_build.cuh:41-60,82",
            "n_queries": 2, "pq_dim": 2, "pq_len": 2, "n_codes": 2, "tolerance": 1e-6,
            "centers": _array(lut, "centers"), "queries": _array(lut, "queries"),
            "expected": _array(lut, "expected_lut"),
        },
        "pq_adc": {
            "file": "src/verification/test_compute_pq_dis.cuh:47-64,93-97",
            "n_data": 4, "pq_dim": 2, "n_codes": 3, "n_queries": 3, "tolerance": 1e-5,
            "codebook_colmajor": [int(x) for x in _array(adc, "h_codebook")],
            "lut": _array(adc, "h_lut"), "expected": _array(adc, "expected_result"),
        },
        "label_predicate": {
            "file": "src/verification/test_filter.cuh:17-57",
            "n_queries": 2, "n_candi": 3, "l": 2,
            "constraints": _array(flt, "h_constrains"),
            "candidate_labels": _array(flt, "h_candi_label"),
            # the old kernel overwrote dropped distances with 0; kept = value unchanged
            "expected_kept": [1 if a == b else 0 for a, b in zip(_array(flt, "expected_dis"), _array(flt, "h_dis"))],
        },
        "select_elements": {
            "file": "src/verification/test_select_element.cuh:62-106",
            "input": _array(sel, "std::vector<float> input"), "n_row": 3, "n_dim_i": 4,
            "indices": [int(x) for x in _array(sel, "std::vector<int> indices")],
            "expected_rows": _array(sel, "expected_output_1"),
            "expected_elements": _array(sel, "expected_output_2"),
        },
    }
    dst = Path(__file__).resolve().parent / "reference_kats.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py REFERENCE_CHECKOUT")
    main(Path(sys.argv[1]))
