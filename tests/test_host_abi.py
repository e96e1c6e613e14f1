"""Host-side logic of the product library that needs no GPU: the C ABI loads and exports
every symbol include/hdgrid.h declares, and the HDGrid.conf / filter.conf readers follow
the reference's parsing rules (src/utils/config_utils.h:33-88, :121-172)."""
import re
from pathlib import Path

import pytest

import hdgrid_b200 as hg

ROOT = Path(__file__).resolve().parents[1]

README_CONF = """enable_multi_gpu = 0
break_down = 1
is_calc_mem_predictor_coeff = 0
pq_dim = 4
n_clusters = 256
lowest_query_batch = 125
label_dim = 1
max_grids = 30000000
mem_bound = 5000000000
path = "dataset/example_dataset/"
clusters = 512
sub_clusters = 10
n_list = 64
sub_lists = 128
exps0 = 30
label_mask = 0
data_width = 1
is_split = 0
n_split = 1
filter_dim = 1
topk = 100
"""

README_FILTER = """l = 5
filter0:
\ttype = 0
\tshift_val = [604800, 0]
filter1:
\ttype = 0
\tshift_val = [30, 30]
filter2:
\ttype = 0
\tshift_val = [107321744, 107321744]
filter3:
\ttype = 1
\tinterval_map = [1, 2, 1, 2, 3, 4, 3, 5, 4, 5]
filter4:
\ttype = 2
\tdiv_value = [10]
"""


def test_every_declared_symbol_is_exported():
    header = (ROOT / "include" / "hdgrid.h").read_text()
    declared = set(re.findall(r"\b(hdg_[a-z_0-9]+)\s*\(", header))
    assert len(declared) >= 20
    for name in sorted(declared):
        assert hasattr(hg.LIB, name), name


def test_version_string():
    assert "sm_100a" in hg.version()


def test_parse_readme_config():
    p = hg.parse_config(README_CONF)
    assert p["pq_dim"] == 4 and p["n_clusters"] == 256 and p["clusters"] == 512
    assert p["sub_clusters"] == 10 and p["n_list"] == 64 and p["sub_lists"] == 128
    assert p["exps0"] == 30 and p["max_grids"] == 30_000_000 and p["topk"] == 100
    assert p["mem_bound"] == 5_000_000_000 and p["break_down"] == 1
    assert p["path"] == "dataset/example_dataset/"


def test_config_keys_case_and_whitespace_and_unknown_keys():
    p = hg.parse_config("  TopK=7\nN_LIST   =  3 \nlabel_dim = 9\nsomething_else = 1\n\n")
    assert p["topk"] == 7 and p["n_list"] == 3


def test_non_integer_value_rejected():
    with pytest.raises(hg.HDGError) as e:
        hg.parse_config("exps0 = 1.5\n")
    assert e.value.status == 1 and "EXPS0" in str(e.value)


def test_parse_readme_filter():
    f = hg.parse_filter(README_FILTER)
    assert f["l"] == 5 and f["type"] == [0, 0, 0, 1, 2]
    assert f["shift_val"][:6] == [604800.0, 0.0, 30.0, 30.0, 107321744.0, 107321744.0]
    assert f["interval_map"] == [1, 2, 1, 2, 3, 4, 3, 5, 4, 5]
    assert f["div_value"][4] == 10


def test_filter_type3_block_and_errors():
    f = hg.parse_filter("l = 2\nfilter0:\ntype = 3\nfilter1:\ntype=3\n")
    assert f["type"] == [3, 3]
    with pytest.raises(hg.HDGError):
        hg.parse_filter("filter0:\ntype = 0\n")  # block before l=
    with pytest.raises(hg.HDGError):
        hg.parse_filter("l = 1\nfilter3:\ntype = 0\n")  # index out of range
    with pytest.raises(hg.HDGError):
        hg.parse_filter("l = 1\nfilter0:\ntype = 2\ndiv_value = [0]\n")


def test_algorithm_names():
    with pytest.raises(hg.HDGError) as e:
        hg.config_factory.create("cagra-post", "/nonexistent")
    assert e.value.status == 6
    with pytest.raises(hg.HDGError) as e:
        hg.config_factory.create("bogus", "/nonexistent")
    assert e.value.status == 1


def test_create_reports_missing_files():
    with pytest.raises(hg.HDGError) as e:
        hg.SuperGridIndex.from_files("/nonexistent/HDGrid.conf", "/nonexistent/filter.conf", "Super-Grid")
    assert e.value.status == 2
