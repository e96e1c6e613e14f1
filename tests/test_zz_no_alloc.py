"""hdg_recover_filters_noalloc: the allocation-free variant of hdg_recover_filters.

Some callers of this library cannot let it allocate device memory while they run -- a host
application whose own allocator owns the GPU's memory, or a serving loop that cannot afford
the device-wide synchronisation cudaMalloc / cudaFree may cause.  For them the variant keeps
the filter's interval-map table in a fixed scratch array inside the library instead of a
per-call cudaMalloc.  This test calls both entry points through the C ABI and requires
identical output on two calls in a row (the second with a different filter and different
labels, so a stale scratch array would show).  The file sorts last so that a failure here
cannot hide any other test in a run that stops at the first failure.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FILTER_A = """l = 3
filter0:
\ttype = 0
\tshift_val = [604800, 0]
filter1:
\ttype = 1
\tinterval_map = [0, 9999, 0, 7499, 0, 4999, 0, 3499, 0, 2499, 0, 1799, 0, 1249, 0, 899, 0, 624, 0, 499]
filter2:
\ttype = 2
\tdiv_value = [10]
"""

FILTER_B = """l = 2
filter0:
\ttype = 1
\tinterval_map = [5, 6, 7, 8, 100, 200]
filter1:
\ttype = 0
\tshift_val = [30, 3]
"""


def _labels(rng, n, l, map_entries):
    x = rng.integers(0, 3_000_000, size=(n, l)).astype(np.float32)
    x[:, 1 if l == 3 else 0] = rng.integers(1, map_entries + 1, size=n)  # valid map rows (label - 1)
    return x


def _run(fn, spec, labels, cuda):
    import torch
    import hdgrid_b200 as hg
    ql = torch.from_numpy(labels).to(cuda)
    out = torch.full((labels.shape[0], 2 * spec.l), float("nan"), device=cuda)
    st = torch.cuda.current_stream().cuda_stream or None
    status = fn(C.byref(spec), ql.data_ptr(), labels.shape[0], out.data_ptr(), st)
    assert status == 0, hg.LIB.hdg_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    import hdgrid_b200 as hg
    rng = np.random.default_rng(5)
    for text, l, entries, n in ((FILTER_A, 3, 10, 4096), (FILTER_B, 2, 3, 777)):
        spec = hg.filter_spec(text)
        labels = _labels(rng, n, l, entries)
        ref = _run(hg.LIB.hdg_recover_filters, spec, labels, cuda)
        got = _run(hg.LIB.hdg_recover_filters_noalloc, spec, labels, cuda)
        assert not np.isnan(got).any()
        # same kernel, same inputs: bit-identical ranges
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_noalloc_rejects_oversized_map(cuda):
    import hdgrid_b200 as hg
    spec = hg.filter_spec(FILTER_B)
    big = (C.c_float * (hg.LIB_NOALLOC_MAP_MAX + 2))()
    spec.n_map = hg.LIB_NOALLOC_MAP_MAX + 2
    spec.interval_map = C.cast(big, C.POINTER(C.c_float))
    labels = np.ones((4, 2), np.float32)
    import torch
    ql = torch.from_numpy(labels).to(cuda)
    out = torch.empty((4, 4), device=cuda)
    status = hg.LIB.hdg_recover_filters_noalloc(C.byref(spec), ql.data_ptr(), 4, out.data_ptr(), None)
    assert status == 1
    assert "exceeds" in hg.LIB.hdg_last_error().decode()


def test_noalloc_out_of_table_labels_after_a_longer_map(cuda):
    """A call whose map is shorter than the previous call's must not read the earlier
    table's leftover entries: labels past the map (including 2^30 and 3e9, where 2 * v + 1
    no longer fits in 32 bits) give the empty box (FLT_MAX, -FLT_MAX) from both entry points,
    here on a non-default stream."""
    import torch
    import hdgrid_b200 as hg
    rng = np.random.default_rng(9)
    long_spec = hg.filter_spec(FILTER_A)
    _run(hg.LIB.hdg_recover_filters_noalloc, long_spec, _labels(rng, 512, 3, 10), cuda)  # fills 20 entries
    spec = hg.filter_spec(FILTER_B)  # 6 map entries: valid labels 1..3
    bad = np.array([4, 5, 11, 1e6, 2.0 ** 30, 1.5e9, 3e9, 0], np.float32)
    labels = np.stack([bad, np.full_like(bad, 1000.0)], axis=1)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        got = _run(hg.LIB.hdg_recover_filters_noalloc, spec, labels, cuda)
        ref = _run(hg.LIB.hdg_recover_filters, spec, labels, cuda)
    fmax = np.float32(np.finfo(np.float32).max)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert (got[:, 0] == fmax).all() and (got[:, 1] == -fmax).all(), got[:, :2]
