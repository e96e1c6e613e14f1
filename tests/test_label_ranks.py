"""Label ranks on the CPU: the thresholds the build derives from a base set's labels
(hdg_label_ranks, host code of the library), and the exactness of the rank boxes built from
them.  The predicate pass rejects a candidate whose rank lies outside the query's rank box, and
the re-rank accepts an entry whose ranks lie inside the inner box, without reading labels; both
must agree with the label test `!(x < lo || x > hi)` (filter.cu:30-64) for every label.  The box
definitions below restate those of the query prologue; the GPU parity tests check the kernels
against the oracle on the same kind of data."""
import math

import numpy as np
import pytest

import hdgrid_b200 as hg


def _rank(thr, x):
    return int(np.searchsorted(thr, np.float32(x), side="right"))


def _boxes(thr, mn, mx, lo, hi):
    """(rank box, inner box) of one label dim, as the prologue computes them."""
    n = len(thr)
    rlo = 0 if math.isnan(lo) else _rank(thr, lo)
    rhi = n if math.isnan(hi) else _rank(thr, hi)
    ilo = 0 if (math.isnan(lo) or mn >= lo) else int(np.searchsorted(thr, np.float32(lo), side="left")) + 1
    ihi = n if (math.isnan(hi) or mx <= hi) else rhi - 1
    return (rlo, rhi), (ilo, ihi)


@pytest.mark.parametrize("l", range(1, 9))
def test_bits_per_dim(l):
    r = hg.label_ranks(np.zeros((10, l), np.float32))
    assert r["bits"] == min(12, (32 - l) // l)
    assert r["bits"] * l + l <= 32


def test_one_rank_per_distinct_value():
    lab = np.array([[5], [1], [3], [3], [9], [1]], np.float32)
    r = hg.label_ranks(lab)
    assert r["thresholds"][0].tolist() == [3.0, 5.0, 9.0]
    assert [_rank(r["thresholds"][0], x) for x in (1, 3, 5, 9)] == [0, 1, 2, 3]
    assert (r["min"][0], r["max"][0]) == (1.0, 9.0)


def test_quantile_thresholds_balance_the_ranks():
    rng = np.random.default_rng(3)
    lab = rng.integers(0, 1_000_000, size=(400_000, 4)).astype(np.float32)
    r = hg.label_ranks(lab)
    for i in range(4):
        t = r["thresholds"][i]
        assert len(t) == (1 << r["bits"]) - 1
        assert np.all(np.diff(t) > 0)
        counts = np.bincount(np.searchsorted(t, lab[:, i], side="right"), minlength=len(t) + 1)
        expect = lab.shape[0] / (len(t) + 1)
        assert counts.min() > 0.8 * expect and counts.max() < 1.2 * expect, (counts.min(), counts.max())


def test_label_range_covers_rows_outside_the_sample():
    # 1,000,000 rows: the sample takes every 3rd row; the extremes sit on unsampled rows
    lab = np.full((1_000_000, 1), 500.0, np.float32)
    lab[::7, 0] = np.arange(len(lab[::7]), dtype=np.float32) % 1000
    lab[1, 0] = -12.5
    lab[2, 0] = 7777.0
    r = hg.label_ranks(lab)
    assert (r["min"][0], r["max"][0]) == (-12.5, 7777.0)


def test_nan_labels_are_left_out():
    lab = np.array([[np.nan], [2.0], [4.0], [np.nan], [8.0]], np.float32)
    r = hg.label_ranks(lab)
    assert r["thresholds"][0].tolist() == [4.0, 8.0]
    assert (r["min"][0], r["max"][0]) == (2.0, 8.0)


def test_rank_boxes_are_exact():
    rng = np.random.default_rng(11)
    n = 50_000
    lab = np.stack([rng.integers(0, 1_000_000, n),            # quantile thresholds
                    (rng.integers(0, 5, n) * 200_000),          # five values: a rank each
                    np.full(n, 500_000),                        # one value
                    rng.normal(0, 1e3, n)], axis=1).astype(np.float32)
    r = hg.label_ranks(lab)
    for i in range(lab.shape[1]):
        thr, mn, mx = r["thresholds"][i], float(r["min"][i]), float(r["max"][i])
        x = lab[:, i]
        ranks = np.searchsorted(thr, x, side="right")
        cands = np.concatenate([x[:40], thr[:40], thr[:40] + 0.5, [mn, mx, mn - 1, mx + 1, -np.inf, np.inf, np.nan]])
        for _ in range(300):
            lo, hi = (float(np.float32(v)) for v in rng.choice(cands, 2))
            (rlo, rhi), (ilo, ihi) = _boxes(thr, mn, mx, lo, hi)
            passes = ~((x < np.float32(lo)) | (x > np.float32(hi)))
            outside = (ranks < rlo) | (ranks > rhi)
            inner = (ranks >= ilo) & (ranks <= ihi)
            assert not np.any(outside & passes), (i, lo, hi)
            assert np.all(passes[inner]), (i, lo, hi)


def test_invalid_arguments():
    with pytest.raises(hg.HDGError):
        hg.label_ranks(np.zeros((4, 9), np.float32))


@pytest.mark.parametrize("l", [1, 2, 3, 4, 5, 6, 7, 8])
def test_guarded_field_range_test(l):
    # The kernels test every dim of a packed rank word at once: with G the guard bits, lo and hi
    # the box's bounds in their fields, ((c | G) - lo) & ((hi | G) - c) & G == G exactly when
    # every field of c lies in [lo, hi] -- including the empty field [1, 0] of an inner box
    # with no rank sure to pass.  Checked here on the 32-bit words of every field width.
    bits = hg.label_ranks(np.zeros((2, l), np.float32))["bits"]
    rng = np.random.default_rng(l)
    top = (1 << bits) - 1
    off = [i * (bits + 1) for i in range(l)]
    G = sum(1 << (o + bits) for o in off)
    mask32 = (1 << 32) - 1
    for _ in range(2000):
        c = rng.integers(0, top + 1, l)
        lo = rng.integers(0, top + 1, l)
        hi = rng.integers(0, top + 1, l)
        empty = rng.random(l) < 0.1
        lo[empty], hi[empty] = 1, 0
        cw = sum(int(v) << o for v, o in zip(c, off))
        low = sum(int(v) << o for v, o in zip(lo, off))
        high = sum(int(v) << o for v, o in zip(hi, off)) | G
        t = (((cw | G) - low) & mask32) & ((high - cw) & mask32)
        assert ((t & G) == G) == bool(np.all((c >= lo) & (c <= hi))), (c, lo, hi)
