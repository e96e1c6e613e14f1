"""CPU oracle for the HDGrid filtered query path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to liboracle.so (oracle/hdg_oracle.cpp), a plain C++ restatement of the
reference's query schedule plus an FP64 filtered brute-force kNN.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it, to check results, never
to produce them.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
_SO = _DIR / "liboracle.so"


def build() -> Path:
    subprocess.run(["make", "-C", str(_DIR), "-s"], check=True)
    return _SO


def _load() -> C.CDLL:
    if not _SO.exists() or _SO.stat().st_mtime < (_DIR / "hdg_oracle.cpp").stat().st_mtime:
        build()
    lib = C.CDLL(str(_SO))
    vp = C.c_void_p
    lib.ora_open.restype = vp
    lib.ora_open.argtypes = [C.c_char_p]
    lib.ora_close.argtypes = [vp]
    lib.ora_last_error.restype = C.c_char_p
    lib.ora_morton_encode.restype = C.c_uint64
    lib.ora_morton_encode.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.ora_grid_id.restype = C.c_int
    lib.ora_grid_id.argtypes = [C.c_float, C.c_uint64, C.c_uint64, C.c_int]
    lib.ora_check_layout.restype = C.c_uint64
    lib.ora_check_layout.argtypes = [vp]
    lib.ora_query.restype = C.c_int
    lib.ora_query.argtypes = [vp, vp, C.c_uint64, vp, C.c_uint32, vp, C.c_uint32, vp, vp, vp, C.c_int, C.c_int]
    lib.ora_query_ex.restype = C.c_int
    lib.ora_query_ex.argtypes = [vp, vp, C.c_uint64, vp, C.c_uint32, vp, C.c_uint32, vp, vp, vp, vp, vp, vp,
                                 C.c_int, C.c_int]
    lib.ora_bruteforce_f64.argtypes = [vp, C.c_uint64, C.c_uint32, vp, C.c_uint32, vp, C.c_uint64, vp, C.c_uint32,
                                       vp, vp, C.c_int]
    lib.ora_pq_lut.argtypes = [vp, vp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp]
    lib.ora_pq_adc.argtypes = [vp, C.c_uint64, vp, C.c_uint64, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp]
    lib.ora_label_mask.argtypes = [vp, vp, C.c_uint32, C.c_uint64, C.c_uint64, vp, C.c_uint64, vp]
    lib.ora_select_elements.argtypes = [vp, C.c_uint64, C.c_uint64, vp, C.c_uint64, C.c_uint64, C.c_int, C.c_float,
                                        vp]
    lib.ora_recover_filters.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int, C.c_int, vp, C.c_uint64, vp]
    lib.ora_cell_boxes.argtypes = [vp, C.c_uint64, C.c_int, vp, vp, vp, vp, vp]
    lib.ora_next_in_box.argtypes = [vp, vp, C.c_uint64, C.c_int, C.c_int, C.c_int, vp, vp]
    lib.ora_grid_shape.restype = C.c_int
    lib.ora_grid_shape.argtypes = [vp, vp, C.c_int, C.c_uint64, C.c_uint64, vp, vp, vp, vp, vp, vp]
    lib.ora_info.argtypes = [vp, vp]
    lib.ora_grid.argtypes = [vp, vp, vp, vp, vp]
    return lib


LIB = _load()


def _p(a: np.ndarray):
    return a.ctypes.data if a is not None else None


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def pq_lut(centers, queries, pq_dim, pq_len, n_codes):
    centers, queries = _c(centers, np.float32), _c(queries, np.float32)
    nq, n_dim = queries.shape
    out = np.empty((nq, pq_dim, n_codes), np.float32)
    LIB.ora_pq_lut(_p(centers), _p(queries), nq, n_dim, pq_dim, pq_len, n_codes, _p(out))
    return out


def pq_adc(codebook_colmajor, tot_data, lut, n_queries, pq_dim, n_codes, indices=None, n_cand=None):
    cb = _c(codebook_colmajor, np.uint8)
    lut = _c(lut, np.float32)
    idx = None if indices is None else _c(indices, np.uint64)
    n_cand = n_cand if n_cand is not None else (idx.shape[1] if idx is not None else tot_data)
    out = np.empty((n_queries, n_cand), np.float32)
    LIB.ora_pq_adc(_p(cb), tot_data, _p(lut), n_queries, pq_dim, n_codes, _p(idx), n_cand, _p(out))
    return out


def label_mask(ranges, labels, indices=None, n_cand=None):
    ranges, labels = _c(ranges, np.float32), _c(labels, np.float32)
    nq = ranges.shape[0]
    l = labels.shape[1]
    idx = None if indices is None else _c(indices, np.uint64)
    n_cand = n_cand if n_cand is not None else (idx.shape[1] if idx is not None else labels.shape[0])
    out = np.empty((nq, n_cand), np.int32)
    LIB.ora_label_mask(_p(ranges), _p(labels), l, labels.shape[0], nq, _p(idx), n_cand, _p(out))
    return out


def select_elements(inp, indices, select_row, invalid=np.finfo(np.float32).max):
    inp = _c(inp, np.float32)
    idx = _c(indices, np.uint64)
    n_row_o, n_dim_o = idx.shape
    n_row_i, n_dim_i = inp.shape
    out = np.empty((n_row_o, n_dim_o, n_dim_i) if select_row else (n_row_o, n_dim_o), np.float32)
    LIB.ora_select_elements(_p(inp), n_row_i, n_dim_i, _p(idx), n_row_o, n_dim_o, int(select_row), float(invalid),
                            _p(out))
    return out


def recover_filters(spec: dict, query_labels, filter_dim: int = 1):
    ql = _c(query_labels, np.float32)
    l = spec["l"]
    t = _c(spec["type"] + [0] * (8 - l), np.int32)
    sh = _c(spec["shift_val"] + [0.0] * (16 - 2 * l), np.float32)
    dv = _c(spec["div_value"] + [0] * (8 - l), np.int32)
    mp = _c(spec["interval_map"] or [0.0], np.float32)
    out = np.empty((ql.shape[0], 2 * l), np.float32)
    LIB.ora_recover_filters(l, _p(t), _p(sh), _p(dv), _p(mp), len(spec["interval_map"]), filter_dim, _p(ql),
                            ql.shape[0], _p(out))
    return out


def morton_encode(coords, dims, max_bits, valid_map):
    c = _c(coords, np.int32)
    return int(LIB.ora_morton_encode(_p(c), dims, max_bits, valid_map))


def grid_id(x: float, left: int, span: int, m: int) -> int:
    return int(LIB.ora_grid_id(float(x), left, span, m))


def grid_shape(mins, maxs, max_grids, label_mask=0):
    mins, maxs = _c(mins, np.float32), _c(maxs, np.float32)
    l = len(mins)
    dims = np.zeros(8, np.int32)
    sh = np.zeros(8, np.int32)
    left = np.zeros(8, np.uint64)
    span = np.zeros(8, np.uint64)
    mb = np.zeros(1, np.int32)
    vm = np.zeros(1, np.int32)
    rc = LIB.ora_grid_shape(_p(mins), _p(maxs), l, max_grids, label_mask, _p(dims), _p(sh), _p(left), _p(span),
                            _p(mb), _p(vm))
    if rc != 0:
        raise ValueError("grid shape infeasible")
    return dict(dims=dims[:l].tolist(), shuffle=sh[:l].tolist(), left=left[:l].tolist(), span=span[:l].tolist(),
                max_bits=int(mb[0]), valid_map=int(vm[0]))


def cell_boxes(boxes, dims, shuffle, left, span):
    """Cell box [n x 2l] i32 of each f32 filter box [n x 2l] on a grid in shuffled order."""
    boxes = _c(boxes, np.float32)
    n, l = boxes.shape[0], boxes.shape[1] // 2
    out = np.empty((n, 2 * l), np.int32)
    dm, sh, lf, sp = _c(dims, np.int32), _c(shuffle, np.int32), _c(left, np.uint64), _c(span, np.uint64)
    LIB.ora_cell_boxes(_p(boxes), n, l, _p(dm), _p(sh), _p(lf), _p(sp), _p(out))
    return out


def next_in_box(cur, boxes, dims, max_bits, valid_map):
    """(next code, found) of the reference's next-in-box jump for each (code, cell box)."""
    cur = _c(cur, np.uint64)
    boxes = _c(boxes, np.int32)
    nx = np.empty(cur.shape[0], np.uint64)
    ok = np.empty(cur.shape[0], np.int32)
    LIB.ora_next_in_box(_p(cur), _p(boxes), cur.shape[0], dims, max_bits, valid_map, _p(nx), _p(ok))
    return nx, ok


def bruteforce_f64(data, labels, queries, ranges, k, threads=0):
    data, labels = _c(data, np.float32), _c(labels, np.float32)
    queries, ranges = _c(queries, np.float32), _c(ranges, np.float32)
    q = queries.shape[0]
    dist = np.empty((q, k), np.float64)
    ids = np.empty((q, k), np.uint64)
    LIB.ora_bruteforce_f64(_p(data), data.shape[0], data.shape[1], _p(labels), labels.shape[1], _p(queries), q,
                           _p(ranges), k, _p(dist), _p(ids), threads)
    return dist, ids


class _Trace(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("box", "cells", "zrange", "list_counts", "probe_clusters", "probe_lists",
                                          "range_start", "range_len", "scalars")]


class OracleIndex:
    """The reference query schedule on an index file written by hdg_save."""

    def __init__(self, path: str):
        self._h = LIB.ora_open(str(path).encode())
        if not self._h:
            raise IOError(LIB.ora_last_error().decode())
        info = np.zeros(17, np.uint64)
        LIB.ora_info(self._h, _p(info))
        (self.n, self.d, self.l, self.M, self.M_pad, self.n_lists, self.clusters, self.tot_cells, self.max_bits,
         self.valid_map, self.topk, self.filter_dim, self.exps0, self.n_list,
         self.sub_lists, self.is_split, self.n_split) = (int(x) for x in info)

    def __del__(self):
        if getattr(self, "_h", None):
            LIB.ora_close(self._h)
            self._h = None

    def grid(self):
        dims = np.zeros(8, np.int32)
        sh = np.zeros(8, np.int32)
        left = np.zeros(8, np.uint64)
        span = np.zeros(8, np.uint64)
        LIB.ora_grid(self._h, _p(dims), _p(sh), _p(left), _p(span))
        l = self.l
        return dict(dims=dims[:l].tolist(), shuffle=sh[:l].tolist(), left=left[:l].tolist(), span=span[:l].tolist())

    def check_layout(self) -> int:
        return int(LIB.ora_check_layout(self._h))

    def query(self, queries, query_labels, data, k, threads=0, trace=True, adc_rotated=False,
              qk=None, n_probe=None, schedule=None, prefix_counts=False):
        """The reference query; qk / n_probe (uint32) and schedule (uint8) are the optional
        per-query arrays of hdg_query_ex.  prefix_counts: per-list counts by the reference's
        inclusion-exclusion over the index's prefix counts instead of a direct count."""
        n_list, sub_lists = self.n_list, self.sub_lists
        qk = None if qk is None else _c(qk, np.uint32)
        n_probe = None if n_probe is None else _c(n_probe, np.uint32)
        schedule = None if schedule is None else _c(schedule, np.uint8)
        queries = _c(queries, np.float32)
        ql = _c(query_labels, np.float32)
        data = _c(data, np.float32)
        q = queries.shape[0]
        l, L = self.l, self.n_lists
        dist = np.empty((q, k), np.float32)
        ids = np.empty((q, k), np.uint64)
        tr = None
        t = {}
        if trace:
            t = dict(box=np.zeros((q, 2 * l), np.float32), cells=np.zeros((q, 2 * l), np.int32),
                     zrange=np.zeros((q, 2), np.uint64), list_counts=np.zeros((q, L), np.uint32),
                     probe_clusters=np.zeros((q, n_list), np.uint32), probe_lists=np.zeros((q, sub_lists), np.uint32),
                     range_start=np.zeros((q, sub_lists * self.n_split), np.uint32),
                     range_len=np.zeros((q, sub_lists * self.n_split), np.uint32),
                     scalars=np.zeros(4, np.float64))
            tr = _Trace(*(t[n].ctypes.data for n, _ in _Trace._fields_))
        opt = [None if a is None else _p(a) for a in (qk, n_probe, schedule)]
        rc = LIB.ora_query_ex(self._h, _p(queries), q, _p(ql), ql.shape[1], _p(data), k, *opt, _p(dist), _p(ids),
                              C.byref(tr) if tr is not None else None, threads,
                              (1 if adc_rotated else 0) | (2 if prefix_counts else 0))
        if rc != 0:
            raise RuntimeError(LIB.ora_last_error().decode())
        return dist, ids, t


class ReferenceStages:
    """The reference's own integer-stage device functions (oracle/_ref/libhdgref.so, built by
    oracle/ref_build.py from a reference checkout), run on the GPU through a small harness:
    the oracle's restatement is checked against them.  Inputs must stay inside what the
    reference code indexes safely (map labels inside the table, a non-zero valid map)."""

    def __init__(self, lib: C.CDLL):
        self.lib = lib
        u64, vp = C.c_uint64, C.c_void_p
        lib.ref_denormalize.argtypes = [vp, u64, u64, vp, vp, vp, u64, vp, u64, vp]
        lib.ref_filter_grid_ranges.argtypes = [vp, u64, C.c_int, vp, vp, vp, vp, vp]
        lib.ref_grid_id.argtypes = [vp, u64, u64, u64, C.c_int, vp]
        lib.ref_morton_encode.argtypes = [vp, u64, C.c_int, C.c_int, C.c_int, vp]
        lib.ref_next_z.argtypes = [vp, vp, u64, C.c_int, C.c_int, C.c_int, vp, vp]

    @staticmethod
    def _ok(rc):
        if rc != 0:
            raise RuntimeError(f"reference stage kernel failed: CUDA error {rc}")

    def denormalize(self, spec: dict, labels, filter_dim: int = 1):
        lab = _c(labels, np.float32)
        l = spec["l"]
        out = np.empty((lab.shape[0], 2 * l), np.float32)
        mp = _c(spec["interval_map"] or [0.0], np.float32)
        sh, ty, dv = _c(spec["shift_val"], np.float32), _c(spec["type"], np.int32), _c(spec["div_value"], np.int32)
        self._ok(self.lib.ref_denormalize(_p(lab), lab.shape[0], lab.shape[1], _p(sh), _p(ty), _p(mp),
                                          len(spec["interval_map"]), _p(dv), l, _p(out)))
        return out

    def filter_grid_ranges(self, boxes, dims, shuffle, left, span):
        boxes = _c(boxes, np.float32)
        n, l = boxes.shape[0], boxes.shape[1] // 2
        out = np.empty((n, 2 * l), np.int32)
        dm, sp, lf, sh = _c(dims, np.int32), _c(span, np.uint64), _c(left, np.uint64), _c(shuffle, np.int32)
        self._ok(self.lib.ref_filter_grid_ranges(_p(boxes), n, l, _p(dm), _p(sp), _p(lf), _p(sh), _p(out)))
        return out

    def grid_id(self, x, left, span, m):
        x = _c(x, np.float32)
        out = np.empty(x.shape[0], np.int32)
        self._ok(self.lib.ref_grid_id(_p(x), x.shape[0], left, span, m, _p(out)))
        return out

    def morton_encode(self, coords, dims, max_bits, valid_map):
        c = _c(coords, np.int32)
        out = np.empty(c.shape[0], np.uint64)
        self._ok(self.lib.ref_morton_encode(_p(c), c.shape[0], dims, max_bits, valid_map, _p(out)))
        return out

    def next_z(self, cur, boxes, dims, max_bits, valid_map):
        cur = _c(cur, np.uint64)
        b = _c(boxes, np.int32)
        nx = np.empty(cur.shape[0], np.uint64)
        ok = np.empty(cur.shape[0], np.int32)
        self._ok(self.lib.ref_next_z(_p(cur), _p(b), cur.shape[0], dims, max_bits, valid_map, _p(nx), _p(ok)))
        return nx, ok


def reference_stages():
    """The reference's integer-stage kernels, or None when oracle/_ref/libhdgref.so is absent."""
    path = _DIR / "_ref" / "libhdgref.so"
    if not path.exists():
        return None
    return ReferenceStages(C.CDLL(str(path)))
