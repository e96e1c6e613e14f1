"""hdgrid_b200 -- B200-native HDGrid ("super-grid") filtered ANN search.

Python mirror of the reference's operator interface over the C ABI of libhdgrid.so
(include/hdgrid.h).  Names follow the reference:

* ``config_factory.create(algorithm, path)``  -- src/index/index-factory.cuh:10-35
* ``index_factory.create(algorithm, config, filter_config_path)`` -- index-factory.cuh:38-87
* ``build_input_t`` / ``query_input_t`` / ``query_output_t`` -- src/core/interfaces.cuh:6-25
* ``SuperGridIndex.build`` / ``.query`` -- index_base_t::build/query (interfaces.cuh:30-31)

Tensors are torch CUDA tensors (device memory and streams only; every computation runs
in the hand-written sm_100a kernels of libhdgrid.so).  There is no CPU fallback: importing
this package without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

_PKG = Path(__file__).resolve().parent
_LIB_PATH = _PKG / "libhdgrid.so"

HDG_OK = 0
HDG_ERR_INVALID_ARG = 1
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "IO", 3: "CUDA", 4: "OOM", 5: "TIMEOUT",
                6: "UNSUPPORTED", 7: "STATE"}
MAX_DIMS = 8

_PARAM_FIELDS = [
    "topk", "filter_dim", "pq_dim", "n_clusters", "exps0", "clusters", "sub_clusters",
    "max_grids", "n_list", "sub_lists", "n_split", "label_mask", "is_split", "break_down",
    "enable_multi_gpu", "mem_bound", "is_calc_mem_predictor_coeff", "lowest_query_batch",
    "data_width", "index_width",
]


class hdg_params(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in _PARAM_FIELDS] + [("path", C.c_char * 512)] + [
        (f, C.c_uint64) for f in ("lut_fp16", "coarse_bf16", "kmeans_iters", "seed", "scan_cpt", "scan_chunk",
                                  "query_graph", "learned", "prefix_rows")]


class hdg_filter_spec(C.Structure):
    _fields_ = [("l", C.c_int32), ("type", C.c_int32 * MAX_DIMS), ("shift_val", C.c_float * (2 * MAX_DIMS)),
                ("div_value", C.c_int32 * MAX_DIMS), ("n_map", C.c_int32), ("interval_map", C.POINTER(C.c_float))]


class hdg_index_info(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in ("n", "d", "l", "M", "M_pad", "n_lists", "clusters", "tot_cells")] + [
        ("grid_dims", C.c_int32 * MAX_DIMS), ("shuffle", C.c_int32 * MAX_DIMS),
        ("label_left", C.c_uint64 * MAX_DIMS), ("label_span", C.c_uint64 * MAX_DIMS),
        ("morton_dims", C.c_int32), ("morton_max_bits", C.c_int32), ("morton_valid_map", C.c_int32),
        ("diff_dim", C.c_int32), ("device_bytes", C.c_uint64), ("prefix_entries", C.c_uint64),
        ("rank_pack_bytes", C.c_uint64), ("rank_bits", C.c_uint64)]


class HDGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{STATUS_NAMES.get(status, status)}] {msg}")
        self.status = status


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(f"{_LIB_PATH} is missing: run `python hdgrid_b200/build_native.py` "
                          "(the package has no CPU fallback)")
    lib = C.CDLL(str(_LIB_PATH))
    vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int32
    sigs = {
        "hdg_create": [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(vp)],
        "hdg_create_from_text": [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(vp)],
        "hdg_destroy": [vp],
        "hdg_parse_config": [C.c_char_p, C.POINTER(hdg_params)],
        "hdg_parse_filter": [C.c_char_p, C.POINTER(hdg_filter_spec)],
        "hdg_get_params": [vp, C.POINTER(hdg_params)],
        "hdg_set_param": [vp, C.c_char_p, u64],
        "hdg_build": [vp, vp, u64, u32, vp, u32, vp],
        "hdg_reserve": [vp, u64],
        "hdg_query": [vp, vp, u64, vp, u32, vp, u32, vp, vp, vp],
        "hdg_query_ex": [vp, vp, u64, vp, u32, vp, u32, vp, vp, vp, vp, vp, vp],
        "hdg_query_status": [vp],
        "hdg_query_features": [vp, vp, u64, vp, u32, vp, u32, vp, vp],
        "hdg_mlp_init": [vp, u64],
        "hdg_mlp_set_weights": [vp, vp, u64],
        "hdg_mlp_get_weights": [vp, vp, u64],
        "hdg_mlp_forward": [vp, vp, u64, vp, vp],
        "hdg_mlp_gradients": [vp, vp, vp, u64, vp, C.POINTER(C.c_double), vp],
        "hdg_mlp_train": [vp, vp, vp, u64, u32, u32, C.c_float, u64, C.POINTER(C.c_double), vp],
        "hdg_autotune": [vp, vp, u64, vp, u32, vp, u32, vp, vp, vp, C.POINTER(C.c_float)],
        "hdg_debug_fetch": [vp, C.c_char_p, vp, C.c_size_t, C.POINTER(C.c_size_t)],
        "hdg_get_info": [vp, C.POINTER(hdg_index_info)],
        "hdg_save": [vp, C.c_char_p],
        "hdg_load": [C.c_char_p, C.POINTER(vp)],
        "hdg_pq_lut": [vp, vp, u64, u32, u32, u32, u32, vp, vp],
        "hdg_pq_adc": [vp, u64, vp, u64, u32, u32, vp, u64, vp, vp],
        "hdg_label_mask": [vp, vp, u32, u64, u64, vp, u64, vp, vp],
        "hdg_recover_filters": [C.POINTER(hdg_filter_spec), vp, u64, vp, vp],
        "hdg_recover_filters_noalloc": [C.POINTER(hdg_filter_spec), vp, u64, vp, vp],
        "hdg_bruteforce_knn": [vp, u64, u32, vp, u32, vp, u64, vp, u32, vp, vp, vp],
        "hdg_bf16_gemm": [vp, u64, vp, u64, u32, vp, u64, vp],
        "hdg_merge_topk": [vp, vp, u64, u32, u32, vp, vp, vp, vp],
        "hdg_label_ranks": [vp, u64, u32, C.POINTER(u32), vp, vp, vp, vp],
    }
    for name, args in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    lib.hdg_last_error.restype = C.c_char_p
    lib.hdg_version.restype = C.c_char_p
    lib.hdg_last_stage_times.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_char_p), C.c_int]
    lib.hdg_last_stage_times.restype = C.c_int
    lib.hdg_last_query_stats.argtypes = [vp, C.POINTER(C.c_uint64), C.c_int]
    lib.hdg_last_query_stats.restype = C.c_int
    lib.hdg_mlp_param_count.restype = C.c_uint64
    lib.hdg_mlp_param_count.argtypes = []
    return lib


LIB = _load()
EXPORTED = [n for n in dir(LIB) if n.startswith("hdg_")]
LIB_NOALLOC_MAP_MAX = 65536  # HDG_NOALLOC_MAP_MAX of include/hdgrid.h


def _check(status: int) -> None:
    if status != HDG_OK:
        raise HDGError(status, LIB.hdg_last_error().decode(errors="replace"))


def _stream_ptr(stream=None) -> Optional[int]:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


def _ptr(t) -> int:
    return t.data_ptr()


def parse_config(text: str) -> dict:
    p = hdg_params()
    _check(LIB.hdg_parse_config(text.encode(), C.byref(p)))
    out = {f: getattr(p, f) for f, _ in hdg_params._fields_ if f != "path"}
    out["path"] = p.path.decode()
    return out


def parse_filter(text: str) -> dict:
    f = hdg_filter_spec()
    _check(LIB.hdg_parse_filter(text.encode(), C.byref(f)))
    l = f.l
    return {"l": l, "type": list(f.type[:l]), "shift_val": list(f.shift_val[:2 * l]),
            "div_value": list(f.div_value[:l]), "interval_map": [f.interval_map[i] for i in range(f.n_map)]}


# ---- the reference's interface types (src/core/interfaces.cuh:6-25) ----------------------

@dataclass
class build_input_t:
    dataset: "torch.Tensor"       # [n x d] f32, cuda
    data_labels: "torch.Tensor"   # [n x l] f32, cuda


@dataclass
class query_input_t:
    dataset: "torch.Tensor"       # [n x d] f32 (used by the exact re-rank)
    queries: "torch.Tensor"       # [q x d] f32
    query_labels: "torch.Tensor"  # [q x l*filter_dim] f32


@dataclass
class query_output_t:
    distances: "torch.Tensor"     # [q x k] f32
    neighbors: "torch.Tensor"     # [q x k] u64 (torch.int64 storage; UINT64_MAX reads as -1)


class Config:
    """Parsed HDGrid.conf (common_config + pq::config_t + super_grid::config_t)."""

    def __init__(self, text: str, source: str = "<text>"):
        self.text = text
        self.source = source
        self.params = parse_config(text)

    def __getattr__(self, k):
        try:
            return self.__dict__["params"][k]
        except KeyError as e:
            raise AttributeError(k) from e


class config_factory:
    @staticmethod
    def create(algorithm: str, search_config_path: str) -> Config:
        _check_algorithm(algorithm)
        return Config(Path(search_config_path).read_text(), search_config_path)


def _check_algorithm(algorithm: str) -> None:
    a = algorithm.lower()
    if a == "super-grid":
        return
    if a in ("pq", "prefilter", "sorting", "parafilter", "ivf-ivf_pq", "grid-ivf_pq", "cagra-post", "ivfpq-post"):
        raise HDGError(6, f"algorithm '{algorithm}' is not implemented by this library (only super-grid)")
    raise HDGError(1, f"Unknown index type: {algorithm}")


class SuperGridIndex:
    """super_grid::index (src/index/2-level_index/Super-Grid-IVF_PQ.cuh:82-110) on one B200."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def from_text(cls, hdgrid_conf: str, filter_conf: str, algorithm: str = "super-grid") -> "SuperGridIndex":
        h = C.c_void_p()
        _check(LIB.hdg_create_from_text(algorithm.encode(), hdgrid_conf.encode(), filter_conf.encode(), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_files(cls, hdgrid_conf_path: str, filter_conf_path: Optional[str] = None,
                   algorithm: str = "super-grid") -> "SuperGridIndex":
        h = C.c_void_p()
        _check(LIB.hdg_create(algorithm.encode(), hdgrid_conf_path.encode(),
                              filter_conf_path.encode() if filter_conf_path else None, C.byref(h)))
        return cls(h.value)

    @classmethod
    def load(cls, path: str) -> "SuperGridIndex":
        h = C.c_void_p()
        _check(LIB.hdg_load(str(path).encode(), C.byref(h)))
        return cls(h.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = globals().get("LIB")
        if h is not None and h.value and lib is not None:  # LIB is gone at interpreter exit
            lib.hdg_destroy(h)
            self._h = C.c_void_p()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def params(self) -> dict:
        p = hdg_params()
        _check(LIB.hdg_get_params(self._h, C.byref(p)))
        out = {f: getattr(p, f) for f, _ in hdg_params._fields_ if f != "path"}
        out["path"] = p.path.decode()
        return out

    def set_param(self, key: str, value: int) -> None:
        _check(LIB.hdg_set_param(self._h, key.encode(), int(value)))

    @property
    def topk(self) -> int:
        return int(self.params["topk"])

    def info(self) -> dict:
        i = hdg_index_info()
        _check(LIB.hdg_get_info(self._h, C.byref(i)))
        l = i.l
        return {"n": i.n, "d": i.d, "l": l, "M": i.M, "M_pad": i.M_pad, "n_lists": i.n_lists,
                "clusters": i.clusters, "tot_cells": i.tot_cells, "grid_dims": list(i.grid_dims[:l]),
                "shuffle": list(i.shuffle[:l]), "label_left": list(i.label_left[:l]),
                "label_span": list(i.label_span[:l]), "morton_dims": i.morton_dims,
                "morton_max_bits": i.morton_max_bits, "morton_valid_map": i.morton_valid_map,
                "diff_dim": i.diff_dim, "device_bytes": i.device_bytes, "prefix_entries": i.prefix_entries,
                "rank_pack_bytes": i.rank_pack_bytes, "rank_bits": i.rank_bits}

    def build(self, build_in: build_input_t, stream=None) -> None:
        ds, lb = build_in.dataset, build_in.data_labels
        _require_cuda_f32(ds, 2)
        _require_cuda_f32(lb, 2)
        _check(LIB.hdg_build(self._h, _ptr(ds), ds.shape[0], ds.shape[1], _ptr(lb), lb.shape[1], _stream_ptr(stream)))

    def reserve(self, max_queries: int) -> None:
        _check(LIB.hdg_reserve(self._h, max_queries))

    def query(self, query_in: query_input_t, query_out: query_output_t, stream=None) -> None:
        q, ql, ds = query_in.queries, query_in.query_labels, query_in.dataset
        _require_cuda_f32(q, 2)
        _require_cuda_f32(ql, 2)
        dist, ids = query_out.distances, query_out.neighbors
        k = dist.shape[1]
        _check(LIB.hdg_query(self._h, _ptr(q), q.shape[0], _ptr(ql), ql.shape[1],
                             _ptr(ds) if ds is not None else None, k, _ptr(dist), _ptr(ids), _stream_ptr(stream)))

    def query_ex(self, query_in: query_input_t, query_out: query_output_t, k=None, n_probe=None,
                 schedule=None, stream=None) -> None:
        """Query with per-query parameters: ``k`` and ``n_probe`` CUDA uint32 tensors and
        ``schedule`` a CUDA uint8 tensor of q entries each (None = the batch value).  The
        output width is the largest k; slots past a query's own k hold id 2**64-1 and +inf."""
        q, ql, ds = query_in.queries, query_in.query_labels, query_in.dataset
        _require_cuda_f32(q, 2)
        _require_cuda_f32(ql, 2)
        dist, ids = query_out.distances, query_out.neighbors
        nq = q.shape[0]

        def arr(t, dtype):
            if t is None:
                return None
            import torch
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()
                    and t.numel() == nq):
                raise HDGError(HDG_ERR_INVALID_ARG, f"per-query array must be a contiguous CUDA {dtype} of {nq}")
            return _ptr(t)

        import torch
        _check(LIB.hdg_query_ex(self._h, _ptr(q), nq, _ptr(ql), ql.shape[1], _ptr(ds) if ds is not None else None,
                                dist.shape[1], arr(k, torch.uint32), arr(n_probe, torch.uint32),
                                arr(schedule, torch.uint8), _ptr(dist), _ptr(ids), _stream_ptr(stream)))

    # ---- learned per-query schedule -------------------------------------------------
    def query_features(self, queries, query_labels, k_max: int, k=None, stream=None):
        """[q x 48] features of each query (CUDA float32 tensor)."""
        import torch
        _require_cuda_f32(queries, 2)
        _require_cuda_f32(query_labels, 2)
        out = torch.empty((queries.shape[0], 48), dtype=torch.float32, device=queries.device)
        if k is not None and not (k.is_cuda and k.dtype == torch.uint32 and k.numel() == queries.shape[0]):
            raise HDGError(HDG_ERR_INVALID_ARG, "k must be a CUDA uint32 tensor of q entries")
        _check(LIB.hdg_query_features(self._h, _ptr(queries), queries.shape[0], _ptr(query_labels),
                                      query_labels.shape[1], _ptr(k) if k is not None else None, k_max, _ptr(out),
                                      _stream_ptr(stream)))
        return out

    def mlp_init(self, seed: int = 1) -> None:
        _check(LIB.hdg_mlp_init(self._h, seed))

    def mlp_weights(self):
        import numpy as np
        w = np.empty(int(LIB.hdg_mlp_param_count()), np.float32)
        _check(LIB.hdg_mlp_get_weights(self._h, w.ctypes.data, w.size))
        return w

    def set_mlp_weights(self, w) -> None:
        import numpy as np
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(LIB.hdg_mlp_set_weights(self._h, w.ctypes.data, w.size))

    def mlp_forward(self, x, stream=None):
        import torch
        _require_cuda_f32(x, 2)
        z = torch.empty((x.shape[0], 2), dtype=torch.float32, device=x.device)
        _check(LIB.hdg_mlp_forward(self._h, _ptr(x), x.shape[0], _ptr(z), _stream_ptr(stream)))
        return z

    def mlp_gradients(self, x, y, stream=None):
        import torch
        _require_cuda_f32(x, 2)
        _require_cuda_f32(y, 2)
        g = torch.empty(int(LIB.hdg_mlp_param_count()), dtype=torch.float32, device=x.device)
        loss = C.c_double()
        _check(LIB.hdg_mlp_gradients(self._h, _ptr(x), _ptr(y), x.shape[0], _ptr(g), C.byref(loss),
                                     _stream_ptr(stream)))
        return g, loss.value

    def mlp_train(self, x, y, epochs: int = 50, batch: int = 1024, lr: float = 2e-3, seed: int = 1,
                  stream=None) -> float:
        _require_cuda_f32(x, 2)
        _require_cuda_f32(y, 2)
        loss = C.c_double()
        _check(LIB.hdg_mlp_train(self._h, _ptr(x), _ptr(y), x.shape[0], epochs, batch, lr, seed, C.byref(loss),
                                 _stream_ptr(stream)))
        return loss.value

    def status(self) -> None:
        """Waits for the last CUDA-graph replay (QUERY_GRAPH=1) and raises its device status."""
        _check(LIB.hdg_query_status(self._h))

    def autotune(self, query_in: query_input_t, query_out: query_output_t, stream=None) -> dict:
        """Times the scan variants on this batch, keeps the fastest (scan_cpt, scan_chunk)."""
        q, ql, ds = query_in.queries, query_in.query_labels, query_in.dataset
        _require_cuda_f32(q, 2)
        _require_cuda_f32(ql, 2)
        dist, ids = query_out.distances, query_out.neighbors
        best = C.c_float()
        _check(LIB.hdg_autotune(self._h, _ptr(q), q.shape[0], _ptr(ql), ql.shape[1],
                                _ptr(ds) if ds is not None else None, dist.shape[1], _ptr(dist), _ptr(ids),
                                _stream_ptr(stream), C.byref(best)))
        p = self.params
        return {"scan_cpt": int(p["scan_cpt"]), "scan_chunk": int(p["scan_chunk"]), "scan_ms": best.value}

    def save(self, path: str) -> None:
        _check(LIB.hdg_save(self._h, str(path).encode()))

    def debug_fetch(self, name: str):
        import numpy as np
        need = C.c_size_t()
        _check(LIB.hdg_debug_fetch(self._h, name.encode(), None, 0, C.byref(need)))
        buf = np.empty(need.value, dtype=np.uint8)
        _check(LIB.hdg_debug_fetch(self._h, name.encode(), buf.ctypes.data, buf.nbytes, None))
        return buf

    def last_query_stats(self) -> dict:
        import struct
        v = (C.c_uint64 * 10)()
        LIB.hdg_last_query_stats(self._h, v, 10)
        return {"queries": v[0], "n_cand_ref": v[1], "n_cand_used": v[2], "coarse_total": v[3], "exact_total": v[4],
                "max_row": v[5], "beta": struct.unpack("f", struct.pack("I", v[6] & 0xFFFFFFFF))[0],
                "schedule": ["pre-filter", "post-filter", "single-dim"][v[7]], "launches": v[8], "dropped": v[9]}

    def stage_times(self) -> dict:
        ms = (C.c_float * 16)()
        names = (C.c_char_p * 16)()
        n = LIB.hdg_last_stage_times(self._h, ms, names, 16)
        return {names[i].decode(): ms[i] for i in range(n)}


class index_factory:
    @staticmethod
    def create(algorithm: str, config: Config, filter_config_path: str) -> SuperGridIndex:
        _check_algorithm(algorithm)
        return SuperGridIndex.from_text(config.text, Path(filter_config_path).read_text(), algorithm)


def _require_cuda_f32(t, ndim: int) -> None:
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.dim() == ndim
            and t.is_contiguous()):
        raise HDGError(1, "expected a contiguous float32 CUDA tensor of rank %d" % ndim)


# ---- kernel-level entry points (the reference kernels' layouts) ---------------------------

def pq_lut(centers, queries, pq_dim: int, pq_len: int, n_codes: int, out, stream=None) -> None:
    _check(LIB.hdg_pq_lut(_ptr(centers), _ptr(queries), queries.shape[0], queries.shape[1], pq_dim, pq_len,
                          n_codes, _ptr(out), _stream_ptr(stream)))


def pq_adc(codebook, tot_data: int, lut, n_queries: int, pq_dim: int, n_codes: int, indices, n_cand: int, out,
           stream=None) -> None:
    _check(LIB.hdg_pq_adc(_ptr(codebook), tot_data, _ptr(lut), n_queries, pq_dim, n_codes,
                          _ptr(indices) if indices is not None else None, n_cand, _ptr(out), _stream_ptr(stream)))


def label_mask(ranges, labels, l: int, n_data: int, n_queries: int, indices, n_cand: int, out, stream=None) -> None:
    _check(LIB.hdg_label_mask(_ptr(ranges), _ptr(labels), l, n_data, n_queries,
                              _ptr(indices) if indices is not None else None, n_cand, _ptr(out), _stream_ptr(stream)))


def filter_spec(filter_conf_text: str) -> hdg_filter_spec:
    f = hdg_filter_spec()
    _check(LIB.hdg_parse_filter(filter_conf_text.encode(), C.byref(f)))
    return f


def recover_filters(filter_conf_text: str, query_labels, out, stream=None) -> None:
    f = filter_spec(filter_conf_text)
    _check(LIB.hdg_recover_filters(C.byref(f), _ptr(query_labels), query_labels.shape[0], _ptr(out),
                                   _stream_ptr(stream)))


def bruteforce_knn(data, labels, queries, ranges, k: int, out_dist, out_ids, stream=None) -> None:
    _check(LIB.hdg_bruteforce_knn(_ptr(data), data.shape[0], data.shape[1], _ptr(labels), labels.shape[1],
                                  _ptr(queries), queries.shape[0], _ptr(ranges), k, _ptr(out_dist), _ptr(out_ids),
                                  _stream_ptr(stream)))


def bf16_gemm(a_bf16, b_bf16, out, stream=None) -> None:
    """out[r][c] = a[r] . b[c] on the tcgen05 tensor cores (bf16 in, f32 out)."""
    _check(LIB.hdg_bf16_gemm(_ptr(a_bf16), a_bf16.shape[0], _ptr(b_bf16), b_bf16.shape[0], a_bf16.shape[1],
                             _ptr(out), out.stride(0), _stream_ptr(stream)))


def version() -> str:
    return LIB.hdg_version().decode()


def label_ranks(labels) -> dict:
    """The label-rank thresholds the build derives from a base set's labels (hdg_label_ranks):
    labels a host [n x l] float32 array.  Returns {"bits", "thresholds" (one ascending array per
    dim), "min", "max"}; a label's rank in dim i is np.searchsorted(thresholds[i], x, "right")."""
    import numpy as np
    lab = np.ascontiguousarray(labels, dtype=np.float32)
    if lab.ndim != 2:
        raise ValueError("labels must be [n x l]")
    n, l = lab.shape
    bits = C.c_uint32(0)
    _check(LIB.hdg_label_ranks(None, 0, l, C.byref(bits), None, None, None, None))
    stride = (1 << bits.value) - 1
    thr = np.zeros((l, stride), np.float32)
    n_thr = np.zeros(l, np.uint32)
    mn = np.zeros(l, np.float32)
    mx = np.zeros(l, np.float32)
    _check(LIB.hdg_label_ranks(lab.ctypes.data, n, l, C.byref(bits), thr.ctypes.data, n_thr.ctypes.data,
                               mn.ctypes.data, mx.ctypes.data))
    return {"bits": bits.value, "thresholds": [thr[i, :n_thr[i]].copy() for i in range(l)], "min": mn, "max": mx}


__all__ = ["Config", "config_factory", "index_factory", "SuperGridIndex", "build_input_t", "query_input_t",
           "query_output_t", "HDGError", "parse_config", "parse_filter", "pq_lut", "pq_adc", "label_mask",
           "recover_filters", "bruteforce_knn", "version", "label_ranks", "EXPORTED", "LIB"]


def merge_topk(dist, ids, k: int, offsets, out_dist, out_ids, stream=None) -> None:
    """Merge of per-data-batch results (hdg_merge_topk): dist / ids [q x k * n_batches] CUDA
    tensors (float32 / int64 holding u64 ids), offsets a CUDA int64 tensor of n_batches."""
    nb = offsets.numel()
    _check(LIB.hdg_merge_topk(_ptr(dist), _ptr(ids), dist.shape[0], k, nb, _ptr(offsets), _ptr(out_dist),
                              _ptr(out_ids), _stream_ptr(stream)))
