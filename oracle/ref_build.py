"""Recipe: the reference's own integer-stage device code, compiled for the GPU -- TEST
INFRASTRUCTURE ONLY.

    python oracle/ref_build.py REFERENCE_CHECKOUT

The reference as a whole does not build here (it needs RAFT/RMM fetched at configure time),
but the device functions of its integer stages are self-contained CUDA.  This recipe reads
them from the checkout where they lie, by file and line range (each range's first line is
checked against the function it must start), writes them into oracle/_ref/ref_stages.cu
after a small header of standard includes, appends a C-ABI harness of its own, and compiles
oracle/_ref/libhdgref.so with nvcc for sm_100a.  Nothing is copied into the repository:
oracle/_ref/ is git-ignored, and only the built library travels to a GPU machine, where
tests/test_gpu_reference_stages.py runs the reference's kernels beside the oracle.

Functions taken (paths inside the HDGrid project):
  src/core/zorder.cuh:13, 23-28      MAX_DIMS, MortonConfig_t
  src/core/zorder.cu:3-34            morton_encode, morton_decode
  src/core/zorder.cu:45-51           point_in_box
  src/core/zorder.cu:67-244          leading_step_diff, set_low_k_bits, getNextZValueBaseline
  src/core/preprocessing.cu:3-32     denormalize_labels_kernel (filter recovery)
  src/index/2-level_index/Super-Grid-IVF_PQ.cu:24-26    get_grid_id_device
  src/index/2-level_index/Super-Grid-IVF_PQ.cu:930-961  get_filter_grid_ranges_kernel
The harness compiles with -DNDEBUG, so the reference's device asserts are not compiled in.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libhdgref.so"
SRC = OUT / "ref_stages.cu"
DEFAULT_CHECKOUT = "/root/reference"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# (file, first line, last line, text the first line must contain, namespace to wrap it in)
RANGES = [
    ("src/core/zorder.cuh", 13, 13, "#define MAX_DIMS", None),
    ("src/core/zorder.cuh", 23, 28, "MortonConfig_t", None),
    ("src/core/zorder.cu", 3, 34, "morton_encode(", None),
    ("src/core/zorder.cu", 45, 51, "point_in_box(", None),
    ("src/core/zorder.cu", 67, 244, "leading_step_diff(", None),
    ("src/core/preprocessing.cu", 3, 32, "denormalize_labels_kernel(", None),
    ("src/index/2-level_index/Super-Grid-IVF_PQ.cu", 24, 26, "get_grid_id_device(", "super_grid"),
    ("src/index/2-level_index/Super-Grid-IVF_PQ.cu", 930, 961, "get_filter_grid_ranges_kernel(", "super_grid"),
]

HEADER = """// Generated by oracle/ref_build.py from a checkout of the reference: its own device
// functions for the integer stages, then this recipe's C-ABI harness.  Test infrastructure.
#include <cassert>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <algorithm>
#include <limits>
#include <cuda_runtime.h>
"""

HARNESS = r"""
// ---- harness (oracle/ref_build.py): host arrays in, host arrays out ----------------------
namespace {
template <typename T>
T* dev_copy(const T* h, size_t n) {
    T* d = nullptr;
    if (cudaMalloc(&d, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
    if (n && h) cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
    return d;
}
int finish(void* out_h, const void* out_d, size_t bytes) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(out_h, out_d, bytes, cudaMemcpyDeviceToHost);
    return (int)e;
}
__global__ void h_grid_id(const float* x, uint64_t n, uint64_t left, uint64_t len, int M, int* out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = super_grid::get_grid_id_device(x[i], left, len, M);
}
__global__ void h_morton(const int* coords, uint64_t n, MortonConfig_t cfg, uint64_t* out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = morton_encode(coords + i * cfg.dims, cfg);
}
__global__ void h_next_z(const uint64_t* cur, const int* boxes, uint64_t n, MortonConfig_t cfg, uint64_t* next,
                         int* ok) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t nx = 0;
    const bool f = getNextZValueBaseline(cur[i], boxes + i * 2 * cfg.dims, nx, cfg);
    ok[i] = f ? 1 : 0;
    next[i] = f ? nx : 0;
}
unsigned blocks_for(uint64_t n) { return (unsigned)((n + 127) / 128); }
}  // namespace

extern "C" {
// denormalize_labels_kernel over n label rows (l values per row; 2l for type 3): out [n x 2l].
int ref_denormalize(const float* data, uint64_t n, uint64_t row_len, const float* shift, const int* types,
                    const float* map, uint64_t n_map, const int* div, uint64_t l, float* out) {
    float* d_data = dev_copy(data, n * row_len);
    float* d_shift = dev_copy(shift, 2 * l);
    int* d_types = dev_copy(types, l);
    float* d_map = dev_copy(map, n_map);
    int* d_div = dev_copy(div, l);
    float* d_out = dev_copy<float>(nullptr, n * 2 * l);
    denormalize_labels_kernel<<<blocks_for(n), 128>>>(d_data, n, d_shift, d_types, d_map, d_div, l, d_out);
    const int rc = finish(out, d_out, sizeof(float) * n * 2 * l);
    cudaFree(d_data); cudaFree(d_shift); cudaFree(d_types); cudaFree(d_map); cudaFree(d_div); cudaFree(d_out);
    return rc;
}
// get_filter_grid_ranges_kernel for n boxes [n x 2 dims] on a shuffled grid: out [n x 2 dims].
int ref_filter_grid_ranges(const float* boxes, uint64_t n, int dims, const int* grid_dims, const uint64_t* spans,
                           const uint64_t* left, const int* shuffle, int* out) {
    float* d_box = dev_copy(boxes, n * 2 * dims);
    int* d_dims = dev_copy(grid_dims, dims);
    uint64_t* d_span = dev_copy(spans, dims);
    uint64_t* d_left = dev_copy(left, dims);
    int* d_sh = dev_copy(shuffle, dims);
    int* d_out = dev_copy<int>(nullptr, n * 2 * dims);
    super_grid::get_filter_grid_ranges_kernel<<<blocks_for(n), 128>>>(d_box, d_out, d_dims, d_span, d_left, dims,
                                                                     (int)n, d_sh);
    const int rc = finish(out, d_out, sizeof(int) * n * 2 * dims);
    cudaFree(d_box); cudaFree(d_dims); cudaFree(d_span); cudaFree(d_left); cudaFree(d_sh); cudaFree(d_out);
    return rc;
}
// get_grid_id_device for n values of one dim.
int ref_grid_id(const float* x, uint64_t n, uint64_t left, uint64_t len, int M, int* out) {
    float* d_x = dev_copy(x, n);
    int* d_out = dev_copy<int>(nullptr, n);
    h_grid_id<<<blocks_for(n), 128>>>(d_x, n, left, len, M, d_out);
    const int rc = finish(out, d_out, sizeof(int) * n);
    cudaFree(d_x); cudaFree(d_out);
    return rc;
}
// morton_encode for n coordinate rows [n x dims].
int ref_morton_encode(const int* coords, uint64_t n, int dims, int max_bits, int valid_map, uint64_t* out) {
    int* d_c = dev_copy(coords, n * dims);
    uint64_t* d_out = dev_copy<uint64_t>(nullptr, n);
    h_morton<<<blocks_for(n), 128>>>(d_c, n, MortonConfig_t{dims, max_bits, valid_map}, d_out);
    const int rc = finish(out, d_out, sizeof(uint64_t) * n);
    cudaFree(d_c); cudaFree(d_out);
    return rc;
}
// getNextZValueBaseline for n (code, cell box [2 dims]) pairs; valid_map must be non-zero and
// max_bits * (set bits of valid_map) <= 64.
int ref_next_z(const uint64_t* cur, const int* boxes, uint64_t n, int dims, int max_bits, int valid_map,
               uint64_t* next, int* ok) {
    uint64_t* d_cur = dev_copy(cur, n);
    int* d_box = dev_copy(boxes, n * 2 * dims);
    uint64_t* d_next = dev_copy<uint64_t>(nullptr, n);
    int* d_ok = dev_copy<int>(nullptr, n);
    h_next_z<<<blocks_for(n), 128>>>(d_cur, d_box, n, MortonConfig_t{dims, max_bits, valid_map}, d_next, d_ok);
    int rc = finish(next, d_next, sizeof(uint64_t) * n);
    if (rc == 0) rc = (int)cudaMemcpy(ok, d_ok, sizeof(int) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_cur); cudaFree(d_box); cudaFree(d_next); cudaFree(d_ok);
    return rc;
}
}  // extern "C"
"""


def extract(checkout: Path) -> str:
    parts = [HEADER]
    for rel, a, b, must, ns in RANGES:
        lines = (checkout / rel).read_text().splitlines()
        if must not in lines[a - 1]:
            raise SystemExit(f"{rel}:{a} does not start {must!r}; the checkout differs from the one this recipe follows")
        body = "\n".join(lines[a - 1:b])
        parts.append(f"// ---- {rel}:{a}-{b}\n" + (f"namespace {ns} {{\n{body}\n}}\n" if ns else body + "\n"))
    parts.append(HARNESS)
    return "\n".join(parts)


def build(checkout: str) -> Path:
    root = Path(checkout)
    OUT.mkdir(exist_ok=True)
    SRC.write_text(extract(root))
    # --expt-relaxed-constexpr / --expt-extended-lambda: what the raft::raft target adds to the
    # reference's own CUDA compile (device code there calls std::numeric_limits<float>::max())
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-DNDEBUG",
           "--expt-relaxed-constexpr", "--expt-extended-lambda", "-shared", "-Xcompiler", "-fPIC", "-w",
           "-o", str(LIB), str(SRC)]
    subprocess.run(cmd, check=True)
    return LIB


def build_if_present() -> Path | None:
    """Builds the library when the reference checkout is on this machine (the build host);
    elsewhere the prebuilt library is used as it is."""
    if not Path(DEFAULT_CHECKOUT, "src", "core", "zorder.cu").exists():
        return LIB if LIB.exists() else None
    src_newer = not LIB.exists() or Path(__file__).stat().st_mtime > LIB.stat().st_mtime
    return build(DEFAULT_CHECKOUT) if src_newer else LIB


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python oracle/ref_build.py REFERENCE_CHECKOUT")
    print(build(sys.argv[1]))
