// Index build: super_grid::index::build (src/index/2-level_index/Super-Grid-IVF_PQ.cu:420-646)
// re-designed for one B200.
//
//  1. label grid shape on the host (calc_grid_shape, :305-412)
//  2. PQ codebooks: per-subspace k-means(256) on a sample, then every point encoded on the
//     GPU (build_pq, src/index/product-quantization.cu:147-212)
//  3. C*S fine centroids by k-means on a sample (the reference's kmeans::fit_predict, :454-463),
//     every point assigned on the GPU; FP64 centroid sums (the only FP64 on the GPU)
//  4. the fine centroids grouped into C clusters of S by a capacity-balanced k-means on the
//     host (the reference's kmeans_balanced::fit_predict, :466-477)
//  5. cell coords + Morton codes of every point on the GPU (get_grid_ids_kernel :28-52,
//     encode_points_kernel zorder.cu:36-43); pool sorted by (list, Morton code, id)
//     (thrust::sort_by_key per list, :607-611, is a stable radix sort over ids in ascending order)
//  6. per-list inclusive prefix counts over the cell grid (HOPS multi_dim_scan,
//     src/core/HOPS.cu:3-74): dense, cell-major with the list index fastest, or -- when that
//     array would be large -- compressed into per-(grid row, list) change points along the diff
//     dim (compress_HOPS_data, Super-Grid-IVF_PQ.cu:209-303).
// k-means results are not pinned by any reference test (RAFT is not vendored), so the
// build uses its own seeded Lloyd iterations.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>

#include "hdg_device.cuh"
#include "hdg_internal.h"

namespace hdg {

// ------------------------------------------------------------------------------------
// k-means kernels
// ------------------------------------------------------------------------------------

// Nearest centre of every row of X: argmin_c (|c|^2 - 2 x.c), FP32, register-tiled.
// Block = 256 threads, 128 rows x 64 centres per tile, K chunks of 32.
constexpr int AT_P = 128, AT_C = 64, AT_K = 32;
__global__ void __launch_bounds__(256) k_assign_nearest(const float* __restrict__ X, uint64_t n,
                                                        int d, const float* __restrict__ Cc,
                                                        const float* __restrict__ cnorm, int k,
                                                        int* __restrict__ out) {
    __shared__ float Xs[AT_K][AT_P + 4];
    __shared__ float Cs[AT_K][AT_C + 4];
    const int t = threadIdx.x;
    const int tx = t & 15;   // centre group (4 centres)
    const int ty = t >> 4;   // row group (8 rows)
    const uint64_t row0 = (uint64_t)blockIdx.x * AT_P;
    float best[8];
    int besti[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        best[i] = INFINITY;
        besti[i] = 0;
    }
    for (int c0 = 0; c0 < k; c0 += AT_C) {
        float acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
        for (int k0 = 0; k0 < d; k0 += AT_K) {
            for (int e = t; e < AT_P * AT_K; e += 256) {
                const int r = e / AT_K, kk = e % AT_K;
                const uint64_t gr = row0 + r;
                Xs[kk][r] = (gr < n && k0 + kk < d) ? X[gr * d + k0 + kk] : 0.f;
            }
            for (int e = t; e < AT_C * AT_K; e += 256) {
                const int r = e / AT_K, kk = e % AT_K;
                const int gc = c0 + r;
                Cs[kk][r] = (gc < k && k0 + kk < d) ? Cc[(uint64_t)gc * d + k0 + kk] : 0.f;
            }
            __syncthreads();
#pragma unroll 4
            for (int kk = 0; kk < AT_K; kk++) {
                float xv[8], cv[4];
#pragma unroll
                for (int i = 0; i < 8; i++) xv[i] = Xs[kk][ty * 8 + i];
#pragma unroll
                for (int j = 0; j < 4; j++) cv[j] = Cs[kk][tx * 4 + j];
#pragma unroll
                for (int i = 0; i < 8; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] = fmaf(xv[i], cv[j], acc[i][j]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = c0 + tx * 4 + j;
            if (c >= k) continue;
            const float cn = cnorm[c];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const float v = cn - 2.f * acc[i][j];
                if (v < best[i]) {
                    best[i] = v;
                    besti[i] = c;
                }
            }
        }
    }
    // reduce across the 16 threads (tx) that share the same 8 rows
#pragma unroll
    for (int i = 0; i < 8; i++) {
        float v = best[i];
        int b = besti[i];
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, v, o, 16);
            const int ob = __shfl_xor_sync(0xffffffffu, b, o, 16);
            if (ov < v || (ov == v && ob < b)) {
                v = ov;
                b = ob;
            }
        }
        const uint64_t gr = row0 + ty * 8 + i;
        if (tx == 0 && gr < n) out[gr] = b;
    }
}

__global__ void k_row_norms(const float* __restrict__ X, uint64_t n, int d, float* __restrict__ out) {
    const uint64_t r = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    float s = 0.f;
    for (int j = lane; j < d; j += 32) {
        const float v = X[r * d + j];
        s = fmaf(v, v, s);
    }
    s = warp_sum(s);
    if (lane == 0) out[r] = s;
}

// FP64 centroid sums (the one place the GPU computes in FP64).
__global__ void k_accumulate(const float* __restrict__ X, uint64_t n, int d,
                             const int* __restrict__ lab, double* __restrict__ sums,
                             unsigned* __restrict__ counts) {
    const uint64_t r = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const int c = lab[r];
    for (int j = lane; j < d; j += 32) atomicAdd(&sums[(uint64_t)c * d + j], (double)X[r * d + j]);
    if (lane == 0) atomicAdd(&counts[c], 1u);
}

__global__ void k_finalize(const double* __restrict__ sums, const unsigned* __restrict__ counts,
                           int k, int d, float* __restrict__ Cc) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)k * d) return;
    const unsigned cnt = counts[e / d];
    if (cnt) Cc[e] = (float)(sums[e] / (double)cnt);
}

// PQ: nearest of 256 codewords per (row, subspace); codebooks [M][256][pq_len].
__global__ void k_pq_assign(const float* __restrict__ X, uint64_t n, int d, int pq_len,
                            const float* __restrict__ cb, uint8_t* __restrict__ out, int out_stride,
                            int* __restrict__ out_int) {
    extern __shared__ float s_cb[];  // [256][pq_len]
    const int m = blockIdx.y;
    for (int e = threadIdx.x; e < kCodes * pq_len; e += blockDim.x)
        s_cb[e] = cb[(uint64_t)m * kCodes * pq_len + e];
    __syncthreads();
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float x[16];
    for (int t = 0; t < pq_len; t++) x[t] = X[r * d + (uint64_t)m * pq_len + t];
    float best = INFINITY;
    int bi = 0;
    for (int c = 0; c < kCodes; c++) {
        float s = 0.f;
        for (int t = 0; t < pq_len; t++) {
            const float df = x[t] - s_cb[c * pq_len + t];
            s = fmaf(df, df, s);
        }
        if (s < best) {
            best = s;
            bi = c;
        }
    }
    if (out) out[r * out_stride + m] = (uint8_t)bi;
    if (out_int) out_int[r * gridDim.y + m] = bi;
}

__global__ void k_pq_accumulate(const float* __restrict__ X, uint64_t n, int d, int pq_len, int M,
                                const int* __restrict__ lab, double* __restrict__ sums,
                                unsigned* __restrict__ counts) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * (uint64_t)M) return;
    const uint64_t r = e / M;
    const int m = (int)(e % M);
    const int c = lab[e];
    const uint64_t base = ((uint64_t)m * kCodes + c) * pq_len;
    for (int t = 0; t < pq_len; t++) atomicAdd(&sums[base + t], (double)X[r * d + (uint64_t)m * pq_len + t]);
    atomicAdd(&counts[(uint64_t)m * kCodes + c], 1u);
}

__global__ void k_gather_rows(const float* __restrict__ X, int d, const uint32_t* __restrict__ rows,
                              uint64_t n_rows, float* __restrict__ out) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_rows * d) return;
    out[e] = X[(uint64_t)rows[e / d] * d + e % d];
}

// Cell coords (shuffled order), flattened cell id and Morton code of every point
// (get_grid_ids_kernel, Super-Grid-IVF_PQ.cu:28-52; encode_points_kernel, zorder.cu:36-43).
__global__ void k_point_cells(const float* __restrict__ labels, uint64_t n, GridMeta g,
                              uint64_t* __restrict__ zcode, uint64_t* __restrict__ cell) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int coords[kMaxDims];
    uint64_t flat = 0;
    for (int i = 0; i < g.l; i++) {
        const float x = labels[r * g.l + g.shuffle[i]];
        int c = grid_id(x, g.left[i], g.span[i], g.grid_dims[i]);
        c = c < g.grid_dims[i] - 1 ? c : g.grid_dims[i] - 1;
        if (c < 0) c = 0;
        coords[i] = c;
        flat += (uint64_t)c * g.cell_stride[i];
    }
    zcode[r] = morton_encode(coords, g.morton_dims, g.morton_max_bits, g.morton_valid_map);
    cell[r] = flat;
}

__global__ void k_count_cells(const uint64_t* __restrict__ cell, const int* __restrict__ list_of,
                              uint64_t n, uint32_t n_lists, uint32_t* __restrict__ prefix) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    atomicAdd(&prefix[cell[r] * n_lists + list_of[r]], 1u);
}

// Counts of the lists [j0, j0 + B) over every cell: dense [cells][B], list fastest.
__global__ void k_count_cells_range(const uint64_t* __restrict__ cell, const int* __restrict__ list_of, uint64_t n,
                                    uint32_t j0, uint32_t B, uint32_t* __restrict__ dense) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t j = (uint32_t)list_of[r];
    if (j >= j0 && j < j0 + B) atomicAdd(&dense[cell[r] * B + (j - j0)], 1u);
}

// Compressed prefix rows (compress_HOPS_data, Super-Grid-IVF_PQ.cu:209-303): the grid's last
// dim of size > 1 (the diff dim, Dd cells, stride 1) runs along a row, every other dim is
// flattened into the row index t, so cell (t, z) is flat t * Dd + z.  For every (t, list j0 + b)
// of the dense inclusive prefix [cells][B] one thread walks z = 0..Dd-1 and keeps the points
// where the value changes.  Without out it writes their number to cnt[t * L + j0 + b]; with out
// it writes them as (z << 32 | value) at out + off[t * L + j0 + b].
__global__ void k_prefix_rows(const uint32_t* __restrict__ dense, uint64_t T, uint32_t Dd, uint32_t B, uint32_t j0,
                              uint32_t L, uint64_t* __restrict__ cnt, const uint64_t* __restrict__ off,
                              uint64_t* __restrict__ out) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T * B) return;
    const uint32_t b = (uint32_t)(e % B);
    const uint64_t t = e / B, r = t * L + j0 + b;
    const uint32_t* p = dense + t * (uint64_t)Dd * B + b;
    uint64_t* o = out ? out + off[r] : nullptr;
    uint32_t prev = 0;
    uint64_t c = 0;
    uint32_t z = 0;
    for (; z + 4 <= Dd; z += 4) {  // four independent loads in flight
        uint32_t v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) v[u] = __ldg(p + (uint64_t)(z + u) * B);
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (v[u] != prev) {
                if (o) o[c] = ((uint64_t)(z + u) << 32) | v[u];
                c++;
                prev = v[u];
            }
    }
    for (; z < Dd; z++) {
        const uint32_t v = __ldg(p + (uint64_t)z * B);
        if (v != prev) {
            if (o) o[c] = ((uint64_t)z << 32) | v;
            c++;
            prev = v;
        }
    }
    if (!out) cnt[r] = c;
}

// Inclusive scan along one grid dim of the cell-major [cells][lists] array.
// One thread per (outer, inner, list) line; consecutive threads = consecutive lists.
__global__ void k_scan_axis(uint32_t* __restrict__ prefix, uint64_t n_lines, uint64_t inner,
                            int axis_len, uint32_t n_lists) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_lines) return;
    const uint64_t list = e % n_lists;
    const uint64_t line = e / n_lists;         // (outer, inner) pair
    const uint64_t in = line % inner, out = line / inner;
    const uint64_t base = (out * axis_len * inner + in) * n_lists + list;
    const uint64_t step = inner * n_lists;
    uint32_t s = 0;
    for (int a = 0; a < axis_len; a++) {
        s += prefix[base + a * step];
        prefix[base + a * step] = s;
    }
}

// Every point's label ranks packed into 32 bits: dim i's rank (thresholds at or below the
// label, by binary search) at bit i * (bits + 1).
__global__ void k_pack_ranks(const float* __restrict__ labels, uint64_t n, int l, const float* __restrict__ thr,
                             uint32_t stride, IndexDev D, uint32_t* __restrict__ out) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint32_t packed = 0;
    for (int i = 0; i < l; i++) {
        const float x = labels[r * l + i];
        const float* t = thr + (uint64_t)i * stride;
        uint32_t lo = 0, hi = D.rank_n[i];
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (t[mid] <= x) lo = mid + 1;
            else hi = mid;
        }
        packed |= lo << (i * (D.rank_bits + 1));
    }
    out[r] = packed;
}

// codes [n][chunks] (16-byte chunks, row-major) -> [chunks][n]: chunk j of point p at j*n + p
__global__ void k_interleave_codes(const uint4* __restrict__ rows, uint64_t n, uint32_t chunks,
                                   uint4* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * chunks) return;
    const uint64_t j = i / n, p = i - j * n;
    out[i] = rows[p * chunks + j];
}

__global__ void k_gather_codes_labels(const uint8_t* __restrict__ codes_by_id, int M_pad,
                                      const float* __restrict__ labels_by_id, int l,
                                      const uint32_t* __restrict__ ids, uint64_t n,
                                      uint8_t* __restrict__ codes, float* __restrict__ labels) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint64_t id = ids[r];
    const uint4* src = reinterpret_cast<const uint4*>(codes_by_id + id * M_pad);
    uint4* dst = reinterpret_cast<uint4*>(codes + r * M_pad);
    for (int v = 0; v < M_pad / 16; v++) dst[v] = src[v];
    for (int i = 0; i < l; i++) labels[r * l + i] = labels_by_id[id * l + i];
}

__global__ void k_to_bf16(const float* __restrict__ x, uint64_t n, __nv_bfloat16* __restrict__ y) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) y[e] = __float2bfloat16_rn(x[e]);
}

// ------------------------------------------------------------------------------------
// host helpers
// ------------------------------------------------------------------------------------

static unsigned blocks_for(uint64_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }

// Lloyd k-means on device rows Xs [ns x d]; centres initialised from the first k rows.
// Returns the centres (device, [k x d]).
static void kmeans_device(const float* Xs, uint64_t ns, int d, int k, int iters, std::mt19937_64& rng,
                          float* centers, cudaStream_t st) {
    DevMem<int> lab(ns);
    DevMem<float> cnorm(k);
    DevMem<double> sums((uint64_t)k * d);
    DevMem<unsigned> counts(k);
    CK(cudaMemcpyAsync(centers, Xs, sizeof(float) * k * d, cudaMemcpyDeviceToDevice, st));
    std::vector<unsigned> h_counts(k);
    for (int it = 0; it < iters; it++) {
        k_row_norms<<<blocks_for(k, 8), 256, 0, st>>>(centers, k, d, cnorm.p);
        k_assign_nearest<<<blocks_for(ns, AT_P), 256, 0, st>>>(Xs, ns, d, centers, cnorm.p, k, lab.p);
        CK(cudaMemsetAsync(sums.p, 0, sizeof(double) * k * d, st));
        CK(cudaMemsetAsync(counts.p, 0, sizeof(unsigned) * k, st));
        k_accumulate<<<blocks_for(ns, 8), 256, 0, st>>>(Xs, ns, d, lab.p, sums.p, counts.p);
        k_finalize<<<blocks_for((uint64_t)k * d, 256), 256, 0, st>>>(sums.p, counts.p, k, d, centers);
        CK(cudaMemcpyAsync(h_counts.data(), counts.p, sizeof(unsigned) * k, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        // re-seed empty clusters from random sample rows
        for (int c = 0; c < k; c++) {
            if (h_counts[c]) continue;
            const uint64_t r = rng() % ns;
            CK(cudaMemcpyAsync(centers + (uint64_t)c * d, Xs + r * d, sizeof(float) * d,
                               cudaMemcpyDeviceToDevice, st));
        }
    }
    CK_LAUNCH();
}

// Capacity-balanced k-means of the fine centroids into C groups of exactly S members
// (stands in for RAFT kmeans_balanced, whose exact algorithm is not vendored).
static void balanced_groups(const std::vector<float>& sub, int L, int d, int C, int S, int iters,
                            std::mt19937_64& rng, std::vector<float>& centers,
                            std::vector<int>& group) {
    centers.assign((size_t)C * d, 0.f);
    std::vector<int> perm(L);
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    for (int c = 0; c < C; c++)
        std::copy(sub.begin() + (size_t)perm[c] * d, sub.begin() + (size_t)(perm[c] + 1) * d,
                  centers.begin() + (size_t)c * d);
    group.assign(L, 0);
    std::vector<std::pair<float, uint64_t>> pairs((size_t)L * C);
    for (int it = 0; it < iters; it++) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < L; i++)
            for (int c = 0; c < C; c++) {
                float s = 0.f;
                for (int j = 0; j < d; j++) {
                    const float df = sub[(size_t)i * d + j] - centers[(size_t)c * d + j];
                    s += df * df;
                }
                pairs[(size_t)i * C + c] = {s, (uint64_t)i * C + c};
            }
        std::sort(pairs.begin(), pairs.end());
        std::vector<int> cap(C, S), done(L, 0);
        int left = L;
        for (const auto& pr : pairs) {
            const int i = (int)(pr.second / C), c = (int)(pr.second % C);
            if (done[i] || cap[c] == 0) continue;
            group[i] = c;
            done[i] = 1;
            cap[c]--;
            if (--left == 0) break;
        }
        std::vector<double> acc((size_t)C * d, 0.0);
        std::vector<int> cnt(C, 0);
        for (int i = 0; i < L; i++) {
            cnt[group[i]]++;
            for (int j = 0; j < d; j++) acc[(size_t)group[i] * d + j] += sub[(size_t)i * d + j];
        }
        for (int c = 0; c < C; c++)
            if (cnt[c])
                for (int j = 0; j < d; j++)
                    centers[(size_t)c * d + j] = (float)(acc[(size_t)c * d + j] / cnt[c]);
    }
}

// Grid shape: calc_grid_shape (Super-Grid-IVF_PQ.cu:305-412), including its integer/float
// conversions.  A dim whose span is 0 gets span 1 (the reference divides by zero there).
GridMeta compute_grid_shape(const std::vector<float>& mins, const std::vector<float>& maxs, int l,
                            uint64_t max_grids, uint64_t label_mask_bits) {
    GridMeta g;
    g.l = l;
    const uint8_t mask = (uint8_t)label_mask_bits;
    const uint8_t label_mask = (uint8_t)(~mask);
    int cnt = 0;
    for (int i = 0; i < l; i++)
        if ((label_mask >> i) & 1) cnt++;
    std::vector<std::pair<uint64_t, int>> span_pairs(l);
    for (int i = 0; i < l; i++) {
        // ceil / floor of the f32 extremes and their difference stay in f32: the reference's
        // `ceil(global_max[i]) - floor(global_min[i])` on float elements resolves to the float
        // overloads under nvcc, so a span above 2^24 is rounded to f32 before the cast
        const float mx = std::ceil(maxs[i]), mn = std::floor(mins[i]);
        HDG_REQUIRE(mn >= 0.0f, HDG_ERR_INVALID_ARG,
                    "labels must be non-negative (label dim " + std::to_string(i) + ")");
        const float diff = mx - mn;
        uint64_t span = (uint64_t)diff;
        if (span == 0) span = 1;
        span_pairs[i] = {span, i};
    }
    int main_grids = (int)std::floor(std::sqrt((double)max_grids));
    std::sort(span_pairs.begin(), span_pairs.end());
    if (l == 1) main_grids = (int)std::min<uint64_t>(max_grids, span_pairs[0].first);
    HDG_REQUIRE(main_grids >= 1, HDG_ERR_INVALID_ARG, "max_grids must be >= 1");
    int remain = 1, remain_cnt = cnt - 1, last_valid = l - 1;
    if (l > 1) remain = (int)(max_grids / (uint64_t)main_grids);
    uint8_t morton_mask = 0xff;
    std::vector<int> dims(l, 1);
    for (int i = 0; i < l; i++) {
        const int id = span_pairs[i].second;
        const uint64_t len = span_pairs[i].first;
        if ((label_mask >> id) & 1) {
            if (remain_cnt == 0) {
                last_valid = i;
                continue;
            }
            int dims_len = (int)std::min<uint64_t>(
                (uint64_t)remain,
                std::min<uint64_t>(len, (uint64_t)std::floor(std::pow((double)main_grids,
                                                                      1.0 / (double)(float)(cnt - 1)))));
            if (remain_cnt == 1) dims_len = (int)std::min<uint64_t>((uint64_t)remain, len);
            remain_cnt--;
            HDG_REQUIRE(dims_len >= 1, HDG_ERR_INVALID_ARG, "max_grids too small for the label dims");
            dims[i] = dims_len;
            remain /= dims_len;
        } else {
            morton_mask &= (uint8_t)~(1 << i);
            dims[i] = 1;
        }
    }
    dims[last_valid] = main_grids;
    g.tot_cells = 1;
    for (int i = 0; i < l; i++) {
        g.grid_dims[i] = dims[i];
        g.tot_cells *= (uint64_t)dims[i];
        g.shuffle[i] = span_pairs[i].second;
        g.span[i] = span_pairs[i].first;
        g.left[i] = (uint64_t)std::floor((double)mins[span_pairs[i].second]);
    }
    uint64_t stride = 1;
    for (int i = l - 1; i >= 0; i--) {
        g.cell_stride[i] = stride;
        stride *= (uint64_t)dims[i];
    }
    g.morton_dims = l;
    const int maxd = *std::max_element(dims.begin(), dims.end());
    g.morton_max_bits = (int)std::ceil(std::log2((double)maxd + 1));
    g.morton_valid_map = morton_mask & (uint8_t)((1u << l) - 1);
    g.diff_dim = l - 1;
    for (int i = l - 1; i >= 0; i--)
        if (dims[i] > 1) {
            g.diff_dim = i;
            break;
        }
    int valid = 0;
    for (int i = 0; i < l; i++)
        if ((g.morton_valid_map >> i) & 1) valid++;
    HDG_REQUIRE(valid * g.morton_max_bits <= 63, HDG_ERR_UNSUPPORTED,
                "Morton code wider than 63 bits; lower max_grids");
    return g;
}

// Dense prefix counts up to this size; beyond it the compressed rows.
constexpr uint64_t kDensePrefixMax = 2ull << 30;

// The compressed per-list prefix rows (the reference's compress_HOPS_data form, built per list
// from a dense HOPS scan, Super-Grid-IVF_PQ.cu:209-303, 527-583).  Lists are taken in chunks of
// B whose dense [cells][B] prefix fits a fixed budget: count, scan along every grid dim, then
// one thread per (grid row, list) keeps the change points along the diff dim.  A first round
// counts each row's change points (their exclusive sum over rows t * L + j gives the offsets),
// a second round rebuilds each chunk and writes the (z << 32 | value) pairs.
static void build_prefix_rows(const GridMeta& g, const uint64_t* d_cell, const int* d_list, uint64_t n, uint32_t L,
                              HostIndex& H, cudaStream_t st) {
    const uint32_t Dd = (uint32_t)g.grid_dims[g.diff_dim];
    HDG_REQUIRE(g.cell_stride[g.diff_dim] == 1 && Dd >= 1 && g.tot_cells % Dd == 0, HDG_ERR_STATE,
                "diff dim of the grid is not its last dim of size > 1");
    const uint64_t T = g.tot_cells / Dd;
    const uint64_t budget = 1ull << 30;
    const uint32_t B = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(L, budget / (g.tot_cells * 4)));
    DevMem<uint32_t> dense(g.tot_cells * B);
    DevMem<uint64_t> cnt(T * L);
    auto chunk = [&](uint32_t j0, uint32_t nb, const uint64_t* off, uint64_t* out) {
        CK(cudaMemsetAsync(dense.p, 0, sizeof(uint32_t) * g.tot_cells * nb, st));
        k_count_cells_range<<<blocks_for(n, 256), 256, 0, st>>>(d_cell, d_list, n, j0, nb, dense.p);
        for (int a = 0; a < g.l; a++) {
            const uint64_t lines = g.tot_cells / (uint64_t)g.grid_dims[a] * nb;
            k_scan_axis<<<blocks_for(lines, 256), 256, 0, st>>>(dense.p, lines, g.cell_stride[a], g.grid_dims[a],
                                                                nb);
        }
        k_prefix_rows<<<blocks_for(T * nb, 128), 128, 0, st>>>(dense.p, T, Dd, nb, j0, L, cnt.p, off, out);
        CK_LAUNCH();
    };
    for (uint32_t j0 = 0; j0 < L; j0 += B) chunk(j0, std::min(B, L - j0), nullptr, nullptr);
    std::vector<uint64_t> hc(T * L);
    CK(cudaMemcpyAsync(hc.data(), cnt.p, sizeof(uint64_t) * hc.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    H.prefix_off.assign(T * L + 1, 0);
    for (uint64_t r = 0; r < T * L; r++) H.prefix_off[r + 1] = H.prefix_off[r] + hc[r];
    const uint64_t E = H.prefix_off.back();
    DevMem<uint64_t> off(T * L + 1), rows(std::max<uint64_t>(E, 1));
    CK(cudaMemcpyAsync(off.p, H.prefix_off.data(), sizeof(uint64_t) * (T * L + 1), cudaMemcpyHostToDevice, st));
    for (uint32_t j0 = 0; j0 < L; j0 += B) chunk(j0, std::min(B, L - j0), off.p, rows.p);
    H.prefix_rows.resize(E);
    if (E) CK(cudaMemcpyAsync(H.prefix_rows.data(), rows.p, sizeof(uint64_t) * E, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    H.prefix.clear();
}

void build_index(hdg_index* idx, const float* d_data, uint64_t n, uint32_t d, const float* d_labels,
                 uint32_t l, cudaStream_t st) {
    const hdg_params& P = idx->params;
    HDG_REQUIRE(d_data && d_labels, HDG_ERR_INVALID_ARG, "null data or labels");
    HDG_REQUIRE((int)l == idx->filter.l, HDG_ERR_INVALID_ARG,
                "label dims differ from filter.conf's l");
    HDG_REQUIRE(P.n_clusters == 256, HDG_ERR_UNSUPPORTED, "only 256-entry PQ codebooks are supported");
    HDG_REQUIRE(P.pq_dim >= 1 && d % P.pq_dim == 0, HDG_ERR_UNSUPPORTED,
                "pq_dim must divide the vector dimension");
    HDG_REQUIRE(d / P.pq_dim <= 16, HDG_ERR_UNSUPPORTED, "pq_len above 16 is not supported");
    const uint64_t C = P.clusters, S = P.sub_clusters, L = C * S;
    HDG_REQUIRE(C >= 1 && S >= 1 && L <= 65536, HDG_ERR_INVALID_ARG, "clusters*sub_clusters out of range");
    HDG_REQUIRE(n >= L && n >= 256 && n < (1ull << 32), HDG_ERR_INVALID_ARG,
                "base set must hold at least max(256, clusters*sub_clusters) points and < 2^32");
    std::mt19937_64 rng(P.seed);
    HostIndex& H = idx->host;
    H = HostIndex();
    H.n = n;
    H.d = d;
    H.l = l;
    H.M = P.pq_dim;
    H.M_pad = align_up(H.M, 16);
    H.pq_len = d / P.pq_dim;
    H.n_lists = L;
    H.C = C;
    const int iters = (int)(P.kmeans_iters ? P.kmeans_iters : 20);

    // ---- 1. grid shape -------------------------------------------------------------
    std::vector<float> hl(n * l);
    CK(cudaMemcpyAsync(hl.data(), d_labels, sizeof(float) * n * l, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<float> mins(l, INFINITY), maxs(l, -INFINITY);
    for (uint64_t r = 0; r < n; r++)
        for (uint32_t i = 0; i < l; i++) {
            mins[i] = std::min(mins[i], hl[r * l + i]);
            maxs[i] = std::max(maxs[i], hl[r * l + i]);
        }
    H.grid = compute_grid_shape(mins, maxs, l, P.max_grids, P.label_mask);
    const GridMeta& g = H.grid;
    // per-list prefix counts: the dense cells x lists array while it stays small, else the
    // compressed rows (PREFIX_ROWS)
    const uint64_t dense_bytes = g.tot_cells * L * 4;
    const bool rows_form = P.prefix_rows == 1 || (P.prefix_rows == 0 && dense_bytes > kDensePrefixMax);
    HDG_REQUIRE(rows_form || dense_bytes <= (16ull << 30), HDG_ERR_UNSUPPORTED,
                "dense prefix-count grid (cells x lists) exceeds 16 GiB; use PREFIX_ROWS or a lower max_grids");

    // ---- sample for training ---------------------------------------------------------
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::shuffle(perm.begin(), perm.end(), rng);
    const uint64_t n_train = std::min<uint64_t>(n, std::max<uint64_t>(65536, 64 * L));
    DevMem<uint32_t> d_perm(n_train);
    CK(cudaMemcpyAsync(d_perm.p, perm.data(), sizeof(uint32_t) * n_train, cudaMemcpyHostToDevice, st));
    DevMem<float> Xs(n_train * d);
    k_gather_rows<<<blocks_for(n_train * d, 256), 256, 0, st>>>(d_data, d, d_perm.p, n_train, Xs.p);

    // ---- 2. PQ codebooks + codes -----------------------------------------------------
    const int M = (int)H.M, pq_len = (int)H.pq_len;
    DevMem<float> pqc((uint64_t)M * kCodes * pq_len);
    {
        const uint64_t n_pq = std::min<uint64_t>(n_train, 65536);
        // initial codewords: first 256 sample rows' slices
        std::vector<float> init((size_t)M * kCodes * pq_len);
        std::vector<float> rows((size_t)kCodes * d);
        CK(cudaMemcpyAsync(rows.data(), Xs.p, sizeof(float) * kCodes * d, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int m = 0; m < M; m++)
            for (int c = 0; c < kCodes; c++)
                for (int t = 0; t < pq_len; t++)
                    init[((size_t)m * kCodes + c) * pq_len + t] = rows[(size_t)c * d + m * pq_len + t];
        CK(cudaMemcpyAsync(pqc.p, init.data(), sizeof(float) * init.size(), cudaMemcpyHostToDevice, st));
        DevMem<int> lab(n_pq * M);
        DevMem<double> sums((uint64_t)M * kCodes * pq_len);
        DevMem<unsigned> counts((uint64_t)M * kCodes);
        std::vector<unsigned> hc((size_t)M * kCodes);
        const size_t smem = sizeof(float) * kCodes * pq_len;
        for (int it = 0; it < iters; it++) {
            k_pq_assign<<<dim3(blocks_for(n_pq, 256), M), 256, smem, st>>>(Xs.p, n_pq, d, pq_len, pqc.p,
                                                                          nullptr, 0, lab.p);
            CK(cudaMemsetAsync(sums.p, 0, sizeof(double) * M * kCodes * pq_len, st));
            CK(cudaMemsetAsync(counts.p, 0, sizeof(unsigned) * M * kCodes, st));
            k_pq_accumulate<<<blocks_for(n_pq * M, 256), 256, 0, st>>>(Xs.p, n_pq, d, pq_len, M, lab.p,
                                                                      sums.p, counts.p);
            k_finalize<<<blocks_for((uint64_t)M * kCodes * pq_len, 256), 256, 0, st>>>(
                sums.p, counts.p, M * kCodes, pq_len, pqc.p);
            CK(cudaMemcpyAsync(hc.data(), counts.p, sizeof(unsigned) * hc.size(), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int m = 0; m < M; m++)
                for (int c = 0; c < kCodes; c++) {
                    if (hc[(size_t)m * kCodes + c]) continue;
                    const uint64_t r = rng() % n_pq;
                    CK(cudaMemcpyAsync(pqc.p + ((uint64_t)m * kCodes + c) * pq_len,
                                       Xs.p + r * d + (uint64_t)m * pq_len, sizeof(float) * pq_len,
                                       cudaMemcpyDeviceToDevice, st));
                }
        }
        H.pq_centers.resize((size_t)M * kCodes * pq_len);
        CK(cudaMemcpyAsync(H.pq_centers.data(), pqc.p, sizeof(float) * H.pq_centers.size(),
                           cudaMemcpyDeviceToHost, st));
    }
    DevMem<uint8_t> codes_by_id(n * H.M_pad);
    CK(cudaMemsetAsync(codes_by_id.p, 0, n * H.M_pad, st));
    k_pq_assign<<<dim3(blocks_for(n, 256), M), 256, sizeof(float) * kCodes * pq_len, st>>>(
        d_data, n, d, pq_len, pqc.p, codes_by_id.p, (int)H.M_pad, nullptr);
    CK_LAUNCH();

    // ---- 3. fine centroids (C*S lists) -------------------------------------------------
    DevMem<float> fine(L * d);
    kmeans_device(Xs.p, n_train, d, (int)L, iters, rng, fine.p, st);
    DevMem<int> list_of_id(n);
    {
        DevMem<float> fnorm(L);
        k_row_norms<<<blocks_for(L, 8), 256, 0, st>>>(fine.p, L, d, fnorm.p);
        k_assign_nearest<<<blocks_for(n, AT_P), 256, 0, st>>>(d_data, n, d, fine.p, fnorm.p, (int)L,
                                                             list_of_id.p);
    }
    std::vector<float> h_fine(L * d);
    CK(cudaMemcpyAsync(h_fine.data(), fine.p, sizeof(float) * L * d, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));

    // ---- 4. group the fine centroids into C clusters of S ------------------------------
    std::vector<int> group;
    balanced_groups(h_fine, (int)L, (int)d, (int)C, (int)S, std::min(iters, 10), rng, H.centers, group);
    // list order: by cluster, then by fine-centroid index (group_by_cluster_id keeps ascending ids)
    std::vector<int> new_of_old(L);
    {
        std::vector<int> order(L);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return group[a] < group[b]; });
        H.sub_centers.resize(L * d);
        for (uint64_t j = 0; j < L; j++) {
            new_of_old[order[j]] = (int)j;
            std::copy(h_fine.begin() + (size_t)order[j] * d, h_fine.begin() + (size_t)(order[j] + 1) * d,
                      H.sub_centers.begin() + j * d);
        }
        H.cluster_off.assign(C + 1, 0);
        for (uint64_t i = 0; i < L; i++) H.cluster_off[group[i] + 1]++;
        for (uint64_t c = 0; c < C; c++) H.cluster_off[c + 1] += H.cluster_off[c];
    }

    // ---- 5. cells, Morton codes, pool order ---------------------------------------------
    DevMem<uint64_t> zc(n), cell(n);
    k_point_cells<<<blocks_for(n, 256), 256, 0, st>>>(d_labels, n, g, zc.p, cell.p);
    std::vector<uint64_t> hz(n);
    std::vector<int> hlist(n);
    CK(cudaMemcpyAsync(hz.data(), zc.p, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hlist.data(), list_of_id.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (uint64_t r = 0; r < n; r++) hlist[r] = new_of_old[hlist[r]];
    H.list_off.assign(L + 1, 0);
    for (uint64_t r = 0; r < n; r++) H.list_off[hlist[r] + 1]++;
    for (uint64_t j = 0; j < L; j++) H.list_off[j + 1] += H.list_off[j];
    H.ids.resize(n);
    {
        std::vector<uint32_t> fill(H.list_off.begin(), H.list_off.end() - 1);
        for (uint64_t r = 0; r < n; r++) H.ids[fill[hlist[r]]++] = (uint32_t)r;  // ascending ids per list
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t j = 0; j < (int64_t)L; j++) {
            auto b = H.ids.begin() + H.list_off[j], e = H.ids.begin() + H.list_off[j + 1];
            std::stable_sort(b, e, [&](uint32_t a, uint32_t c) { return hz[a] < hz[c]; });
        }
    }
    H.zcodes.resize(n);
    for (uint64_t r = 0; r < n; r++) H.zcodes[r] = hz[H.ids[r]];

    // ---- 6. prefix counts ------------------------------------------------------------------
    if (rows_form) {
        DevMem<int> dl(n);
        CK(cudaMemcpyAsync(dl.p, hlist.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        build_prefix_rows(g, cell.p, dl.p, n, (uint32_t)L, H, st);
    } else {
        DevMem<uint32_t> prefix(g.tot_cells * L);
        DevMem<int> dl(n);
        CK(cudaMemcpyAsync(dl.p, hlist.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(prefix.p, 0, sizeof(uint32_t) * g.tot_cells * L, st));
        k_count_cells<<<blocks_for(n, 256), 256, 0, st>>>(cell.p, dl.p, n, (uint32_t)L, prefix.p);
        for (int a = 0; a < g.l; a++) {
            const uint64_t inner = g.cell_stride[a];
            const uint64_t lines = g.tot_cells / (uint64_t)g.grid_dims[a] * L;
            k_scan_axis<<<blocks_for(lines, 256), 256, 0, st>>>(prefix.p, lines, inner, g.grid_dims[a],
                                                                (uint32_t)L);
        }
        H.prefix.resize(g.tot_cells * L);
        CK(cudaMemcpyAsync(H.prefix.data(), prefix.p, sizeof(uint32_t) * H.prefix.size(),
                           cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }

    // ---- pool-ordered codes and labels ---------------------------------------------------
    {
        DevMem<uint32_t> dids(n);
        CK(cudaMemcpyAsync(dids.p, H.ids.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
        DevMem<uint8_t> codes(n * H.M_pad);
        DevMem<float> labels(n * l);
        k_gather_codes_labels<<<blocks_for(n, 256), 256, 0, st>>>(codes_by_id.p, (int)H.M_pad, d_labels,
                                                                 (int)l, dids.p, n, codes.p, labels.p);
        H.codes.resize(n * H.M_pad);
        H.labels.resize(n * l);
        CK(cudaMemcpyAsync(H.codes.data(), codes.p, H.codes.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(H.labels.data(), labels.p, sizeof(float) * H.labels.size(),
                           cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    CK_LAUNCH();
    upload_index(idx, st);
}

// Label-rank thresholds of n rows of l label dims (host memory, row-major [n][l]): per dim,
// the distinct values of a strided sample of at most 262,144 rows when they fit in 2^bits - 1
// thresholds (one rank per value), else the sample's quantiles (equal counts per rank); thr
// [l][2^bits - 1], n_thr [l], and each dim's smallest and largest label over every row.  NaN
// labels are left out of all of them.
void label_rank_thresholds(const float* labels, uint64_t n, int l, int bits, float* thr, uint32_t* n_thr, float* mn,
                           float* mx) {
    const uint32_t stride = (1u << bits) - 1u;
    const uint64_t step = std::max<uint64_t>(1, n / 262144);
#pragma omp parallel for
    for (int i = 0; i < l; i++) {
        std::vector<float> v;
        v.reserve(n / step + 1);
        for (uint64_t r = 0; r < n; r += step) {
            const float x = labels[r * l + i];
            if (!std::isnan(x)) v.push_back(x);
        }
        std::sort(v.begin(), v.end());
        float lo = INFINITY, hi = -INFINITY;  // over every label, not the sample
        for (uint64_t r = 0; r < n; r++) {
            const float x = labels[r * l + i];
            lo = std::min(lo, x);
            hi = std::max(hi, x);
        }
        mn[i] = lo;
        mx[i] = hi;
        std::vector<float> u(v);
        u.erase(std::unique(u.begin(), u.end()), u.end());
        float* t = thr + (size_t)i * stride;
        uint32_t m = 0;
        if (u.size() <= stride + 1) {
            for (size_t k = 1; k < u.size(); k++) t[m++] = u[k];
        } else {
            for (uint32_t k = 1; k <= stride; k++) {
                const float x = v[(size_t)((uint64_t)k * v.size() / (stride + 1))];
                if (m == 0 || x > t[m - 1]) t[m++] = x;
            }
        }
        n_thr[i] = m;
    }
}

// Copy the host index into one device arena and fill idx->dev.
void upload_index(hdg_index* idx, cudaStream_t st) {
    HostIndex& H = idx->host;
    struct Part {
        const void* src;
        size_t bytes;
        void** dst;
    };
    uint16_t* cb = nullptr;
    uint16_t* scb = nullptr;
    float* cn = nullptr;
    IndexDev& D = idx->dev;
    D = IndexDev();
    std::vector<std::pair<size_t, size_t>> offs;
    size_t total = 0;
    auto reserve = [&](size_t bytes) {
        const size_t o = total;
        total += align_up(bytes ? bytes : 1, 256);
        return o;
    };
    const size_t o_c = reserve(H.centers.size() * 4), o_sc = reserve(H.sub_centers.size() * 4);
    const size_t o_cb = reserve(H.centers.size() * 2), o_scb = reserve(H.sub_centers.size() * 2);
    const size_t o_cn = reserve((H.C + H.n_lists) * 4);
    const size_t o_co = reserve(H.cluster_off.size() * 4), o_lo = reserve(H.list_off.size() * 4);
    GridMeta gp = H.grid;
    // label-rank thresholds, so that a rank box is about as tight as the labels
    const int rbits = H.n && !H.labels.empty() ? rank_bits_for((int)H.l) : 0;
    const uint32_t rstride = rbits ? (1u << rbits) - 1u : 0u;
    std::vector<float> rthr((size_t)H.l * rstride);
    uint32_t rn[kMaxDims] = {0};
    float rmin[kMaxDims] = {0.f}, rmax[kMaxDims] = {0.f};
    if (rbits) label_rank_thresholds(H.labels.data(), H.n, (int)H.l, rbits, rthr.data(), rn, rmin, rmax);
    const size_t o_z = reserve(H.zcodes.size() * 8), o_id = reserve(H.ids.size() * 4);
    const size_t o_pk = reserve(rbits ? H.n * 4 : 0), o_rt = reserve(rthr.size() * 4);
    const size_t o_code = reserve(H.codes.size() + 64), o_lab = reserve(H.labels.size() * 4);
    // a dense prefix count never exceeds its list's size: 16 bits suffice when no list passes 65535
    uint32_t max_list = 0;
    for (uint64_t j = 0; j + 1 < H.list_off.size(); j++) max_list = std::max(max_list, H.list_off[j + 1] - H.list_off[j]);
    const bool pre16 = !H.prefix.empty() && max_list <= 0xffffu;
    const size_t o_pq = reserve(H.pq_centers.size() * 4), o_pre = reserve(H.prefix.size() * (pre16 ? 2 : 4));
    const size_t o_poff = reserve(H.prefix_off.size() * 8), o_prow = reserve(H.prefix_rows.size() * 8);
    idx->arena.reset();
    idx->arena.ensure(total);
    char* base = static_cast<char*>(idx->arena.ptr);
    auto up = [&](size_t off, const void* src, size_t bytes) {
        if (bytes) CK(cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st));
        return base + off;
    };
    D.centers = (const float*)up(o_c, H.centers.data(), H.centers.size() * 4);
    D.sub_centers = (const float*)up(o_sc, H.sub_centers.data(), H.sub_centers.size() * 4);
    cb = (uint16_t*)(base + o_cb);
    scb = (uint16_t*)(base + o_scb);
    cn = (float*)(base + o_cn);
    D.cluster_off = (const uint32_t*)up(o_co, H.cluster_off.data(), H.cluster_off.size() * 4);
    D.list_off = (const uint32_t*)up(o_lo, H.list_off.data(), H.list_off.size() * 4);
    D.zcodes = (const uint64_t*)up(o_z, H.zcodes.data(), H.zcodes.size() * 8);
    D.ids = (const uint32_t*)up(o_id, H.ids.data(), H.ids.size() * 4);
    D.labels_nan = std::any_of(H.labels.begin(), H.labels.end(), [](float v) { return std::isnan(v); }) ? 1u : 0u;
    {
        // pool-ordered rows -> 16-byte chunk planes (the scan's coalesced layout)
        DevMem<uint8_t> rows(std::max<size_t>(H.codes.size(), 16));
        if (!H.codes.empty()) {
            CK(cudaMemcpyAsync(rows.p, H.codes.data(), H.codes.size(), cudaMemcpyHostToDevice, st));
            const uint64_t chunks = H.M_pad / 16;
            k_interleave_codes<<<blocks_for(H.n * chunks, 256), 256, 0, st>>>(
                reinterpret_cast<const uint4*>(rows.p), H.n, (uint32_t)chunks, reinterpret_cast<uint4*>(base + o_code));
            CK_LAUNCH();
        }
        CK(cudaStreamSynchronize(st));
        D.codes = (const uint8_t*)(base + o_code);
    }
    D.labels = (const float*)up(o_lab, H.labels.data(), H.labels.size() * 4);
    D.rank_bits = (uint32_t)rbits;
    D.rank_stride = rstride;
    D.rank_guard = D.rank_full = 0;
    for (int i = 0; i < kMaxDims; i++) {
        D.rank_n[i] = i < (int)H.l ? rn[i] : 0u;
        D.rank_min[i] = i < (int)H.l ? rmin[i] : 0.f;
        D.rank_max[i] = i < (int)H.l ? rmax[i] : 0.f;
    }
    for (int i = 0; rbits && i < (int)H.l; i++) {
        D.rank_guard |= 1u << (i * (rbits + 1) + rbits);
        D.rank_full |= rn[i] << (i * (rbits + 1));
    }
    D.rank_thr = rbits ? (const float*)up(o_rt, rthr.data(), rthr.size() * 4) : nullptr;
    D.rankpack = rbits ? reinterpret_cast<const uint32_t*>(base + o_pk) : nullptr;
    if (rbits) {
        k_pack_ranks<<<blocks_for(H.n, 256), 256, 0, st>>>(D.labels, H.n, (int)H.l, D.rank_thr, rstride, D,
                                                         reinterpret_cast<uint32_t*>(base + o_pk));
        CK_LAUNCH();
        CK(cudaStreamSynchronize(st));  // rthr is read by the copy
    }
    D.pq_centers = (const float*)up(o_pq, H.pq_centers.data(), H.pq_centers.size() * 4);
    if (!H.prefix_off.empty()) {  // the compressed rows form
        D.prefix = nullptr;
        D.prefix16 = nullptr;
        D.prefix_off = (const uint64_t*)up(o_poff, H.prefix_off.data(), H.prefix_off.size() * 8);
        D.prefix_rows = (const uint64_t*)up(o_prow, H.prefix_rows.data(), H.prefix_rows.size() * 8);
    } else {
        D.prefix = nullptr;
        D.prefix16 = nullptr;
        if (pre16) {
            std::vector<uint16_t> p16(H.prefix.size());
#pragma omp parallel for
            for (int64_t i = 0; i < (int64_t)H.prefix.size(); i++) p16[i] = (uint16_t)H.prefix[i];
            D.prefix16 = (const uint16_t*)up(o_pre, p16.data(), p16.size() * 2);
            CK(cudaStreamSynchronize(st));  // p16 is read by the copy
        } else {
            D.prefix = (const uint32_t*)up(o_pre, H.prefix.data(), H.prefix.size() * 4);
        }
        D.prefix_off = D.prefix_rows = nullptr;
    }
    k_to_bf16<<<blocks_for(H.centers.size(), 256), 256, 0, st>>>(D.centers, H.centers.size(),
                                                                reinterpret_cast<__nv_bfloat16*>(cb));
    k_to_bf16<<<blocks_for(H.sub_centers.size(), 256), 256, 0, st>>>(
        D.sub_centers, H.sub_centers.size(), reinterpret_cast<__nv_bfloat16*>(scb));
    k_row_norms<<<blocks_for(H.C, 8), 256, 0, st>>>(D.centers, H.C, (int)H.d, cn);
    k_row_norms<<<blocks_for(H.n_lists, 8), 256, 0, st>>>(D.sub_centers, H.n_lists, (int)H.d, cn + H.C);
    D.centers_bf16 = cb;
    D.sub_centers_bf16 = scb;
    D.cnorm = cn;
    D.n = (uint32_t)H.n;
    D.d = (uint32_t)H.d;
    D.l = (uint32_t)H.l;
    D.M = (uint32_t)H.M;
    D.M_pad = (uint32_t)H.M_pad;
    D.pq_len = (uint32_t)H.pq_len;
    D.n_lists = (uint32_t)H.n_lists;
    D.C = (uint32_t)H.C;
    D.S_max = 0;
    for (uint64_t c = 0; c < H.C; c++)
        D.S_max = std::max<uint32_t>(D.S_max, H.cluster_off[c + 1] - H.cluster_off[c]);
    idx->grid = gp;
    CK(cudaStreamSynchronize(st));
    CK_LAUNCH();
    idx->built = true;
    (void)offs;
}

}  // namespace hdg
