// The filtered query path: super_grid::index::query
// (src/index/2-level_index/Super-Grid-IVF_PQ.cu:985-1249) as five B200 kernels.
//
//   k_prologue   per query: filter recovery (preprocessing.cu:3-32) -> f32 box, cell box
//                (:930-961), Morton corners (:903-928, zorder.cu:3-15), per-list filtered
//                counts by 2^d-corner inclusion-exclusion over the dense prefix counts
//                (:693-765) and per-cluster sums (:767-790).
//   k_coarse     per query: exact f32 L2 to the non-empty clusters, top n_list
//                (::refine, :1034-1042); their non-empty lists, exact L2 to the list
//                centroids, top sub_lists (select_sub_clusters, :849-901); Morton interval
//                [lower_bound(zlo), lower_bound(zhi+1)) inside every probed list (zorder.cu:656-685).
//   k_batch      batch sums for the post-filter candidate budget beta (:1198-1222).
//   k_scan       per query: LUT in shared memory (product-quantization.cu:4-35), ADC over the
//                contiguous Z-ordered candidate ranges (:37-77), optional fused label predicate
//                (filter.cu:30-64), block top-K (RAFT select_k in the reference).
//   k_refine     per query: label predicate on the ADC top-n_cand (post-filter, :1227-1236),
//                exact f32 re-rank and top-k (refine.cu:36-120).
// There is no dense [q x max_row_len] candidate table and no host round trip except the
// one scalar read for the batch-wide candidate budget.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include "hdg_device.cuh"
#include "hdg_internal.h"

namespace hdg {

constexpr int kThreads = 256;
constexpr uint32_t kInvalid = 0xffffffffu;
constexpr int kMaxCand = 8192 - kThreads;  // largest ADC top-K kept in shared memory

struct Workspace {
    float* box;              // [q x 2l]
    int* cells;              // [q x 2l]
    uint64_t* zrange;        // [q x 2]
    uint32_t* list_counts;   // [q x L]
    uint32_t* cluster_counts;// [q x C]
    uint32_t* probe_clusters;// [q x Pc]
    uint32_t* probe_lists;   // [q x Ps]
    uint32_t* range_start;   // [q x Ps]
    uint32_t* range_len;     // [q x Ps]
    uint32_t* qstat;         // [q x 4]: cand_total, exact_total, n_lists, n_clusters
    uint64_t* scal;          // [8]
    uint32_t* cand_pool;     // [q x kcand]
    uint32_t* cand_count;    // [q]
    uint64_t kcand;
};

// ------------------------------------------------------------------------------------
// k_prologue
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_prologue(IndexDev D, GridMeta g, FilterDev f,
                                                       const float* __restrict__ qlabels,
                                                       int label_cols, Workspace w) {
    extern __shared__ uint32_t s_counts[];  // [L]
    __shared__ float s_box[2 * kMaxDims];
    __shared__ int s_cells[2 * kMaxDims];
    __shared__ uint64_t s_corner[1 << kMaxDims];
    __shared__ int s_sign[1 << kMaxDims];
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x;
    const int l = g.l;
    const uint32_t L = D.n_lists;
    if (t < l) {
        float lo, hi;
        recover_dim(f, qlabels + qi * label_cols, t, &lo, &hi);
        s_box[2 * t] = lo;
        s_box[2 * t + 1] = hi;
        w.box[qi * 2 * l + 2 * t] = lo;
        w.box[qi * 2 * l + 2 * t + 1] = hi;
    }
    __syncthreads();
    if (t < l) {
        const int od = g.shuffle[t];
        int lo, hi;
        cell_range(s_box[2 * od], s_box[2 * od + 1], g.left[t], g.span[t], g.grid_dims[t], &lo, &hi);
        s_cells[2 * t] = lo;
        s_cells[2 * t + 1] = hi;
        w.cells[qi * 2 * l + 2 * t] = lo;
        w.cells[qi * 2 * l + 2 * t + 1] = hi;
    }
    __syncthreads();
    if (t == 0) {
        int clo[kMaxDims], chi[kMaxDims];
        for (int i = 0; i < l; i++) {
            clo[i] = s_cells[2 * i];
            chi[i] = s_cells[2 * i + 1];
        }
        w.zrange[qi * 2] = morton_encode(clo, g.morton_dims, g.morton_max_bits, g.morton_valid_map);
        w.zrange[qi * 2 + 1] = morton_encode(chi, g.morton_dims, g.morton_max_bits, g.morton_valid_map);
    }
    // corners of the cell box over the valid (unmasked) dims (get_prefix_sum_device :693-724)
    const int dv = __popc(g.morton_valid_map);
    const int n_corner = 1 << dv;
    for (int mask = t; mask < n_corner; mask += blockDim.x) {
        int sign = 1, vi = 0;
        bool zero = false;
        uint64_t flat = 0;
        for (int i = 0; i < l; i++) {
            int c = 0;
            if ((g.morton_valid_map >> i) & 1) {
                if ((mask >> vi) & 1) {
                    c = s_cells[2 * i] - 1;
                    sign = -sign;
                    if (c < 0) zero = true;
                } else {
                    c = s_cells[2 * i + 1];
                }
                vi++;
            }
            flat += (uint64_t)(c < 0 ? 0 : c) * g.cell_stride[i];
        }
        s_corner[mask] = flat;
        s_sign[mask] = zero ? 0 : sign;
    }
    __syncthreads();
    for (uint32_t j = t; j < L; j += blockDim.x) {
        long long acc = 0;
        for (int m = 0; m < n_corner; m++) {
            const int sg = s_sign[m];
            if (sg) acc += (long long)sg * (long long)D.prefix[s_corner[m] * L + j];
        }
        s_counts[j] = (uint32_t)acc;
        w.list_counts[qi * L + j] = (uint32_t)acc;
    }
    __syncthreads();
    for (uint32_t c = t; c < D.C; c += blockDim.x) {
        uint32_t s = 0;
        for (uint32_t j = D.cluster_off[c]; j < D.cluster_off[c + 1]; j++) s += s_counts[j];
        w.cluster_counts[qi * D.C + c] = s;
    }
}

// ------------------------------------------------------------------------------------
// k_coarse
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float seq_l2_v4(const float* __restrict__ q, const float* __restrict__ c,
                                           int d) {
    // sequential f32 sum in dimension order, 16-byte loads of the centroid row
    float s = 0.f;
    const float4* c4 = reinterpret_cast<const float4*>(c);
    for (int i = 0; i < d / 4; i++) {
        const float4 v = __ldg(c4 + i);
        float t0 = __fsub_rn(q[4 * i], v.x);
        s = __fadd_rn(s, __fmul_rn(t0, t0));
        t0 = __fsub_rn(q[4 * i + 1], v.y);
        s = __fadd_rn(s, __fmul_rn(t0, t0));
        t0 = __fsub_rn(q[4 * i + 2], v.z);
        s = __fadd_rn(s, __fmul_rn(t0, t0));
        t0 = __fsub_rn(q[4 * i + 3], v.w);
        s = __fadd_rn(s, __fmul_rn(t0, t0));
    }
    for (int i = d & ~3; i < d; i++) {
        const float t0 = __fsub_rn(q[i], c[i]);
        s = __fadd_rn(s, __fmul_rn(t0, t0));
    }
    return s;
}

__device__ __forceinline__ uint32_t lower_bound_u64(const uint64_t* __restrict__ a, uint32_t n,
                                                    uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kThreads) k_coarse(IndexDev D, const float* __restrict__ queries,
                                                     int Pc, int Ps, int sort_n1, int sort_n2,
                                                     Workspace w) {
    extern __shared__ uint64_t s_keys[];  // [max(sort_n1, sort_n2)] then query vector
    float* s_q = reinterpret_cast<float*>(s_keys + max(sort_n1, sort_n2));
    __shared__ uint32_t s_chosen[1024];
    __shared__ uint32_t s_red[2];
    __shared__ int s_nvalid;
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x;
    const int d = D.d;
    for (int i = t; i < d; i += blockDim.x) s_q[i] = queries[qi * d + i];
    if (t == 0) {
        s_nvalid = 0;
        s_red[0] = s_red[1] = 0;
    }
    __syncthreads();
    // clusters with a non-zero filtered count (filter_none_zero_data :1027-1028)
    for (int c = t; c < sort_n1; c += blockDim.x) {
        uint64_t key = ~0ull;
        if (c < (int)D.C && w.cluster_counts[qi * D.C + c] > 0) {
            key = ((uint64_t)float_key(seq_l2_v4(s_q, D.centers + (uint64_t)c * d, d)) << 32) | (uint32_t)c;
            atomicAdd(&s_nvalid, 1);
        }
        s_keys[c] = key;
    }
    __syncthreads();
    block_bitonic_sort(s_keys, sort_n1);
    const int npc = min(Pc, s_nvalid);
    for (int i = t; i < Pc; i += blockDim.x) {
        const uint32_t c = i < npc ? (uint32_t)s_keys[i] : kInvalid;
        w.probe_clusters[qi * Pc + i] = c;
        if (i < 1024) s_chosen[i] = c;
    }
    __syncthreads();
    if (t == 0) s_nvalid = 0;
    __syncthreads();
    // the non-empty lists of the chosen clusters
    const uint32_t Smax = D.S_max;
    for (int e = t; e < sort_n2; e += blockDim.x) {
        uint64_t key = ~0ull;
        const int i = e / Smax, jj = e % Smax;
        if (i < npc) {
            const uint32_t c = s_chosen[i];
            const uint32_t j = D.cluster_off[c] + jj;
            if (j < D.cluster_off[c + 1] && w.list_counts[qi * D.n_lists + j] > 0) {
                key = ((uint64_t)float_key(seq_l2_v4(s_q, D.sub_centers + (uint64_t)j * d, d)) << 32) | j;
                atomicAdd(&s_nvalid, 1);
            }
        }
        s_keys[e] = key;
    }
    __syncthreads();
    block_bitonic_sort(s_keys, sort_n2);
    const int nps = min(Ps, s_nvalid);
    const uint64_t zlo = w.zrange[qi * 2], zhi = w.zrange[qi * 2 + 1];
    uint32_t my_cand = 0, my_exact = 0;
    for (int i = t; i < Ps; i += blockDim.x) {
        uint32_t list = kInvalid, start = 0, len = 0;
        if (i < nps) {
            list = (uint32_t)s_keys[i];
            const uint32_t off = D.list_off[list], size = D.list_off[list + 1] - off;
            const uint32_t lo = lower_bound_u64(D.zcodes + off, size, zlo);
            const uint32_t hi = lower_bound_u64(D.zcodes + off, size, zhi + 1);
            start = off + lo;
            len = hi - lo;
            my_cand += len;
            my_exact += w.list_counts[qi * D.n_lists + list];
        }
        w.probe_lists[qi * Ps + i] = list;
        w.range_start[qi * Ps + i] = start;
        w.range_len[qi * Ps + i] = len;
    }
    atomicAdd(&s_red[0], my_cand);
    atomicAdd(&s_red[1], my_exact);
    __syncthreads();
    if (t == 0) {
        w.qstat[qi * 4 + 0] = s_red[0];
        w.qstat[qi * 4 + 1] = s_red[1];
        w.qstat[qi * 4 + 2] = nps;
        w.qstat[qi * 4 + 3] = npc;
    }
}

// Batch sums: scal[0] = sum of candidate-range sizes, scal[1] = sum of exact filtered
// counts of the probed lists, scal[2] = max candidates of one query.
__global__ void k_batch(const uint32_t* __restrict__ qstat, uint64_t q, uint64_t* __restrict__ scal) {
    __shared__ unsigned long long s[3];
    if (threadIdx.x == 0) s[0] = s[1] = s[2] = 0;
    __syncthreads();
    unsigned long long a = 0, b = 0, m = 0;
    for (uint64_t i = threadIdx.x; i < q; i += blockDim.x) {
        a += qstat[i * 4];
        b += qstat[i * 4 + 1];
        m = max(m, (unsigned long long)qstat[i * 4]);
    }
    atomicAdd(&s[0], a);
    atomicAdd(&s[1], b);
    atomicMax(&s[2], m);
    __syncthreads();
    if (threadIdx.x == 0) {
        scal[0] = s[0];
        scal[1] = s[1];
        scal[2] = s[2];
    }
}

// ------------------------------------------------------------------------------------
// block top-K over u64 keys (distance key << 32 | payload) in shared memory
// ------------------------------------------------------------------------------------
struct TopK {
    uint64_t* buf;
    int cap;   // power of two, >= K + blockDim
    int K;
    int* cnt;
    uint64_t* thresh;
};

// Called by all threads after a chunk has been appended and the block synchronised.
__device__ __forceinline__ void topk_maybe_compact(TopK& tk, bool force) {
    const int c = *tk.cnt;
    __syncthreads();  // every thread has read the count before anyone appends again
    if (!force && c <= tk.cap - (int)blockDim.x) return;  // uniform decision
    for (int i = c + threadIdx.x; i < tk.cap; i += blockDim.x) tk.buf[i] = ~0ull;
    __syncthreads();
    block_bitonic_sort(tk.buf, tk.cap);
    if (threadIdx.x == 0) {
        const int nc = min(c, tk.K);
        *tk.cnt = nc;
        if (nc == tk.K) *tk.thresh = tk.buf[tk.K - 1];
    }
    __syncthreads();
}

__device__ __forceinline__ void topk_push(TopK& tk, uint64_t key) {
    if (key < *tk.thresh) {
        const int pos = atomicAdd(tk.cnt, 1);
        tk.buf[pos] = key;
    }
}

// ------------------------------------------------------------------------------------
// k_scan: LUT + ADC (+ predicate) + top-K over the Morton candidate ranges
// ------------------------------------------------------------------------------------
enum ScanMode { kPre = 0, kPost = 1, kL1 = 2 };

template <bool kFp16>
__global__ void __launch_bounds__(kThreads) k_scan(IndexDev D, const float* __restrict__ queries,
                                                   int Ps, int mode, int K, int cap, int lbl,
                                                   Workspace w, float* __restrict__ out_dist,
                                                   uint64_t* __restrict__ out_ids, int k_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int M = D.M, pq_len = D.pq_len, d = D.d;
    uint64_t* s_buf = reinterpret_cast<uint64_t*>(smem);                  // [cap]
    float* s_q = reinterpret_cast<float*>(s_buf + cap);                   // [d]
    uint32_t* s_pre = reinterpret_cast<uint32_t*>(s_q + d);               // [Ps + 1]
    uint32_t* s_start = s_pre + (Ps + 1);                                 // [Ps]
    float* s_lut = reinterpret_cast<float*>(s_start + Ps + ((Ps + 1) & 1) + 2);  // [M x 256]
    __half* s_lut16 = reinterpret_cast<__half*>(s_lut);
    __shared__ int s_cnt;
    __shared__ uint64_t s_thresh;
    __shared__ float s_box[2 * kMaxDims];
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x;
    for (int i = t; i < d; i += blockDim.x) s_q[i] = queries[qi * d + i];
    if (t < 2 * lbl) s_box[t] = w.box[qi * 2 * lbl + t];
    if (t == 0) {
        s_cnt = 0;
        s_thresh = ~0ull;
        uint32_t acc = 0;
        for (int i = 0; i < Ps; i++) {
            s_pre[i] = acc;
            acc += w.range_len[qi * Ps + i];
            s_start[i] = w.range_start[qi * Ps + i];
        }
        s_pre[Ps] = acc;
    }
    __syncthreads();
    // LUT[m][c] = sum_t (C[m][c][t] - q[m*pq_len+t])^2, sequential FMA accumulation
    for (int e = t; e < M * kCodes; e += blockDim.x) {
        const int m = e / kCodes;
        const float* cw = D.pq_centers + (uint64_t)e * pq_len;
        float s = 0.f;
        for (int tt = 0; tt < pq_len; tt++) {
            const float df = __fsub_rn(cw[tt], s_q[m * pq_len + tt]);
            s = fmaf(df, df, s);
        }
        if (kFp16)
            s_lut16[e] = __float2half_rn(s);
        else
            s_lut[e] = s;
    }
    __syncthreads();
    TopK tk{s_buf, cap, K, &s_cnt, &s_thresh};
    const uint32_t total = s_pre[Ps];
    const int Mv = D.M_pad / 16;
    for (uint32_t base = 0; base < total; base += blockDim.x) {
        const uint32_t e = base + t;
        if (e < total) {
            // range r with s_pre[r] <= e < s_pre[r+1]
            int lo = 0, hi = Ps - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_pre[mid] <= e)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const uint32_t pool = s_start[lo] + (e - s_pre[lo]);
            bool pass = true;
            if (mode == kPre) {
                const float* lab = D.labels + (uint64_t)pool * lbl;
                for (int i = 0; i < lbl; i++) {
                    const float v = lab[i];
                    if (v < s_box[2 * i] || v > s_box[2 * i + 1]) {
                        pass = false;
                        break;
                    }
                }
            }
            if (pass) {
                const uint4* cp = reinterpret_cast<const uint4*>(D.codes + (uint64_t)pool * D.M_pad);
                float sum = 0.f;
                for (int v = 0; v < Mv; v++) {
                    const uint4 cv = __ldg(cp + v);
                    const uint32_t wv[4] = {cv.x, cv.y, cv.z, cv.w};
#pragma unroll
                    for (int b = 0; b < 16; b++) {
                        const int m = v * 16 + b;
                        if (m < M) {
                            const uint32_t code = (wv[b >> 2] >> (8 * (b & 3))) & 0xffu;
                            sum += kFp16 ? __half2float(s_lut16[m * kCodes + code]) : s_lut[m * kCodes + code];
                        }
                    }
                }
                topk_push(tk, ((uint64_t)float_key(sum) << 32) | pool);
            }
        }
        __syncthreads();
        topk_maybe_compact(tk, false);
    }
    __syncthreads();
    topk_maybe_compact(tk, true);
    const int nres = s_cnt;
    if (mode == kPre) {
        for (int i = t; i < k_out; i += blockDim.x) {
            if (i < nres) {
                const uint64_t key = s_buf[i];
                out_dist[qi * k_out + i] = key_float((uint32_t)(key >> 32));
                out_ids[qi * k_out + i] = D.ids[(uint32_t)key];
            } else {
                out_dist[qi * k_out + i] = INFINITY;
                out_ids[qi * k_out + i] = ~0ull;
            }
        }
    } else {
        for (int i = t; i < K; i += blockDim.x)
            w.cand_pool[qi * w.kcand + i] = i < nres ? (uint32_t)s_buf[i] : kInvalid;
        if (t == 0) w.cand_count[qi] = nres;
    }
}

// ------------------------------------------------------------------------------------
// k_refine: post-filter predicate, exact f32 L2, top-k
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_refine(IndexDev D, const float* __restrict__ queries,
                                                     const float* __restrict__ data, int K, int cap,
                                                     int apply_pred, int lbl, Workspace w,
                                                     float* __restrict__ out_dist,
                                                     uint64_t* __restrict__ out_ids, int k_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(smem);      // [cap]
    uint32_t* s_surv = reinterpret_cast<uint32_t*>(s_keys + cap); // [K]
    float* s_q = reinterpret_cast<float*>(s_surv + K + (K & 1)); // [d]
    __shared__ float s_box[2 * kMaxDims];
    __shared__ int s_ns;
    __shared__ int s_wsum[kThreads / 32];
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int d = D.d;
    for (int i = t; i < d; i += blockDim.x) s_q[i] = queries[qi * d + i];
    if (t < 2 * lbl) s_box[t] = w.box[qi * 2 * lbl + t];
    if (t == 0) s_ns = 0;
    __syncthreads();
    const int nc = min((int)w.cand_count[qi], K);
    // order-preserving compaction of the candidates that pass the predicate
    for (int base = 0; base < nc; base += blockDim.x) {
        const int e = base + t;
        bool keep = false;
        uint32_t pool = kInvalid;
        if (e < nc) {
            pool = w.cand_pool[qi * w.kcand + e];
            keep = pool != kInvalid;
            if (keep && apply_pred) {
                const float* lab = D.labels + (uint64_t)pool * lbl;
                for (int i = 0; i < lbl; i++) {
                    const float v = lab[i];
                    if (v < s_box[2 * i] || v > s_box[2 * i + 1]) {
                        keep = false;
                        break;
                    }
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_wsum[warp] = __popc(bal);
        __syncthreads();
        int before = 0;
        for (int i = 0; i < warp; i++) before += s_wsum[i];
        if (keep) s_surv[s_ns + before + __popc(bal & ((1u << lane) - 1))] = pool;
        __syncthreads();
        if (t == 0) {
            int tot = 0;
            for (int i = 0; i < (int)(blockDim.x / 32); i++) tot += s_wsum[i];
            s_ns += tot;
        }
        __syncthreads();
    }
    const int ns = s_ns;
    // exact distances, one warp per survivor
    for (int i = warp; i < cap; i += blockDim.x / 32) {
        uint64_t key = ~0ull;
        if (i < ns) {
            const uint32_t id = D.ids[s_surv[i]];
            const float* row = data + (uint64_t)id * d;
            float s = 0.f;
            for (int j = lane; j < d; j += 32) {
                const float df = s_q[j] - __ldg(row + j);
                s = fmaf(df, df, s);
            }
            s = warp_sum(s);
            key = ((uint64_t)float_key(s) << 32) | id;
        }
        if (lane == 0) s_keys[i] = key;
    }
    __syncthreads();
    block_bitonic_sort(s_keys, cap);
    for (int i = t; i < k_out; i += blockDim.x) {
        if (i < ns) {
            const uint64_t key = s_keys[i];
            out_dist[qi * k_out + i] = key_float((uint32_t)(key >> 32));
            out_ids[qi * k_out + i] = (uint32_t)key;
        } else {
            out_dist[qi * k_out + i] = INFINITY;
            out_ids[qi * k_out + i] = ~0ull;
        }
    }
}

// ------------------------------------------------------------------------------------
// host orchestration
// ------------------------------------------------------------------------------------
static Workspace carve(hdg_index* idx, uint64_t q, uint64_t kcand, bool record) {
    const hdg_params& P = idx->params;
    const uint64_t l = idx->dev.l, L = idx->dev.n_lists, C = idx->dev.C;
    const uint64_t Pc = std::max<uint64_t>(1, P.n_list), Ps = std::max<uint64_t>(1, P.sub_lists);
    size_t off = 0;
    char* base = static_cast<char*>(idx->work.ptr);
    auto take = [&](const char* name, size_t bytes) -> void* {
        const size_t o = off;
        off += align_up(bytes ? bytes : 1, 256);
        if (record) idx->work_layout[name] = {o, bytes};
        return base ? base + o : nullptr;
    };
    Workspace w{};
    w.box = (float*)take("box", q * 2 * l * 4);
    w.cells = (int*)take("cells", q * 2 * l * 4);
    w.zrange = (uint64_t*)take("zrange", q * 2 * 8);
    w.list_counts = (uint32_t*)take("list_counts", q * L * 4);
    w.cluster_counts = (uint32_t*)take("cluster_counts", q * C * 4);
    w.probe_clusters = (uint32_t*)take("probe_clusters", q * Pc * 4);
    w.probe_lists = (uint32_t*)take("probe_lists", q * Ps * 4);
    w.range_start = (uint32_t*)take("range_start", q * Ps * 4);
    w.range_len = (uint32_t*)take("range_len", q * Ps * 4);
    w.qstat = (uint32_t*)take("qstat", q * 4 * 4);
    w.scal = (uint64_t*)take("scalars", 8 * 8);
    w.cand_count = (uint32_t*)take("cand_count", q * 4);
    w.cand_pool = (uint32_t*)take("cand_pool", q * kcand * 4);
    w.kcand = kcand;
    if (!base) idx->work.bytes = std::max(idx->work.bytes, off);  // size probe
    return w;
}

static size_t workspace_bytes(hdg_index* idx, uint64_t q, uint64_t kcand) {
    size_t off = 0;
    void* saved = idx->work.ptr;
    idx->work.ptr = nullptr;
    const size_t before = idx->work.bytes;
    idx->work.bytes = 0;
    carve(idx, q, kcand, false);
    off = idx->work.bytes;
    idx->work.ptr = saved;
    idx->work.bytes = before;
    return off;
}

void reserve_workspace(hdg_index* idx, uint64_t q, uint64_t kcand) {
    HDG_REQUIRE(idx->built, HDG_ERR_STATE, "index not built");
    const size_t need = workspace_bytes(idx, q, kcand);
    if (idx->work.ptr && idx->work.bytes >= need) return;
    idx->work.reset();
    idx->work.ensure(need);
    idx->work_queries = q;
}

FilterDev filter_dev(const hdg_index* idx) {
    FilterDev f{};
    f.l = idx->filter.l;
    f.filter_dim = (int)std::max<uint64_t>(1, idx->params.filter_dim);
    for (int i = 0; i < kMaxDims; i++) {
        f.type[i] = idx->filter.type[i];
        f.div_value[i] = idx->filter.div_value[i] ? idx->filter.div_value[i] : 1;
        f.shift_val[2 * i] = idx->filter.shift_val[2 * i];
        f.shift_val[2 * i + 1] = idx->filter.shift_val[2 * i + 1];
    }
    f.n_map = (int)idx->filter.interval_map.size();
    f.map = static_cast<const float*>(idx->map_buf.ptr);
    return f;
}

void upload_filter(hdg_index* idx) {
    const auto& m = idx->filter.interval_map;
    idx->map_buf.reset();
    idx->map_buf.ensure(std::max<size_t>(16, m.size() * 4));
    if (!m.empty()) CK(cudaMemcpy(idx->map_buf.ptr, m.data(), m.size() * 4, cudaMemcpyHostToDevice));
}

namespace {
struct StageTimer {
    hdg_index* idx;
    cudaStream_t st;
    bool on;
    std::vector<cudaEvent_t> ev;
    std::vector<std::string> names;
    StageTimer(hdg_index* i, cudaStream_t s, bool enabled) : idx(i), st(s), on(enabled) { mark(""); }
    void mark(const char* name) {
        if (!on) return;
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        CK(cudaEventRecord(e, st));
        ev.push_back(e);
        names.push_back(name);
    }
    void finish() {
        if (!on) return;
        CK(cudaEventSynchronize(ev.back()));
        idx->stage_names.clear();
        idx->stage_ms.clear();
        for (size_t i = 1; i < ev.size(); i++) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[i - 1], ev[i]));
            idx->stage_names.push_back(names[i]);
            idx->stage_ms.push_back(ms);
        }
    }
    ~StageTimer() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};
}  // namespace

void run_query(hdg_index* idx, const float* d_queries, uint64_t q, const float* d_query_labels,
               uint32_t label_cols, const float* d_data, uint32_t k, float* d_dist, uint64_t* d_ids,
               cudaStream_t st) {
    HDG_REQUIRE(idx->built, HDG_ERR_STATE, "index not built");
    HDG_REQUIRE(q > 0 && q < (1ull << 31), HDG_ERR_INVALID_ARG, "query count out of range");
    HDG_REQUIRE(d_queries && d_query_labels && d_dist && d_ids, HDG_ERR_INVALID_ARG, "null pointer");
    HDG_REQUIRE(k >= 1 && k <= 4096, HDG_ERR_INVALID_ARG, "k must be in [1, 4096]");
    const hdg_params& P = idx->params;
    const IndexDev& D = idx->dev;
    const int l = (int)D.l;
    const int fd = (int)std::max<uint64_t>(1, P.filter_dim);
    HDG_REQUIRE(label_cols == (uint32_t)(l * fd), HDG_ERR_INVALID_ARG,
                "query label columns must equal l * filter_dim");
    const int Pc = (int)std::max<uint64_t>(1, P.n_list);
    const int Ps = (int)std::max<uint64_t>(1, P.sub_lists);
    HDG_REQUIRE(Pc <= 1024 && Ps <= 2048, HDG_ERR_UNSUPPORTED, "n_list <= 1024 and sub_lists <= 2048");
    const uint64_t exps0 = P.exps0;
    const int mode = exps0 <= 1 ? kPre : (l > 1 ? kPost : kL1);
    HDG_REQUIRE(mode != kPost || d_data, HDG_ERR_INVALID_ARG, "d_data is required for the re-rank");
    HDG_REQUIRE(mode != kL1 || d_data, HDG_ERR_INVALID_ARG, "d_data is required for the re-rank");
    HDG_REQUIRE(D.n_lists <= 32768, HDG_ERR_UNSUPPORTED, "at most 32768 inverted lists");
    const uint64_t k_l1 = exps0 * k;
    // The candidate buffer is sized for the largest budget up front, so a query never
    // reallocates between its stages (and never allocates once hdg_reserve has run).
    const uint64_t kcand = mode == kPre ? 1 : (uint64_t)kMaxCand;
    if (!idx->work.ptr || idx->work.bytes < workspace_bytes(idx, q, kcand))
        reserve_workspace(idx, q, kcand);
    Workspace w = carve(idx, q, kcand, true);
    const FilterDev f = filter_dev(idx);
    StageTimer tm(idx, st, P.break_down != 0);

    const size_t sm_pro = sizeof(uint32_t) * D.n_lists;
    if (sm_pro > 48 * 1024)
        CK(cudaFuncSetAttribute(k_prologue, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_pro));
    k_prologue<<<(unsigned)q, kThreads, sm_pro, st>>>(D, idx->grid, f, d_query_labels, (int)label_cols, w);
    CK_LAUNCH();
    tm.mark("prologue");

    const int sort_n1 = (int)next_pow2(std::max<uint32_t>(D.C, 2));
    const int sort_n2 = (int)next_pow2(std::max<uint32_t>((uint32_t)Pc * D.S_max, 2));
    const size_t sm_co = sizeof(uint64_t) * std::max(sort_n1, sort_n2) + sizeof(float) * D.d;
    HDG_REQUIRE(sm_co <= 200 * 1024, HDG_ERR_UNSUPPORTED, "coarse selection does not fit shared memory");
    if (sm_co > 48 * 1024)
        CK(cudaFuncSetAttribute(k_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_co));
    k_coarse<<<(unsigned)q, kThreads, sm_co, st>>>(D, d_queries, Pc, Ps, sort_n1, sort_n2, w);
    CK_LAUNCH();
    tm.mark("coarse");

    uint64_t K = k;
    float beta = 0.f;
    if (mode == kPost) {
        k_batch<<<1, 1024, 0, st>>>(w.qstat, q, w.scal);
        CK_LAUNCH();
        uint64_t sc[3];
        CK(cudaMemcpyAsync(sc, w.scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        // beta = coarse / real; n_cand = min(exps0*k*beta, max_row_len) (:1219-1222)
        const uint64_t coarse = sc[0], real = sc[1], max_row = sc[2];
        if (real == 0) {
            K = max_row;
            beta = INFINITY;
        } else {
            beta = (float)coarse / (float)real;
            const float want = (float)(exps0 * (uint64_t)k) * beta;
            const uint64_t nc = want >= 1.8e19f ? ~0ull : (uint64_t)want;
            K = std::min<uint64_t>(nc, max_row);
        }
        tm.mark("budget");
    } else if (mode == kL1) {
        K = k_l1;
    }
    idx->last_ncand = K;
    if (mode != kPre) {
        K = std::min<uint64_t>(K, (uint64_t)kMaxCand);
        if (K == 0) K = 1;
    }
    idx->last_beta = beta;
    idx->last_q = q;

    const int cap = (int)next_pow2((uint32_t)K + kThreads);
    const bool fp16 = P.lut_fp16 != 0;
    const size_t lut_bytes = (size_t)D.M * kCodes * (fp16 ? 2 : 4);
    const size_t sm_scan = sizeof(uint64_t) * cap + sizeof(float) * D.d + sizeof(uint32_t) * (2 * Ps + 4) + 16 +
                           lut_bytes;
    HDG_REQUIRE(sm_scan <= 227 * 1024, HDG_ERR_UNSUPPORTED, "scan working set exceeds shared memory");
    if (fp16) {
        CK(cudaFuncSetAttribute(k_scan<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_scan));
        k_scan<true><<<(unsigned)q, kThreads, sm_scan, st>>>(D, d_queries, Ps, mode, (int)K, cap, l, w,
                                                             d_dist, d_ids, (int)k);
    } else {
        CK(cudaFuncSetAttribute(k_scan<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_scan));
        k_scan<false><<<(unsigned)q, kThreads, sm_scan, st>>>(D, d_queries, Ps, mode, (int)K, cap, l, w,
                                                              d_dist, d_ids, (int)k);
    }
    CK_LAUNCH();
    tm.mark("scan");
    if (mode != kPre) {
        const int rcap = (int)next_pow2((uint32_t)std::max<uint64_t>(K, k));
        const size_t sm_ref = sizeof(uint64_t) * rcap + sizeof(uint32_t) * (K + 1) + sizeof(float) * D.d + 16;
        CK(cudaFuncSetAttribute(k_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_ref));
        k_refine<<<(unsigned)q, kThreads, sm_ref, st>>>(D, d_queries, d_data, (int)K, rcap,
                                                       mode == kPost ? 1 : 0, l, w, d_dist, d_ids, (int)k);
        CK_LAUNCH();
        tm.mark("refine");
    }
    tm.finish();
}

}  // namespace hdg
