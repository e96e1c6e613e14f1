// The filtered query path: super_grid::index::query
// (src/index/2-level_index/Super-Grid-IVF_PQ.cu:985-1249) as B200 kernels.
//
//   k_prologue   per query: filter recovery (preprocessing.cu:3-32) -> f32 box, cell box
//                (:930-961), label-rank box, Morton corners (:903-928, zorder.cu:3-15), per-list filtered
//                counts by 2^d-corner inclusion-exclusion over the dense prefix counts
//                (:693-765) and per-cluster sums (:767-790).
//   k_coarse     per query: exact f32 L2 to the non-empty clusters, top n_list
//                (::refine, :1034-1042); their non-empty lists, exact L2 to the list
//                centroids, top sub_lists (select_sub_clusters, :849-901); Morton interval
//                [lower_bound(zlo), lower_bound(zhi+1)) inside every probed list (zorder.cu:656-685).
//   k_batch      candidate offsets, work items and the batch sums of the post-filter budget
//                beta (:1198-1222).
//   k_pre_scan   predicate-first queries: label-rank box test, then the label predicate
//                (filter.cu:30-64), survivors listed for the ADC (prefiltering.cu:36-51).
//   k_lut        per query PQ lookup table (build_pq_lut_kernel, product-quantization.cu:4-35).
//   k_scan       persistent streaming ADC over the contiguous Z-ordered candidate ranges
//                (compute_batched_L2_distance_kernel, :37-77) with the LUT in shared memory,
//                optional fused label predicate (filter.cu:30-64); one f32 per candidate.
//   k_select     per query: the K smallest (distance, position) pairs (RAFT select_k in the
//                reference) by a two-pass histogram select.
//   k_refine     per query: label predicate on the ADC top-n_cand (post-filter, :1227-1236),
//                exact f32 re-rank and top-k (refine.cu:36-120).
// There is no dense [q x max_row_len] candidate table and one host round trip per batch
// (the candidate total and the batch-wide budget).
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "hdg_device.cuh"
#include "hdg_internal.h"

namespace hdg {

constexpr int kThreads = 256;
constexpr uint32_t kInvalid = 0xffffffffu;
constexpr uint32_t kChunk = 32768;  // default candidates per scan work item (SCAN_CHUNK)
constexpr int kBins = 4096;         // select histogram
constexpr int kBCap = 4096;         // boundary-bin buffer of the select
constexpr uint32_t kPreChunk = 8192; // candidates per work item of the predicate pass

struct Workspace {
    float* box;              // [q x 2l]
    int* cells;              // [q x 2l]
    uint32_t* rank_box;      // [q x 4] rank box (low ranks, high ranks | guard bits), inner box (same)
    uint64_t* zrange;        // [q x 2]
    uint32_t* list_counts;   // [q x L]
    uint32_t* cluster_counts;// [q x C]
    uint32_t* probe_clusters;// [q x Pc]
    uint32_t* probe_lists;   // [q x Ps]
    uint32_t* range_start;   // [q x Ps]
    uint32_t* range_len;     // [q x Ps]
    uint32_t* range_pre;     // [q x (Ps + 1)] exclusive prefix of range_len (last: the candidate total)
    uint32_t* qstat;         // [q x 4]: cand_total, exact_total, n_lists, n_clusters
    uint64_t* scal;          // [8]: cand sum, exact sum, max cand, items, beta (f32 bits),
                             //      queries dropped by a capacity, kept candidates, selected sum
    uint64_t* qoff;          // [q + 1] candidate offsets into dist
    uint32_t* item_off;      // [q + 1] work-item offsets of the ADC scan
    uint32_t* pitem_off;     // [q + 1] work-item offsets of the predicate pass (predicate-first queries)
    uint32_t* mm;            // [q x 2] min / max finite distance key
    uint32_t* nfin;          // [q] finite distances (predicate passed)
    uint32_t* lab_read;      // [q] candidates of the predicate pass whose labels were read
    uint32_t* rank_read;     // [q] candidates of the predicate pass whose label ranks were read
    uint32_t* counter;       // [4] work counters: ADC scan, refine, predicate pass
    float* lut;              // [q x G x 256 x 32] f32, or __half when lut16
    int lut16;               // LUT stored in FP16 (LUT_FP16=1); the scan sums in FP32
    uint32_t* qbud;          // [q] candidate budget n_cand of each query (k_batch)
    uint64_t* soff;          // [q + 1] offsets of the queries' selections in cand_pool
    uint32_t* cand_pool;     // [soff[q]] selected candidates: min(n_cand, candidates) per query
    uint32_t* cand_count;    // [q]
    uint64_t sel_cap;        // cand_pool capacity in entries
    uint32_t* ritem_off;     // [q + 1] refine work-item offsets (k_refine_plan)
    uint32_t* rdone;         // [q] refine items finished per query
    uint32_t* rsurv;         // [q] rows re-ranked exactly per query (predicate survivors of the selection)
    uint32_t* rlab;          // [q] selected entries whose labels the re-rank read (the ranks left them open)
    uint64_t* rpart;         // [refine items x k_max] best keys of each refine item
    int surv_list;           // 1: the predicate pass lists each predicate-first query's survivors
    float* dist;             // [sum of candidates]
    uint32_t* spos;          // [sum of candidates] candidate position of each entry of a compact row
    float* S;                // [q x (C + L)] tensor-core dot products (nullptr: exact path only)
    uint64_t ldS;
    float* qnorm;            // [q] squared query norms
    void* qbf;               // [q x d] bf16 queries
    int* gemm_err;           // tensor-core wait expiry flag
    float* feats;            // [q x 48] learned-schedule features
    uint32_t* lq_ps;         // [q] lists to probe predicted by the learned schedule
    uint8_t* lq_sched;       // [q] predicate-first flag predicted by the learned schedule
    // per-query parameters (nullptr: the batch-wide value)
    const uint32_t* qk;      // [q] k of each query (<= k_max)
    const uint32_t* qps;     // [q] lists probed (<= sub_lists)
    const uint8_t* qsched;   // [q] 0 = the index's reference schedule, 1 = predicate-first + re-rank
    uint32_t k_max;          // output row stride
    int mode;                // batch schedule: 0 pre-filter (exps0 <= 1), 1 post-filter, 2 single dim
    uint32_t exps0;
    uint32_t chunk;          // candidates per scan work item
    int is_split;            // IS_SPLIT: trimmed Morton sub-ranges per probed list
    int nsplit;              // sub-ranges per probed list (n_split when is_split, else 1)
    uint64_t cap;            // distance-buffer capacity in candidates
};

enum ScanMode { kPre = 0, kPost = 1, kL1 = 2 };

__device__ __forceinline__ uint32_t q_k(const Workspace& w, uint64_t qi) {
    return w.qk ? max(1u, min(w.qk[qi], w.k_max)) : w.k_max;
}
__device__ __forceinline__ int q_sched(const Workspace& w, uint64_t qi) { return w.qsched ? (int)w.qsched[qi] : 0; }
// true when query qi evaluates the label predicate inside the scan
__device__ __forceinline__ bool q_prefilter(const Workspace& w, uint64_t qi) {
    return w.mode == kPre || q_sched(w, qi) == 1;
}
// true when query qi's row is compact: the predicate pass lists its survivors (position and
// pool row), the ADC scan replaces each pool row by the survivor's distance
__device__ __forceinline__ bool compacts(const Workspace& w, uint64_t qi) { return w.surv_list && q_prefilter(w, qi); }
// Candidate budget n_cand of query qi given the batch's beta and max_row_len: the query's k for
// the reference pre-filter schedule (exps0 <= 1), exps0 * k for the single-dim schedule and the
// predicate-first schedule, and the reference's min(exps0 * k * beta, max_row_len) for the
// post-filter schedule (Super-Grid-IVF_PQ.cu:1219-1222), with no further cap.  Here k is the
// call's k (the width of the output rows): the reference has one topk per batch, so a batch
// whose queries ask for different k runs as a batch of the largest k whose rows are cut to
// each query's k.  k_batch evaluates it once per query into w.qbud.
__device__ __forceinline__ uint64_t budget_of(const Workspace& w, uint64_t qi, float beta, uint64_t max_row) {
    if (w.mode == kPre) return q_k(w, qi);
    const uint32_t k = w.k_max;
    uint64_t K;
    if (w.mode == kL1 || q_sched(w, qi) == 1) {
        K = (uint64_t)w.exps0 * k;
    } else if (!(beta < INFINITY)) {
        K = max_row;
    } else {
        const float want = (float)((uint64_t)w.exps0 * k) * beta;
        K = want >= 1.8e19f ? ~0ull : (uint64_t)want;
        K = min(K, max_row);
    }
    return max((uint64_t)1, min(K, (uint64_t)0xffffffffu));
}
__device__ __forceinline__ uint32_t q_budget(const Workspace& w, uint64_t qi) { return w.qbud[qi]; }
// A compact row (predicate survivors) that its budget takes whole: the selection is the row
// itself -- its distance slots still hold the survivors' pool rows, as the ADC scan leaves such
// a row alone -- so the select skips it and the re-rank reads the row in place.  (nfin: the
// row's survivors, which the select does not change, unlike cand_count.)
__device__ __forceinline__ bool takes_row(const Workspace& w, uint64_t qi) {
    return compacts(w, qi) && w.nfin[qi] <= q_budget(w, qi);
}
// The selected candidates (pool rows) of query qi: its row of the selection buffer, or its
// distance row when it takes the row whole
__device__ __forceinline__ uint32_t* sel_row(const Workspace& w, uint64_t qi) {
    return takes_row(w, qi) ? reinterpret_cast<uint32_t*>(w.dist + w.qoff[qi]) : w.cand_pool + w.soff[qi];
}

// Warp-wide sum / maximum of a u64 (every lane gets it)
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// Slot of this lane among the lanes of its warp where f holds, taken from the counter *ctr
// with one atomic per warp (~0u where f is false).  Every lane of the warp must call it.
__device__ __forceinline__ uint32_t warp_reserve(bool f, uint32_t* ctr) {
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (!bal) return ~0u;
    const int lane = threadIdx.x & 31, leader = __ffs(bal) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(ctr, (uint32_t)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, leader);
    return f ? base + __popc(bal & ((1u << lane) - 1u)) : ~0u;
}

// Appends v at the next free slot of dst (counter *ctr) where f holds; every lane calls it.
__device__ __forceinline__ void warp_append(bool f, uint32_t v, uint32_t* ctr, uint32_t* dst) {
    const uint32_t slot = warp_reserve(f, ctr);
    if (f) dst[slot] = v;
}

// Inclusive sum of x over the block (blockDim.x a multiple of 32, <= 1024); s_w: 32 words of
// shared scratch that no other thread touches until the following barrier.
__device__ __forceinline__ unsigned long long block_inclusive_sum(unsigned long long x, unsigned long long* s_w,
                                                                  unsigned long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long y = lane < nw ? s_w[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long z = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += z;
        }
        s_w[lane] = y;
    }
    __syncthreads();
    *total = s_w[nw - 1];
    return x + (warp ? s_w[warp - 1] : 0);
}

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
    __shared__ uint32_t s_rank[4];
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x;
    const int l = g.l;
    const uint32_t L = D.n_lists;
    if (t < 4) s_rank[t] = 0;
    if (t < l) {
        float lo, hi;
        recover_dim(f, qlabels + qi * label_cols, t, &lo, &hi);
        s_box[2 * t] = lo;
        s_box[2 * t + 1] = hi;
        w.box[qi * 2 * l + 2 * t] = lo;
        w.box[qi * 2 * l + 2 * t + 1] = hi;
    }
    __syncthreads();
    if (t < l && D.rankpack) {
        // The rank box of label dim t: a rank below that of lo holds labels below a threshold
        // <= lo, a rank above that of hi labels at or above a threshold > hi.  The inner box:
        // ranks whose labels all lie in [lo, hi] -- above the rank of the largest threshold
        // below lo (or every rank when the dim's smallest label is >= lo), and below the rank
        // of hi (or every rank when its largest label is <= hi).  NaN bounds reject nothing.
        const float blo = s_box[2 * t], bhi = s_box[2 * t + 1];
        const float* thr = D.rank_thr + (uint64_t)t * D.rank_stride;
        const uint32_t n = D.rank_n[t];
        auto count = [&](float x, bool le) {  // thresholds <= x (le) or < x
            uint32_t a = 0, b = n;
            while (a < b) {
                const uint32_t m = (a + b) >> 1;
                if (le ? thr[m] <= x : thr[m] < x) a = m + 1;
                else b = m;
            }
            return a;
        };
        const uint32_t rlo = isnan(blo) ? 0u : count(blo, true), rhi = isnan(bhi) ? n : count(bhi, true);
        const int ilo = isnan(blo) || D.rank_min[t] >= blo ? 0 : (int)count(blo, false) + 1;
        const int ihi = isnan(bhi) || D.rank_max[t] <= bhi ? (int)n : (int)rhi - 1;
        const bool empty = ilo > ihi;  // no rank is sure to pass: the field's box [1, 0]
        const int off = t * (int)(D.rank_bits + 1);
        if (rlo) atomicOr(&s_rank[0], rlo << off);
        atomicOr(&s_rank[1], rhi << off);
        if (empty || ilo) atomicOr(&s_rank[2], (empty ? 1u : (uint32_t)ilo) << off);
        if (!empty && ihi) atomicOr(&s_rank[3], (uint32_t)ihi << off);
    }
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
        w.rank_box[qi * 4] = s_rank[0];
        w.rank_box[qi * 4 + 1] = s_rank[1] | D.rank_guard;
        w.rank_box[qi * 4 + 2] = s_rank[2];
        w.rank_box[qi * 4 + 3] = s_rank[3] | D.rank_guard;
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
    if (D.prefix16) {  // dense in 16 bits: eight lists per 16-byte load when L allows, else two per 4 bytes
        if ((L & 7) == 0) {
            for (uint32_t jo = t; 8 * jo < L; jo += blockDim.x) {
                long long a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for (int m = 0; m < n_corner; m++) {
                    const int sg = s_sign[m];
                    if (!sg) continue;
                    const uint4 v = reinterpret_cast<const uint4*>(D.prefix16 + s_corner[m] * L)[jo];
                    const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int h = 0; h < 4; h++) {
                        a[2 * h] += (long long)sg * (long long)(wv[h] & 0xffffu);
                        a[2 * h + 1] += (long long)sg * (long long)(wv[h] >> 16);
                    }
                }
#pragma unroll
                for (int h = 0; h < 8; h++) s_counts[8 * jo + h] = (uint32_t)a[h];
                uint4* lc = reinterpret_cast<uint4*>(w.list_counts + qi * L + 8 * jo);
                lc[0] = make_uint4((uint32_t)a[0], (uint32_t)a[1], (uint32_t)a[2], (uint32_t)a[3]);
                lc[1] = make_uint4((uint32_t)a[4], (uint32_t)a[5], (uint32_t)a[6], (uint32_t)a[7]);
            }
        } else if ((L & 1) == 0) {
            for (uint32_t jp = t; 2 * jp < L; jp += blockDim.x) {
                long long a0 = 0, a1 = 0;
                for (int m = 0; m < n_corner; m++) {
                    const int sg = s_sign[m];
                    if (!sg) continue;
                    const uint32_t v = reinterpret_cast<const uint32_t*>(D.prefix16 + s_corner[m] * L)[jp];
                    a0 += (long long)sg * (long long)(v & 0xffffu);
                    a1 += (long long)sg * (long long)(v >> 16);
                }
                s_counts[2 * jp] = (uint32_t)a0;
                s_counts[2 * jp + 1] = (uint32_t)a1;
                w.list_counts[qi * L + 2 * jp] = (uint32_t)a0;
                w.list_counts[qi * L + 2 * jp + 1] = (uint32_t)a1;
            }
        } else {
            for (uint32_t j = t; j < L; j += blockDim.x) {
                long long acc = 0;
                for (int m = 0; m < n_corner; m++) {
                    const int sg = s_sign[m];
                    if (sg) acc += (long long)sg * (long long)D.prefix16[s_corner[m] * L + j];
                }
                s_counts[j] = (uint32_t)acc;
                w.list_counts[qi * L + j] = (uint32_t)acc;
            }
        }
    } else if (D.prefix) {  // dense: one coalesced row of L counts per corner
        for (uint32_t j = t; j < L; j += blockDim.x) {
            long long acc = 0;
            for (int m = 0; m < n_corner; m++) {
                const int sg = s_sign[m];
                if (sg) acc += (long long)sg * (long long)D.prefix[s_corner[m] * L + j];
            }
            s_counts[j] = (uint32_t)acc;
            w.list_counts[qi * L + j] = (uint32_t)acc;
        }
    } else {
        // compressed rows (query_compressed_sum_device, Super-Grid-IVF_PQ.cu:648-691): the corner
        // at flat cell t * Dd + z reads list j's row t, the last change point at or before z
        const uint32_t Dd = (uint32_t)g.grid_dims[g.diff_dim];
        for (uint32_t j = t; j < L; j += blockDim.x) {
            long long acc = 0;
            for (int m = 0; m < n_corner; m++) {
                const int sg = s_sign[m];
                if (!sg) continue;
                const uint64_t r = (s_corner[m] / Dd) * L + j;
                const uint32_t z = (uint32_t)(s_corner[m] % Dd);
                const uint64_t b0 = D.prefix_off[r];
                uint64_t lo = b0, hi = D.prefix_off[r + 1];
                while (lo < hi) {  // first change point past z
                    const uint64_t mid = (lo + hi) >> 1;
                    if ((uint32_t)(D.prefix_rows[mid] >> 32) <= z) lo = mid + 1;
                    else hi = mid;
                }
                if (lo > b0) acc += (long long)sg * (long long)(uint32_t)D.prefix_rows[lo - 1];
            }
            s_counts[j] = (uint32_t)acc;
            w.list_counts[qi * L + j] = (uint32_t)acc;
        }
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

// N lower_bounds (key k[i] in the sorted a[i][0, n[i])) with their searches interleaved so the
// dependent loads overlap; each result equals lower_bound_u64's
template <int N>
__device__ __forceinline__ void lower_bound_u64_multi(const uint64_t* const (&a)[N], const uint32_t (&n)[N],
                                                      const uint64_t (&k)[N], uint32_t (&r)[N]) {
    uint32_t lo[N], hi[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        lo[i] = 0;
        hi[i] = n[i];
    }
    for (;;) {
        bool any = false;
        uint64_t v[N];
        uint32_t m[N];
#pragma unroll
        for (int i = 0; i < N; i++) {
            m[i] = (lo[i] + hi[i]) >> 1;
            v[i] = lo[i] < hi[i] ? a[i][m[i]] : 0;
        }
#pragma unroll
        for (int i = 0; i < N; i++) {
            if (lo[i] < hi[i]) {
                if (v[i] < k[i]) lo[i] = m[i] + 1;
                else hi[i] = m[i];
            }
            any |= lo[i] < hi[i];
        }
        if (!any) break;
    }
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = lo[i];
}

// One sub-range of a probed list's Morton interval [lo, hi) when is_split = 1.
// get_query_end_points_kernel (zorder.cu:596-654) cuts the interval into
// min(len, n_split) near-equal parts; zorder_range_query_kernel (:474-594) then moves each
// part's start forward by up to three next-in-box jumps and drops the part when a jump fails
// or lands past the part's last code.  (The reference reads the probed list as
// candidates[c] instead of candidates[q * n + c], :500; the list of this query is used.)
// Empty parts get start kInvalid.
__device__ void split_subrange(const uint64_t* __restrict__ z, uint32_t off, uint32_t lo, uint32_t hi, int s,
                               int ns, const int* box, const GridMeta& g, uint32_t* start, uint32_t* len) {
    const uint32_t n = hi - lo;
    const uint32_t nsp = min(n, (uint32_t)ns);
    if (n == 0 || (uint32_t)s >= nsp) {
        *start = kInvalid;
        *len = 0;
        return;
    }
    const uint32_t qn = n / nsp, r = n % nsp;
    uint32_t a = off + lo + (uint32_t)s * qn + min((uint32_t)s, r);
    const uint32_t b = a + qn + ((uint32_t)s < r ? 1u : 0u);
    const uint64_t zmax = z[b - 1];
    uint64_t cur = z[a];
    bool valid = true;
    for (int jump = 0; jump < 3; jump++) {
        const uint32_t idx = a + lower_bound_u64(z + a, b - a, cur);
        if (idx >= b) break;
        a = idx;
        int c[kMaxDims];
        morton_decode(z[idx], c, g.morton_dims, g.morton_max_bits, g.morton_valid_map);
        if (cells_in_box(c, box, g.morton_dims)) break;
        uint64_t nz = 0;
        if (!next_code_in_box(z[idx], box, g.morton_dims, g.morton_max_bits, g.morton_valid_map, &nz) || nz >= zmax) {
            valid = false;
            break;
        }
        cur = nz;
    }
    *start = a;
    *len = valid ? b - a : 0;
}


// Band [lo, hi] around the exact f32 distance of query qi to centroid col (clusters first,
// then lists) from the tensor-core dot product S: |(|q|^2 + |c|^2 - 2 q.c) - exact| is below
// 2 * 2^-8 |q||c| for BF16-rounded inputs, plus f32 rounding of the norms and sums; the band
// doubles both terms.
__device__ __forceinline__ void approx_band(const IndexDev& D, const Workspace& w, uint64_t qi, uint32_t col,
                                            float* lo, float* hi) {
    coarse_band(w.qnorm[qi], D.cnorm[col], w.S[qi * w.ldS + col], lo, hi);
}

// One block of kCoarseThreads per query: the query's phases are serial (selections, searches),
// so smaller blocks keep more queries in flight per SM
constexpr int kCoarseThreads = 128;
__global__ void __launch_bounds__(kCoarseThreads) k_coarse(IndexDev D, GridMeta g, const float* __restrict__ queries,
                                                     int Pc, int Ps, int sort_n1, int sort_n2,
                                                     Workspace w) {
    extern __shared__ uint64_t s_keys[];  // [max(sort_n1, sort_n2)], then the bands' lows, the query vector
    float* s_lo = reinterpret_cast<float*>(s_keys + max(sort_n1, sort_n2));
    float* s_q = s_lo + max(sort_n1, sort_n2);
    __shared__ uint32_t s_chosen[1024];
    __shared__ uint32_t s_red[2];
    __shared__ uint32_t s_wc[32];
    __shared__ unsigned long long s_scan[32];
    __shared__ uint32_t s_hist[256];
    __shared__ unsigned long long s_sel[4];
    __shared__ int s_nvalid;
    __shared__ float s_bound;
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x;
    const int d = D.d;
    const bool est = w.S != nullptr;  // tensor-core estimates of the centroid distances
    for (int i = t; i < d; i += blockDim.x) s_q[i] = queries[qi * d + i];
    if (t == 0) {
        s_nvalid = 0;
        s_red[0] = s_red[1] = 0;
    }
    __syncthreads();
    // One pass over the clusters: those with a non-zero filtered count (filter_none_zero_data
    // :1027-1028) get a key -- the upper end of their estimate band and the cluster -- and the
    // band's lower end; the others ~0.  When all of them fit in n_list the ranking cannot change
    // the chosen set: no distances needed.
    {
        uint32_t nz = 0;
        for (int c = t; c < sort_n1; c += blockDim.x) {
            uint64_t key = ~0ull;
            if (c < (int)D.C && w.cluster_counts[qi * D.C + c] > 0) {
                float lo = 0.f, hi = 0.f;
                if (est) approx_band(D, w, qi, c, &lo, &hi);
                key = ((uint64_t)float_key(hi) << 32) | (uint32_t)c;
                s_lo[c] = lo;
                nz++;
            }
            s_keys[c] = key;
        }
        nz = __reduce_add_sync(0xffffffffu, nz);  // one shared atomic per warp
        if ((t & 31) == 0 && nz) atomicAdd(&s_nvalid, (int)nz);
    }
    __syncthreads();
    const bool all_c = s_nvalid <= Pc;
    // With the tensor-core estimates, only clusters whose lower bound is below the n_list-th
    // smallest upper bound can be in the exact top n_list; only those get exact distances.
    const bool prune_c = !all_c && est;
    if (prune_c) {
        const uint64_t kth = block_select_smallest(s_keys, sort_n1, Pc, s_hist, s_wc, s_sel, false);
        if (t == 0) s_bound = key_float((uint32_t)(kth >> 32));
        __syncthreads();
    }
    for (int c = t; c < sort_n1; c += blockDim.x) {
        uint64_t key = s_keys[c];
        if (key != ~0ull) {
            if (all_c) key = (uint32_t)key;
            else if (prune_c && s_lo[c] > s_bound) key = ~0ull;
            else key = ((uint64_t)float_key(seq_l2_v4(s_q, D.centers + (uint64_t)c * d, d)) << 32) | (uint32_t)c;
        }
        s_keys[c] = key;
    }
    __syncthreads();
    // with every non-empty cluster taken the keys hold no distance: cluster order, compacted;
    // otherwise the n_list smallest (distance, cluster) keys, a set in no particular order
    if (all_c) block_compact_keys(s_keys, sort_n1, s_wc);
    else block_select_smallest(s_keys, sort_n1, Pc, s_hist, s_wc, s_sel);
    const int npc = min(Pc, s_nvalid);
    for (int i = t; i < Pc; i += blockDim.x) {
        const uint32_t c = i < npc ? (uint32_t)s_keys[i] : kInvalid;
        w.probe_clusters[qi * Pc + i] = c;
        if (i < 1024) s_chosen[i] = c;
    }
    __syncthreads();
    if (t == 0) s_nvalid = 0;
    __syncthreads();
    // the same for the non-empty lists of the chosen clusters
    const uint32_t Smax = D.S_max;
    // list slot e = chosen cluster e / Smax, its list e % Smax (shifts when Smax is a power of two)
    const bool sm_pow2 = (Smax & (Smax - 1)) == 0;
    const int sm_shift = __ffs((int)Smax) - 1;
    {
        uint32_t nzl = 0;
        for (int e = t; e < sort_n2; e += blockDim.x) {
            uint64_t key = ~0ull;
            const int i = sm_pow2 ? (e >> sm_shift) : e / (int)Smax, jj = sm_pow2 ? (e & (int)(Smax - 1)) : e % (int)Smax;
            if (i < npc) {
                const uint32_t c = s_chosen[i], j = D.cluster_off[c] + jj;
                if (j < D.cluster_off[c + 1] && w.list_counts[qi * D.n_lists + j] > 0) {
                    float lo = 0.f, hi = 0.f;
                    if (est) approx_band(D, w, qi, D.C + j, &lo, &hi);
                    key = ((uint64_t)float_key(hi) << 32) | j;
                    s_lo[e] = lo;
                    nzl++;
                }
            }
            s_keys[e] = key;
        }
        nzl = __reduce_add_sync(0xffffffffu, nzl);
        if ((t & 31) == 0 && nzl) atomicAdd(&s_nvalid, (int)nzl);
    }
    __syncthreads();
    // lists probed by this query: sub_lists, or the query's own n_probe when given
    const int Psq = w.qps ? max(1, min(Ps, (int)w.qps[qi])) : Ps;
    const bool all_l = s_nvalid <= Psq;
    const bool prune_l = !all_l && est;
    if (prune_l) {
        const uint64_t kth = block_select_smallest(s_keys, sort_n2, Psq, s_hist, s_wc, s_sel, false);
        if (t == 0) s_bound = key_float((uint32_t)(kth >> 32));
        __syncthreads();
    }
    for (int e = t; e < sort_n2; e += blockDim.x) {
        uint64_t key = s_keys[e];
        if (key != ~0ull) {
            const uint32_t j = (uint32_t)key;
            if (all_l) key = j;
            else if (prune_l && s_lo[e] > s_bound) key = ~0ull;
            else key = ((uint64_t)float_key(seq_l2_v4(s_q, D.sub_centers + (uint64_t)j * d, d)) << 32) | j;
        }
        s_keys[e] = key;
    }
    __syncthreads();
    // every list taken: the keys carry no distance, compacted (in list-id order when the chosen
    // clusters are in cluster order too); otherwise the sub_lists smallest (distance, list) keys
    if (all_l) block_compact_keys(s_keys, sort_n2, s_wc);
    else block_select_smallest(s_keys, sort_n2, Psq, s_hist, s_wc, s_sel);
    const int nps = min(Psq, s_nvalid);
    // the probed lists in list-id (= pool) order, so candidate positions follow pool order:
    // marked in a bitmap over the lists (s_chosen is free again), then emitted word by word
    if (!(all_l && all_c)) {
        if (D.n_lists <= 32u * 1024u) {
            const int W = (int)((D.n_lists + 31) / 32);
            for (int i = t; i < W; i += blockDim.x) s_chosen[i] = 0;
            __syncthreads();
            for (int i = t; i < nps; i += blockDim.x) {
                const uint32_t j = (uint32_t)s_keys[i];
                atomicOr(&s_chosen[j >> 5], 1u << (j & 31));
            }
            __syncthreads();
            unsigned long long run = 0;
            for (int b0 = 0; b0 < W; b0 += blockDim.x) {
                const int i = b0 + t;
                const uint32_t word = i < W ? s_chosen[i] : 0u;
                const unsigned long long x = (unsigned long long)__popc(word);
                unsigned long long tot = 0;
                uint32_t at = (uint32_t)(run + block_inclusive_sum(x, s_scan, &tot) - x);
                for (uint32_t m = word; m; m &= m - 1) s_keys[at++] = (uint32_t)(32 * i + __ffs((int)m) - 1);
                run += tot;
                __syncthreads();  // s_scan is reused by the next chunk
            }
        } else {
            const int sort_n3 = (int)next_pow2_dev((uint32_t)max(nps, 2));
            for (int i = t; i < sort_n3; i += blockDim.x)
                s_keys[i] = i < nps ? (uint64_t)(uint32_t)s_keys[i] : ~0ull;
            __syncthreads();
            block_bitonic_sort(s_keys, sort_n3);
        }
    }
    const uint64_t zlo = w.zrange[qi * 2], zhi = w.zrange[qi * 2 + 1];
    uint32_t my_cand = 0, my_exact = 0;
    const int ns = w.nsplit;
    int box[2 * kMaxDims];
    if (w.is_split)
        for (int i = 0; i < 2 * g.l; i++) box[i] = w.cells[qi * 2 * g.l + i];
    // two probed lists per thread and step: their four Morton bound searches interleaved
    for (int i0 = t; i0 < Ps; i0 += 2 * blockDim.x) {
        const uint64_t* arr[4];
        uint32_t nn[4], rr[4], list[2], off[2];
        uint64_t kk[4];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = i0 + u * (int)blockDim.x;
            uint32_t size = 0;
            list[u] = kInvalid;
            off[u] = 0;
            if (i < nps) {
                list[u] = (uint32_t)s_keys[i];
                off[u] = D.list_off[list[u]];
                size = D.list_off[list[u] + 1] - off[u];
            }
            arr[2 * u] = arr[2 * u + 1] = D.zcodes + off[u];
            nn[2 * u] = nn[2 * u + 1] = size;
            kk[2 * u] = zlo;
            kk[2 * u + 1] = zhi + 1;
        }
        lower_bound_u64_multi<4>(arr, nn, kk, rr);
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = i0 + u * (int)blockDim.x;
            if (i >= Ps) break;
            const uint32_t lo = rr[2 * u], hi = rr[2 * u + 1];
            uint32_t start = 0, len = 0;
            if (i < nps) {
                start = off[u] + lo;
                len = hi - lo;
                my_exact += w.list_counts[qi * D.n_lists + list[u]];
            }
            w.probe_lists[qi * Ps + i] = list[u];
            const uint64_t r0 = (qi * Ps + i) * (uint64_t)ns;
            if (!w.is_split) {
                w.range_start[r0] = start;
                w.range_len[r0] = len;
                my_cand += len;
            } else {
                for (int sp = 0; sp < ns; sp++) {
                    uint32_t st = kInvalid, ln = 0;
                    if (i < nps) split_subrange(D.zcodes, off[u], lo, hi, sp, ns, box, g, &st, &ln);
                    w.range_start[r0 + sp] = st;
                    w.range_len[r0 + sp] = ln;
                    my_cand += ln;
                }
            }
        }
    }
    atomicAdd(&s_red[0], my_cand);
    atomicAdd(&s_red[1], my_exact);
    __syncthreads();
    // the exclusive prefix of the ranges' lengths (its last entry the candidate total): the
    // predicate pass, the scan and the select find a position's range by searching it
    {
        // (the ranges past the probed lists' are empty: their prefix is the total)
        const int Rq = Ps * ns, Rn = nps * ns;
        const uint32_t* len = w.range_len + qi * Rq;
        uint32_t* pre = w.range_pre + qi * (Rq + 1);
        unsigned long long run = 0;
        for (int b0 = 0; b0 < Rn; b0 += blockDim.x) {
            const int i = b0 + t;
            const unsigned long long x = i < Rn ? len[i] : 0;
            unsigned long long tot = 0;
            const unsigned long long inc = block_inclusive_sum(x, s_scan, &tot);
            if (i < Rn) pre[i] = (uint32_t)(run + inc - x);
            run += tot;
            __syncthreads();  // s_scan is reused by the next chunk
        }
        for (int i = Rn + t; i <= Rq; i += blockDim.x) pre[i] = (uint32_t)run;
    }
    if (t == 0) {
        w.qstat[qi * 4 + 0] = s_red[0];
        w.qstat[qi * 4 + 1] = s_red[1];
        w.qstat[qi * 4 + 2] = nps;
        w.qstat[qi * 4 + 3] = npc;
    }
}


// ------------------------------------------------------------------------------------
// k_batch: per-query candidate offsets and work items, batch sums (one block)
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_batch(uint64_t q, Workspace w) {
    __shared__ unsigned long long s_tot[32], s_items[32], s_pitems[32], s_sel[32];
    __shared__ unsigned long long s_red[3], s_drop[2];
    __shared__ float s_beta;
    const int t = threadIdx.x;
    if (t == 0) s_red[0] = s_red[1] = s_red[2] = s_drop[0] = s_drop[1] = 0;
    __syncthreads();
    const uint64_t per = (q + blockDim.x - 1) / blockDim.x;
    const uint64_t b = t * per, e = min(q, b + per);
    // a predicate-first query of the predicate pass has predicate items over its candidates
    // (its ADC items follow from its survivors, k_scan_plan); any other query has ADC items
    auto n_items = [&](uint64_t i, uint32_t c) { return compacts(w, i) ? 0u : (c + w.chunk - 1) / w.chunk; };
    auto n_pitems = [&](uint64_t i, uint32_t c) { return compacts(w, i) ? (c + kPreChunk - 1) / kPreChunk : 0u; };
    unsigned long long cand = 0, items = 0, pitems = 0, exact = 0, mx = 0;
    for (uint64_t i = b; i < e; i++) {
        const uint32_t c = w.qstat[i * 4];
        cand += c;
        items += n_items(i, c);
        pitems += n_pitems(i, c);
        exact += w.qstat[i * 4 + 1];
        mx = max(mx, (unsigned long long)c);
    }
    unsigned long long tot_c = 0, tot_i = 0, tot_p = 0;
    unsigned long long rc = block_inclusive_sum(cand, s_tot, &tot_c) - cand;
    unsigned long long ri = block_inclusive_sum(items, s_items, &tot_i) - items;
    unsigned long long rp = block_inclusive_sum(pitems, s_pitems, &tot_p) - pitems;
    unsigned long long dropped = 0, kept = 0;
    for (uint64_t i = b; i < e; i++) {
        const uint32_t c = w.qstat[i * 4];
        w.qoff[i] = rc;
        w.item_off[i] = (uint32_t)ri;
        w.pitem_off[i] = (uint32_t)rp;
        // queries past the distance capacity (a prefix cut: offsets grow with i) get no
        // candidates; the batch's beta and max_row above still count them
        if (rc + c > w.cap) {
            if (c) {
                w.qstat[i * 4] = 0;
                dropped++;
            }
        } else {
            kept += c;
        }
        ri += n_items(i, c);
        rp += n_pitems(i, c);
        rc += c;
        w.mm[2 * i] = 0xffffffffu;
        w.mm[2 * i + 1] = 0u;
        w.nfin[i] = 0;
        w.lab_read[i] = 0;
        w.rank_read[i] = 0;
        w.cand_count[i] = 0;
    }
    if (e == q && b < e) {
        w.qoff[q] = rc;
        w.item_off[q] = (uint32_t)ri;
        w.pitem_off[q] = (uint32_t)rp;
    }
    // one shared atomic per warp (1,024 threads on one word would serialise)
    cand = warp_sum_u64(cand);
    exact = warp_sum_u64(exact);
    mx = warp_max_u64(mx);
    if ((t & 31) == 0) {
        atomicAdd(&s_red[0], cand);
        atomicAdd(&s_red[1], exact);
        atomicMax(&s_red[2], mx);
    }
    __syncthreads();
    if (t == 0) {
        w.scal[0] = s_red[0];
        w.scal[1] = s_red[1];
        w.scal[2] = s_red[2];
        w.scal[3] = tot_i + tot_p;
        // beta = coarse / real as the reference computes it (Super-Grid-IVF_PQ.cu:1219)
        const float beta = s_red[1] == 0 ? INFINITY : __fdiv_rn((float)s_red[0], (float)s_red[1]);
        w.scal[4] = __float_as_uint(beta);
        s_beta = beta;
        w.counter[0] = 0;
        w.counter[2] = 0;
    }
    __syncthreads();
    // each query's budget n_cand, now that the batch's beta and max_row are known, and the
    // offset of its selection (min(n_cand, candidates) entries) in cand_pool
    const float beta = s_beta;
    const uint64_t max_row = s_red[2];
    unsigned long long sel = 0;
    for (uint64_t i = b; i < e; i++) {
        const uint64_t K = budget_of(w, i, beta, max_row);
        w.qbud[i] = (uint32_t)K;
        sel += min(K, (uint64_t)w.qstat[i * 4]);
    }
    unsigned long long tot_s = 0;
    unsigned long long rs = block_inclusive_sum(sel, s_sel, &tot_s) - sel;
    for (uint64_t i = b; i < e; i++) {
        const uint32_t c = w.qstat[i * 4];
        const uint64_t si = min((uint64_t)w.qbud[i], (uint64_t)c);
        w.soff[i] = rs;
        if (rs + si > w.sel_cap && c) {  // past the selection capacity: no candidates either
            w.qstat[i * 4] = 0;
            dropped++;
            kept -= c;
        }
        rs += si;
    }
    if (e == q && b < e) w.soff[q] = rs;
    dropped = warp_sum_u64(dropped);
    kept = warp_sum_u64(kept);
    if ((t & 31) == 0) {
        atomicAdd(&s_drop[0], dropped);
        atomicAdd(&s_drop[1], kept);
    }
    __syncthreads();
    if (t == 0) {
        w.scal[5] = s_drop[0];
        w.scal[6] = s_drop[1];
        w.scal[7] = tot_s;
    }
}

// ------------------------------------------------------------------------------------
// k_lut: LUT[q][g][c][j] = sum_t (C[m][c][t] - x[q][m*pq_len + t])^2, m = 32g + j
// (build_pq_lut_kernel, product-quantization.cu:4-35; the reference's `ans += (c-q)*(c-q)`
// is an FMA under nvcc's default contraction), zero for m >= M.
// ------------------------------------------------------------------------------------
constexpr int kLutQ = 64;          // queries per k_lut block
constexpr int kLutMaxPqLen = 6;    // staged codebook group fits shared memory up to this pq_len

// one LUT entry, FP32 or rounded to FP16 (round to nearest even)
__device__ __forceinline__ void store_lut(float* lut, int f16, uint64_t i, float v) {
    if (f16)
        reinterpret_cast<__half*>(lut)[i] = __float2half_rn(v);
    else
        lut[i] = v;
}

// Block = (64 queries, one group of 32 subspaces).  The group's codebook is staged once in
// shared memory as [c*pq_len + t][33] (conflict-free stores from coalesced global reads and
// conflict-free lane reads); lane = subspace column j, so a warp stores one contiguous
// 128-byte LUT row per codeword.
__global__ void __launch_bounds__(512) k_lut(IndexDev D, const float* __restrict__ queries, uint64_t q, int G,
                                             float* __restrict__ lut, int f16, const uint32_t* __restrict__ item_off) {
    extern __shared__ float smem_lut[];
    // a block none of whose queries has ADC work stages nothing
    {
        const uint64_t qt = (uint64_t)blockIdx.x * kLutQ + threadIdx.x;
        const bool need = threadIdx.x < kLutQ && qt < q && item_off[qt + 1] != item_off[qt];
        if (!__syncthreads_or(need)) return;
    }
    const int g = blockIdx.y, pq_len = D.pq_len, d = D.d, M = D.M;
    float* s_cb = smem_lut;                          // [(c * pq_len + t) * 33 + j]
    const int n = 32 * kCodes * pq_len;
    const float* src = D.pq_centers + (uint64_t)(32 * g) * kCodes * pq_len;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int j = e / (kCodes * pq_len), rem = e - j * (kCodes * pq_len);
        s_cb[rem * 33 + j] = (32 * g + j < M) ? __ldg(src + e) : 0.f;
    }
    __syncthreads();
    // one warp per query: lane j keeps the query's slice of subspace 32g+j in registers
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int m = 32 * g + lane;
    const bool real = m < M;
    for (int qq = warp; qq < kLutQ; qq += nw) {
        const uint64_t qi = (uint64_t)blockIdx.x * kLutQ + qq;
        if (qi >= q) break;
        if (item_off[qi + 1] == item_off[qi]) continue;  // no ADC work: no LUT
        float qv[kLutMaxPqLen];
#pragma unroll
        for (int t = 0; t < kLutMaxPqLen; t++)
            qv[t] = (real && t < pq_len) ? queries[qi * d + (uint64_t)m * pq_len + t] : 0.f;
        const uint64_t row0 = (qi * G + g) * (kCodes * 32);
        for (int c = 0; c < kCodes; c++) {
            float s = 0.f;
#pragma unroll
            for (int t = 0; t < kLutMaxPqLen; t++) {
                if (t < pq_len) {
                    const float df = __fsub_rn(s_cb[(c * pq_len + t) * 33 + lane], qv[t]);
                    s = fmaf(df, df, s);
                }
            }
            store_lut(lut, f16, row0 + c * 32 + lane, real ? s : 0.f);
        }
    }
}

// Fallback for long subspaces: one query per block, thread = codeword, transposed store.
__global__ void __launch_bounds__(256) k_lut_plain(IndexDev D, const float* __restrict__ queries, int G,
                                                   float* __restrict__ lut, int f16,
                                                   const uint32_t* __restrict__ item_off) {
    extern __shared__ float s_q[];     // [d]
    __shared__ float s_t[kCodes][33];  // [c][j]
    const uint64_t qi = blockIdx.x;
    if (item_off[qi + 1] == item_off[qi]) return;  // no ADC work: no LUT (block-uniform)
    const int g = blockIdx.y, d = D.d, pq_len = D.pq_len, c = threadIdx.x;
    for (int i = threadIdx.x; i < d; i += blockDim.x) s_q[i] = queries[qi * d + i];
    __syncthreads();
    for (int j = 0; j < 32; j++) {
        const int m = g * 32 + j;
        float s = 0.f;
        if (m < (int)D.M) {
            const float* cw = D.pq_centers + ((uint64_t)m * kCodes + c) * pq_len;
            for (int tt = 0; tt < pq_len; tt++) {
                const float df = __fsub_rn(__ldg(cw + tt), s_q[m * pq_len + tt]);
                s = fmaf(df, df, s);
            }
        }
        s_t[c][j] = s;
    }
    __syncthreads();
    const uint64_t row0 = (qi * G + g) * (kCodes * 32);
    for (int e = threadIdx.x; e < kCodes * 32; e += blockDim.x) store_lut(lut, f16, row0 + e, s_t[e >> 5][e & 31]);
}

// ------------------------------------------------------------------------------------
// k_scan: persistent ADC stream
// ------------------------------------------------------------------------------------
// Shared-memory LUT layout (fast path): for each group g of 32 subspaces a [256][64] f32
// table whose columns 32..63 repeat 0..31.  Lane r rotates its candidate's 32 code bytes of
// the group left by r, so at step s it looks up subspace (r + s) mod 32 at column r + s:
// the 32 lanes of a warp read 32 different banks, the column offset 4*s is an immediate,
// and no wrap-around arithmetic is needed.

// (a0, a1) += (b0, b1) as one packed FP32x2 add (round to nearest, like two FADDs)
__device__ __forceinline__ void add_f32x2(float& a0, float& a1, float b0, float b1) {
    asm("{\n\t.reg .b64 ra, rb;\n\tmov.b64 ra, {%0, %1};\n\tmov.b64 rb, {%2, %3};\n\t"
        "add.rn.f32x2 ra, ra, rb;\n\tmov.b64 {%0, %1}, ra;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "f"(b0), "f"(b1));
}

// rotate 8 words left by R words (out[i] = in[(i + R) & 7]) with selects only
__device__ __forceinline__ void rotate_words(uint32_t (&w)[8], uint32_t R) {
    uint32_t t[8];
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = (R & 1) ? w[(i + 1) & 7] : w[i];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = (R & 2) ? t[(i + 2) & 7] : t[i];
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = (R & 4) ? w[(i + 4) & 7] : w[i];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = t[i];
}

struct ScanShared {
    int item, query;
};

// ADC of one candidate's 32-subspace group g in the fast path's lane-rotated order (the
// same loads, rotation and lookups as the interleaved loop of k_scan_fast)
__device__ __forceinline__ void adc_group1(const uint4* cp, uint64_t n_pts, int g, uint32_t R, uint32_t sh,
                                           uint32_t lane4, const float* s_lut, float& s0, float& s1) {
    const uint4 a = __ldg(cp + (2 * g) * n_pts), b = __ldg(cp + (2 * g + 1) * n_pts);
    uint32_t wv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    rotate_words(wv, R);
    uint32_t x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = __funnelshift_r(wv[i], wv[(i + 1) & 7], sh);
    const char* L = reinterpret_cast<const char*>(s_lut + g * (kCodes * 64));
#pragma unroll
    for (int st = 0; st < 32; st += 2) {
        const uint32_t a0 = __byte_perm(x[st >> 2], lane4, 0x5504u | ((st & 3) << 4));
        const uint32_t a1 = __byte_perm(x[st >> 2], lane4, 0x5504u | (((st + 1) & 3) << 4));
        add_f32x2(s0, s1, reinterpret_cast<const float*>(L + a0)[st], reinterpret_cast<const float*>(L + a1)[st + 1]);
    }
}

// Loads the query's range table (prefix of the range lengths and range starts) into shared
// memory.  All threads; ends with a barrier.
__device__ __forceinline__ void scan_load_query(const Workspace& w, int Ps, int qq, uint32_t* s_pre,
                                                uint32_t* s_start) {
    const uint32_t* pre = w.range_pre + (uint64_t)qq * (Ps + 1);
    for (int i = threadIdx.x; i <= Ps; i += blockDim.x) s_pre[i] = pre[i];
    for (int i = threadIdx.x; i < Ps; i += blockDim.x) s_start[i] = w.range_start[(uint64_t)qq * Ps + i];
    __syncthreads();
}

// ------------------------------------------------------------------------------------
// k_pre_scan: the label predicate of the predicate-first queries, ahead of their ADC
// ------------------------------------------------------------------------------------
// A predicate-first query (query_prefilter, prefiltering.cu:36-51; the learned schedule's
// predicate-first flag) keeps only its candidates that pass the label predicate
// (filter.cu:30-64), and only those need an ADC distance.  This pass runs before the ADC scan:
// one warp per work item (kPreChunk consecutive candidate positions of one query), no
// shared-memory LUT, so it runs at full occupancy and streams the candidates' packed label
// ranks and labels.  A lane tests positions lane, lane + 32, ... of every step of 32 * J:
//   1. the candidate's label ranks against the query's rank box, all dims in one guarded-field
//      range test: a rank outside the box proves that the label test fails, so the candidate
//      is rejected without reading its labels;
//   2. the labels of the other candidates against the query's f32 box, 128 per batch from a
//      per-warp queue, so that a batch's label loads are all useful;
//   3. the survivors are staged per warp and appended to the query's row 32 at a time -- the
//      candidate position into spos and the pool row into the distance slot, which the ADC
//      scan then overwrites with the survivor's distance.
// The row's order depends on timing; the distance of each survivor does not (the ADC order
// follows its position) and the select orders ties by position.
constexpr int kPreThreads = 256;
constexpr int kPreRingWords = 4 * 128 + 2 * 512 + 2 * 64;  // shared words per warp: labels, queue, survivors

// Largest i in [0, n) with a[i] <= key (a nondecreasing, a[0] <= key), by 32-way rounds.
// Every lane of the warp calls it and gets the answer.
__device__ __forceinline__ int warp_find_le(const uint32_t* a, int n, uint32_t key) {
    const int lane = threadIdx.x & 31;
    int lo = 0, len = n;
    while (len > 1) {
        const int step = (len + 31) >> 5;
        const int off = lane * step;
        const bool ok = off < len && a[lo + off] <= key;
        const unsigned b = __ballot_sync(0xffffffffu, ok);  // bit 0 set: a[lo] <= key
        const int j = 31 - __clz(b);
        lo += j * step;
        len = min(step, len - j * step);
    }
    return lo;
}

// Per-warp rings in shared memory: word i of entry s at ring[i * size + s], head h and tail t
// warp-uniform and free-running (entries t - h).

// Appends (a, b) of the lanes where f holds at the ring's tail.  All lanes.
template <uint32_t SIZE>
__device__ __forceinline__ void ring_push(uint32_t* ring, uint32_t& t, bool f, uint32_t a, uint32_t b) {
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (f) {
        const uint32_t s = (t + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u))) & (SIZE - 1);
        ring[s] = a;
        ring[SIZE + s] = b;
    }
    t += __popc(bal);
}

// 16-byte asynchronous global -> shared copy (cp.async, cached in L2 only) and its groups
__device__ __forceinline__ void cp16_async(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One predicate-pass work item: positions [e0, e1) of one query (R ranges, prefix pre, starts
// start; r0 the range of e0).  CHECK: test the rank box first (lo_f / hi_g / gd: the box's low
// ranks, its high ranks with the guard bits set, the guard bits), LAB4: four 16-byte-aligned
// label dims.  qr: [2][512] ring of rank-passed candidates (without CHECK: of survivors), sr:
// [2][64] survivor ring, lst: [128] staged labels (LAB4).  n_chk / n_read: candidates whose
// ranks / labels were read (warp totals).
template <bool CHECK, bool LAB4>
__device__ __forceinline__ void pre_span(const IndexDev& D, int lbl, const float* bx_s, uint32_t lo_f, uint32_t hi_g,
                                         uint32_t gd,
                                         const uint32_t* pre, const uint32_t* start, int R, int r0, uint32_t e0,
                                         uint32_t e1, uint32_t* qr, uint32_t* sr, float4* lst, uint32_t* ctr,
                                         uint32_t* drow, uint32_t* prow, uint32_t& n_read, uint32_t& n_chk) {
    constexpr int J = 8;  // windows of 32 positions in one step
    constexpr uint32_t QS = 512, SS = 64, LB = 128;
    const int lane = threadIdx.x & 31;
    const uint32_t* ranks = D.rankpack;
    const float4* lab4 = reinterpret_cast<const float4*>(D.labels);
    // Position -> pool row (warp-uniform state): the current range rc holds positions up to
    // nb1 (pool row = bc + position), the next non-empty range from nb1 up to nb2 (bn).  A step
    // with at most one range start inside reads the two bases; a window with more (ranges
    // shorter than 32) walks per lane.
    int rc = r0, rn = r0;
    uint32_t nb1 = pre[r0 + 1], bc = start[r0] - pre[r0], nb2 = 0xffffffffu, bn = 0;
    const uint32_t total = pre[R];
    auto find_next = [&]() {  // the first non-empty range after rc (none past the last position)
        int r = nb1 < total ? rc + 1 : R;
        while (r < R && pre[r + 1] == nb1) r++;
        rn = r;
        nb2 = r < R ? pre[r + 1] : 0xffffffffu;
        bn = r < R ? start[r] - nb1 : 0u;
    };
    find_next();
    auto advance_to = [&](uint32_t p) {  // the state at the range of position p
        while (nb1 <= p && nb1 < e1) {
            rc = rn;
            nb1 = nb2;
            bc = bn;
            find_next();
        }
    };
    // (the box stays in shared memory: the label tests are rare and the registers go to loads in flight)
    auto box4 = [&](const float4& v) {
        const float4 b0 = reinterpret_cast<const float4*>(bx_s)[0], b1 = reinterpret_cast<const float4*>(bx_s)[1];
        return !(v.x < b0.x || v.x > b0.y) && !(v.y < b0.z || v.y > b0.w) && !(v.z < b1.x || v.z > b1.y) &&
               !(v.w < b1.z || v.w > b1.w);
    };
    // the label predicate of the candidate at pool row p (a NaN label passes, as in the reference)
    auto label_ok = [&](uint32_t p) -> bool {
        if (LAB4) return box4(__ldg(lab4 + p));
        bool ok = true;
        const float* lab = D.labels + (uint64_t)p * lbl;
        for (int i = 0; i < lbl; i++) {
            const float v = __ldg(lab + i);
            if (v < bx_s[2 * i] || v > bx_s[2 * i + 1]) ok = false;
        }
        return ok;
    };
    // m (<= 32) entries from a ring's head to the query's row: position into spos, pool row
    // into the distance slot
    auto flush = [&](const uint32_t* ring, uint32_t size, uint32_t h, int m) {
        __syncwarp();
        uint32_t at = 0;
        if (lane == 0) at = atomicAdd(ctr, (uint32_t)m);
        at = __shfl_sync(0xffffffffu, at, 0);
        if (lane < m) {
            const uint32_t s = (h + lane) & (size - 1);
            prow[at + lane] = ring[s];
            drow[at + lane] = ring[size + s];
        }
        __syncwarp();
    };
    uint32_t sh = 0, st = 0;
    auto stage_surv = [&](bool f, uint32_t e, uint32_t p) {
        ring_push<SS>(sr, st, f, e, p);
        if (st - sh >= 32) {
            flush(sr, SS, sh, 32);
            sh += 32;
        }
    };
    // Label batches (CHECK): qr holds [qh, qi) whose labels are on their way into lst, then
    // [qi, qt) queued.  issue() starts the next batch's 16-byte label copies (cp.async: no
    // registers held while they fly), consume() tests a batch once its copies have landed.
    uint32_t qh = 0, qi = 0, qt = 0;
    auto issue = [&](uint32_t m) {
        __syncwarp();  // the pushes of every lane are visible
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint32_t k = lane + 32u * u;
            if (LAB4 && k < m) cp16_async(lst + k, lab4 + qr[QS + ((qi + k) & (QS - 1))]);
        }
        if (LAB4) cp_commit();
        qi += m;
    };
    auto consume = [&]() {
        const uint32_t m = qi - qh;
        if (LAB4) cp_wait<0>();
        __syncwarp();  // every lane's copies have landed
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint32_t k = lane + 32u * u;
            const bool v = k < m;
            const uint32_t s = (qh + k) & (QS - 1);
            const uint32_t e = v ? qr[s] : 0u, p = v ? qr[QS + s] : 0u;
            bool ok = false;
            if (v) ok = LAB4 ? box4(lst[k]) : label_ok(p);
            stage_surv(ok, e, p);
        }
        qh = qi;
        __syncwarp();  // lst and the consumed ring slots are free again
    };
    // one pass past the last step drains the queue (a single copy of the label-batch code)
    for (uint32_t eb = e0;; eb += 32u * J) {
        const bool last_pass = eb >= e1;
        if (CHECK) {
            // test the batch in flight, start the next one; drain more only when the ring has no
            // room for this step's pushes (or, after the last step, until it is empty)
            for (;;) {
                if (qi != qh) consume();
                const uint32_t pend = qt - qh;
                if (pend >= LB || (last_pass && pend > 0)) issue(min(LB, pend));
                if (last_pass ? qi == qh : qt - qh <= QS - 32u * J) break;
            }
        }
        if (last_pass) break;
        uint32_t pp[J];
        bool pv[J];
        const uint32_t last = min(e1, eb + 32u * J) - 1;  // the step's last position
        if (last < nb1 && eb + 32u * J <= e1) {  // a whole step inside the current range
#pragma unroll
            for (int j = 0; j < J; j++) {
                pv[j] = true;
                pp[j] = bc + eb + 32u * j + lane;
            }
            advance_to(eb + 32u * J);
        } else if (last < nb2) {  // at most one range starts inside the step
#pragma unroll
            for (int j = 0; j < J; j++) {
                const uint32_t e = eb + 32u * j + lane;
                pv[j] = e < e1;
                pp[j] = pv[j] ? (e < nb1 ? bc : bn) + e : 0u;
            }
            advance_to(eb + 32u * J);
        } else {
#pragma unroll
            for (int j = 0; j < J; j++) {
                const uint32_t p = eb + 32u * j, e = p + lane;  // the window [p, p + 32)
                pv[j] = e < e1;
                uint32_t base;
                if (p + 31u < nb2) {
                    base = e < nb1 ? bc : bn;
                } else {  // two or more ranges start inside the window
                    int r = rc;
                    if (pv[j])
                        while (pre[r + 1] <= e) r++;
                    base = start[r] - pre[r];
                }
                pp[j] = pv[j] ? base + e : 0u;
                advance_to(p + 32u);
            }
        }
        if constexpr (CHECK) {
            uint32_t c[J];
#pragma unroll
            for (int j = 0; j < J; j++) c[j] = pv[j] ? __ldg(ranks + pp[j]) : 0u;
#pragma unroll
            for (int j = 0; j < J; j++) {
                // every field at or above its low bound and at or below its high bound: the
                // guard bit above a field survives both subtractions exactly then
                const uint32_t t = ((c[j] | gd) - lo_f) & (hi_g - c[j]);
                ring_push<QS>(qr, qt, pv[j] && (t & gd) == gd, eb + 32u * j + lane, pp[j]);
            }
        } else {
            if (LAB4) {
                // four 16-byte label loads in flight at a time
#pragma unroll
                for (int j0 = 0; j0 < J; j0 += 4) {
                    float4 v[4];
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        v[j] = pv[j0 + j] ? __ldg(lab4 + pp[j0 + j]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        ring_push<QS>(qr, qt, pv[j0 + j] && box4(v[j]), eb + 32u * (j0 + j) + lane, pp[j0 + j]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < J; j++)
                    ring_push<QS>(qr, qt, pv[j] && label_ok(pp[j]), eb + 32u * j + lane, pp[j]);
            }
            while (qt - qh >= 32) {
                flush(qr, QS, qh, 32);
                qh += 32;
            }
        }
    }
    if (CHECK) {
        n_read += qt;  // every rank-passed candidate had its labels read
        n_chk += e1 - e0;
        for (;;) {
            if (qi != qh) consume();
            if (qt == qh) break;
            issue(min(LB, qt - qh));
        }
        if (st != sh) flush(sr, SS, sh, (int)(st - sh));
    } else {
        n_read += e1 - e0;
        while (qt != qh) {
            const int m = (int)min(32u, qt - qh);
            flush(qr, QS, qh, m);
            qh += (uint32_t)m;
        }
    }
}

// The pass without the rank test (queries with most candidates inside the cell box, or an index
// with NaN labels) is called out of line, so that the hot loop with the test stays compact in
// the instruction cache
template <bool LAB4>
__device__ __noinline__ void pre_span_labels(const IndexDev& D, int lbl, const float* bx_s, const uint32_t* pre,
                                             const uint32_t* start, int R, int r0, uint32_t e0, uint32_t e1,
                                             uint32_t* qr, uint32_t* sr, float4* lst, uint32_t* ctr, uint32_t* drow,
                                             uint32_t* prow, uint32_t& n_read, uint32_t& n_chk) {
    pre_span<false, LAB4>(D, lbl, bx_s, 0u, 0u, 0u, pre, start, R, r0, e0, e1, qr, sr, lst, ctr, drow, prow, n_read,
                          n_chk);
}

template <bool LAB4>
__global__ void __launch_bounds__(kPreThreads, 4) k_pre_scan(IndexDev D, int R, int lbl, uint64_t q, Workspace w) {
    constexpr int NW = kPreThreads / 32;
    extern __shared__ __align__(16) uint32_t s_rings[];  // per warp: staged labels, queue ring, survivor ring
    __shared__ __align__(16) float s_bx[NW][2 * kMaxDims];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const uint32_t n_items = w.pitem_off[q];
    for (;;) {
        __syncwarp();  // the previous item's reads of the warp's tables are done
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(&w.counter[2], 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n_items) break;
        const int qq = warp_find_le(w.pitem_off, (int)q, item);
        const uint32_t total = w.qstat[(uint64_t)qq * 4];
        const uint32_t e0 = (item - w.pitem_off[qq]) * kPreChunk;
        if (e0 >= total) continue;  // a query cut by a capacity
        const uint32_t e1 = min(total, e0 + kPreChunk);
        if (lane < 2 * lbl) s_bx[wp][lane] = w.box[(uint64_t)qq * 2 * lbl + lane];
        // The query's rank box (label ranks: see IndexDev) rejects a candidate whose labels
        // must fail without reading them.  Skipped when it rejects nothing, when the index holds
        // NaN labels (a NaN passes the label test), or when the query's count of points in its
        // cell box over the probed lists says that most candidates pass anyway.
        const uint32_t inbox = w.qstat[(uint64_t)qq * 4 + 1];
        const uint32_t rlo = w.rank_box[4 * qq], rhi = w.rank_box[4 * qq + 1];
        const bool use = D.rankpack && !D.labels_nan && (rlo != 0 || rhi != (D.rank_full | D.rank_guard)) &&
                         (uint64_t)inbox * 16 < (uint64_t)total * 12;
        __syncwarp();  // s_bx is written
        const uint32_t* pre = w.range_pre + (uint64_t)qq * (R + 1);
        const uint32_t* start = w.range_start + (uint64_t)qq * R;
        const int r0 = warp_find_le(pre, R, e0);
        uint32_t* ctr = &w.cand_count[qq];
        uint32_t* drow = reinterpret_cast<uint32_t*>(w.dist + w.qoff[qq]);
        uint32_t* prow = w.spos + w.qoff[qq];
        uint32_t n_read = 0, n_chk = 0;
        const float* bxs = s_bx[wp];
        float4* lst = reinterpret_cast<float4*>(s_rings + (size_t)wp * kPreRingWords);
        uint32_t* qr = reinterpret_cast<uint32_t*>(lst + 128);
        uint32_t* sr = qr + 2 * 512;
        if (use)
            pre_span<true, LAB4>(D, lbl, bxs, rlo, rhi, D.rank_guard, pre, start, R, r0, e0, e1, qr, sr, lst, ctr,
                                 drow, prow, n_read, n_chk);
        else
            pre_span_labels<LAB4>(D, lbl, bxs, pre, start, R, r0, e0, e1, qr, sr, lst, ctr, drow, prow, n_read,
                                  n_chk);
        if (lane == 0 && n_read) atomicAdd(&w.lab_read[qq], n_read);
        if (lane == 0 && n_chk) atomicAdd(&w.rank_read[qq], n_chk);
    }
}

// ADC work items once the predicate pass has listed the survivors: a compact row has
// cand_count entries, any other row one per candidate position.  One block.
__global__ void __launch_bounds__(1024) k_scan_plan(uint64_t q, Workspace w) {
    __shared__ unsigned long long s_w[32];
    const int t = threadIdx.x;
    const uint64_t per = (q + blockDim.x - 1) / blockDim.x;
    const uint64_t b = t * per, e = min(q, b + per);
    auto n_items = [&](uint64_t i) {
        uint32_t c = compacts(w, i) ? w.cand_count[i] : w.qstat[i * 4];
        // a compact row that its budget takes whole needs no ADC distance (the select takes
        // every survivor and the re-rank orders them), unless the distances are the output
        // (the reference's pre-filter schedule)
        if (compacts(w, i) && w.mode != kPre && c <= w.qbud[i]) c = 0;
        return (c + w.chunk - 1) / w.chunk;
    };
    // such a row's survivors all count as passed (the ADC scan counts them for the others)
    for (uint64_t i = b; i < e; i++)
        if (compacts(w, i) && w.mode != kPre && w.cand_count[i] <= w.qbud[i]) w.nfin[i] = w.cand_count[i];
    unsigned long long items = 0;
    for (uint64_t i = b; i < e; i++) items += n_items(i);
    unsigned long long tot = 0;
    unsigned long long r = block_inclusive_sum(items, s_w, &tot) - items;
    for (uint64_t i = b; i < e; i++) {
        w.item_off[i] = (uint32_t)r;
        r += n_items(i);
    }
    if (e == q && b < e) w.item_off[q] = (uint32_t)r;
    if (t == 0) w.counter[0] = 0;
}

// Fast path (M a multiple of 32).  The CTA computes the query's LUT straight into shared
// memory when it switches query (codeword-major loads, one subspace per lane), then streams
// candidates; CPT candidates per thread are interleaved step by step so every thread keeps
// CPT independent load->add chains in flight.  A candidate at position e sums from subspace
// (e mod 32) of each group: for a full row that is the lane, for a compact row (the predicate
// pass's survivors) it comes from the survivor's recorded position.
template <int G, int NT, int CPT>
__global__ void __launch_bounds__(NT, (G == 1 && CPT == 1) ? 2 : 1) k_scan_fast(IndexDev D, int Ps, uint64_t q,
                                                                                 Workspace w) {
    extern __shared__ __align__(16) float s_lut[];  // [G][256][64]
    uint32_t* s_pre = reinterpret_cast<uint32_t*>(s_lut + G * kCodes * 64);  // [Ps + 1]
    uint32_t* s_start = s_pre + Ps + 1;                                       // [Ps]
    __shared__ ScanShared s;
    const int t = threadIdx.x, lane = t & 31;
    const uint32_t n_items = w.item_off[q];
    int cur = -1;
    for (;;) {
        if (t == 0) {
            const int item = (int)atomicAdd(w.counter, 1u);
            s.item = item;
            if (item < (int)n_items) {  // largest query with item_off <= item
                int lo = 0, hi = (int)q - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (w.item_off[mid] <= (uint32_t)item) lo = mid;
                    else hi = mid - 1;
                }
                s.query = lo;
            }
        }
        __syncthreads();
        const int item = s.item;
        if (item >= (int)n_items) break;
        const int qq = s.query;
        const bool compact = compacts(w, qq);
        const uint32_t total = compact ? w.cand_count[qq] : w.qstat[(uint64_t)qq * 4];
        const uint32_t e0 = (uint32_t)(item - w.item_off[qq]) * w.chunk;
        if (e0 >= total) {  // a query cut by the distance capacity
            __syncthreads();
            continue;
        }
        if (qq != cur) {
            if (w.lut16) {  // FP16 entries widened to FP32 in shared memory
                const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const __half*>(w.lut) +
                                                                  (uint64_t)qq * G * kCodes * 32);
                for (int e = t; e < G * kCodes * 4; e += NT) {
                    const uint4 v = __ldg(src + e);
                    const int row = e >> 2, col = (e & 3) * 8;
                    const __half2* h = reinterpret_cast<const __half2*>(&v);
                    const float2 f0 = __half22float2(h[0]), f1 = __half22float2(h[1]);
                    const float2 f2 = __half22float2(h[2]), f3 = __half22float2(h[3]);
                    float4* dstl = reinterpret_cast<float4*>(s_lut + row * 64 + col);
                    dstl[0] = make_float4(f0.x, f0.y, f1.x, f1.y);
                    dstl[1] = make_float4(f2.x, f2.y, f3.x, f3.y);
                    dstl[8] = dstl[0];
                    dstl[9] = dstl[1];
                }
            } else {
                const float4* src = reinterpret_cast<const float4*>(w.lut + (uint64_t)qq * G * kCodes * 32);
                for (int e = t; e < G * kCodes * 8; e += NT) {
                    const float4 v = __ldg(src + e);
                    const int row = e >> 3, col = (e & 7) * 4;  // row = g*256 + c
                    float4* dstl = reinterpret_cast<float4*>(s_lut + row * 64 + col);
                    dstl[0] = v;
                    dstl[8] = v;  // columns 32..63 repeat 0..31
                }
            }
            // a query's rows are all compact or all full: a compact query needs no range table
            if (!compact) scan_load_query(w, Ps, qq, s_pre, s_start);  // ends with a barrier
            else __syncthreads();
            cur = qq;
        }
        const uint32_t e1 = min(total, e0 + w.chunk);
        float* dst = w.dist + w.qoff[qq];
        const uint32_t* srow = reinterpret_cast<const uint32_t*>(dst);  // compact: the survivors' pool rows
        const uint32_t* sp = w.spos + w.qoff[qq];
        uint32_t kmin = 0xffffffffu, kmax = 0u, nf = 0;
        // each warp takes a contiguous span of the item (a multiple of 32 * CPT entries, so in
        // a full row position mod 32 stays the lane), so a lane's walk to its candidate's range
        // crosses few range boundaries per step
        constexpr uint32_t kStep = 32u * CPT;
        const uint32_t span = ((e1 - e0 + NT / 32 - 1) / (NT / 32) + kStep - 1) / kStep * kStep;
        const uint32_t wb = e0 + (uint32_t)(t >> 5) * span;
        const uint32_t we = min(e1, wb + span);
        int r[CPT];
#pragma unroll
        for (int u = 0; u < CPT; u++) {
            r[u] = 0;
            if (compact) continue;
            const uint32_t e = wb + lane + u * 32;
            int lo = 0, hi = Ps - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_pre[mid] <= e) lo = mid;
                else hi = mid - 1;
            }
            r[u] = lo;
        }
        const uint4* planes = reinterpret_cast<const uint4*>(D.codes);
        const uint64_t n_pts = D.n;
        for (uint32_t eb = wb + lane; eb < we; eb += kStep) {
            const uint4* cp[CPT];
            bool live[CPT];
            uint32_t rot[CPT];
            float sum[CPT], sum1[CPT];  // even / odd steps, added at the end
#pragma unroll
            for (int u = 0; u < CPT; u++) {
                const uint32_t e = eb + u * 32;
                live[u] = e < we;
                sum[u] = sum1[u] = 0.f;
                uint32_t row = 0;  // a dead lane reads row 0 (in bounds), result discarded
                rot[u] = (uint32_t)lane;
                if (live[u]) {
                    if (compact) {
                        row = srow[e];
                        rot[u] = sp[e] & 31u;
                    } else {
                        while (s_pre[r[u] + 1] <= e) r[u]++;
                        row = s_start[r[u]] + (e - s_pre[r[u]]);
                    }
                }
                cp[u] = planes + row;  // chunk j of this point at cp[u][j * n_pts]
            }
#pragma unroll
            for (int g = 0; g < G; g++) {
                uint32_t x[CPT][8];
#pragma unroll
                for (int u = 0; u < CPT; u++) {
                    const uint4 a = __ldg(cp[u] + (2 * g) * n_pts), b = __ldg(cp[u] + (2 * g + 1) * n_pts);
                    uint32_t wv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
                    rotate_words(wv, rot[u] >> 2);
                    const uint32_t sh = 8u * (rot[u] & 3u);
#pragma unroll
                    for (int i = 0; i < 8; i++) x[u][i] = __funnelshift_r(wv[i], wv[(i + 1) & 7], sh);
                }
                const char* L = reinterpret_cast<const char*>(s_lut + g * (kCodes * 64));
#pragma unroll
                for (int st = 0; st < 32; st += 2) {
#pragma unroll
                    for (int u = 0; u < CPT; u++) {
                        // one PRMT builds the byte offset c*256 + rot*4 (code byte -> byte 1,
                        // the column byte -> byte 0); the step's column is the immediate
                        const uint32_t c4 = 4u * rot[u];
                        const uint32_t a0 = __byte_perm(x[u][st >> 2], c4, 0x5504u | ((st & 3) << 4));
                        const uint32_t a1 = __byte_perm(x[u][st >> 2], c4, 0x5504u | (((st + 1) & 3) << 4));
                        add_f32x2(sum[u], sum1[u], reinterpret_cast<const float*>(L + a0)[st],
                                  reinterpret_cast<const float*>(L + a1)[st + 1]);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < CPT; u++) {
                sum[u] += sum1[u];
                if (!live[u]) continue;
                const uint32_t e = eb + u * 32;
                if (sum[u] < INFINITY) {
                    const uint32_t key = float_key(sum[u]);
                    kmin = min(kmin, key);
                    kmax = max(kmax, key);
                    nf++;
                }
                dst[e] = sum[u];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
            kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
            nf += __shfl_xor_sync(0xffffffffu, nf, o);
        }
        if (lane == 0 && nf) {
            atomicMin(&w.mm[2 * qq], kmin);
            atomicMax(&w.mm[2 * qq + 1], kmax);
            atomicAdd(&w.nfin[qq], nf);
        }
        __syncthreads();
    }
}
// Generic ADC (any M): natural subspace order, LUT [G][256][32] in shared memory.
__global__ void __launch_bounds__(512) k_scan_generic(IndexDev D, int G, int Ps, int pre, int lbl, uint64_t q,
                                                      Workspace w) {
    extern __shared__ __align__(16) float s_lut[];  // [G][256][32]
    uint32_t* s_pre = reinterpret_cast<uint32_t*>(s_lut + G * kCodes * 32);
    uint32_t* s_start = s_pre + Ps + 1;
    __shared__ ScanShared s;
    __shared__ float s_box[2 * kMaxDims];
    const int t = threadIdx.x, lane = t & 31;
    const uint32_t n_items = w.item_off[q];
    const int M = D.M;
    int cur = -1;
    for (;;) {
        if (t == 0) {
            const int item = (int)atomicAdd(w.counter, 1u);
            s.item = item;
            if (item < (int)n_items) {
                int lo = 0, hi = (int)q - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (w.item_off[mid] <= (uint32_t)item) lo = mid;
                    else hi = mid - 1;
                }
                s.query = lo;
            }
        }
        __syncthreads();
        const int item = s.item;
        if (item >= (int)n_items) break;
        const int qq = s.query;
        const uint32_t total = w.qstat[(uint64_t)qq * 4];
        const uint32_t e0 = (uint32_t)(item - w.item_off[qq]) * w.chunk;
        if (e0 >= total) {  // a query cut by the distance capacity
            __syncthreads();
            continue;
        }
        if (qq != cur) {
            const uint64_t src0 = (uint64_t)qq * G * kCodes * 32;
            if (w.lut16) {
                const __half* src = reinterpret_cast<const __half*>(w.lut) + src0;
                for (int e = t; e < G * kCodes * 32; e += blockDim.x) s_lut[e] = __half2float(src[e]);
            } else {
                const float* src = w.lut + src0;
                for (int e = t; e < G * kCodes * 32; e += blockDim.x) s_lut[e] = src[e];
            }
            if (t < 2 * lbl) s_box[t] = w.box[(uint64_t)qq * 2 * lbl + t];
            scan_load_query(w, Ps, qq, s_pre, s_start);  // ends with a barrier
            cur = qq;
        }
        const uint32_t e1 = min(total, e0 + w.chunk);
        float* dst = w.dist + w.qoff[qq];
        const bool preq = pre || q_prefilter(w, qq);
        uint32_t kmin = 0xffffffffu, kmax = 0u, nf = 0;
        for (uint32_t e = e0 + t; e < e1; e += blockDim.x) {
            int lo = 0, hi = Ps - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_pre[mid] <= e) lo = mid;
                else hi = mid - 1;
            }
            const uint32_t pool = s_start[lo] + (e - s_pre[lo]);
            bool pass = true;
            if (preq) {
                const float* lab = D.labels + (uint64_t)pool * lbl;
                for (int i = 0; i < lbl; i++) {
                    const float v = lab[i];
                    if (v < s_box[2 * i] || v > s_box[2 * i + 1]) pass = false;
                }
            }
            float sum = INFINITY;
            if (pass) {
                sum = 0.f;
                const uint4* cp = reinterpret_cast<const uint4*>(D.codes) + pool;
                for (int j = 0; j * 16 < M; j++) {
                    const uint4 v = __ldg(cp + (uint64_t)j * D.n);
                    const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
                    for (int b = 0; b < 16 && j * 16 + b < M; b++) {
                        const int m = j * 16 + b;
                        const uint32_t c = (wv[b >> 2] >> (8 * (b & 3))) & 0xffu;
                        sum += s_lut[(m >> 5) * (kCodes * 32) + c * 32 + (m & 31)];
                    }
                }
                const uint32_t key = float_key(sum);
                kmin = min(kmin, key);
                kmax = max(kmax, key);
                nf++;
            }
            dst[e] = sum;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
            kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
            nf += __shfl_xor_sync(0xffffffffu, nf, o);
        }
        if (lane == 0 && nf) {
            atomicMin(&w.mm[2 * qq], kmin);
            atomicMax(&w.mm[2 * qq + 1], kmax);
            atomicAdd(&w.nfin[qq], nf);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------
// k_select: the K smallest (distance, position) pairs of one query
// ------------------------------------------------------------------------------------
// Pass 1 histograms the finite distances over kBins linear bins between the query's
// min and max; pass 2 emits every candidate below the bin that holds the K-th and gathers
// that boundary bin, which is sorted by (distance key, position).  A boundary bin larger
// than kBCap is split again over its own min/max (at most kMaxLevels levels); a bin whose
// entries all share one distance is resolved by position order.
constexpr int kMaxLevels = 4;
constexpr int kSelThreads = 512;

struct SelLevel {
    float lo, inv;
    int bin;
};

__device__ __forceinline__ int sel_bin(float d, float lo, float inv) {
    const int b = (int)__fmul_rn(__fsub_rn(d, lo), inv);
    return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
}

__device__ __forceinline__ uint32_t pos_to_pool(const uint32_t* s_pre, const uint32_t* s_start, int Ps,
                                                uint32_t e) {
    int lo = 0, hi = Ps - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_pre[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return s_start[lo] + (e - s_pre[lo]);
}

__global__ void __launch_bounds__(kSelThreads) k_select(IndexDev D, int Ps, int Kcap, int sorted_out, Workspace w,
                                                        float* __restrict__ out_dist,
                                                        uint64_t* __restrict__ out_ids, int k_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* s_hist = reinterpret_cast<uint32_t*>(smem);                   // [kBins]
    uint64_t* s_bbuf = reinterpret_cast<uint64_t*>(s_hist + kBins);         // [kBCap]
    uint64_t* s_sel = s_bbuf + kBCap;                                        // [sel_cap] (sorted mode)
    const int sel_cap = sorted_out ? (int)next_pow2_dev((uint32_t)max(Kcap, 2)) : 0;
    // this query's budget: its k for the sorted pre-filter output, else the candidate budget
    const int K = sorted_out ? (int)q_k(w, blockIdx.x) : (int)q_budget(w, blockIdx.x);
    uint32_t* s_pre = reinterpret_cast<uint32_t*>(s_sel + sel_cap);        // [Ps + 1]
    uint32_t* s_start = s_pre + Ps + 1;                                      // [Ps]
    __shared__ uint32_t s_warp[32];
    __shared__ SelLevel s_lv[kMaxLevels];
    __shared__ int s_bin;
    __shared__ uint32_t s_below, s_cntb, s_out, s_nb, s_bmin, s_bmax, s_need;
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x;
    // A predicate-first query of the predicate pass has a compact row: its survivors' distances
    // in arrival order with their candidate positions beside them (cand_count entries); any
    // other query's row holds one distance per candidate position.
    const bool compact = compacts(w, qi);
    if (!sorted_out && takes_row(w, qi)) return;  // the selection is the row (cand_count entries)
    const uint32_t total = compact ? w.cand_count[qi] : w.qstat[qi * 4];
    const float* dist = w.dist + w.qoff[qi];
    const uint32_t* prow = compact ? w.spos + w.qoff[qi] : nullptr;
    {
        const uint32_t* rpre = w.range_pre + qi * (Ps + 1);
        for (int i = t; i <= Ps; i += blockDim.x) s_pre[i] = rpre[i];
        for (int i = t; i < Ps; i += blockDim.x) s_start[i] = w.range_start[qi * Ps + i];
    }
    if (t == 0) s_out = 0;
    __syncthreads();
    const uint32_t nfin = w.nfin[qi];
    const uint32_t need0 = min((uint32_t)K, nfin);
    uint32_t* sel_dst = sorted_out ? nullptr : w.cand_pool + w.soff[qi];
    // candidate position of row entry e (e < total)
    auto posof = [&](uint32_t e) { return prow ? prow[e] : e; };
    // Selected entries are recorded by candidate position; positions become pool slots once the
    // selection is complete, in one divergence-free loop over the K entries (converting at
    // emit time made nearly every warp of the pass run the range search for one lane).  Ties in
    // distance are broken by the lower position.
    auto emit = [&](uint32_t pos, float d) {
        const uint32_t at = atomicAdd(&s_out, 1u);
        if (sorted_out)
            s_sel[at] = ((uint64_t)float_key(d) << 32) | pos;
        else
            sel_dst[at] = pos;
    };
    auto inside = [&](float d, int nlv) {
        for (int l = 0; l < nlv; l++)
            if (sel_bin(d, s_lv[l].lo, s_lv[l].inv) != s_lv[l].bin) return false;
        return true;
    };
    // First bin of s_hist whose cumulative count reaches need: s_bin, s_below (count before
    // it) and s_cntb (its count).  Warp 0 scans; the caller synchronises.
    auto find_bin = [&](uint32_t need) {
        if (t < 32) {
            uint32_t run = 0, below = 0;
            int found = -1;
            for (int base = 0; base < kBins && found < 0; base += 32) {
                const uint32_t v = s_hist[base + t];
                uint32_t x = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                    if (t >= o) x += y;
                }
                const unsigned hit = __ballot_sync(0xffffffffu, run + x >= need);
                if (hit) {
                    const int l0 = __ffs(hit) - 1;
                    found = base + l0;
                    below = run + __shfl_sync(0xffffffffu, x - v, l0);
                }
                run += __shfl_sync(0xffffffffu, x, 31);
            }
            if (t == 0) {
                s_bin = found;
                s_below = below;
                s_cntb = found >= 0 ? s_hist[found] : 0;
            }
        }
    };
    if (need0 > 0 && nfin <= (uint32_t)K) {
        // every finite candidate is selected (the loop bound is block-uniform so that every
        // lane reaches the warp appends)
        for (uint32_t base = 0; base < total; base += blockDim.x) {
            const uint32_t e = base + t;
            const float d = e < total ? dist[e] : INFINITY;
            const bool f = d < INFINITY;
            const uint32_t p = f ? posof(e) : 0u;
            if (sorted_out) {
                if (f) emit(p, d);
            } else {
                warp_append(f, p, &s_out, sel_dst);
            }
        }
        __syncthreads();
    } else if (need0 > 0) {
        float lo = key_float(w.mm[2 * qi]), hi = key_float(w.mm[2 * qi + 1]);
        uint32_t need = need0;
        for (int level = 0; level < kMaxLevels; level++) {
            const float inv = hi > lo ? (float)kBins / (hi - lo) : 0.f;
            for (int i = t; i < kBins; i += blockDim.x) s_hist[i] = 0;
            if (t == 0) {
                s_bmin = 0xffffffffu;
                s_bmax = 0u;
                s_nb = 0;
            }
            __syncthreads();
            for (uint32_t e0 = t; e0 < total; e0 += 4 * blockDim.x) {
                float dv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {  // four independent loads in flight per thread
                    const uint32_t e = e0 + u * blockDim.x;
                    dv[u] = e < total ? __ldg(dist + e) : INFINITY;
                }
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (dv[u] < INFINITY && inside(dv[u], level)) atomicAdd(&s_hist[sel_bin(dv[u], lo, inv)], 1u);
            }
            __syncthreads();
            find_bin(need);
            __syncthreads();
            const int b = s_bin;
            const bool fits = s_cntb <= (uint32_t)kBCap;
            for (uint32_t e0 = 0; e0 < total; e0 += 4 * blockDim.x) {  // block-uniform bound
                float dv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const uint32_t e = e0 + t + u * blockDim.x;
                    dv[u] = e < total ? __ldg(dist + e) : INFINITY;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const float d = dv[u];
                    const uint32_t e = e0 + t + u * blockDim.x;
                    const bool in = d < INFINITY && inside(d, level);
                    const int bb = in ? sel_bin(d, lo, inv) : kBins;
                    const uint32_t p = bb <= b ? posof(e) : 0u;
                    if (!sorted_out) warp_append(bb < b, p, &s_out, sel_dst);
                    if (!in) continue;
                    if (bb < b) {
                        if (sorted_out) emit(p, d);
                    } else if (bb == b) {
                        if (fits) {
                            const uint32_t at = atomicAdd(&s_nb, 1u);
                            s_bbuf[at] = ((uint64_t)float_key(d) << 32) | p;
                        } else {
                            atomicMin(&s_bmin, float_key(d));
                            atomicMax(&s_bmax, float_key(d));
                        }
                    }
                }
            }
            __syncthreads();
            need -= s_below;
            if (fits) {
                // the boundary bin, sorted by (distance, position)
                const int nb = (int)s_nb;
                const int n2 = (int)next_pow2_dev((uint32_t)max(nb, 2));
                for (int i = nb + t; i < n2; i += blockDim.x) s_bbuf[i] = ~0ull;
                __syncthreads();
                block_bitonic_sort(s_bbuf, n2);
                for (uint32_t i = t; i < need; i += blockDim.x) {
                    const uint64_t key = s_bbuf[i];
                    emit((uint32_t)key, key_float((uint32_t)(key >> 32)));
                }
                __syncthreads();
                break;
            }
            if (s_bmin == s_bmax || level == kMaxLevels - 1) {
                // one distance value (or no levels left): the boundary bin's entries (of that
                // one distance) are taken in position order
                const uint32_t tie_key = s_bmin;
                const bool one = s_bmin == s_bmax;
                const int nlv = level;
                auto tie = [&](float d) {
                    return d < INFINITY && inside(d, nlv) && sel_bin(d, lo, inv) == b && (!one || float_key(d) == tie_key);
                };
                if (t == 0) s_need = need;
                __syncthreads();
                if (!compact) {
                    // row order is position order: the first s_need tie entries of the row
                    for (uint32_t base = 0; base < total && s_need > 0; base += blockDim.x) {
                        const uint32_t e = base + t;
                        bool f = false;
                        float d = 0.f;
                        if (e < total) {
                            d = dist[e];
                            f = tie(d);
                        }
                        const unsigned bal = __ballot_sync(0xffffffffu, f);
                        if ((t & 31) == 0) s_warp[t >> 5] = __popc(bal);
                        __syncthreads();
                        uint32_t before = 0;
                        for (int i = 0; i < (t >> 5); i++) before += s_warp[i];
                        const uint32_t rank = before + __popc(bal & ((1u << (t & 31)) - 1));
                        if (f && rank < s_need) emit(e, d);
                        __syncthreads();
                        if (t == 0) {
                            uint32_t tot = 0;
                            for (int i = 0; i < (int)(blockDim.x >> 5); i++) tot += s_warp[i];
                            s_need = s_need > tot ? s_need - tot : 0;
                        }
                        __syncthreads();
                    }
                } else {
                    // a compact row is in arrival order: the s_need smallest positions among
                    // the tie entries, by a radix select over positions (kBins bins per level;
                    // positions are unique, so a one-position bin holds one entry)
                    uint32_t plo = 0, phi = w.qstat[qi * 4];
                    for (;;) {
                        const uint32_t binw = max(1u, (phi - plo + kBins - 1) / kBins);
                        for (int i = t; i < kBins; i += blockDim.x) s_hist[i] = 0;
                        __syncthreads();
                        for (uint32_t e = t; e < total; e += blockDim.x) {
                            const float d = dist[e];
                            const uint32_t p = prow[e];
                            if (tie(d) && p >= plo && p < phi) atomicAdd(&s_hist[(p - plo) / binw], 1u);
                        }
                        __syncthreads();
                        find_bin(s_need);
                        __syncthreads();
                        const int pb = s_bin;
                        const bool last = binw == 1;
                        for (uint32_t e = t; e < total; e += blockDim.x) {
                            const float d = dist[e];
                            const uint32_t p = prow[e];
                            if (!tie(d) || p < plo || p >= phi) continue;
                            const int bin = (int)((p - plo) / binw);
                            if (bin < pb || (last && bin == pb)) emit(p, d);
                        }
                        __syncthreads();
                        if (last || pb < 0) break;
                        if (t == 0) s_need -= s_below;
                        plo += (uint32_t)pb * binw;
                        phi = min(phi, plo + binw);
                        __syncthreads();
                    }
                }
                break;
            }
            if (t == 0) {
                s_lv[level].lo = lo;
                s_lv[level].inv = inv;
                s_lv[level].bin = b;
            }
            lo = key_float(s_bmin);
            hi = key_float(s_bmax);
            __syncthreads();
        }
    }
    __syncthreads();
    const uint32_t nsel = s_out;
    if (!sorted_out) {
        uint32_t* pool = w.cand_pool + w.soff[qi];
        for (uint32_t i = t; i < nsel; i += blockDim.x) pool[i] = pos_to_pool(s_pre, s_start, Ps, pool[i]);
        if (t == 0) w.cand_count[qi] = nsel;
        return;
    }
    const int n2 = (int)next_pow2_dev((uint32_t)max((int)nsel, 2));
    for (int i = nsel + t; i < n2; i += blockDim.x) s_sel[i] = ~0ull;
    __syncthreads();
    block_bitonic_sort(s_sel, n2);
    for (int i = t; i < k_out; i += blockDim.x) {
        if (i < (int)nsel) {
            const uint64_t key = s_sel[i];
            out_dist[qi * k_out + i] = key_float((uint32_t)(key >> 32));
            out_ids[qi * k_out + i] = D.ids[pos_to_pool(s_pre, s_start, Ps, (uint32_t)key)];
        } else {
            out_dist[qi * k_out + i] = INFINITY;
            out_ids[qi * k_out + i] = ~0ull;
        }
    }
}

// ------------------------------------------------------------------------------------
// k_refine: post-filter predicate, exact f32 L2, top-k
// ------------------------------------------------------------------------------------
// A query's selection (min(n_cand, candidates) entries, which the reference's uncapped
// budget can put in the hundreds of thousands) is cut into work items of kRefChunk entries;
// k_refine_plan lays them out and a persistent k_refine takes them from a counter.  An item
// compacts its predicate survivors, computes their exact distances and keeps its best k;
// a query with one item writes its output row directly, otherwise every item leaves its
// best k in the partial buffer and the last item of the query to finish merges them.
constexpr uint32_t kRefChunk = 4096;


__global__ void __launch_bounds__(1024) k_refine_plan(uint64_t q, Workspace w) {
    __shared__ unsigned long long s_w[32];
    const int t = threadIdx.x;
    const uint64_t per = (q + blockDim.x - 1) / blockDim.x;
    const uint64_t b = t * per, e = min(q, b + per);
    unsigned long long items = 0;
    for (uint64_t i = b; i < e; i++) items += max(1u, (w.cand_count[i] + kRefChunk - 1) / kRefChunk);
    unsigned long long tot = 0;
    unsigned long long r = block_inclusive_sum(items, s_w, &tot) - items;
    for (uint64_t i = b; i < e; i++) {
        w.ritem_off[i] = (uint32_t)r;
        r += max(1u, (w.cand_count[i] + kRefChunk - 1) / kRefChunk);
        w.rdone[i] = 0;
        w.rsurv[i] = 0;
        w.rlab[i] = 0;
    }
    if (e == q && b < e) w.ritem_off[q] = (uint32_t)r;
    if (t == 0) w.counter[1] = 0;
}

// Scratch of the re-rank's selections (shared memory)
struct RefSel {
    uint32_t* hist;            // [256]
    uint32_t* wc;              // [32]
    unsigned long long* sel;   // [4]
};

// Keeps the kq smallest of the c keys in s_keys (c > kq) in s_keys[0, kq), in no order, and
// returns the kq-th smallest; the rest of [0, c) becomes ~0.  All threads.
__device__ __forceinline__ uint64_t keep_smallest(uint64_t* s_keys, int c, int kq, const RefSel& rs) {
    return block_select_smallest(s_keys, c, kq, rs.hist, rs.wc, rs.sel);
}

// Sorts s_keys[0, m) ascending (padding to the next power of two with ~0).  All threads.
__device__ __forceinline__ void sort_prefix(uint64_t* s_keys, int m) {
    const int n2 = (int)next_pow2_dev((uint32_t)max(m, 2));
    for (int i = m + threadIdx.x; i < n2; i += blockDim.x) s_keys[i] = ~0ull;
    __syncthreads();
    block_bitonic_sort(s_keys, n2);
}

// Adds the keys below the running k-th to s_keys in rounds of at most cap - kq keys; between
// rounds the buffer keeps its kq smallest.  get(i) gives key i of n; all threads.
template <typename Get>
__device__ __forceinline__ void topk_rounds(uint64_t* s_keys, int cap, int kq, int n, int* s_cnt, uint64_t* s_th,
                                            const RefSel& rs, Get get) {
    const int per_round = max(cap - kq, 1);
    for (int r0 = 0; r0 < n; r0 += per_round) {
        const int r1 = min(n, r0 + per_round);
        for (int i = r0 + (int)threadIdx.x; i < r1; i += blockDim.x) {
            const uint64_t key = get(i);
            if (key < *s_th) s_keys[atomicAdd(s_cnt, 1)] = key;
        }
        __syncthreads();
        const int c = *s_cnt;
        __syncthreads();
        if (r1 < n && c > kq) {
            const uint64_t kth = keep_smallest(s_keys, c, kq, rs);
            if (threadIdx.x == 0) {
                *s_cnt = kq;
                *s_th = kth;
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kThreads, 5) k_refine(IndexDev D, const float* __restrict__ queries,
                                                     const float* __restrict__ data, int cap, int apply_pred,
                                                     int lbl, uint64_t q, Workspace w, float* __restrict__ out_dist,
                                                     uint64_t* __restrict__ out_ids, int k_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(smem);           // [cap]
    float* s_q = reinterpret_cast<float*>(s_keys + cap);             // [d]
    __shared__ float s_box[2 * kMaxDims];
    __shared__ int s_wsum[kThreads / 32];
    __shared__ int s_cnt, s_ns, s_item, s_qi, s_last;
    __shared__ uint64_t s_th;
    __shared__ uint32_t s_rb[4];
    __shared__ uint32_t s_rhist[256], s_rwc[32];
    __shared__ unsigned long long s_rsel[4];
    const RefSel rs{s_rhist, s_rwc, s_rsel};
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nw = kThreads / 32;
    const int d = D.d;
    const uint32_t n_items = w.ritem_off[q];
    int cur = -1;
    for (;;) {
        if (t == 0) {
            const int item = (int)atomicAdd(&w.counter[1], 1u);
            s_item = item;
            if (item < (int)n_items) {  // largest query with ritem_off <= item
                int lo = 0, hi = (int)q - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (w.ritem_off[mid] <= (uint32_t)item) lo = mid;
                    else hi = mid - 1;
                }
                s_qi = lo;
            }
        }
        __syncthreads();
        const int item = s_item;
        if (item >= (int)n_items) break;
        const uint64_t qi = (uint64_t)s_qi;
        if ((int)qi != cur) {
            for (int i = t; i < d; i += blockDim.x) s_q[i] = queries[qi * d + i];
            if (t < 2 * lbl) s_box[t] = w.box[qi * 2 * lbl + t];
            if (t < 4) s_rb[t] = w.rank_box[qi * 4 + t];
            cur = (int)qi;
        }
        if (t == 0) {
            s_cnt = 0;
            s_ns = 0;
            s_th = ~0ull;
        }
        __syncthreads();
        const uint32_t it0 = w.ritem_off[qi], nq_items = w.ritem_off[qi + 1] - it0;
        const uint32_t c0 = (uint32_t)(item - (int)it0) * kRefChunk;
        const int nc = (int)(min(w.cand_count[qi], c0 + kRefChunk) - min(w.cand_count[qi], c0));
        const int kq = (int)q_k(w, qi);
        const bool pred_q = apply_pred && q_sched(w, qi) == 0;  // predicate-first queries already passed it
        // label ranks decide most entries: outside the rank box fails, inside the inner box passes
        const bool ranks = D.rankpack && !D.labels_nan;
        const uint32_t gd = D.rank_guard;
        uint32_t* list = sel_row(w, qi) + c0;
        // 1. the predicate survivors, compacted in place as original ids (each chunk is read
        //    before the barrier and written at or below its own start)
        uint32_t n_lab = 0;
        // a row taken whole holds valid pool rows only (the predicate pass listed them): no
        // compaction, just the ids, four lookups in flight per thread and no barrier
        const bool whole = takes_row(w, qi);
        if (whole) {
            for (int e0 = t; e0 < nc; e0 += 4 * kThreads) {
                uint32_t p[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int e = e0 + u * kThreads;
                    p[u] = e < nc ? list[e] : 0u;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) p[u] = __ldg(D.ids + p[u]);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int e = e0 + u * kThreads;
                    if (e < nc) list[e] = p[u];
                }
            }
            if (t == 0) s_ns = nc;
        }
        for (int base = 0; !whole && base < nc; base += kThreads) {
            const int e = base + t;
            bool keep = false;
            uint32_t pool = kInvalid;
            if (e < nc) {
                pool = list[e];
                keep = pool != kInvalid;
                if (keep && pred_q) {
                    bool sure = false;
                    if (ranks) {
                        const uint32_t c = __ldg(D.rankpack + pool);
                        const uint32_t to = ((c | gd) - s_rb[0]) & (s_rb[1] - c);
                        const uint32_t ti = ((c | gd) - s_rb[2]) & (s_rb[3] - c);
                        keep = (to & gd) == gd;
                        sure = (ti & gd) == gd;
                    }
                    if (keep && !sure) {
                        n_lab++;
                        const float* lab = D.labels + (uint64_t)pool * lbl;
                        for (int i = 0; i < lbl; i++) {
                            const float v = lab[i];
                            if (v < s_box[2 * i] || v > s_box[2 * i + 1]) keep = false;
                        }
                    }
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) s_wsum[warp] = __popc(bal);
            __syncthreads();
            int before = s_ns, tot = 0;
            for (int i = 0; i < nw; i++) {
                before += i < warp ? s_wsum[i] : 0;
                tot += s_wsum[i];
            }
            if (keep) list[before + __popc(bal & ((1u << lane) - 1))] = D.ids[pool];
            __syncthreads();
            if (t == 0) s_ns += tot;
        }
        n_lab = __reduce_add_sync(0xffffffffu, n_lab);
        if (lane == 0 && n_lab) atomicAdd(&w.rlab[qi], n_lab);
        __syncthreads();
        const int ns = s_ns;
        if (t == 0 && ns) atomicAdd(&w.rsurv[qi], (uint32_t)ns);
        // 2. exact distances in rounds of cap - kq rows: every warp takes rows of the round, the
        //    keys (distance, id) below the running k-th go to the buffer, which is sorted and cut
        //    to kq after each round
        const int per_round = max(cap - kq, 1);
        // rows 16-byte aligned with d % 4 == 0: four rows per warp at a time, 8 lanes per row,
        // 16-byte loads, four independent partial sums per lane (the gathers are latency-bound:
        // this keeps ~6 KB per warp in flight instead of one 128-byte load per lane)
        const bool vec4 = (d & 3) == 0 && (reinterpret_cast<uintptr_t>(data) & 15) == 0;
        for (int r0 = 0; r0 < ns; r0 += per_round) {
            const int r1 = min(ns, r0 + per_round);
            if (vec4) {
                const int g = lane >> 3, sl = lane & 7, d4 = d >> 2;
                const float4* q4 = reinterpret_cast<const float4*>(s_q);
                for (int i0 = r0 + warp * 4; i0 < r1; i0 += nw * 4) {
                    const int i = i0 + g;
                    const bool ok = i < r1;
                    const uint32_t id = ok ? list[i] : list[r0];
                    const float4* row = reinterpret_cast<const float4*>(data + (uint64_t)id * d);
                    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
                    int j = sl;
                    for (; j + 24 < d4; j += 32) {
                        const float4 x0 = __ldg(row + j), x1 = __ldg(row + j + 8), x2 = __ldg(row + j + 16),
                                     x3 = __ldg(row + j + 24);
                        const float4 y0 = q4[j], y1 = q4[j + 8], y2 = q4[j + 16], y3 = q4[j + 24];
                        a0 = fmaf(y0.x - x0.x, y0.x - x0.x, a0);
                        a0 = fmaf(y0.y - x0.y, y0.y - x0.y, a0);
                        a0 = fmaf(y0.z - x0.z, y0.z - x0.z, a0);
                        a0 = fmaf(y0.w - x0.w, y0.w - x0.w, a0);
                        a1 = fmaf(y1.x - x1.x, y1.x - x1.x, a1);
                        a1 = fmaf(y1.y - x1.y, y1.y - x1.y, a1);
                        a1 = fmaf(y1.z - x1.z, y1.z - x1.z, a1);
                        a1 = fmaf(y1.w - x1.w, y1.w - x1.w, a1);
                        a2 = fmaf(y2.x - x2.x, y2.x - x2.x, a2);
                        a2 = fmaf(y2.y - x2.y, y2.y - x2.y, a2);
                        a2 = fmaf(y2.z - x2.z, y2.z - x2.z, a2);
                        a2 = fmaf(y2.w - x2.w, y2.w - x2.w, a2);
                        a3 = fmaf(y3.x - x3.x, y3.x - x3.x, a3);
                        a3 = fmaf(y3.y - x3.y, y3.y - x3.y, a3);
                        a3 = fmaf(y3.z - x3.z, y3.z - x3.z, a3);
                        a3 = fmaf(y3.w - x3.w, y3.w - x3.w, a3);
                    }
                    for (; j < d4; j += 8) {
                        const float4 x = __ldg(row + j), y = q4[j];
                        a0 = fmaf(y.x - x.x, y.x - x.x, a0);
                        a0 = fmaf(y.y - x.y, y.y - x.y, a0);
                        a0 = fmaf(y.z - x.z, y.z - x.z, a0);
                        a0 = fmaf(y.w - x.w, y.w - x.w, a0);
                    }
                    float sq = (a0 + a1) + (a2 + a3);
                    sq += __shfl_xor_sync(0xffffffffu, sq, 4);
                    sq += __shfl_xor_sync(0xffffffffu, sq, 2);
                    sq += __shfl_xor_sync(0xffffffffu, sq, 1);
                    const uint64_t key = ((uint64_t)float_key(sq) << 32) | id;
                    if (ok && sl == 0 && key < s_th) s_keys[atomicAdd(&s_cnt, 1)] = key;
                }
            } else {
                for (int i = r0 + warp; i < r1; i += nw) {
                    const uint32_t id = list[i];
                    const float* row = data + (uint64_t)id * d;
                    float sq = 0.f;
                    for (int j = lane; j < d; j += 32) {
                        const float df = s_q[j] - __ldg(row + j);
                        sq = fmaf(df, df, sq);
                    }
                    sq = warp_sum(sq);
                    const uint64_t key = ((uint64_t)float_key(sq) << 32) | id;
                    if (lane == 0 && key < s_th) s_keys[atomicAdd(&s_cnt, 1)] = key;
                }
            }
            __syncthreads();
            const int c = s_cnt;
            __syncthreads();
            if (r1 < ns && c > kq) {  // more rows follow: keep the kq best
                const uint64_t kth = keep_smallest(s_keys, c, kq, rs);
                if (t == 0) {
                    s_cnt = kq;
                    s_th = kth;
                }
                __syncthreads();
            }
        }
        int c = s_cnt;
        __syncthreads();
        if (c > kq) keep_smallest(s_keys, c, kq, rs);
        sort_prefix(s_keys, min(c, kq));
        bool write_out = nq_items == 1;
        if (!write_out) {
            // this item's best kq keys go to its partial row; the query's last item merges
            uint64_t* part = w.rpart + (uint64_t)item * k_out;
            for (int i = t; i < kq; i += blockDim.x) part[i] = i < c ? s_keys[i] : ~0ull;
            __threadfence();
            __syncthreads();
            if (t == 0) s_last = atomicAdd(&w.rdone[qi], 1u) == nq_items - 1;
            __syncthreads();
            if (s_last) {
                __threadfence();  // the other items' partial rows are visible past their counts
                if (t == 0) {
                    s_cnt = 0;
                    s_th = ~0ull;
                }
                __syncthreads();
                const uint64_t* rows = w.rpart + (uint64_t)it0 * k_out;
                topk_rounds(s_keys, cap, kq, (int)nq_items * kq, &s_cnt, &s_th, rs,
                            [&](int i) { return __ldcg(rows + (uint64_t)(i / kq) * k_out + (i % kq)); });
                c = s_cnt;
                __syncthreads();
                if (c > kq) keep_smallest(s_keys, c, kq, rs);
                sort_prefix(s_keys, min(c, kq));
                write_out = true;
            }
        }
        if (write_out) {
            for (int i = t; i < k_out; i += blockDim.x) {
                if (i < min(c, kq) && s_keys[i] != ~0ull) {
                    const uint64_t key = s_keys[i];
                    out_dist[qi * k_out + i] = key_float((uint32_t)(key >> 32));
                    out_ids[qi * k_out + i] = (uint32_t)key;
                } else {
                    out_dist[qi * k_out + i] = INFINITY;
                    out_ids[qi * k_out + i] = ~0ull;
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------
// host orchestration
// ------------------------------------------------------------------------------------
static uint32_t lut_groups(const IndexDev& D) { return (D.M + 31) / 32; }

static Workspace carve(hdg_index* idx, QueryCtx& cx, uint64_t q, bool record) {
    const hdg_params& P = idx->params;
    const uint64_t l = idx->dev.l, L = idx->dev.n_lists, C = idx->dev.C;
    const uint64_t Pc = std::max<uint64_t>(1, P.n_list), Ps = std::max<uint64_t>(1, P.sub_lists);
    const uint64_t G = lut_groups(idx->dev);
    size_t off = 0;
    char* base = static_cast<char*>(cx.work.ptr);
    auto take = [&](const char* name, size_t bytes) -> void* {
        const size_t o = off;
        off += align_up(bytes ? bytes : 1, 256);
        if (record) cx.layout[name] = {o, bytes};
        return base ? base + o : nullptr;
    };
    Workspace w{};
    w.box = (float*)take("box", q * 2 * l * 4);
    w.cells = (int*)take("cells", q * 2 * l * 4);
    w.rank_box = (uint32_t*)take("rank_box", q * 4 * 4);
    w.zrange = (uint64_t*)take("zrange", q * 2 * 8);
    w.list_counts = (uint32_t*)take("list_counts", q * L * 4);
    w.cluster_counts = (uint32_t*)take("cluster_counts", q * C * 4);
    w.probe_clusters = (uint32_t*)take("probe_clusters", q * Pc * 4);
    w.probe_lists = (uint32_t*)take("probe_lists", q * Ps * 4);
    const uint64_t ns = P.is_split ? std::max<uint64_t>(1, P.n_split) : 1;
    w.range_start = (uint32_t*)take("range_start", q * Ps * ns * 4);
    w.range_len = (uint32_t*)take("range_len", q * Ps * ns * 4);
    w.range_pre = (uint32_t*)take("range_pre", q * (Ps * ns + 1) * 4);
    w.is_split = P.is_split ? 1 : 0;
    w.nsplit = (int)ns;
    w.qstat = (uint32_t*)take("qstat", q * 4 * 4);
    w.scal = (uint64_t*)take("scalars", 8 * 8);
    w.qoff = (uint64_t*)take("qoff", (q + 1) * 8);
    w.item_off = (uint32_t*)take("item_off", (q + 1) * 4);
    w.pitem_off = (uint32_t*)take("pre_items", (q + 1) * 4);
    w.mm = (uint32_t*)take("minmax", q * 2 * 4);
    w.nfin = (uint32_t*)take("nfin", q * 4);
    w.lab_read = (uint32_t*)take("labels_read", q * 4);
    w.rank_read = (uint32_t*)take("ranks_read", q * 4);
    w.counter = (uint32_t*)take("counter", 16);
    w.lut16 = P.lut_fp16 != 0;
    w.lut = (float*)take("lut", q * G * kCodes * 32 * (w.lut16 ? 2 : 4));
    w.cand_count = (uint32_t*)take("cand_count", q * 4);
    w.qbud = (uint32_t*)take("budget", q * 4);
    w.soff = (uint64_t*)take("sel_off", (q + 1) * 8);
    w.ritem_off = (uint32_t*)take("refine_items", (q + 1) * 4);
    w.rdone = (uint32_t*)take("refine_done", q * 4);
    w.rsurv = (uint32_t*)take("refine_rows", q * 4);
    w.rlab = (uint32_t*)take("refine_labels_read", q * 4);
    w.ldS = C + L;
    w.S = (float*)take("gemm_s", q * (C + L) * 4);
    w.qnorm = (float*)take("qnorm", q * 4);
    w.qbf = take("qbf", q * idx->dev.d * 2);
    w.gemm_err = (int*)take("gemm_err", 16);
    w.feats = (float*)take("features", q * kMlpFeatures * 4);
    w.lq_ps = (uint32_t*)take("learned_nprobe", q * 4);
    w.lq_sched = (uint8_t*)take("learned_schedule", q);
    w.dist = static_cast<float*>(cx.dist_buf.ptr);
    w.spos = static_cast<uint32_t*>(cx.pos_buf.ptr);
    w.cand_pool = static_cast<uint32_t*>(cx.sel_buf.ptr);
    w.sel_cap = cx.sel_buf.bytes / 4;
    w.rpart = static_cast<uint64_t*>(cx.part_buf.ptr);
    if (!base) cx.work.bytes = std::max(cx.work.bytes, off);  // size probe
    return w;
}

// Partial rows of the refine items: at most one item per query plus one per kRefChunk
// entries of the selection buffer, k keys each.
static size_t part_bytes(const QueryCtx& cx, uint64_t q, uint32_t k) {
    return (q + (cx.sel_buf.bytes / 4) / kRefChunk + 1) * (size_t)k * 8;
}
static void invalidate_ctx_graphs(QueryCtx& cx);
static void ensure_part_buf(QueryCtx& cx, uint64_t q, uint32_t k) {
    const size_t need = part_bytes(cx, q, k);
    if (cx.part_buf.bytes >= need) return;
    invalidate_ctx_graphs(cx);
    cx.part_buf.reset();
    cx.part_buf.ensure(need);
}

// The per-candidate rows: one f32 distance and one u32 position per candidate, same capacity.
static void resize_rows(QueryCtx& cx, size_t bytes) {
    cx.dist_buf.reset();
    cx.pos_buf.reset();
    cx.dist_buf.ensure(bytes);
    cx.pos_buf.ensure(bytes);
}

static size_t workspace_bytes(hdg_index* idx, QueryCtx& cx, uint64_t q) {
    void* saved = cx.work.ptr;
    cx.work.ptr = nullptr;
    const size_t before = cx.work.bytes;
    cx.work.bytes = 0;
    carve(idx, cx, q, false);
    const size_t need = cx.work.bytes;
    cx.work.ptr = saved;
    cx.work.bytes = before;
    return need;
}

static void reserve_ctx(hdg_index* idx, QueryCtx& cx, uint64_t q) {
    HDG_REQUIRE(idx->built, HDG_ERR_STATE, "index not built");
    const size_t need = workspace_bytes(idx, cx, q);
    if (cx.work.ptr && cx.work.bytes >= need) return;
    cx.work.reset();
    cx.work.ensure(need);
    cx.work_queries = q;
}

// The query context of a stream (created on first use); it becomes the last one used.
static QueryCtx& query_ctx(hdg_index* idx, cudaStream_t st) {
    std::lock_guard<std::mutex> g(idx->ctx_mu);
    auto& slot = idx->ctxs[static_cast<void*>(st)];
    if (!slot) slot.reset(new QueryCtx());
    idx->last_ctx = slot.get();
    return *slot;
}

void reserve_workspace(hdg_index* idx, uint64_t q, cudaStream_t st) {
    QueryCtx& cx = query_ctx(idx, st);
    std::lock_guard<std::mutex> g(cx.mu);
    reserve_ctx(idx, cx, q);
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

// Stage times from consecutive recorded events (the first marks the start).
static void store_stage_times(hdg_index* idx, const std::vector<cudaEvent_t>& ev,
                              const std::vector<std::string>& names) {
    std::lock_guard<std::mutex> g(idx->stats_mu);
    idx->stage_names.clear();
    idx->stage_ms.clear();
    for (size_t i = 1; i < ev.size(); i++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[i - 1], ev[i]));
        idx->stage_names.push_back(names[i]);
        idx->stage_ms.push_back(ms);
    }
}

namespace {
// Events between the stages of one query batch.  On the plain path they are recorded on
// the stream and read by finish(); while a CUDA graph is captured (keep != nullptr) they
// become external event-record nodes of the graph, owned by its entry, and every replay
// records them again, so the stage times of each replay can be read once it completes.
struct StageTimer {
    hdg_index* idx;
    cudaStream_t st;
    bool on;
    std::vector<cudaEvent_t> ev;
    std::vector<std::string> names;
    std::vector<cudaEvent_t>* keep;
    std::vector<std::string>* keep_names;
    StageTimer(hdg_index* i, cudaStream_t s, bool enabled, std::vector<cudaEvent_t>* k = nullptr,
               std::vector<std::string>* kn = nullptr)
        : idx(i), st(s), on(enabled), keep(k), keep_names(kn) {
        mark("");
    }
    void mark(const char* name) {
        if (!on) return;
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        if (keep) {
            keep->push_back(e);
            keep_names->push_back(name);
            CK(cudaEventRecordWithFlags(e, st, cudaEventRecordExternal));
        } else {
            ev.push_back(e);
            names.push_back(name);
            CK(cudaEventRecord(e, st));
        }
    }
    void finish() {
        if (!on || keep) return;
        CK(cudaEventSynchronize(ev.back()));
        store_stage_times(idx, ev, names);
    }
    ~StageTimer() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

template <typename K>
int occupancy_blocks(K kernel, int threads, size_t smem) {
    int nb = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem));
    return std::max(nb, 1);
}

}  // namespace

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    }
    return n;
}

struct QueryCall {
    const float* queries;
    uint64_t q;
    const float* qlabels;
    uint32_t label_cols;
    const float* data;
    uint32_t k;
    float* dist;
    uint64_t* ids;
    const uint32_t* qk;
    const uint32_t* qps;
    const uint8_t* qsched;
};

struct GraphEntry {
    uint64_t key[24];
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> stage_ev;     // event-record nodes between the stages (break_down=1)
    std::vector<std::string> stage_names;
    uint64_t q = 0, launches = 0;
    int mode = 0;
    uint32_t k = 0;
};

struct GraphState {
    std::vector<GraphEntry> entries;
    cudaStream_t stream = nullptr;  // capture and replay stream
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    uint64_t* pinned = nullptr;     // [8] scalars + [8] gemm status of the last replay
    bool pending = false;
    GraphEntry last;                // description of the last replay (stats)
};

static void destroy_entry(GraphEntry& e) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    for (auto ev : e.stage_ev) cudaEventDestroy(ev);
    e.exec = nullptr;
    e.stage_ev.clear();
    e.stage_names.clear();
}

void release_graphs(GraphState* g) {
    if (!g) return;
    for (auto& e : g->entries) destroy_entry(e);
    if (g->ev_in) cudaEventDestroy(g->ev_in);
    if (g->ev_out) cudaEventDestroy(g->ev_out);
    if (g->stream) cudaStreamDestroy(g->stream);
    if (g->pinned) cudaFreeHost(g->pinned);
    delete g;
}

static void invalidate_ctx_graphs(QueryCtx& cx) {
    if (!cx.graphs) return;
    if (cx.graphs->pending) cudaEventSynchronize(cx.graphs->ev_out);
    for (auto& e : cx.graphs->entries) destroy_entry(e);
    cx.graphs->entries.clear();
    cx.graphs->pending = false;
}

void invalidate_graphs(hdg_index* idx) {
    std::lock_guard<std::mutex> g(idx->ctx_mu);
    for (auto& kv : idx->ctxs) {
        std::lock_guard<std::mutex> gc(kv.second->mu);
        invalidate_ctx_graphs(*kv.second);
    }
}

// The stats of a query from its batch scalars (scal of k_batch).
static void fill_stats(hdg_index* idx, uint64_t q, uint32_t k, int mode, uint64_t exps0, const uint64_t* sc,
                       uint64_t launches) {
    std::lock_guard<std::mutex> g(idx->stats_mu);
    const uint64_t coarse = sc[0], real = sc[1], max_row = sc[2];
    const uint32_t bb = (uint32_t)sc[4];
    float beta;
    std::memcpy(&beta, &bb, 4);
    if (mode != kPost) beta = 0.f;
    uint64_t K = k;  // the budget of a query with the batch k and the reference schedule
    if (mode == kPost) {
        if (real == 0) {
            K = max_row;
        } else {
            const float want = (float)(exps0 * (uint64_t)k) * beta;
            K = std::min<uint64_t>(want >= 1.8e19f ? ~0ull : (uint64_t)want, max_row);
        }
    } else if (mode == kL1) {
        K = exps0 * k;
    }
    idx->last_ncand = K;  // no cap: the budget the reference computes is the one used
    idx->last_beta = beta;
    idx->last_q = q;
    uint32_t bits;
    std::memcpy(&bits, &beta, 4);
    const uint64_t s[10] = {q, idx->last_ncand, K, coarse, real, max_row, bits, (uint64_t)mode, launches, sc[5]};
    std::memcpy(idx->last_stats, s, sizeof(s));
}

// Enqueues one query batch on st.  sync_sizing: one host read after k_batch sizes the
// distance buffer and fills the stats (the plain path).  Otherwise nothing waits on the
// host (the CUDA-graph path): the distance buffer keeps its capacity, queries past it are
// cut by k_batch, and the scalars and the GEMM status word are copied to pinned memory.
static void enqueue_query(hdg_index* idx, QueryCtx& cx, const QueryCall& c, cudaStream_t st, bool sync_sizing,
                          uint64_t* pinned, uint64_t* launches_out, int* mode_out, uint64_t* coarse_out = nullptr,
                          uint64_t* sel_out = nullptr, GraphEntry* capture = nullptr) {
    const uint64_t q = c.q;
    const uint32_t k = c.k;
    HDG_REQUIRE(idx->built, HDG_ERR_STATE, "index not built");
    HDG_REQUIRE(q > 0 && q < (1ull << 31), HDG_ERR_INVALID_ARG, "query count out of range");
    HDG_REQUIRE(c.queries && c.qlabels && c.dist && c.ids, HDG_ERR_INVALID_ARG, "null pointer");
    HDG_REQUIRE(k >= 1 && k <= 2048, HDG_ERR_INVALID_ARG, "k must be in [1, 2048]");
    const hdg_params& P = idx->params;
    const IndexDev& D = idx->dev;
    const int l = (int)D.l;
    const int fd = (int)std::max<uint64_t>(1, P.filter_dim);
    HDG_REQUIRE(c.label_cols == (uint32_t)(l * fd), HDG_ERR_INVALID_ARG,
                "query label columns must equal l * filter_dim");
    const int Pc = (int)std::max<uint64_t>(1, P.n_list);
    const int Ps = (int)std::max<uint64_t>(1, P.sub_lists);
    HDG_REQUIRE(Pc <= 1024 && Ps <= 2048, HDG_ERR_UNSUPPORTED, "n_list <= 1024 and sub_lists <= 2048");
    HDG_REQUIRE(D.n_lists <= 32768, HDG_ERR_UNSUPPORTED, "at most 32768 inverted lists");
    const uint64_t exps0 = P.exps0;
    const int mode = exps0 <= 1 ? kPre : (l > 1 ? kPost : kL1);
    if (mode_out) *mode_out = mode;
    HDG_REQUIRE(mode == kPre || c.data, HDG_ERR_INVALID_ARG, "d_data is required for the re-rank");
    HDG_REQUIRE(mode != kPre || !c.qsched, HDG_ERR_INVALID_ARG,
                "per-query schedules need exps0 > 1 (the pre-filter schedule has no re-rank)");
    if (!cx.work.ptr || cx.work.bytes < workspace_bytes(idx, cx, q)) {
        HDG_REQUIRE(sync_sizing, HDG_ERR_STATE, "workspace too small for a captured query");
        reserve_ctx(idx, cx, q);
    }
    Workspace w = carve(idx, cx, q, true);
    const uint32_t G = lut_groups(D);
    const bool fast = (D.M % 32 == 0) && G <= 3;
    w.surv_list = fast ? 1 : 0;  // the fast path lists the predicate-first queries' survivors
    w.qk = c.qk;
    w.qps = c.qps;
    w.qsched = c.qsched;
    w.k_max = k;
    w.mode = mode;
    w.exps0 = (uint32_t)std::min<uint64_t>(exps0, 1u << 20);
    w.chunk = P.scan_chunk ? (uint32_t)P.scan_chunk : kChunk;
    w.cap = sync_sizing ? ~0ull : cx.dist_buf.bytes / 4;
    if (sync_sizing) w.sel_cap = ~0ull;  // sized after k_batch
    const FilterDev f = filter_dev(idx);
    StageTimer tm(idx, st, P.break_down != 0 && (sync_sizing || capture), capture ? &capture->stage_ev : nullptr,
                  capture ? &capture->stage_names : nullptr);

    const size_t sm_pro = sizeof(uint32_t) * D.n_lists;
    if (sm_pro > 48 * 1024)
        CK(cudaFuncSetAttribute(k_prologue, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_pro));
    uint64_t launches = 0;  // kernels of this query, reported in the stats
    k_prologue<<<(unsigned)q, kThreads, sm_pro, st>>>(D, idx->grid, f, c.qlabels, (int)c.label_cols, w);
    CK_LAUNCH();
    launches++;
    tm.mark("prologue");
    const int sort_n1 = (int)next_pow2(std::max<uint32_t>(D.C, 2));
    const int sort_n2 = (int)next_pow2(std::max<uint32_t>((uint32_t)Pc * D.S_max, 2));
    const size_t sm_co = (sizeof(uint64_t) + sizeof(float)) * std::max(sort_n1, sort_n2) + sizeof(float) * D.d;
    HDG_REQUIRE(sm_co <= 200 * 1024, HDG_ERR_UNSUPPORTED, "coarse selection does not fit shared memory");
    if (sm_co > 48 * 1024)
        CK(cudaFuncSetAttribute(k_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_co));
    // tensor-core estimates of every query-centroid dot product, used to prune the exact
    // ranking when n_list or sub_lists leaves part of the candidates out (COARSE_BF16=1)
    const bool use_gemm = P.coarse_bf16 != 0 && D.d % 8 == 0 && (Pc < (int)D.C || Ps < Pc * (int)D.S_max);
    CK(cudaMemsetAsync(w.gemm_err, 0, sizeof(int), st));
    if (use_gemm) {
        rows_to_bf16(c.queries, q, (int)D.d, w.qbf, w.qnorm, st);
        umma_dot(w.qbf, q, D.centers_bf16, D.C, (int)D.d, w.S, w.ldS, w.gemm_err, st);
        umma_dot(w.qbf, q, D.sub_centers_bf16, D.n_lists, (int)D.d, w.S + D.C, w.ldS, w.gemm_err, st);
        launches += 3;
        tm.mark("coarse_gemm");
    } else {
        w.S = nullptr;
    }
    if (P.learned && !c.qps && !c.qsched) {
        // the learned schedule: per-query lists to probe and predicate-first flag
        HDG_REQUIRE(idx->mlp_ready, HDG_ERR_STATE, "LEARNED=1 but the index holds no trained model");
        // the features' 16 nearest centroids are pruned by the tensor-core products when present
        learned_features(idx, c.queries, q, w.box, w.cluster_counts, c.qk, k, w.feats, st, w.S, w.ldS, w.qnorm);
        learned_infer(idx, w.feats, q, w.lq_ps, w.lq_sched, mode != kPre, (uint32_t)Ps, nullptr, st);
        w.qps = w.lq_ps;
        w.qsched = mode != kPre ? w.lq_sched : nullptr;
        launches += 2;
        tm.mark("learned");
    }

    k_coarse<<<(unsigned)q, kCoarseThreads, sm_co, st>>>(D, idx->grid, c.queries, Pc, Ps, sort_n1, sort_n2, w);
    CK_LAUNCH();
    launches++;
    tm.mark("coarse");

    // candidate offsets, work items, batch sums, beta and the per-query budgets' inputs
    k_batch<<<1, 1024, 0, st>>>(q, w);
    CK_LAUNCH();
    launches++;
    uint64_t sc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (sync_sizing) {
        int gemm_err = 0;
        CK(cudaMemcpyAsync(sc, w.scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&gemm_err, w.gemm_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        HDG_REQUIRE(gemm_err == 0, HDG_ERR_TIMEOUT, "tensor-core wait expired in the coarse GEMM");
        const uint64_t coarse = sc[0], selected = sc[7];
        if (coarse_out) *coarse_out = coarse;
        if (sel_out) *sel_out = selected;
        if (cx.dist_buf.bytes < std::max<uint64_t>(coarse, 1) * 4) {
            invalidate_ctx_graphs(cx);  // their distance pointer dies with the old buffer
            resize_rows(cx, std::max<uint64_t>(coarse, 1) * 4 * 5 / 4);
        }
        if (cx.sel_buf.bytes < std::max<uint64_t>(selected, 1) * 4) {
            invalidate_ctx_graphs(cx);  // and their selection pointer with this one
            cx.sel_buf.reset();
            cx.sel_buf.ensure(std::max<uint64_t>(selected, 1) * 4 * 5 / 4);
        }
        ensure_part_buf(cx, q, k);
    } else {
        HDG_REQUIRE(cx.dist_buf.ptr && cx.sel_buf.ptr && cx.part_buf.bytes >= part_bytes(cx, q, k), HDG_ERR_STATE,
                    "no candidate buffers for a captured query");
    }
    w.dist = static_cast<float*>(cx.dist_buf.ptr);
    w.spos = static_cast<uint32_t*>(cx.pos_buf.ptr);
    w.cand_pool = static_cast<uint32_t*>(cx.sel_buf.ptr);
    w.rpart = static_cast<uint64_t*>(cx.part_buf.ptr);
    tm.mark("budget");

    const int pre = mode == kPre ? 1 : 0;
    // candidate ranges per query: one per probed list, or n_split per list when is_split
    const int R = Ps * w.nsplit;
    const size_t sm_tab = sizeof(uint32_t) * (2 * R + 1);
    if (!sync_sizing || sc[3] > 0) {
        if (fast && (pre || w.qsched)) {
            // the predicate pass of the predicate-first queries, then the ADC items that
            // follow from their survivors
            const bool lab4 = l == 4 && (reinterpret_cast<uintptr_t>(D.labels) & 15) == 0;
            auto launch_pre = [&](auto kern) {
                const size_t smp = sizeof(uint32_t) * kPreRingWords * (kPreThreads / 32);
                CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
                const int blocks = sm_count() * occupancy_blocks(kern, kPreThreads, smp);
                kern<<<blocks, kPreThreads, smp, st>>>(D, R, l, q, w);
            };
            if (lab4) launch_pre(k_pre_scan<true>);
            else launch_pre(k_pre_scan<false>);
            CK_LAUNCH();
            k_scan_plan<<<1, 1024, 0, st>>>(q, w);
            CK_LAUNCH();
            launches += 2;
            tm.mark("predicate");
        }
        {
            // the LUTs of the queries that have ADC work items (a predicate-first query whose
            // budget takes every survivor has none)
            if (D.pq_len <= (uint32_t)kLutMaxPqLen) {
                const size_t sm = sizeof(float) * kCodes * D.pq_len * 33;
                CK(cudaFuncSetAttribute(k_lut, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                k_lut<<<dim3((unsigned)((q + kLutQ - 1) / kLutQ), G), 512, sm, st>>>(D, c.queries, q, (int)G, w.lut,
                                                                                    w.lut16, w.item_off);
            } else {
                k_lut_plain<<<dim3((unsigned)q, G), 256, sizeof(float) * D.d, st>>>(D, c.queries, (int)G, w.lut,
                                                                                  w.lut16, w.item_off);
            }
            CK_LAUNCH();
            launches++;
            tm.mark("lut");
        }
        if (fast) {
            // threads x candidates-per-thread (SCAN_CPT, chosen by the autotuner; 0 = 1)
            const int cpt = (P.scan_cpt == 1 || P.scan_cpt == 2 || P.scan_cpt == 4) ? (int)P.scan_cpt : 1;
            const size_t sm = sizeof(float) * G * kCodes * 64 + sm_tab;
            HDG_REQUIRE(sm <= 227 * 1024, HDG_ERR_UNSUPPORTED, "scan tables exceed shared memory");
            auto launch = [&](auto kern, int nt) {
                CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                const int blocks = sm_count() * occupancy_blocks(kern, nt, sm);
                kern<<<blocks, nt, sm, st>>>(D, R, q, w);
            };
            if (G == 1) {
                if (cpt == 1) launch(k_scan_fast<1, 512, 1>, 512);
                else if (cpt == 2) launch(k_scan_fast<1, 512, 2>, 512);
                else launch(k_scan_fast<1, 256, 4>, 256);
            } else if (G == 2) {
                if (cpt == 1) launch(k_scan_fast<2, 512, 1>, 512);
                else if (cpt == 2) launch(k_scan_fast<2, 512, 2>, 512);
                else launch(k_scan_fast<2, 256, 4>, 256);
            } else {
                if (cpt == 1) launch(k_scan_fast<3, 1024, 1>, 1024);
                else if (cpt == 2) launch(k_scan_fast<3, 512, 2>, 512);
                else launch(k_scan_fast<3, 256, 4>, 256);
            }
        } else {
            const size_t sm = sizeof(float) * G * kCodes * 32 + sm_tab;
            HDG_REQUIRE(sm <= 227 * 1024, HDG_ERR_UNSUPPORTED, "scan tables exceed shared memory");
            CK(cudaFuncSetAttribute(k_scan_generic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            const int blocks = sm_count() * occupancy_blocks(k_scan_generic, 512, sm);
            k_scan_generic<<<blocks, 512, sm, st>>>(D, (int)G, R, pre, l, q, w);
        }
        CK_LAUNCH();
        launches++;
    }
    tm.mark("scan");

    const int sorted_out = mode == kPre ? 1 : 0;
    const size_t sm_sel = sizeof(uint32_t) * kBins + sizeof(uint64_t) * kBCap +
                          (sorted_out ? sizeof(uint64_t) * next_pow2(std::max<uint32_t>(k, 2)) : 0) + sm_tab + 16;
    CK(cudaFuncSetAttribute(k_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_sel));
    k_select<<<(unsigned)q, kSelThreads, sm_sel, st>>>(D, R, (int)k, sorted_out, w, c.dist, c.ids, (int)k);
    CK_LAUNCH();
    launches++;
    tm.mark("select");
    if (mode != kPre) {
        k_refine_plan<<<1, 1024, 0, st>>>(q, w);
        CK_LAUNCH();
        const int rcap = (int)next_pow2(k + 4 * kThreads);  // rounds of rcap - k exact distances
        const size_t sm_ref = sizeof(uint64_t) * rcap + sizeof(float) * D.d + 16;
        CK(cudaFuncSetAttribute(k_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_ref));
        // persistent over the refine items; no more CTAs than queries are useful for small batches
        const uint64_t blocks = std::min<uint64_t>((uint64_t)sm_count() * occupancy_blocks(k_refine, kThreads, sm_ref),
                                                   q + (cx.sel_buf.bytes / 4) / kRefChunk + 1);
        k_refine<<<(unsigned)blocks, kThreads, sm_ref, st>>>(D, c.queries, c.data, rcap, mode == kPost ? 1 : 0, l, q,
                                                            w, c.dist, c.ids, (int)k);
        CK_LAUNCH();
        launches += 2;
        tm.mark("refine");
    }
    if (!sync_sizing && pinned) {
        CK(cudaMemcpyAsync(pinned, w.scal, 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(pinned + 8, w.gemm_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    if (launches_out) *launches_out = launches;
    if (sync_sizing) fill_stats(idx, q, k, mode, exps0, sc, launches);
    tm.finish();
}

static hdg_status finish_ctx(hdg_index* idx, QueryCtx& cx) {
    GraphState* g = cx.graphs;
    if (!g || !g->pending) return HDG_OK;
    CK(cudaEventSynchronize(g->ev_out));
    g->pending = false;
    fill_stats(idx, g->last.q, g->last.k, g->last.mode, idx->params.exps0, g->pinned, g->last.launches);
    if (!g->last.stage_ev.empty()) store_stage_times(idx, g->last.stage_ev, g->last.stage_names);
    if (static_cast<int>(g->pinned[8] & 0xffffffffu) != 0) return HDG_ERR_TIMEOUT;
    if (g->pinned[5] != 0) return HDG_ERR_OOM;
    return HDG_OK;
}

hdg_status finish_async_query(hdg_index* idx) {
    std::vector<QueryCtx*> all;
    {
        std::lock_guard<std::mutex> g(idx->ctx_mu);
        for (auto& kv : idx->ctxs) all.push_back(kv.second.get());
    }
    hdg_status worst = HDG_OK;
    for (QueryCtx* cx : all) {
        std::lock_guard<std::mutex> g(cx->mu);
        const hdg_status s = finish_ctx(idx, *cx);
        if (worst == HDG_OK) worst = s;
    }
    return worst;
}

static void make_graph_key(const hdg_index* idx, const QueryCtx& cx, const QueryCall& c, uint64_t* key) {
    const hdg_params& P = idx->params;
    const uint64_t v[24] = {(uint64_t)c.queries, c.q, (uint64_t)c.qlabels, c.label_cols, (uint64_t)c.data, c.k,
                            (uint64_t)c.dist, (uint64_t)c.ids, (uint64_t)c.qk, (uint64_t)c.qps, (uint64_t)c.qsched,
                            (uint64_t)cx.work.ptr, cx.work.bytes, (uint64_t)cx.dist_buf.ptr,
                            cx.dist_buf.bytes, P.n_list, P.sub_lists, P.exps0, P.lut_fp16, P.coarse_bf16,
                            P.scan_cpt, P.scan_chunk, P.filter_dim, P.learned | (P.is_split << 8) | (P.n_split << 16)};
    std::memcpy(key, v, sizeof(v));
}

void run_query(hdg_index* idx, const float* d_queries, uint64_t q, const float* d_query_labels,
               uint32_t label_cols, const float* d_data, uint32_t k, float* d_dist, uint64_t* d_ids,
               cudaStream_t st, const uint32_t* d_k, const uint32_t* d_nprobe, const uint8_t* d_sched) {
    const QueryCall c{d_queries, q, d_query_labels, label_cols, d_data, k, d_dist, d_ids, d_k, d_nprobe, d_sched};
    QueryCtx& cx = query_ctx(idx, st);
    std::lock_guard<std::mutex> lock(cx.mu);  // one query at a time per stream
    if (idx->params.query_graph == 0) {
        finish_ctx(idx, cx);
        enqueue_query(idx, cx, c, st, true, nullptr, nullptr, nullptr);
        return;
    }
    if (!cx.graphs) {
        GraphState* g = new GraphState();
        cx.graphs = g;
        CK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&g->ev_in, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&g->ev_out, cudaEventDisableTiming));
        CK(cudaMallocHost(reinterpret_cast<void**>(&g->pinned), 16 * sizeof(uint64_t)));
        std::memset(g->pinned, 0, 16 * sizeof(uint64_t));
    }
    GraphState* g = cx.graphs;
    finish_ctx(idx, cx);  // the pinned status words are reused by this replay
    uint64_t key[24];
    make_graph_key(idx, cx, c, key);
    GraphEntry* hit = nullptr;
    for (auto& e : g->entries)
        if (std::memcmp(e.key, key, sizeof(key)) == 0) hit = &e;
    if (!hit) {
        // first call of this shape: the plain path computes this call's results and sizes
        // the buffers; the captured graph serves the next calls
        uint64_t coarse = 0, selected = 0;
        enqueue_query(idx, cx, c, st, true, nullptr, nullptr, nullptr, &coarse, &selected);
        const uint64_t need = std::max<uint64_t>(coarse, 1) * 4 * 5 / 4;  // 1.25x this batch
        if (cx.dist_buf.bytes < need) {
            invalidate_ctx_graphs(cx);
            resize_rows(cx, need);
        }
        const uint64_t need_sel = std::max<uint64_t>(selected, 1) * 4 * 5 / 4;
        if (cx.sel_buf.bytes < need_sel) {
            invalidate_ctx_graphs(cx);
            cx.sel_buf.reset();
            cx.sel_buf.ensure(need_sel);
        }
        ensure_part_buf(cx, q, k);
        make_graph_key(idx, cx, c, key);
        CK(cudaStreamSynchronize(st));
        GraphEntry e;
        std::memcpy(e.key, key, sizeof(key));
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed));
        try {
            enqueue_query(idx, cx, c, g->stream, false, g->pinned, &e.launches, &e.mode, nullptr, nullptr, &e);
        } catch (...) {
            cudaStreamEndCapture(g->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            destroy_entry(e);
            throw;
        }
        CK(cudaStreamEndCapture(g->stream, &graph));
        const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) destroy_entry(e);
        CK(ie);
        e.q = q;
        e.k = k;
        if (g->entries.size() >= 8) {
            destroy_entry(g->entries.front());
            g->entries.erase(g->entries.begin());
        }
        g->entries.push_back(e);
        return;
    }
    CK(cudaEventRecord(g->ev_in, st));
    CK(cudaStreamWaitEvent(g->stream, g->ev_in, 0));
    CK(cudaGraphLaunch(hit->exec, g->stream));
    CK(cudaEventRecord(g->ev_out, g->stream));
    CK(cudaStreamWaitEvent(st, g->ev_out, 0));
    g->last = *hit;
    g->pending = true;
}

void query_features(hdg_index* idx, const float* d_queries, uint64_t q, const float* d_query_labels,
                    uint32_t label_cols, const uint32_t* d_k, uint32_t k_max, float* d_feats, cudaStream_t st) {
    HDG_REQUIRE(idx->built, HDG_ERR_STATE, "index not built");
    HDG_REQUIRE(q > 0 && q < (1ull << 31), HDG_ERR_INVALID_ARG, "query count out of range");
    HDG_REQUIRE(d_queries && d_query_labels && d_feats, HDG_ERR_INVALID_ARG, "null pointer");
    const IndexDev& D = idx->dev;
    const int fd = (int)std::max<uint64_t>(1, idx->params.filter_dim);
    HDG_REQUIRE(label_cols == (uint32_t)(D.l * fd), HDG_ERR_INVALID_ARG,
                "query label columns must equal l * filter_dim");
    QueryCtx& cx = query_ctx(idx, st);
    std::lock_guard<std::mutex> lock(cx.mu);
    if (!cx.work.ptr || cx.work.bytes < workspace_bytes(idx, cx, q)) reserve_ctx(idx, cx, q);
    Workspace w = carve(idx, cx, q, true);
    const FilterDev f = filter_dev(idx);
    const size_t sm_pro = sizeof(uint32_t) * D.n_lists;
    if (sm_pro > 48 * 1024)
        CK(cudaFuncSetAttribute(k_prologue, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_pro));
    k_prologue<<<(unsigned)q, kThreads, sm_pro, st>>>(D, idx->grid, f, d_query_labels, (int)label_cols, w);
    CK_LAUNCH();
    learned_features(idx, d_queries, q, w.box, w.cluster_counts, d_k, k_max, d_feats, st);
}

void autotune_query(hdg_index* idx, const float* d_queries, uint64_t q, const float* d_query_labels,
                    uint32_t label_cols, const float* d_data, uint32_t k, float* d_dist, uint64_t* d_ids,
                    cudaStream_t st, float* best_ms) {
    hdg_params& P = idx->params;
    const uint64_t saved_bd = P.break_down, saved_graph = P.query_graph;
    P.break_down = 1;
    P.query_graph = 0;
    const QueryCall c{d_queries, q, d_query_labels, label_cols, d_data, k, d_dist, d_ids, nullptr, nullptr, nullptr};
    float best = INFINITY;
    uint64_t best_cpt = 1, best_chunk = kChunk;
    QueryCtx& cx = query_ctx(idx, st);
    std::unique_lock<std::mutex> lock(cx.mu);
    try {
        enqueue_query(idx, cx, c, st, true, nullptr, nullptr, nullptr);  // warm-up, buffers sized
        const uint64_t cpts[3] = {1, 2, 4};
        const uint64_t chunks[4] = {8192, 16384, 32768, 65536};
        for (uint64_t cpt : cpts)
            for (uint64_t ch : chunks) {
                P.scan_cpt = cpt;
                P.scan_chunk = ch;
                float t = INFINITY;
                for (int rep = 0; rep < 2; rep++) {  // the faster of two runs
                    enqueue_query(idx, cx, c, st, true, nullptr, nullptr, nullptr);
                    float s = 0.f;
                    std::lock_guard<std::mutex> gs(idx->stats_mu);
                    for (size_t i = 0; i < idx->stage_names.size(); i++)
                        if (idx->stage_names[i] == "scan") s = idx->stage_ms[i];
                    t = std::min(t, s);
                }
                if (t < best) {
                    best = t;
                    best_cpt = cpt;
                    best_chunk = ch;
                }
            }
    } catch (...) {
        P.break_down = saved_bd;
        P.query_graph = saved_graph;
        throw;
    }
    P.scan_cpt = best_cpt;
    P.scan_chunk = best_chunk;
    P.break_down = saved_bd;
    P.query_graph = saved_graph;
    lock.unlock();
    invalidate_graphs(idx);
    if (best_ms) *best_ms = best;
}

}  // namespace hdg
