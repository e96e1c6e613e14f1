// Kernel-level entry points that keep the reference kernels' data layouts, so the
// reference's known-answer tests (src/verification/test_*.cuh) can run through the GPU.
//   pq_lut          build_pq_lut_kernel            (src/index/product-quantization.cu:4-35)
//   pq_adc          compute_batched_L2_distance_kernel (product-quantization.cu:37-77)
//   label_mask      label_matrix_by_filter_indices_kernel (src/core/filter.cu:30-64)
//   recover_filters denormalize_labels_kernel      (src/core/preprocessing.cu:3-32)
//   bruteforce_knn  brute_forece_vector_search     (src/verification/ground_truth.cuh:165-232),
//                   with the filter.conf predicate instead of its hard-coded window.
#include <cfloat>
#include <mutex>
#include <vector>

#include "hdg_device.cuh"
#include "hdg_internal.h"

namespace hdg {

static unsigned nblk(uint64_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }

__global__ void k_pq_lut(const float* __restrict__ centers, const float* __restrict__ queries, uint64_t nq,
                         uint32_t n_dim, uint32_t pq_dim, uint32_t pq_len, uint32_t n_codes,
                         float* __restrict__ lut) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nq * pq_dim * n_codes) return;
    const uint64_t q = e / ((uint64_t)pq_dim * n_codes);
    const uint32_t m = (uint32_t)((e / n_codes) % pq_dim);
    const uint32_t c = (uint32_t)(e % n_codes);
    float s = 0.f;
    for (uint32_t t = 0; t < pq_len; t++) {
        if (m * pq_len + t >= n_dim) break;
        const float df = __fsub_rn(centers[((uint64_t)m * n_codes + c) * pq_len + t],
                                   queries[q * n_dim + m * pq_len + t]);
        s = fmaf(df, df, s);
    }
    lut[e] = s;
}

__global__ void k_pq_adc(const uint8_t* __restrict__ codebook, uint64_t tot_data, const float* __restrict__ lut,
                         uint64_t nq, uint32_t pq_dim, uint32_t n_codes, const uint64_t* __restrict__ indices,
                         uint64_t n_cand, float* __restrict__ dist) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nq * n_cand) return;
    const uint64_t q = e / n_cand, j = e % n_cand;
    const uint64_t idx = indices ? indices[e] : j;
    if (idx >= tot_data) {
        dist[e] = FLT_MAX;
        return;
    }
    float s = 0.f;
    for (uint32_t m = 0; m < pq_dim; m++)
        s += lut[(q * pq_dim + m) * n_codes + codebook[(uint64_t)m * tot_data + idx]];
    dist[e] = s;
}

__global__ void k_label_mask(const float* __restrict__ ranges, const float* __restrict__ labels, uint32_t l,
                             uint64_t n_data, uint64_t nq, const uint64_t* __restrict__ indices,
                             uint64_t n_cand, int32_t* __restrict__ mask) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nq * n_cand) return;
    const uint64_t q = e / n_cand, j = e % n_cand;
    const uint64_t idx = indices ? indices[e] : j;
    if (idx >= n_data) {
        mask[e] = 0;
        return;
    }
    int ok = 1;
    for (uint32_t i = 0; i < l; i++) {
        const float v = labels[idx * l + i];
        if (v < ranges[q * 2 * l + 2 * i] || v > ranges[q * 2 * l + 2 * i + 1]) {
            ok = 0;
            break;
        }
    }
    mask[e] = ok;
}

__global__ void k_recover(FilterDev f, const float* __restrict__ qlabels, uint64_t nq, float* __restrict__ out) {
    const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    for (int i = 0; i < f.l; i++) {
        float lo, hi;
        recover_dim(f, qlabels + q * f.l * f.filter_dim, i, &lo, &hi);
        out[q * 2 * f.l + 2 * i] = lo;
        out[q * 2 * f.l + 2 * i + 1] = hi;
    }
}

void pq_lut(const float* centers, const float* queries, uint64_t nq, uint32_t n_dim, uint32_t pq_dim,
            uint32_t pq_len, uint32_t n_codes, float* lut, cudaStream_t st) {
    const uint64_t n = nq * pq_dim * n_codes;
    if (!n) return;
    k_pq_lut<<<nblk(n, 256), 256, 0, st>>>(centers, queries, nq, n_dim, pq_dim, pq_len, n_codes, lut);
    CK_LAUNCH();
}
void pq_adc(const uint8_t* codebook, uint64_t tot_data, const float* lut, uint64_t nq, uint32_t pq_dim,
            uint32_t n_codes, const uint64_t* indices, uint64_t n_cand, float* dist, cudaStream_t st) {
    if (!nq || !n_cand) return;
    k_pq_adc<<<nblk(nq * n_cand, 256), 256, 0, st>>>(codebook, tot_data, lut, nq, pq_dim, n_codes, indices,
                                                      n_cand, dist);
    CK_LAUNCH();
}
void label_mask(const float* ranges, const float* labels, uint32_t l, uint64_t n_data, uint64_t nq,
                const uint64_t* indices, uint64_t n_cand, int32_t* mask, cudaStream_t st) {
    if (!nq || !n_cand) return;
    k_label_mask<<<nblk(nq * n_cand, 256), 256, 0, st>>>(ranges, labels, l, n_data, nq, indices, n_cand, mask);
    CK_LAUNCH();
}
void recover_filters(const FilterDev& f, const float* qlabels, uint64_t nq, float* ranges, cudaStream_t st) {
    if (!nq) return;
    k_recover<<<nblk(nq, 128), 128, 0, st>>>(f, qlabels, nq, ranges);
    CK_LAUNCH();
}

// ---- allocation-free filter recovery ---------------------------------------------------
// Scratch for the interval-map table of hdg_recover_filters_noalloc: a fixed array in the
// library's own device memory, present on every GPU that loads the library until the
// process exits.  Host code must not pass `g_noalloc_map` itself to a kernel (on the host it
// is only a stand-in symbol); it passes the device address fetched below.
static __device__ __align__(256) float g_noalloc_map[HDG_NOALLOC_MAP_MAX];

namespace {
std::mutex g_noalloc_mu;
std::vector<float*> g_noalloc_ptr;  // per device ordinal, filled on first use
}  // namespace

// Device address of the scratch array on the current device.  The first call on a device
// resolves it with cudaGetSymbolAddress (that device must be current); later calls reuse it.
static float* noalloc_map_scratch() {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if ((int)g_noalloc_ptr.size() <= dev) g_noalloc_ptr.resize(dev + 1, nullptr);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_map));
        g_noalloc_ptr[dev] = static_cast<float*>(p);
    }
    return g_noalloc_ptr[dev];
}

void recover_filters_noalloc(const FilterDev& f0, const float* host_map, const float* qlabels, uint64_t nq,
                             float* ranges, cudaStream_t st) {
    HDG_REQUIRE(f0.n_map >= 0 && f0.n_map <= HDG_NOALLOC_MAP_MAX, HDG_ERR_INVALID_ARG,
                "interval map of " + std::to_string(f0.n_map) + " entries exceeds the " +
                    std::to_string(HDG_NOALLOC_MAP_MAX) + "-entry limit of hdg_recover_filters_noalloc");
    FilterDev f = f0;
    f.map = noalloc_map_scratch();
    // the whole used prefix is rewritten every call, so nothing has to start at zero
    if (f.n_map) CK(cudaMemcpyAsync(const_cast<float*>(f.map), host_map, sizeof(float) * f.n_map,
                                    cudaMemcpyHostToDevice, st));
    recover_filters(f, qlabels, nq, ranges, st);
}

// ---- filtered exact kNN ------------------------------------------------------------------
// Block = 256 threads, 32 queries x 64 base vectors per tile, each thread a 2 x 4 register
// tile of f32 distances; per-query top-k buffers in shared memory with a running threshold.
constexpr int BF_Q = 32, BF_V = 64, BF_K = 32, BF_CAP = 512;

__device__ void warp_bitonic_sort(uint64_t* keys, int n) {
    const int lane = threadIdx.x & 31;
    for (int k = 2; k <= n; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < (n >> 1); i += 32) {
                const int lo = 2 * i - (i & (j - 1)), hi = lo + j;
                const bool up = (lo & k) == 0;
                const uint64_t a = keys[lo], b = keys[hi];
                if ((a > b) == up) {
                    keys[lo] = b;
                    keys[hi] = a;
                }
            }
            __syncwarp();
        }
}

__global__ void __launch_bounds__(256) k_bruteforce(const float* __restrict__ data, uint64_t n, uint32_t d,
                                                    const float* __restrict__ labels, uint32_t l,
                                                    const float* __restrict__ queries, uint64_t nq,
                                                    const float* __restrict__ ranges, uint32_t k,
                                                    float* __restrict__ out_dist, uint64_t* __restrict__ out_ids) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* s_buf = reinterpret_cast<uint64_t*>(smem);  // [BF_Q][BF_CAP]
    __shared__ float s_qt[BF_K][BF_Q + 1];
    __shared__ float s_vt[BF_K][BF_V + 4];
    __shared__ float s_lab[BF_V][kMaxDims];
    __shared__ float s_rng[BF_Q][2 * kMaxDims];
    __shared__ int s_cnt[BF_Q];
    __shared__ uint64_t s_th[BF_Q];
    __shared__ int s_need;
    const int t = threadIdx.x, warp = t >> 5;
    const int tq = t >> 4;  // 16 query pairs
    const int tv = t & 15;  // 16 vector quads
    const uint64_t q0 = (uint64_t)blockIdx.x * BF_Q;
    for (int e = t; e < BF_Q * 2 * (int)l; e += blockDim.x) {
        const int qq = e / (2 * l), c = e % (2 * l);
        s_rng[qq][c] = (q0 + qq < nq) ? ranges[(q0 + qq) * 2 * l + c] : 1.f;
    }
    if (t < BF_Q) {
        s_cnt[t] = 0;
        s_th[t] = ~0ull;
    }
    const int K = (int)k;
    for (uint64_t v0 = 0; v0 < n; v0 += BF_V) {
        float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
        for (uint32_t k0 = 0; k0 < d; k0 += BF_K) {
            __syncthreads();
            for (int e = t; e < BF_Q * BF_K; e += blockDim.x) {
                const int qq = e / BF_K, kk = e % BF_K;
                s_qt[kk][qq] = (q0 + qq < nq && k0 + kk < d) ? queries[(q0 + qq) * d + k0 + kk] : 0.f;
            }
            for (int e = t; e < BF_V * BF_K; e += blockDim.x) {
                const int vv = e / BF_K, kk = e % BF_K;
                s_vt[kk][vv] = (v0 + vv < n && k0 + kk < d) ? data[(v0 + vv) * d + k0 + kk] : 0.f;
            }
            if (k0 == 0)
                for (int e = t; e < BF_V * (int)l; e += blockDim.x) {
                    const int vv = e / l, c = e % l;
                    s_lab[vv][c] = (v0 + vv < n) ? labels[(v0 + vv) * l + c] : 0.f;
                }
            __syncthreads();
#pragma unroll 8
            for (int kk = 0; kk < BF_K; kk++) {
                const float a0 = s_qt[kk][2 * tq], a1 = s_qt[kk][2 * tq + 1];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const float b = s_vt[kk][4 * tv + j];
                    const float d0 = a0 - b, d1 = a1 - b;
                    acc[0][j] = fmaf(d0, d0, acc[0][j]);
                    acc[1][j] = fmaf(d1, d1, acc[1][j]);
                }
            }
        }
        // predicate + threshold + append (each query gets at most 64 appends per tile)
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int qq = 2 * tq + i;
            if (q0 + qq >= nq) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int vv = 4 * tv + j;
                const uint64_t id = v0 + vv;
                if (id >= n) continue;
                bool pass = true;
                for (uint32_t c = 0; c < l; c++) {
                    const float lv = s_lab[vv][c];
                    if (lv < s_rng[qq][2 * c] || lv > s_rng[qq][2 * c + 1]) pass = false;
                }
                if (!pass) continue;
                const uint64_t key = ((uint64_t)float_key(acc[i][j]) << 32) | (uint32_t)id;
                if (key < s_th[qq]) {
                    const int pos = atomicAdd(&s_cnt[qq], 1);
                    s_buf[qq * BF_CAP + pos] = key;
                }
            }
        }
        __syncthreads();
        if (t == 0) {
            int need = 0;
            for (int qq = 0; qq < BF_Q; qq++) need |= (s_cnt[qq] > BF_CAP - BF_V) ? 1 : 0;
            s_need = need;
        }
        __syncthreads();
        if (s_need) {
            for (int qq = warp; qq < BF_Q; qq += 8) {
                const int c = s_cnt[qq];
                if (c <= BF_CAP - BF_V) continue;
                uint64_t* buf = s_buf + qq * BF_CAP;
                for (int i = c + (t & 31); i < BF_CAP; i += 32) buf[i] = ~0ull;
                __syncwarp();
                warp_bitonic_sort(buf, BF_CAP);
                if ((t & 31) == 0) {
                    s_cnt[qq] = min(c, K);
                    if (c >= K) s_th[qq] = buf[K - 1];
                }
                __syncwarp();
            }
        }
    }
    __syncthreads();
    for (int qq = warp; qq < BF_Q; qq += 8) {
        if (q0 + qq >= nq) continue;
        const int c = s_cnt[qq];
        uint64_t* buf = s_buf + qq * BF_CAP;
        for (int i = c + (t & 31); i < BF_CAP; i += 32) buf[i] = ~0ull;
        __syncwarp();
        warp_bitonic_sort(buf, BF_CAP);
        const uint64_t q = q0 + qq;
        for (int i = (t & 31); i < K; i += 32) {
            const uint64_t key = buf[i];
            if (i < c && key != ~0ull) {
                out_dist[q * k + i] = key_float((uint32_t)(key >> 32));
                out_ids[q * k + i] = (uint32_t)key;
            } else {
                out_dist[q * k + i] = INFINITY;
                out_ids[q * k + i] = ~0ull;
            }
        }
    }
}

void bruteforce_knn(const float* data, uint64_t n, uint32_t d, const float* labels, uint32_t l,
                    const float* queries, uint64_t q, const float* ranges, uint32_t k, float* dist,
                    uint64_t* ids, cudaStream_t st) {
    HDG_REQUIRE(k >= 1 && k <= 256, HDG_ERR_UNSUPPORTED, "bruteforce k must be in [1, 256]");
    HDG_REQUIRE(l >= 1 && l <= (uint32_t)kMaxDims && d >= 1, HDG_ERR_INVALID_ARG, "bad dims");
    HDG_REQUIRE(n < (1ull << 32), HDG_ERR_INVALID_ARG, "n must be < 2^32");
    if (!q) return;
    const size_t sm = sizeof(uint64_t) * BF_Q * BF_CAP;
    CK(cudaFuncSetAttribute(k_bruteforce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_bruteforce<<<nblk(q, BF_Q), 256, sm, st>>>(data, n, d, labels, l, queries, q, ranges, k, dist, ids);
    CK_LAUNCH();
}

}  // namespace hdg

namespace hdg {

// ---- merge of per-data-batch results (merge_intermediate_result, src/core/merge_res.cu:18-56)
// Row r of (dist, ids) holds n_batches blocks of k results, block b from an index built on
// base rows [offset_b, ...): ids are shifted by offset_b (invalid ids stay invalid), the
// k smallest (distance, id) of the row are kept, ascending.
namespace {
__global__ void k_merge_topk(const float* __restrict__ dist, const uint64_t* __restrict__ ids, uint32_t k,
                             uint32_t nb, const uint64_t* __restrict__ offsets, int n2, float* __restrict__ out_dist,
                             uint64_t* __restrict__ out_ids) {
    extern __shared__ uint64_t s_key[];            // [n2] (distance key << 32 | slot)
    uint64_t* s_id = s_key + n2;                    // [k * nb] shifted ids
    const uint64_t r = blockIdx.x;
    const uint32_t w = k * nb;
    for (uint32_t i = threadIdx.x; i < (uint32_t)n2; i += blockDim.x) {
        uint64_t key = ~0ull;
        if (i < w) {
            const uint64_t id = ids[r * w + i];
            const bool ok = id != ~0ull;
            const uint64_t sid = ok ? id + offsets[i / k] : ~0ull;
            s_id[i] = sid;
            // ties by the shifted id: the slot order of equal distances follows the id
            key = ok ? ((uint64_t)float_key(dist[r * w + i]) << 32) | i : ~0ull;
        }
        s_key[i] = key;
    }
    __syncthreads();
    block_bitonic_sort(s_key, n2);
    // equal distance keys are ordered by slot; re-order each run of equal keys by id
    if (threadIdx.x == 0) {
        for (uint32_t i = 0; i + 1 < (uint32_t)min(n2, (int)w) && i < k; i++) {  // runs reaching the top k
            uint32_t j = i + 1;
            while (j < w && (s_key[j] >> 32) == (s_key[i] >> 32) && s_key[j] != ~0ull) j++;
            for (uint32_t a = i + 1; a < j; a++)  // insertion sort on the (short) tie run
                for (uint32_t b2 = a; b2 > i && s_id[(uint32_t)s_key[b2]] < s_id[(uint32_t)s_key[b2 - 1]]; b2--) {
                    const uint64_t tmp = s_key[b2];
                    s_key[b2] = s_key[b2 - 1];
                    s_key[b2 - 1] = tmp;
                }
            i = j - 1;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) {
        const uint64_t key = s_key[i];
        const bool ok = key != ~0ull;
        out_dist[r * k + i] = ok ? key_float((uint32_t)(key >> 32)) : INFINITY;
        out_ids[r * k + i] = ok ? s_id[(uint32_t)key] : ~0ull;
    }
}
}  // namespace

void merge_topk(const float* dist, const uint64_t* ids, uint64_t q, uint32_t k, uint32_t nb, const uint64_t* offsets,
                float* out_dist, uint64_t* out_ids, cudaStream_t st) {
    HDG_REQUIRE(k >= 1 && nb >= 1 && (uint64_t)k * nb <= 8192, HDG_ERR_UNSUPPORTED, "k * n_batches must be <= 8192");
    const int n2 = (int)next_pow2(std::max<uint32_t>(k * nb, 2));
    const size_t sm = sizeof(uint64_t) * (n2 + (size_t)k * nb);
    CK(cudaFuncSetAttribute(k_merge_topk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_merge_topk<<<(unsigned)q, 256, sm, st>>>(dist, ids, k, nb, offsets, n2, out_dist, out_ids);
    CK_LAUNCH();
}

}  // namespace hdg
