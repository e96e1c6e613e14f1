// Learned per-query schedule: query features and a BF16 MLP (48 -> 128 -> 128 -> 2) with
// hand-written forward, backward and Adam kernels.
//
// The network predicts, per query, z0 = log2 of the number of inverted lists to probe and
// z1 = the logit of the predicate-first flag (1: label predicate inside the ADC pass, a budget
// of exps0 * k and an exact re-rank; 0: the index's own schedule,
// Super-Grid-IVF_PQ.cu:1151-1241).  It replaces the batch-wide n_list / sub_lists choice of
// super_grid::index::query for each query; the plain schedule stays the fallback.
//
// Precision: weights, inputs and hidden activations are rounded to BF16 (round to nearest
// even), every dot product accumulates in FP32, the optimiser keeps FP32 master weights.
//
// Features (48 per query, all scale-free):
//   [0, 8)   normalised filter bounds (lo, hi) of label dims 0..3: (x - left) / span in [0, 1]
//   [8, 12)  log10 of the normalised box width of dims 0..3, divided by 7
//   [12, 28) the 16 nearest coarse-centroid distances: log1p(d_0), then log1p(d_j) - log1p(d_0)
//   [28, 44) filtered point counts of those 16 clusters (the grid-cell histogram counts of the
//            query's cell box summed over each cluster's lists), log1p(count) / log1p(N)
//   [44]     log1p(filtered points over all lists) / log1p(N)   (selectivity estimate)
//   [45]     fraction of clusters holding any filtered point
//   [46]     k of the query / 100
//   [47]     log1p(filtered points of the 16 nearest clusters) / log1p(N)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "hdg_device.cuh"
#include "hdg_internal.h"

namespace hdg {

namespace {

constexpr int kTile = 32;  // samples per forward block

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

struct Params {
    const float* master;          // fp32 parameters (biases are read from here)
    const __nv_bfloat16* w;       // bf16 copies of the parameters (weights are read from here)
};

// ---- features --------------------------------------------------------------------------
// One 128-thread block per query (its phases are serial; small blocks keep more queries in flight)
__global__ void __launch_bounds__(128) k_features(IndexDev D, GridMeta g, const float* __restrict__ queries,
                                                  const float* __restrict__ box, const uint32_t* __restrict__ cc,
                                                  const uint32_t* __restrict__ qk, uint32_t k_max, int sort_n,
                                                  const float* __restrict__ S, uint64_t ldS,
                                                  const float* __restrict__ qnorm, float* __restrict__ feats) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(smem);         // [sort_n]
    uint32_t* s_cand = reinterpret_cast<uint32_t*>(s_keys + sort_n);  // [sort_n]
    float* s_q = reinterpret_cast<float*>(s_cand + sort_n);        // [d]
    float* s_lo = s_q + D.d;                                         // [sort_n] the bands' lows
    __shared__ int s_ncand;
    __shared__ float s_bound;
    __shared__ float s_f[kMlpFeatures];
    __shared__ uint32_t s_hist[256], s_wc[32];
    __shared__ unsigned long long s_sel[4];
    __shared__ unsigned long long s_tot;
    __shared__ unsigned s_nz;
    const uint64_t qi = blockIdx.x;
    const int t = threadIdx.x, d = D.d, C = D.C, l = g.l;
    for (int i = t; i < d; i += blockDim.x) s_q[i] = queries[qi * d + i];
    if (t == 0) {
        s_tot = 0;
        s_nz = 0;
    }
    __syncthreads();
    unsigned long long tot = 0;
    unsigned nz = 0;
    for (int c = t; c < sort_n; c += blockDim.x) {
        if (c < C) {
            const uint32_t n = cc[qi * C + c];
            tot += n;
            nz += n > 0;
        } else {
            s_keys[c] = ~0ull;
        }
    }
    // centroid distances, one warp per centroid: the lanes read a row with coalesced loads
    // (the features only rank and log-scale these distances; no summation order is implied)
    // Four centroids per warp and step keep four independent row loads in flight; each
    // centroid's sum is formed exactly as with one per step (per-lane FMA chain, warp sum).
    const int lane = t & 31, warp = t >> 5, nw = blockDim.x >> 5;
    // With the coarse stage's tensor-core products S, only a centroid whose lower bound lies
    // within the 16th smallest upper bound can be among the 16 nearest (the 16 with the
    // smallest upper bounds are at or below it), so only those get exact distances: the same
    // 16 keys, each computed the same way
    const int kn = min(16, C);
    int n_ex = C;
    if (S) {
        for (int c = t; c < sort_n; c += blockDim.x) {
            uint64_t key = ~0ull;
            if (c < C) {
                float lo, hi;
                coarse_band(qnorm[qi], D.cnorm[c], S[qi * ldS + c], &lo, &hi);
                key = ((uint64_t)float_key(hi) << 32) | (uint32_t)c;
                s_lo[c] = lo;
            }
            s_keys[c] = key;
        }
        if (t == 0) s_ncand = 0;
        __syncthreads();
        // (only the k-th is needed: the keys stay in place)
        const uint64_t kth = block_select_smallest(s_keys, sort_n, kn, s_hist, s_wc, s_sel, false);
        if (t == 0) s_bound = key_float((uint32_t)(kth >> 32));
        __syncthreads();
        for (int c = t; c < sort_n; c += blockDim.x) {
            if (c < C && s_lo[c] <= s_bound) s_cand[atomicAdd(&s_ncand, 1)] = (uint32_t)c;
            s_keys[c] = ~0ull;
        }
        __syncthreads();
        n_ex = s_ncand;
    }
    auto cid = [&](int k) { return S ? (int)s_cand[k] : k; };
    constexpr int kCU = 4;
    for (int c0 = warp; c0 < n_ex; c0 += kCU * nw) {
        const float* row[kCU];
        float sq[kCU];
#pragma unroll
        for (int u = 0; u < kCU; u++) {
            row[u] = D.centers + (uint64_t)cid(min(c0 + u * nw, n_ex - 1)) * d;
            sq[u] = 0.f;
        }
        for (int i = lane; i < d; i += 32) {
            const float qv = s_q[i];
#pragma unroll
            for (int u = 0; u < kCU; u++) {
                const float df = qv - __ldg(row[u] + i);
                sq[u] = fmaf(df, df, sq[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < kCU; u++) {
            const float v = warp_sum(sq[u]);
            if (lane == 0 && c0 + u * nw < n_ex) {
                const int c = cid(c0 + u * nw);
                s_keys[c] = ((uint64_t)float_key(v) << 32) | (uint32_t)c;
            }
        }
    }
    atomicAdd(&s_tot, tot);
    atomicAdd(&s_nz, nz);
    __syncthreads();
    // the 16 nearest centroids (keys distinct: the centroid index is their low word), in order
    block_select_smallest(s_keys, sort_n, kn, s_hist, s_wc, s_sel);
    block_bitonic_sort(s_keys, (int)next_pow2_dev((uint32_t)max(kn, 2)));
    const float lnN = logf(1.f + (float)D.n);
    if (t < 16) {
        const int j = min(t, C - 1);
        const float dj = key_float((uint32_t)(s_keys[j] >> 32));
        const float d0 = key_float((uint32_t)(s_keys[0] >> 32));
        s_f[12 + t] = t == 0 ? log1pf(d0) : log1pf(dj) - log1pf(d0);
        const uint32_t c = (uint32_t)s_keys[j];
        s_f[28 + t] = t < C ? log1pf((float)cc[qi * C + c]) / lnN : 0.f;
    } else if (t < 20) {
        const int i = t - 16;  // original label dim
        float lo = 0.f, hi = 1.f;
        if (i < l) {
            int sd = 0;
            for (int s = 0; s < l; s++)
                if (g.shuffle[s] == i) sd = s;
            const float left = (float)g.left[sd], span = fmaxf((float)g.span[sd], 1.f);
            lo = fminf(fmaxf((box[qi * 2 * l + 2 * i] - left) / span, 0.f), 1.f);
            hi = fminf(fmaxf((box[qi * 2 * l + 2 * i + 1] - left) / span, 0.f), 1.f);
        }
        s_f[2 * i] = lo;
        s_f[2 * i + 1] = hi;
        s_f[8 + i] = log10f(fmaxf(hi - lo, 1e-7f)) / 7.f;
    }
    __syncthreads();
    if (t == 0) {
        float near = 0.f;
        for (int j = 0; j < 16 && j < C; j++) near += (float)cc[qi * C + (uint32_t)s_keys[j]];
        s_f[44] = log1pf((float)s_tot) / lnN;
        s_f[45] = (float)s_nz / (float)C;
        s_f[46] = (float)(qk ? max(1u, min(qk[qi], k_max)) : k_max) / 100.f;
        s_f[47] = log1pf(near) / lnN;
    }
    __syncthreads();
    if (t < kMlpFeatures) feats[qi * kMlpFeatures + t] = s_f[t];
}

// ---- forward ---------------------------------------------------------------------------
// 128 threads (one hidden unit each), persistent over tiles of kTile samples: the weights are
// staged once per block, unit-major with rows padded by one word (49 and 129), so that both
// the staging writes and the reads of unit t's row across the threads are conflict-free;
// inputs are broadcast.
struct FwdOut {
    float* z;            // [n x 2]
    float* a1;           // [n x 128] hidden 1 (bf16-rounded), training only
    float* a2;           // [n x 128] hidden 2, training only
    uint32_t* nprobe;    // inference: per-query lists to probe
    uint8_t* sched;      // inference: per-query schedule flag
    int allow_sched;
    uint32_t max_probe;
};

__global__ void __launch_bounds__(kMlpHidden) k_mlp_forward(Params P, const float* __restrict__ x, uint64_t n,
                                                            FwdOut o) {
    constexpr int S1 = kMlpFeatures + 1, S2 = kMlpHidden + 1;  // padded weight rows
    constexpr int SH = kTile + 4;  // activation rows: 16-byte aligned, 4-way conflicts at most on the writes
    extern __shared__ __align__(16) float sm[];
    float* w1p = sm;                                   // [128][49]: unit-major W1
    float* w2p = w1p + kMlpHidden * S1;                // [128][129]
    float* w3 = w2p + kMlpHidden * S2;                 // [2][128]
    float* xs = w3 + kMlpOut * kMlpHidden;             // [48][kTile]: feature-major inputs
    float* h1 = xs + kMlpFeatures * kTile;             // [128][SH]: unit-major activations
    float* h2 = h1 + kMlpHidden * SH;                  // [128][SH]
    const int t = threadIdx.x;
    for (int e = t; e < kMlpHidden * kMlpFeatures; e += blockDim.x)
        w1p[(e / kMlpFeatures) * S1 + e % kMlpFeatures] = __bfloat162float(P.w[kMlpW1 + e]);
    for (int e = t; e < kMlpHidden * kMlpHidden; e += blockDim.x)
        w2p[(e / kMlpHidden) * S2 + e % kMlpHidden] = __bfloat162float(P.w[kMlpW2 + e]);
    for (int e = t; e < kMlpOut * kMlpHidden; e += blockDim.x) w3[e] = __bfloat162float(P.w[kMlpW3 + e]);
    const float bias1 = P.master[kMlpB1 + t], bias2 = P.master[kMlpB2 + t];
    // one hidden layer: acc[b] = sum over r of w[r] * in[r][b], in order r = 0, 1, ... (the
    // sample's inputs read four at a time as broadcasts)
    auto layer = [&](const float* wrow, const float* in, int rows, int ld, float (&acc)[kTile]) {
#pragma unroll
        for (int b = 0; b < kTile; b++) acc[b] = 0.f;
        for (int r = 0; r < rows; r++) {
            const float wv = wrow[r];
            const float4* v = reinterpret_cast<const float4*>(in + r * ld);
#pragma unroll
            for (int b4 = 0; b4 < kTile / 4; b4++) {
                const float4 a = v[b4];
                acc[4 * b4] = fmaf(wv, a.x, acc[4 * b4]);
                acc[4 * b4 + 1] = fmaf(wv, a.y, acc[4 * b4 + 1]);
                acc[4 * b4 + 2] = fmaf(wv, a.z, acc[4 * b4 + 2]);
                acc[4 * b4 + 3] = fmaf(wv, a.w, acc[4 * b4 + 3]);
            }
        }
    };
    for (uint64_t b0 = (uint64_t)blockIdx.x * kTile; b0 < n; b0 += (uint64_t)gridDim.x * kTile) {
        __syncthreads();  // the weights are staged; the previous tile's reads are done
        for (int e = t; e < kTile * kMlpFeatures; e += blockDim.x) {
            const int i = e / kTile, b = e % kTile;
            xs[e] = b0 + b < n ? bf16r(x[(b0 + b) * kMlpFeatures + i]) : 0.f;
        }
        __syncthreads();
        float acc[kTile];
        layer(w1p + t * S1, xs, kMlpFeatures, kTile, acc);
#pragma unroll
        for (int b = 0; b < kTile; b++) h1[t * SH + b] = bf16r(fmaxf(acc[b] + bias1, 0.f));
        __syncthreads();
        layer(w2p + t * S2, h1, kMlpHidden, SH, acc);
#pragma unroll
        for (int b = 0; b < kTile; b++) h2[t * SH + b] = bf16r(fmaxf(acc[b] + bias2, 0.f));
        __syncthreads();
        if (o.a1) {
            for (int e = t; e < kTile * kMlpHidden; e += blockDim.x) {
                const int b = e / kMlpHidden, u = e % kMlpHidden;
                if (b0 + b < n) {
                    o.a1[(b0 + b) * kMlpHidden + u] = h1[u * SH + b];
                    o.a2[(b0 + b) * kMlpHidden + u] = h2[u * SH + b];
                }
            }
        }
        if (t < kTile * kMlpOut) {
            const int b = t >> 1, c = t & 1;
            float z = 0.f;
            for (int j2 = 0; j2 < kMlpHidden; j2++) z = fmaf(w3[c * kMlpHidden + j2], h2[j2 * SH + b], z);
            z += P.master[kMlpB3 + c];
            const uint64_t bi = b0 + b;
            if (bi < n) {
                if (o.z) o.z[bi * kMlpOut + c] = z;
                if (c == 0 && o.nprobe) {
                    const float p = exp2f(fminf(fmaxf(z, 0.f), 20.f));
                    o.nprobe[bi] = (uint32_t)min((float)o.max_probe, fmaxf(1.f, rintf(p)));
                }
                if (c == 1 && o.sched) o.sched[bi] = (o.allow_sched && z > 0.f) ? 1 : 0;
            }
        }
    }
}

// ---- loss and backward -----------------------------------------------------------------
// loss = mean over the batch of (z0 - y0)^2 + BCE(sigmoid(z1), y1)
__global__ void k_loss_grad(const float* __restrict__ z, const float* __restrict__ y, uint64_t n,
                            float* __restrict__ dz, double* __restrict__ loss) {
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (b < n) {
        const float z0 = z[2 * b], z1 = z[2 * b + 1], y0 = y[2 * b], y1 = y[2 * b + 1];
        const float inv = 1.f / (float)n;
        dz[2 * b] = 2.f * (z0 - y0) * inv;
        const float s = 1.f / (1.f + expf(-z1));
        dz[2 * b + 1] = (s - y1) * inv;
        // numerically stable BCE with logits: max(z,0) - z*y + log(1 + exp(-|z|))
        l = (double)(z0 - y0) * (z0 - y0) + (double)(fmaxf(z1, 0.f) - z1 * y1 + log1pf(expf(-fabsf(z1))));
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / (double)n);
}

// dW[o][i] = sum_b dY[b][o] * X[b][i], db[o] = sum_b dY[b][o]; one block per output row o
__global__ void __launch_bounds__(128) k_grad_w(const float* __restrict__ dy, int n_out, const float* __restrict__ xin,
                                                int n_in, uint64_t n, float* __restrict__ dw, float* __restrict__ db) {
    const int o = blockIdx.x, t = threadIdx.x;
    for (int i = t; i < n_in; i += blockDim.x) {
        float s = 0.f;
        for (uint64_t b = 0; b < n; b++) s = fmaf(dy[b * n_out + o], xin[b * n_in + i], s);
        dw[(uint64_t)o * n_in + i] = s;
    }
    if (t < 32) {
        float s = 0.f;
        for (uint64_t b = t; b < n; b += 32) s += dy[b * n_out + o];
        for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
        if (t == 0) db[o] = s;
    }
}

// dX[b][j] = (sum_o dY[b][o] * W[o][j]) * (A[b][j] > 0); one block per sample
__global__ void __launch_bounds__(128) k_grad_x(const float* __restrict__ dy, int n_out,
                                                const __nv_bfloat16* __restrict__ w, int n_in,
                                                const float* __restrict__ a, uint64_t n, float* __restrict__ dx) {
    const uint64_t b = blockIdx.x;
    for (int j = threadIdx.x; j < n_in; j += blockDim.x) {
        float s = 0.f;
        for (int o = 0; o < n_out; o++) s = fmaf(dy[b * n_out + o], __bfloat162float(w[(uint64_t)o * n_in + j]), s);
        dx[b * n_in + j] = a[b * n_in + j] > 0.f ? s : 0.f;
    }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ pw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    pw[i] = __float2bfloat16_rn(pi);
}

__global__ void k_to_bf16_params(const float* __restrict__ p, int n, __nv_bfloat16* __restrict__ pw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pw[i] = __float2bfloat16_rn(p[i]);
}

__global__ void k_gather_batch(const float* __restrict__ x, const float* __restrict__ y,
                               const uint32_t* __restrict__ idx, uint64_t n, float* __restrict__ xb,
                               float* __restrict__ yb) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * kMlpFeatures) return;
    const uint64_t b = e / kMlpFeatures, i = e % kMlpFeatures;
    const uint64_t src = idx[b];
    xb[e] = x[src * kMlpFeatures + i];
    if (i < kMlpOut) yb[b * kMlpOut + i] = y[src * kMlpOut + i];
}

// model buffer: master | adam m | adam v | grad (fp32, kMlpParams each) | bf16 copy
struct ModelPtrs {
    float *master, *m, *v, *grad;
    __nv_bfloat16* w;
};

ModelPtrs model_ptrs(hdg_index* idx) {
    if (!idx->mlp.ptr) {
        idx->mlp.ensure(sizeof(float) * 4 * kMlpParams + sizeof(__nv_bfloat16) * kMlpParams + 256);
        CK(cudaMemset(idx->mlp.ptr, 0, idx->mlp.bytes));
    }
    float* base = static_cast<float*>(idx->mlp.ptr);
    ModelPtrs p;
    p.master = base;
    p.m = base + kMlpParams;
    p.v = base + 2 * kMlpParams;
    p.grad = base + 3 * kMlpParams;
    p.w = reinterpret_cast<__nv_bfloat16*>(base + 4 * kMlpParams);
    return p;
}

size_t forward_smem() {
    return sizeof(float) * ((kMlpFeatures + 1) * kMlpHidden + (kMlpHidden + 1) * kMlpHidden + kMlpOut * kMlpHidden +
                            kTile * kMlpFeatures + 2 * (kTile + 4) * kMlpHidden);
}

void launch_forward(const ModelPtrs& mp, const float* x, uint64_t n, const FwdOut& o, cudaStream_t st) {
    const size_t sm = forward_smem();
    CK(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    // persistent over the tiles: as many blocks as fit at once (each stages the weights once)
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_forward, kMlpHidden, sm));
    const uint64_t tiles = (n + kTile - 1) / kTile;
    const uint64_t blocks = std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)sm_count() * std::max(per_sm, 1)));
    k_mlp_forward<<<(unsigned)blocks, kMlpHidden, sm, st>>>(Params{mp.master, mp.w}, x, n, o);
    CK_LAUNCH();
}

// backward of one batch into mp.grad (forward activations a1, a2 and outputs z given)
void launch_backward(const ModelPtrs& mp, const float* x, const float* y, uint64_t n, const float* z,
                     const float* a1, const float* a2, float* dz, float* dh2, float* dh1, double* loss,
                     cudaStream_t st) {
    k_loss_grad<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(z, y, n, dz, loss);
    CK_LAUNCH();
    k_grad_w<<<kMlpOut, 128, 0, st>>>(dz, kMlpOut, a2, kMlpHidden, n, mp.grad + kMlpW3, mp.grad + kMlpB3);
    CK_LAUNCH();
    k_grad_x<<<(unsigned)n, 128, 0, st>>>(dz, kMlpOut, mp.w + kMlpW3, kMlpHidden, a2, n, dh2);
    CK_LAUNCH();
    k_grad_w<<<kMlpHidden, 128, 0, st>>>(dh2, kMlpHidden, a1, kMlpHidden, n, mp.grad + kMlpW2, mp.grad + kMlpB2);
    CK_LAUNCH();
    k_grad_x<<<(unsigned)n, 128, 0, st>>>(dh2, kMlpHidden, mp.w + kMlpW2, kMlpHidden, a1, n, dh1);
    CK_LAUNCH();
    // the layer-1 input is the bf16-rounded feature row, as in the forward pass
    k_grad_w<<<kMlpHidden, 128, 0, st>>>(dh1, kMlpHidden, x, kMlpFeatures, n, mp.grad + kMlpW1, mp.grad + kMlpB1);
    CK_LAUNCH();
}

__global__ void k_round_rows(const float* __restrict__ x, uint64_t n, float* __restrict__ out) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) out[e] = bf16r(x[e]);
}

}  // namespace

void learned_features(hdg_index* idx, const float* d_queries, uint64_t q, const float* box, const uint32_t* cc,
                      const uint32_t* qk, uint32_t k_max, float* feats, cudaStream_t st, const float* S, uint64_t ldS,
                      const float* qnorm) {
    const IndexDev& D = idx->dev;
    const int sort_n = (int)next_pow2(std::max<uint32_t>(D.C, 16));
    const size_t sm = (sizeof(uint64_t) + sizeof(uint32_t) + sizeof(float)) * sort_n + sizeof(float) * D.d;
    HDG_REQUIRE(sm <= 200 * 1024, HDG_ERR_UNSUPPORTED, "feature kernel does not fit shared memory");
    CK(cudaFuncSetAttribute(k_features, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_features<<<(unsigned)q, 128, sm, st>>>(D, idx->grid, d_queries, box, cc, qk, k_max, sort_n, S, ldS, qnorm,
                                             feats);
    CK_LAUNCH();
}

void learned_infer(hdg_index* idx, const float* feats, uint64_t q, uint32_t* nprobe, uint8_t* sched, int allow_sched,
                   uint32_t max_probe, float* z, cudaStream_t st) {
    HDG_REQUIRE(idx->mlp_ready, HDG_ERR_STATE, "no trained model in this index");
    const ModelPtrs mp = model_ptrs(idx);
    FwdOut o{z, nullptr, nullptr, nprobe, sched, allow_sched, max_probe};
    launch_forward(mp, feats, q, o, st);
}

void mlp_init(hdg_index* idx, uint64_t seed) {
    const ModelPtrs mp = model_ptrs(idx);
    std::vector<float> p(kMlpParams, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int count) {  // He-uniform for the ReLU layers
        const float a = std::sqrt(6.f / (float)fan_in);
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < count; i++) p[off + i] = u(rng);
    };
    fill(kMlpW1, kMlpFeatures, kMlpHidden * kMlpFeatures);
    fill(kMlpW2, kMlpHidden, kMlpHidden * kMlpHidden);
    fill(kMlpW3, kMlpHidden, kMlpOut * kMlpHidden);
    mlp_set(idx, p.data(), kMlpParams);
}

void mlp_set(hdg_index* idx, const float* host, size_t count) {
    HDG_REQUIRE(count == (size_t)kMlpParams, HDG_ERR_INVALID_ARG, "wrong parameter count for the MLP");
    const ModelPtrs mp = model_ptrs(idx);
    CK(cudaMemcpy(mp.master, host, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    CK(cudaMemset(mp.m, 0, sizeof(float) * 2 * kMlpParams));
    k_to_bf16_params<<<(kMlpParams + 255) / 256, 256>>>(mp.master, kMlpParams, mp.w);
    CK_LAUNCH();
    CK(cudaDeviceSynchronize());
    idx->mlp_step = 0;
    idx->mlp_ready = true;
}

void mlp_get(hdg_index* idx, float* host, size_t count) {
    HDG_REQUIRE(idx->mlp_ready, HDG_ERR_STATE, "no model in this index");
    HDG_REQUIRE(count == (size_t)kMlpParams, HDG_ERR_INVALID_ARG, "wrong parameter count for the MLP");
    const ModelPtrs mp = model_ptrs(idx);
    CK(cudaMemcpy(host, mp.master, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
}

void mlp_forward(hdg_index* idx, const float* d_x, uint64_t n, float* d_z, cudaStream_t st) {
    HDG_REQUIRE(idx->mlp_ready, HDG_ERR_STATE, "no model in this index");
    const ModelPtrs mp = model_ptrs(idx);
    launch_forward(mp, d_x, n, FwdOut{d_z, nullptr, nullptr, nullptr, nullptr, 0, 0}, st);
}

double mlp_gradients(hdg_index* idx, const float* d_x, const float* d_y, uint64_t n, float* d_grad, cudaStream_t st) {
    HDG_REQUIRE(idx->mlp_ready, HDG_ERR_STATE, "no model in this index");
    HDG_REQUIRE(n > 0, HDG_ERR_INVALID_ARG, "empty batch");
    const ModelPtrs mp = model_ptrs(idx);
    DevMem<float> z(n * kMlpOut), a1(n * kMlpHidden), a2(n * kMlpHidden), dz(n * kMlpOut);
    DevMem<float> dh2(n * kMlpHidden), dh1(n * kMlpHidden), xr(n * kMlpFeatures);
    DevMem<double> loss(1);
    CK(cudaMemsetAsync(loss.p, 0, sizeof(double), st));
    k_round_rows<<<(unsigned)((n * kMlpFeatures + 255) / 256), 256, 0, st>>>(d_x, n * kMlpFeatures, xr.p);
    CK_LAUNCH();
    launch_forward(mp, xr.p, n, FwdOut{z.p, a1.p, a2.p, nullptr, nullptr, 0, 0}, st);
    launch_backward(mp, xr.p, d_y, n, z.p, a1.p, a2.p, dz.p, dh2.p, dh1.p, loss.p, st);
    CK(cudaMemcpyAsync(d_grad, mp.grad, sizeof(float) * kMlpParams, cudaMemcpyDeviceToDevice, st));
    double h = 0.0;
    CK(cudaMemcpyAsync(&h, loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return h;
}

double mlp_train(hdg_index* idx, const float* d_x, const float* d_y, uint64_t n, uint32_t epochs, uint32_t batch,
                 float lr, uint64_t seed, cudaStream_t st) {
    HDG_REQUIRE(idx->mlp_ready, HDG_ERR_STATE, "initialise or load the model first");
    HDG_REQUIRE(n > 0 && batch > 0 && epochs > 0, HDG_ERR_INVALID_ARG, "empty training run");
    const ModelPtrs mp = model_ptrs(idx);
    const uint64_t B = std::min<uint64_t>(batch, n);
    DevMem<float> xb(B * kMlpFeatures), xr(B * kMlpFeatures), yb(B * kMlpOut), z(B * kMlpOut);
    DevMem<float> a1(B * kMlpHidden), a2(B * kMlpHidden), dz(B * kMlpOut), dh2(B * kMlpHidden), dh1(B * kMlpHidden);
    DevMem<uint32_t> perm(n);
    DevMem<double> loss(1);
    std::vector<uint32_t> order(n);
    for (uint64_t i = 0; i < n; i++) order[i] = (uint32_t)i;
    std::mt19937_64 rng(seed);
    double last = 0.0;
    for (uint32_t ep = 0; ep < epochs; ep++) {
        std::shuffle(order.begin(), order.end(), rng);
        CK(cudaMemcpyAsync(perm.p, order.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(loss.p, 0, sizeof(double), st));
        uint64_t steps = 0;
        for (uint64_t s = 0; s + B <= n || (s < n && steps == 0); s += B) {
            const uint64_t nb = std::min<uint64_t>(B, n - s);
            k_gather_batch<<<(unsigned)((nb * kMlpFeatures + 255) / 256), 256, 0, st>>>(d_x, d_y, perm.p + s, nb,
                                                                                        xb.p, yb.p);
            CK_LAUNCH();
            k_round_rows<<<(unsigned)((nb * kMlpFeatures + 255) / 256), 256, 0, st>>>(xb.p, nb * kMlpFeatures,
                                                                                      xr.p);
            CK_LAUNCH();
            launch_forward(mp, xr.p, nb, FwdOut{z.p, a1.p, a2.p, nullptr, nullptr, 0, 0}, st);
            launch_backward(mp, xr.p, yb.p, nb, z.p, a1.p, a2.p, dz.p, dh2.p, dh1.p, loss.p, st);
            idx->mlp_step++;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)idx->mlp_step), c2 = 1.f - std::pow(b2, (float)idx->mlp_step);
            k_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(mp.master, mp.grad, mp.m, mp.v, kMlpParams, lr, b1, b2,
                                                             1e-8f, c1, c2, mp.w);
            CK_LAUNCH();
            steps++;
        }
        double h = 0.0;
        CK(cudaMemcpyAsync(&h, loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        last = h / (double)std::max<uint64_t>(steps, 1);
    }
    return last;
}

}  // namespace hdg
