// Device-side building blocks shared by the build and query kernels.
//
// The integer stages (filter box, cell ids, Morton codes) follow the reference's float
// semantics exactly so that cell boxes, Morton codes and counts are bit-identical:
//   - filter recovery: denormalize_labels_kernel (src/core/preprocessing.cu:3-32)
//   - cell id: get_grid_id_device (src/index/2-level_index/Super-Grid-IVF_PQ.cu:24-26)
//   - cell box: get_filter_grid_ranges_kernel (Super-Grid-IVF_PQ.cu:930-961)
//   - Morton: morton_encode (src/core/zorder.cu:3-15)
// A C-style float->uint64 cast on the GPU is cvt.rzi.u64.f32, which saturates
// (negatives -> 0, >= 2^64 -> UINT64_MAX, NaN -> 2^63); the kernels use the same cast as the
// reference, so they agree with it on every input.
#pragma once
#include <cfloat>
#include <climits>
#include <cstdint>

#include "hdg_index.h"

namespace hdg {

// ---- filter recovery (preprocessing.cu:13-30) --------------------------------------
// x points at the query's label row; returns [lo, hi] for label dim i.
__device__ __forceinline__ void recover_dim(const FilterDev& f, const float* row, int i, float* lo,
                                            float* hi) {
    const int t = f.type[i];
    if (t == 0) {
        // max(float, double) promotes to double; the result is rounded back to f32.
        const float x = row[i];
        const double sl = fmax((double)f.shift_val[2 * i], 1e-7);
        const double sr = fmax((double)f.shift_val[2 * i + 1], 1e-7);
        *lo = (float)((double)x - sl);
        *hi = (float)((double)x + sr);
    } else if (t == 1) {
        // the f32 -> s32 conversion saturates (a label >= 2^31 gives INT_MAX); the bound is
        // checked in 64 bits so that 2 * v + 1 cannot wrap for labels of 2^30 and above
        const int v = (int)(row[i] - 1.0f);
        if (v >= 0 && 2 * (int64_t)v + 1 < (int64_t)f.n_map) {
            *lo = f.map[2 * v];
            *hi = f.map[2 * v + 1];
        } else {  // out-of-table label: the reference reads out of bounds; empty box here
            *lo = FLT_MAX;
            *hi = -FLT_MAX;
        }
    } else if (t == 2) {
        const int v = (int)row[i];  // saturating, like the map type
        const int dv = f.div_value[i];
        // INT_MIN / -1 is the one quotient that overflows: kept as INT_MIN
        *lo = (float)((v == INT_MIN && dv == -1) ? v : v / dv);
        *hi = FLT_MAX;
    } else {
        // type 3 reads a [lo, hi] pair from a filter_dim = 2 label row (preprocessing.cu:27-28)
        *lo = row[2 * i];
        *hi = row[2 * i + 1];
    }
}

// ---- grid cells (Super-Grid-IVF_PQ.cu:24-26) ----------------------------------------
// ((uint64_t)((x - l) * M)) / len, returned as int (truncating), float arithmetic.
__device__ __forceinline__ int grid_id(float x, uint64_t left, uint64_t len, int M) {
    const float t = __fmul_rn(__fsub_rn(x, (float)left), (float)M);
    const uint64_t u = (uint64_t)t;  // saturating cvt.rzi.u64.f32
    return (int)(u / len);
}

// Cell box of one shuffled dim (Super-Grid-IVF_PQ.cu:947-960).
__device__ __forceinline__ void cell_range(float box_lo, float box_hi, uint64_t left, uint64_t span,
                                           int M, int* out_lo, int* out_hi) {
    const uint64_t blo = (uint64_t)box_lo;  // saturating
    const uint64_t bhi = (uint64_t)box_hi;
    const float l = (float)(blo > left ? blo : left);
    const uint64_t rr = left + span;
    const float r = (float)(bhi < rr ? bhi : rr);
    const int gl = grid_id(l, left, span, M);
    const int gr = grid_id(r, left, span, M);
    int hi = gr < M - 1 ? gr : M - 1;
    int lo = hi < gl ? hi : gl;
    // The int truncation can only go negative when the uint64 cell value reaches 2^31,
    // where the reference indexes out of bounds; clamp to a valid cell instead.
    if (hi < 0) hi = 0;
    if (lo < 0) lo = 0;
    *out_hi = hi;
    *out_lo = lo;
}

// ---- Morton (zorder.cu:3-15): MSB-first bit interleave over valid dims -------------
__device__ __forceinline__ uint64_t morton_encode(const int* coords, int dims, int max_bits,
                                                  int valid_map) {
    uint64_t code = 0;
    for (int b = 0; b < max_bits; ++b) {
        for (int i = 0; i < dims; ++i) {
            if (!((valid_map >> i) & 1)) continue;
            const int bit = (coords[i] >> (max_bits - 1 - b)) & 1;
            code = (code << 1) | (uint64_t)bit;
        }
    }
    return code;
}

// ---- Morton decode and the next in-box code (zorder.cu:17-34, 83-243) -----------------
__device__ __forceinline__ void morton_decode(uint64_t code, int* coords, int dims, int max_bits, int valid_map) {
    const int active = __popc(valid_map);
    for (int i = 0; i < dims; ++i) coords[i] = 0;
    for (int b = 0; b < max_bits; ++b) {
        int j = 0;
        for (int i = 0; i < dims; ++i) {
            if (!((valid_map >> i) & 1)) continue;
            const int shift = (max_bits - 1 - b) * active + (active - 1 - j);
            coords[i] |= (int)((code >> shift) & 1) << (max_bits - 1 - b);
            j++;
        }
    }
}

// box: [lo, hi] cell pairs of every dim (masked dims included, as the reference checks them)
__device__ __forceinline__ bool cells_in_box(const int* c, const int* box, int dims) {
    for (int i = 0; i < dims; ++i)
        if (c[i] < box[2 * i] || c[i] > box[2 * i + 1]) return false;
    return true;
}

__device__ __forceinline__ int with_low_bits(int target, int source, int k) {
    const uint64_t m = (1ull << k) - 1;
    return (int)(((uint64_t)(int64_t)target & ~m) | ((uint64_t)(int64_t)source & m));
}

// The smallest code the reference's getNextZValueBaseline (zorder.cu:83-243) jumps to from
// cur: cur + 1 when that decodes inside the box; otherwise the lowest violating bit of
// cur + 1 is carried per its left/right-violation rules.  Returns false when no jump
// exists.  The steps, including which bits count as "safe", are the reference's; the
// result decides which candidate sub-ranges exist, so it has to match bit for bit.
__device__ inline bool next_code_in_box(uint64_t cur, const int* box, int dims, int max_bits, int valid_map,
                                        uint64_t* next) {
    const uint64_t nisp = cur + 1;
    int c[kMaxDims];
    morton_decode(nisp, c, dims, max_bits, valid_map);
    if (cells_in_box(c, box, dims)) {
        *next = nisp;
        return true;
    }
    const int active = __popc(valid_map);
    int flag[kMaxDims], out_step[kMaxDims], save_min[kMaxDims], save_max[kMaxDims], vdim[kMaxDims];
    int j = 0;
    for (int i = 0; i < dims; ++i) {
        flag[i] = 0;
        if (!((valid_map >> i) & 1)) continue;
        vdim[j++] = i;
        out_step[i] = save_min[i] = save_max[i] = max_bits;
        for (int s = 0; s < max_bits; ++s) {  // first differing bit against the low corner
            const int sh = max_bits - 1 - s;
            const int lb = (box[2 * i] >> sh) & 1, cb = (c[i] >> sh) & 1;
            if (cb < lb) {
                flag[i] = -1;
                out_step[i] = s;
                break;
            }
            if (cb > lb) break;
        }
        if (flag[i] == 0) {
            for (int s = 0; s < max_bits; ++s) {  // ... and against the high corner
                const int sh = max_bits - 1 - s;
                const int hb = (box[2 * i + 1] >> sh) & 1, cb = (c[i] >> sh) & 1;
                if (cb > hb) {
                    flag[i] = 1;
                    out_step[i] = s;
                    break;
                }
                if (cb < hb) break;
            }
        }
        if (flag[i] != -1) {
            for (int s = 0; s < max_bits; ++s) {
                const int sh = max_bits - 1 - s;
                if (((c[i] >> sh) & 1) > ((box[2 * i] >> sh) & 1)) {
                    save_min[i] = s;
                    break;
                }
            }
        }
        if (flag[i] != 1) {
            for (int s = 0; s < max_bits; ++s) {
                const int sh = max_bits - 1 - s;
                if (((c[i] >> sh) & 1) < ((box[2 * i + 1] >> sh) & 1)) {
                    save_max[i] = s;
                    break;
                }
            }
        }
    }
    int change = 0;
    j = 0;
    for (int i = 0; i < dims; ++i) {
        if (!((valid_map >> i) & 1)) continue;
        if (out_step[i] < max_bits) change = max(change, (max_bits - 1 - out_step[i]) * active + (active - 1 - j));
        j++;
    }
    int d = vdim[active - 1 - (change % active)];
    if (flag[d] == 1) {
        int found = -1;
        for (int bp = change + 1; bp < max_bits * active; ++bp) {
            const int a = active - 1 - (bp % active);
            if (bp <= (max_bits - 1 - save_max[vdim[a]]) * active + (active - 1 - a) && ((nisp >> bp) & 1ull) == 0) {
                found = bp;
                break;
            }
        }
        if (found < 0) return false;
        change = found;
        d = vdim[active - 1 - (change % active)];
        save_min[d] = max_bits - 1 - (change / active);
        flag[d] = 0;
    }
    const int blocks = change / active;
    j = 0;
    for (int i = 0; i < dims; ++i) {
        if (!((valid_map >> i) & 1)) continue;
        if (flag[i] >= 0) {
            const int bits = blocks + (vdim[j] > d ? 1 : 0);
            c[i] = change <= (max_bits - 1 - save_min[i]) * active + (active - 1 - j) ? with_low_bits(c[i], 0, bits)
                                                                                    : with_low_bits(c[i], box[2 * i], bits);
        } else {
            c[i] = box[2 * i];
        }
        j++;
    }
    *next = morton_encode(c, dims, max_bits, valid_map) | (1ull << change);
    return true;
}

// ---- distances --------------------------------------------------------------------
// Exact f32 L2 in the reference's order (refine.cu:71-88 with d <= 512): each squared
// difference rounded to f32, then summed sequentially in dimension order.
__device__ __forceinline__ float seq_l2(const float* __restrict__ a, const float* __restrict__ b,
                                        int d) {
    float s = 0.f;
    for (int i = 0; i < d; ++i) {
        const float t = __fsub_rn(a[i], b[i]);
        s = __fadd_rn(s, __fmul_rn(t, t));
    }
    return s;
}

// Monotone map float -> u32 (ascending order preserved, +inf largest finite key).
__device__ __forceinline__ uint32_t float_key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// In-place ascending bitonic sort of n (power of two) u64 keys in shared memory.
// Must be called by all threads of the block.
__device__ __forceinline__ void block_bitonic_sort(uint64_t* keys, int n) {
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < (n >> 1); i += blockDim.x) {
                const int lo = 2 * i - (i & (j - 1));
                const int hi = lo + j;
                const bool up = ((lo & k) == 0);
                const uint64_t a = keys[lo], b = keys[hi];
                if ((a > b) == up) {
                    keys[lo] = b;
                    keys[hi] = a;
                }
            }
            __syncthreads();
        }
    }
}

// Stable in-place compaction of the keys that are not ~0 to the front of keys[0, n) (the
// rest set to ~0); all threads of the block.  s_wc: 32 words of shared scratch.
__device__ __forceinline__ void block_compact_keys(uint64_t* keys, int n, uint32_t* s_wc) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nw = blockDim.x >> 5;
    uint32_t base = 0;
    for (int r = 0; r < n; r += blockDim.x) {
        const int e = r + t;
        const uint64_t v = e < n ? keys[e] : ~0ull;
        const bool f = v != ~0ull;
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) s_wc[warp] = __popc(bal);
        __syncthreads();  // every read of this round is done before any write
        uint32_t off = 0, tot = 0;
        for (int i = 0; i < nw; i++) {
            const uint32_t c = s_wc[i];
            off += i < warp ? c : 0u;
            tot += c;
        }
        // the destination is below r + blockDim.x: no later round's key is overwritten
        if (f) keys[base + off + __popc(bal & ((1u << lane) - 1u))] = v;
        __syncthreads();
        base += tot;
    }
    for (int e = (int)base + t; e < n; e += blockDim.x) keys[e] = ~0ull;
    __syncthreads();
}

// The k smallest keys of keys[0, n) (the keys other than ~0 distinct, at least k of them):
// compacted to keys[0, k) in their original relative order, the rest set to ~0; returns the
// k-th smallest (compact = false: only returns it, the keys stay as they are).  A radix select over 8-bit digits from the most significant one, stopping
// once one key is left in the chosen digit's bin, then one compaction.  All threads; s_hist:
// 256 words, s_wc: 32 words, s_sel: 4 words of shared scratch.
__device__ __forceinline__ uint64_t block_select_smallest(uint64_t* keys, int n, int k, uint32_t* s_hist, uint32_t* s_wc,
                                          unsigned long long* s_sel, bool compact = true) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    // the bytes above the highest one where the smallest and largest key differ are common to
    // every key: the select starts below them
    if (t == 0) {
        s_sel[0] = ~0ull;
        s_sel[1] = 0ull;
    }
    __syncthreads();
    unsigned long long kmin = ~0ull, kmax = 0ull;
    for (int i = t; i < n; i += blockDim.x) {
        const uint64_t v = keys[i];
        if (v != ~0ull) {
            kmin = min(kmin, (unsigned long long)v);
            kmax = max(kmax, (unsigned long long)v);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if (lane == 0) {
        atomicMin(&s_sel[0], kmin);
        atomicMax(&s_sel[1], kmax);
    }
    __syncthreads();
    const uint64_t lo_all = s_sel[0], diff = lo_all ^ s_sel[1];
    const int top = diff ? (63 - __clzll((long long)diff)) / 8 * 8 : 0;  // shift of the highest differing byte
    uint64_t pmask = top >= 56 ? 0ull : ~0ull << (top + 8);
    uint64_t prefix = lo_all & pmask;
    __syncthreads();  // every thread has read s_sel before it is reused
    uint32_t need = (uint32_t)k, cnt = 0;
    for (int shift = top; shift >= 0; shift -= 8) {
        for (int i = t; i < 256; i += blockDim.x) s_hist[i] = 0;
        __syncthreads();
        for (int i = t; i < n; i += blockDim.x) {
            const uint64_t v = keys[i];
            if (v != ~0ull && (v & pmask) == prefix) atomicAdd(&s_hist[(v >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (warp == 0) {  // lane l scans bins 8l .. 8l + 7
            uint32_t c[8], sum = 0;
#pragma unroll
            for (int b = 0; b < 8; b++) {
                c[b] = s_hist[8 * lane + b];
                sum += c[b];
            }
            uint32_t incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            uint32_t run = incl - sum;
            if (run < need && need <= incl) {
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    if (run < need && need <= run + c[b]) {
                        s_sel[0] = (unsigned long long)(8 * lane + b);
                        s_sel[1] = need - run;
                        s_sel[2] = c[b];
                    }
                    run += c[b];
                }
            }
        }
        __syncthreads();
        prefix |= (uint64_t)s_sel[0] << shift;
        pmask |= 255ull << shift;
        need = (uint32_t)s_sel[1];
        cnt = (uint32_t)s_sel[2];
        if (cnt == 1) break;  // one key left with this prefix: the k-th
    }
    __syncthreads();  // every thread has read s_sel
    for (int i = t; i < n; i += blockDim.x) {
        const uint64_t v = keys[i];
        if (v != ~0ull && (v & pmask) == prefix) s_sel[3] = v;
    }
    __syncthreads();
    const uint64_t kth = s_sel[3];
    if (!compact) return kth;
    for (int i = t; i < n; i += blockDim.x)
        if (keys[i] > kth) keys[i] = ~0ull;
    __syncthreads();
    block_compact_keys(keys, n, s_wc);
    return kth;
}

// Band [lo, hi] around the exact f32 squared distance between a query and a centroid from
// their squared norms qn, cn and a BF16 tensor-core dot product s: |(qn + cn - 2 s) - exact| is
// below 2 * 2^-8 sqrt(qn cn) for BF16-rounded inputs, plus f32 rounding of the norms and sums;
// the band doubles both terms.
__device__ __forceinline__ void coarse_band(float qn, float cn, float s, float* lo, float* hi) {
    const float a = qn + cn - 2.f * s;
    const float e = 0.015625f * sqrtf(qn * cn) + 1e-4f * (qn + cn);
    *lo = a - e;
    *hi = a + e;
}

__device__ __forceinline__ uint32_t next_pow2_dev(uint32_t x) {
    return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace hdg
