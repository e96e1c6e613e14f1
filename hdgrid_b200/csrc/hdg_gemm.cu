// BF16 tcgen05 GEMM for the coarse assignment: S[q][n] = Q[q] . Cn[n] with FP32 accumulation
// in tensor memory.  It replaces the per-query FP32 distance loops of ::refine
// (src/core/refine.cu:36-75) for the ranking step of k_coarse; the chosen set is still
// decided by exact FP32 distances re-checked inside a provable error band.
//
// One CTA = 128 queries x 128 centroids, 128 threads.  K runs in chunks of 64 through two
// shared-memory stages: all threads copy chunk kc+1 of A (queries) and B (centroids) with
// cp.async (16 bytes, zero-filled past the matrix edges) into the K-major "no swizzle"
// canonical UMMA layout (8-row x 16-byte core matrices; K chunks of 8 elements LBO bytes
// apart, 8-row groups SBO bytes apart) while the tensor core runs chunk kc: one elected
// thread issues four tcgen05.mma (M=128, N=128, K=16) per chunk and a tcgen05.commit to the
// stage's mbarrier, which is waited on only before that stage is refilled.  The epilogue
// reads the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows of the
// tile) and writes S.  Every wait is bounded: on expiry the kernel records an error in *err,
// lets its own copies land and stops instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <mutex>

#include "hdg_internal.h"

namespace hdg {

constexpr int GM = 128, GN = 128, GK = 64;  // tile
constexpr int kGemmThreads = 128;
constexpr uint32_t kStage = 16 * 1024;         // one 128 x 64 bf16 chunk in the canonical layout
constexpr uint32_t kLBO = (GM / 8) * 128;      // bytes between the two 8-element K chunks
constexpr uint32_t kSBO = 128;                 // bytes between 8-row groups
constexpr long long kSpinLimit = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle UMMA shared-memory descriptor (layout of cute::UMMA::SmemDescriptor:
// start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46), version 1 [46,48), layout 0 [61,64)).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3fff);
    d |= (uint64_t)((kLBO >> 4) & 0x3fff) << 16;
    d |= (uint64_t)((kSBO >> 4) & 0x3fff) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: F32 accumulate, BF16 A and B, both K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(GN >> 3) << 17) |
                            ((uint32_t)(GM >> 4) << 24);

// element (row, k) of a GM x GK chunk -> byte offset in the canonical layout
__device__ __forceinline__ uint32_t canon_off(int row, int k) {
    return (uint32_t)(k >> 3) * kLBO + (uint32_t)(row >> 3) * kSBO + (uint32_t)(row & 7) * 16u +
           (uint32_t)(k & 7) * 2u;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (long long it = 0; it < kSpinLimit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// out[r][n] = sum_k A[r][k] * B[n][k]; A [rows x d] bf16, B [cols x d] bf16, out row stride ldo.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}

// out[r][n] = sum_k A[r][k] * B[n][k]; A [rows x d] bf16, B [cols x d] bf16, out row stride ldo.
__global__ void __launch_bounds__(kGemmThreads) k_umma_dot(const __nv_bfloat16* __restrict__ A, uint64_t rows,
                                                           const __nv_bfloat16* __restrict__ B, uint64_t cols,
                                                           int d, float* __restrict__ out, uint64_t ldo,
                                                           int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];  // stage s: A at 2s*kStage, B at (2s+1)*kStage
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const uint64_t r0 = (uint64_t)blockIdx.x * GM, c0 = (uint64_t)blockIdx.y * GN;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t bar[2] = {smem_u32(&s_bar[0]), smem_u32(&s_bar[1])};
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(GN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar[0]), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar[1]), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    // chunk kc -> stage s: every 16-byte piece of the 128 x 64 tiles of A and B
    auto load = [&](int kc, int st) {
        const int k0 = kc * GK;
        const uint32_t sa = sbase + (uint32_t)(2 * st) * kStage, sb = sa + kStage;
        for (int p = t; p < GM * (GK / 8); p += kGemmThreads) {
            const int row = p >> 3, kk = (p & 7) * 8;
            const bool kin = k0 + kk < d;
            const bool va = kin && r0 + row < rows, vb = kin && c0 + row < cols;
            cp_async16(sa + canon_off(row, kk), va ? (const void*)(A + (r0 + row) * d + k0 + kk) : (const void*)A, va);
            cp_async16(sb + canon_off(row, kk), vb ? (const void*)(B + (c0 + row) * d + k0 + kk) : (const void*)B, vb);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    uint32_t phase[2] = {0u, 0u};
    const int nchunks = (d + GK - 1) / GK;
    load(0, 0);
    for (int kc = 0; kc < nchunks; kc++) {
        const int st = kc & 1;
        if (kc + 1 < nchunks) {
            const int s1 = st ^ 1;
            if (kc >= 1) {  // stage s1 was read by chunk kc - 1's MMAs
                if (!mbar_wait(bar[s1], phase[s1])) s_fail = 1;
                phase[s1] ^= 1u;
            }
            load(kc + 1, s1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (s_fail) break;
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t sa = sbase + (uint32_t)(2 * st) * kStage, sb = sa + kStage;
#pragma unroll
            for (int ks = 0; ks < GK / 16; ks++) {
                const uint64_t da = umma_desc(sa + ks * 2 * kLBO);
                const uint64_t db = umma_desc(sb + ks * 2 * kLBO);
                const uint32_t acc = (kc > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar[st])
                         : "memory");
        }
    }
    // the last commit covers every earlier MMA of this thread
    if (!s_fail) {
        const int st = (nchunks - 1) & 1;
        if (!mbar_wait(bar[st], phase[st])) s_fail = 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!s_fail) {
        const uint64_t row = r0 + warp * 32 + lane;
        for (int cb = 0; cb < GN; cb += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < rows)
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (c0 + cb + j < cols) out[row * ldo + c0 + cb + j] = __uint_as_float(v[j]);
        }
    } else if (t == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GN));
}

// ---- TMA-fed variant ----------------------------------------------------------------
// The same product with the operands brought in by the Tensor Memory Accelerator: K chunks of
// 64 bf16 (128 bytes) per row land in shared memory through cp.async.bulk.tensor (no
// multicast: the tensor maps cover this GPU's buffers only) with the 128-byte swizzle that
// the UMMA K-major SW128 descriptor reads (8-row groups 1024 bytes apart; a K step of 16
// elements advances the start address by 32 bytes inside the swizzle atom).  A ring of
// kTStages stages has a full barrier (TMA transaction bytes) and an empty barrier
// (tcgen05.commit after the stage's MMAs) each; one thread issues the loads and the MMAs.
// BN = 64 or 128 output columns per CTA (64 when 128-wide tiles would leave SMs idle).
constexpr int kTStages = 4;
constexpr uint32_t kTileA = GM * GK * 2;  // 16 KB per stage

__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3fff);
    d |= (uint64_t)1 << 16;                   // leading byte offset (unused by K-major SW128)
    d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset: 8 rows x 128 bytes
    d |= (uint64_t)1 << 46;                   // descriptor version (sm100)
    d |= (uint64_t)2 << 61;                   // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads) k_umma_tma(const __grid_constant__ CUtensorMap mapA, uint64_t rows,
                                                           const __grid_constant__ CUtensorMap mapB, uint64_t cols,
                                                           int d, float* __restrict__ out, uint64_t ldo,
                                                           int* __restrict__ err) {
    extern __shared__ unsigned char smem_raw[];  // kTStages x (A tile, B tile), 1024-aligned inside
    __shared__ __align__(8) uint64_t s_full[kTStages], s_empty[kTStages], s_done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    constexpr uint32_t kTileB = BN * GK * 2;
    constexpr uint32_t kIdescT = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                 ((uint32_t)(GM >> 4) << 24);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int r0 = (int)(blockIdx.x * GM), c0 = (int)(blockIdx.y * BN);
    const uint32_t sbase = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const int nchunks = (d + GK - 1) / GK;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        s_fail = 0;
        for (int i = 0; i < kTStages; i++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_full[i])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_empty[i])), "r"(1));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_done)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    if (t == 0) {
        int issued = 0;  // chunks whose loads were issued
        auto issue = [&](int kc) {
            const int st = kc % kTStages;
            const uint32_t sa = sbase + (uint32_t)st * (kTileA + kTileB), sb = sa + kTileA;
            const uint32_t fb = smem_u32(&s_full[st]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(kTileA + kTileB)
                         : "memory");
            tma_load_2d(sa, &mapA, kc * GK, r0, fb);
            tma_load_2d(sb, &mapB, kc * GK, c0, fb);
            issued = kc + 1;
        };
        for (int kc = 0; kc < nchunks && kc < kTStages; kc++) issue(kc);
        bool ok = true;
        int committed = 0;  // chunks whose MMAs were committed
        for (int kc = 0; kc < nchunks && ok; kc++) {
            const int st = kc % kTStages;
            const uint32_t ph = (uint32_t)(kc / kTStages) & 1u;
            if (!mbar_wait(smem_u32(&s_full[st]), ph)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t sa = sbase + (uint32_t)st * (kTileA + kTileB), sb = sa + kTileA;
#pragma unroll
            for (int ks = 0; ks < GK / 16; ks++) {
                const uint64_t da = umma_desc_sw128(sa + ks * 32);
                const uint64_t db = umma_desc_sw128(sb + ks * 32);
                const uint32_t acc = (kc > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(kIdescT), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&s_empty[st]))
                         : "memory");
            committed = kc + 1;
            if (kc + kTStages < nchunks) {  // refill this stage once its MMAs have read it
                if (!mbar_wait(smem_u32(&s_empty[st]), ph)) {
                    ok = false;
                    break;
                }
                issue(kc + kTStages);
            }
        }
        if (ok) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&s_done))
                         : "memory");
        } else {
            // a wait expired: record it, then let the loads and MMAs already issued finish
            // (bounded waits) before the shared memory and TMEM are given back
            s_fail = 1;
            for (int kc = committed; kc < issued; kc++)
                mbar_wait(smem_u32(&s_full[kc % kTStages]), (uint32_t)(kc / kTStages) & 1u);
            if (committed > 0) {
                const int kc = committed - 1;
                mbar_wait(smem_u32(&s_empty[kc % kTStages]), (uint32_t)(kc / kTStages) & 1u);
            }
        }
    }
    __syncthreads();
    bool ok = s_fail == 0;
    if (ok && !mbar_wait(smem_u32(&s_done), 0)) ok = false;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
        const uint64_t row = (uint64_t)r0 + warp * 32 + lane;
        const bool vec = (ldo % 4 == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
        for (int cb = 0; cb < BN; cb += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row >= rows) continue;
            const uint64_t col = (uint64_t)c0 + cb;
            float* o = out + row * ldo + col;
            if (vec && col + 16 <= cols) {
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    *reinterpret_cast<float4*>(o + j) = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                                     __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
            } else {
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (col + j < cols) o[j] = __uint_as_float(v[j]);
            }
        }
    } else if (t == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

__global__ void k_f32_to_bf16_rows(const float* __restrict__ x, uint64_t n, __nv_bfloat16* __restrict__ y,
                                   float* __restrict__ norms, int d) {
    const uint64_t r = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    float s = 0.f;
    for (int j = lane; j < d; j += 32) {
        const float v = x[r * d + j];
        y[r * d + j] = __float2bfloat16_rn(v);
        s = fmaf(v, v, s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0 && norms) norms[r] = s;
}

size_t umma_smem_bytes() { return 4 * kStage; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link needed).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    HDG_REQUIRE(fn != nullptr, HDG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    return fn;
}

// Tensor map of a row-major bf16 [n x d] matrix read in boxes of 64 (K) x box_rows, 128-byte
// swizzle, zero fill past the edges.
static CUtensorMap bf16_rows_map(const void* base, uint64_t n, int d, uint32_t box_rows) {
    HDG_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0 && d % 8 == 0, HDG_ERR_UNSUPPORTED,
                "TMA operands need 16-byte aligned rows");
    CUtensorMap m;
    const cuuint64_t gdim[2] = {(cuuint64_t)d, (cuuint64_t)n};
    const cuuint64_t gstride[1] = {(cuuint64_t)d * 2};
    const cuuint32_t box[2] = {(cuuint32_t)GK, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_tiled()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), gdim, gstride,
                                      box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    HDG_REQUIRE(r == CUDA_SUCCESS, HDG_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return m;
}

// S [rows x cols] (row stride ldo) = A . B^T in BF16 with FP32 accumulation, TMA-fed.
void umma_dot_tma(const void* A_bf16, uint64_t rows, const void* B_bf16, uint64_t cols, int d, float* out,
                  uint64_t ldo, int* err, cudaStream_t st, int sm_count) {
    HDG_REQUIRE(d % 8 == 0, HDG_ERR_UNSUPPORTED, "tensor-core coarse GEMM needs d % 8 == 0");
    HDG_REQUIRE(rows < (1ull << 31) && cols < (1ull << 31), HDG_ERR_UNSUPPORTED, "GEMM operand too large");
    if (!rows || !cols) return;
    const uint64_t row_tiles = (rows + GM - 1) / GM;
    // 128-wide column tiles unless they would leave SMs without two CTAs each
    const bool narrow = row_tiles * ((cols + 127) / 128) < (uint64_t)(2 * sm_count);
    const CUtensorMap ma = bf16_rows_map(A_bf16, rows, d, GM);
    auto launch = [&](auto kern, uint32_t bn) {
        const CUtensorMap mb = bf16_rows_map(B_bf16, cols, d, bn);
        const int sm = (int)(kTStages * (kTileA + bn * GK * 2) + 1024);
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        dim3 grid((unsigned)row_tiles, (unsigned)((cols + bn - 1) / bn));
        kern<<<grid, kGemmThreads, sm, st>>>(ma, rows, mb, cols, d, out, ldo, err);
    };
    if (narrow) launch(k_umma_tma<64>, 64);
    else launch(k_umma_tma<128>, 128);
    CK_LAUNCH();
}

// S [rows x cols] (row stride ldo) = A . B^T in BF16 with FP32 accumulation (the TMA-fed kernel).
void umma_dot(const void* A_bf16, uint64_t rows, const void* B_bf16, uint64_t cols, int d, float* out,
              uint64_t ldo, int* err, cudaStream_t st) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    umma_dot_tma(A_bf16, rows, B_bf16, cols, d, out, ldo, err, st, sms);
}

// The cp.async-fed kernel above, kept beside the TMA one for comparison runs.
void umma_dot_cp_async(const void* A_bf16, uint64_t rows, const void* B_bf16, uint64_t cols, int d, float* out,
                       uint64_t ldo, int* err, cudaStream_t st) {
    HDG_REQUIRE(d % 8 == 0, HDG_ERR_UNSUPPORTED, "tensor-core coarse GEMM needs d % 8 == 0");
    if (!rows || !cols) return;
    const int sm = (int)umma_smem_bytes();
    CK(cudaFuncSetAttribute(k_umma_dot, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    dim3 grid((unsigned)((rows + GM - 1) / GM), (unsigned)((cols + GN - 1) / GN));
    k_umma_dot<<<grid, kGemmThreads, sm, st>>>(static_cast<const __nv_bfloat16*>(A_bf16), rows,
                                               static_cast<const __nv_bfloat16*>(B_bf16), cols, d, out, ldo, err);
    CK_LAUNCH();
}

void rows_to_bf16(const float* x, uint64_t n, int d, void* y, float* norms, cudaStream_t st) {
    if (!n) return;
    k_f32_to_bf16_rows<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(x, n, static_cast<__nv_bfloat16*>(y), norms, d);
    CK_LAUNCH();
}

}  // namespace hdg
