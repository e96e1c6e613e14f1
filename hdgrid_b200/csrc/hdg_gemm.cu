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
#include <cuda_bf16.h>

#include <cstdint>

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

// S [rows x cols] (row stride ldo) = A . B^T in BF16 with FP32 accumulation.
void umma_dot(const void* A_bf16, uint64_t rows, const void* B_bf16, uint64_t cols, int d, float* out,
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
