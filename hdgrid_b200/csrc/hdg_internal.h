// Internal declarations shared by the translation units of libhdgrid.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "hdg_index.h"

namespace hdg {

inline void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        const hdg_status s = (e == cudaErrorMemoryAllocation) ? HDG_ERR_OOM : HDG_ERR_CUDA;
        throw Error(s, std::string(what) + " failed: " + cudaGetErrorString(e) + " (" + file + ":" +
                           std::to_string(line) + ")");
    }
}
#define CK(x) ::hdg::check_cuda((x), #x, __FILE__, __LINE__)
#define CK_LAUNCH() ::hdg::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// RAII device allocation used by the build (never on the query path).
template <typename T>
struct DevMem {
    T* p = nullptr;
    explicit DevMem(uint64_t count) {
        if (count) CK(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count));
    }
    ~DevMem() {
        if (p) cudaFree(p);
    }
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
};

GridMeta compute_grid_shape(const std::vector<float>& mins, const std::vector<float>& maxs, int l,
                            uint64_t max_grids, uint64_t label_mask_bits);
void build_index(hdg_index* idx, const float* d_data, uint64_t n, uint32_t d, const float* d_labels,
                 uint32_t l, cudaStream_t st);
void upload_index(hdg_index* idx, cudaStream_t st);
void upload_filter(hdg_index* idx);
FilterDev filter_dev(const hdg_index* idx);
void reserve_workspace(hdg_index* idx, uint64_t q, cudaStream_t st = nullptr);
void run_query(hdg_index* idx, const float* d_queries, uint64_t q, const float* d_query_labels,
               uint32_t label_cols, const float* d_data, uint32_t k, float* d_dist, uint64_t* d_ids,
               cudaStream_t st, const uint32_t* d_k = nullptr, const uint32_t* d_nprobe = nullptr,
               const uint8_t* d_sched = nullptr);
int sm_count();  // SMs of the current device
// per-dim label-rank thresholds and label ranges of a base set (hdg_build.cu)
void label_rank_thresholds(const float* labels, uint64_t n, int l, int bits, float* thr, uint32_t* n_thr, float* mn,
                           float* mx);
// learned per-query schedule (hdg_learned.cu): 48 features -> 128 -> 128 -> 2 BF16 MLP,
// parameters W1 [128 x 48], b1, W2 [128 x 128], b2, W3 [2 x 128], b3 in one f32 vector
constexpr int kMlpFeatures = 48, kMlpHidden = 128, kMlpOut = 2;
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpHidden * kMlpFeatures;
constexpr int kMlpW2 = kMlpB1 + kMlpHidden;
constexpr int kMlpB2 = kMlpW2 + kMlpHidden * kMlpHidden;
constexpr int kMlpW3 = kMlpB2 + kMlpHidden;
constexpr int kMlpB3 = kMlpW3 + kMlpOut * kMlpHidden;
constexpr int kMlpParams = kMlpB3 + kMlpOut;
// S / ldS / qnorm: the coarse stage's tensor-core products and the queries' squared norms,
// which narrow the exact centroid distances to the candidates of the 16 nearest (nullptr: all)
void learned_features(hdg_index* idx, const float* d_queries, uint64_t q, const float* box, const uint32_t* cc,
                      const uint32_t* qk, uint32_t k_max, float* feats, cudaStream_t st, const float* S = nullptr,
                      uint64_t ldS = 0, const float* qnorm = nullptr);
void learned_infer(hdg_index* idx, const float* feats, uint64_t q, uint32_t* nprobe, uint8_t* sched, int allow_sched,
                   uint32_t max_probe, float* z, cudaStream_t st);
void mlp_init(hdg_index* idx, uint64_t seed);
void mlp_set(hdg_index* idx, const float* host, size_t count);
void mlp_get(hdg_index* idx, float* host, size_t count);
void mlp_forward(hdg_index* idx, const float* d_x, uint64_t n, float* d_z, cudaStream_t st);
double mlp_gradients(hdg_index* idx, const float* d_x, const float* d_y, uint64_t n, float* d_grad, cudaStream_t st);
double mlp_train(hdg_index* idx, const float* d_x, const float* d_y, uint64_t n, uint32_t epochs, uint32_t batch,
                 float lr, uint64_t seed, cudaStream_t st);
// query features of a batch: the prologue (filter boxes, per-list counts) then k_features
void query_features(hdg_index* idx, const float* d_queries, uint64_t q, const float* d_query_labels,
                    uint32_t label_cols, const uint32_t* d_k, uint32_t k_max, float* d_feats, cudaStream_t st);
void invalidate_graphs(hdg_index* idx);
// waits for the last graph replay's status words; HDG_ERR_TIMEOUT (coarse GEMM wait
// expired) or HDG_ERR_OOM (queries cut by the distance capacity) when they report one
hdg_status finish_async_query(hdg_index* idx);
// the autotuner: times the scan's (threads x candidates-per-thread, chunk) variants on
// this batch and keeps the fastest in params.scan_cpt / params.scan_chunk
void autotune_query(hdg_index* idx, const float* d_queries, uint64_t q, const float* d_query_labels,
                    uint32_t label_cols, const float* d_data, uint32_t k, float* d_dist, uint64_t* d_ids,
                    cudaStream_t st, float* best_ms);
void save_index(const hdg_index* idx, const std::string& path);
hdg_index* load_index(const std::string& path);

// kernel-level entry points (hdg_kernels_ref.cu)
void pq_lut(const float* centers, const float* queries, uint64_t nq, uint32_t n_dim, uint32_t pq_dim,
            uint32_t pq_len, uint32_t n_codes, float* lut, cudaStream_t st);
void pq_adc(const uint8_t* codebook, uint64_t tot_data, const float* lut, uint64_t nq, uint32_t pq_dim,
            uint32_t n_codes, const uint64_t* indices, uint64_t n_cand, float* dist, cudaStream_t st);
void label_mask(const float* ranges, const float* labels, uint32_t l, uint64_t n_data, uint64_t nq,
                const uint64_t* indices, uint64_t n_cand, int32_t* mask, cudaStream_t st);
void recover_filters(const FilterDev& f, const float* qlabels, uint64_t nq, float* ranges,
                     cudaStream_t st);
void recover_filters_noalloc(const FilterDev& f, const float* host_map, const float* qlabels, uint64_t nq,
                             float* ranges, cudaStream_t st);
// tcgen05 BF16 GEMM (hdg_gemm.cu)
void umma_dot(const void* A_bf16, uint64_t rows, const void* B_bf16, uint64_t cols, int d, float* out,
              uint64_t ldo, int* err, cudaStream_t st);
void umma_dot_tma(const void* A_bf16, uint64_t rows, const void* B_bf16, uint64_t cols, int d, float* out,
                  uint64_t ldo, int* err, cudaStream_t st, int sm_count);
void umma_dot_cp_async(const void* A_bf16, uint64_t rows, const void* B_bf16, uint64_t cols, int d, float* out,
                       uint64_t ldo, int* err, cudaStream_t st);
void rows_to_bf16(const float* x, uint64_t n, int d, void* y, float* norms, cudaStream_t st);
void merge_topk(const float* dist, const uint64_t* ids, uint64_t q, uint32_t k, uint32_t nb, const uint64_t* offsets,
                float* out_dist, uint64_t* out_ids, cudaStream_t st);
void bruteforce_knn(const float* data, uint64_t n, uint32_t d, const float* labels, uint32_t l,
                    const float* queries, uint64_t q, const float* ranges, uint32_t k, float* dist,
                    uint64_t* ids, cudaStream_t st);

}  // namespace hdg
