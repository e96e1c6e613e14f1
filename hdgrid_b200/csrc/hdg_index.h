// Device-resident layout of a built HDGrid index and the host object that owns it.
//
// HBM layout (one arena per index, 256-byte aligned sub-buffers):
//   centers      f32 [C x d]            coarse centroids (src/index/2-level_index/Super-Grid-IVF_PQ.cuh:77)
//   sub_centers  f32 [L x d]            one centroid per inverted list, grouped by cluster (:72)
//   centers_bf16 / sub_centers_bf16     BF16 copies for the tensor-core coarse GEMM
//   cnorm        f32 [C + L]            squared norms of the centroids (GEMM epilogue)
//   cluster_off  u32 [C + 1]            list range of each cluster (sub_cluster_offsets/counts, :78-79)
//   list_off     u32 [L + 1]            pool range of each list (zorder_array_offsets/lengthes, :70-71)
//   zcodes       u64 [N]                Morton code of every point, sorted inside each list (:69)
//   ids          u32 [N]                original point id in pool order (zorder_node_arrays, :68)
//   codes        u8  [M_pad/16][N][16]  PQ codes in pool order as 16-byte chunk planes: bytes
//                                       16j..16j+15 of point p at (j*N + p)*16, so the lanes of a
//                                       warp scanning consecutive pool positions load one
//                                       contiguous 512-byte span per chunk (the saved file and
//                                       HostIndex keep the row-major [N x M_pad] form)
//   labels       f32 [N x l]            labels in pool order (read by the fused predicate)
//   pq_centers   f32 [M x 256 x pq_len] PQ codebooks (pq::index_data_t::centers, product-quantization.cuh:9)
//   prefix       u32 [cells x L]        inclusive multi-dim prefix counts per list, cell-major,
//                                       list fastest (dense form of compressed_sums, :67), or
//   prefix_off   u64 [T x L + 1]        the compressed form: for grid row t (every dim but the
//   prefix_rows  u64 [E]                diff dim, T rows) and list j, the change points of the
//                                       inclusive prefix along the diff dim, (coordinate << 32 |
//                                       count) ascending, at [prefix_off[t*L+j], prefix_off[t*L+j+1])
// L = C*S inverted lists; N points; M PQ subspaces; M_pad = M rounded up to 16.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "hdg_common.h"

namespace hdg {

constexpr int kMaxDims = HDG_MAX_LABEL_DIMS;
constexpr int kCodes = 256;

// Label grid + Morton configuration (calc_grid_shape, Super-Grid-IVF_PQ.cu:305-412).
// Dims are stored in "shuffled" order (label dims sorted by span, ascending).
struct GridMeta {
    int l = 0;
    int grid_dims[kMaxDims] = {0};
    int shuffle[kMaxDims] = {0};          // shuffled position -> original label dim
    uint64_t left[kMaxDims] = {0};        // floor(min label)
    uint64_t span[kMaxDims] = {0};        // ceil(max) - floor(min)
    uint64_t cell_stride[kMaxDims] = {0}; // row-major strides, last dim fastest
    uint64_t tot_cells = 0;
    int morton_dims = 0, morton_max_bits = 0, morton_valid_map = 0;
    int diff_dim = 0;
};

// Bits per label-rank field: l fields of b bits, each with its guard bit, in 32 bits; at most
// 12 (4095 thresholds per dim); 0 when l fields do not fit.
inline int rank_bits_for(int l) {
    if (l <= 0) return 0;
    const int b = (32 - l) / l;
    return b < 1 ? 0 : (b > 12 ? 12 : b);
}

// filter.conf on the device (passed by value; the map table lives in the arena).
struct FilterDev {
    int l;
    int filter_dim;
    int type[kMaxDims];
    float shift_val[2 * kMaxDims];
    int div_value[kMaxDims];
    int n_map;
    const float* map;
};

struct IndexDev {
    uint32_t n, d, l, M, M_pad, pq_len, n_lists, C, S_max;
    const float* centers;
    const float* sub_centers;
    const uint16_t* centers_bf16;
    const uint16_t* sub_centers_bf16;
    const float* cnorm;
    const uint32_t* cluster_off;
    const uint32_t* list_off;
    const uint64_t* zcodes;
    // Label ranks (derived at upload, not stored in the index file): per label dim i, up to
    // 2^rank_bits - 1 ascending thresholds rank_thr[i * rank_stride + k], k < rank_n[i]; a
    // label's rank is the number of thresholds at or below it.  rankpack holds every point's
    // ranks in pool order, dim i in bits [i * (rank_bits + 1), +rank_bits) with a zero guard bit
    // above (rank_guard = the guard bits; rank_full = every rank_n[i] in its field).  The labels
    // of rank r lie in [thr[r - 1], thr[r]), with rank_min / rank_max (the smallest and largest
    // label of the dim) closing the two ends.  A rank outside the query's rank box proves that
    // the label test fails; a rank inside its inner box proves that it passes.  Only the others
    // need their labels read.  rankpack = nullptr when the label dims do not fit 32 bits.
    const uint32_t* rankpack;
    const float* rank_thr;
    uint32_t rank_n[kMaxDims];
    float rank_min[kMaxDims], rank_max[kMaxDims];
    uint32_t rank_bits, rank_stride, rank_guard, rank_full;
    uint32_t labels_nan;           // some label is NaN (passes every label test, in any cell)
    const uint32_t* ids;
    const uint8_t* codes;
    const float* labels;
    const float* pq_centers;
    const uint32_t* prefix;        // dense prefix counts (nullptr when the rows form or prefix16 is used)
    const uint16_t* prefix16;      // the dense counts in 16 bits, kept when no list exceeds 65535 points
    const uint64_t* prefix_off;    // compressed rows (nullptr when dense)
    const uint64_t* prefix_rows;
};

// Host-side copy of every index array (build output, save/load payload).
struct HostIndex {
    uint64_t n = 0, d = 0, l = 0, M = 0, M_pad = 0, pq_len = 0, n_lists = 0, C = 0;
    GridMeta grid;
    std::vector<float> centers, sub_centers, pq_centers;
    std::vector<uint32_t> cluster_off, list_off, ids, prefix;
    std::vector<uint64_t> prefix_off, prefix_rows;  // compressed rows (prefix empty), see above
    std::vector<uint64_t> zcodes;
    std::vector<uint8_t> codes;
    std::vector<float> labels;
};

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    void reset();
    void ensure(size_t b);  // grow-only cudaMalloc
    ~DeviceBuffer() { reset(); }
};

struct GraphState;                 // captured query graphs (hdg_query.cu)
void release_graphs(GraphState* g);

// Query state of one stream: the workspace, the distance buffer and the captured graphs.
// Calls on different streams use different contexts and may run concurrently; calls on one
// stream take `mu` in turn.
struct QueryCtx {
    DeviceBuffer work;              // per-query workspace
    DeviceBuffer dist_buf;          // one f32 ADC distance per scanned candidate
    DeviceBuffer pos_buf;           // u32 candidate positions of compact rows (same capacity)
    DeviceBuffer sel_buf;           // u32 selected candidates: min(n_cand, candidates) per query
    DeviceBuffer part_buf;          // u64 best keys of the refine work items
    uint64_t work_queries = 0;
    std::map<std::string, std::pair<size_t, size_t>> layout;  // name -> (offset, bytes)
    GraphState* graphs = nullptr;   // QUERY_GRAPH=1: graphs keyed by pointers and sizes
    std::mutex mu;
    QueryCtx() = default;
    QueryCtx(const QueryCtx&) = delete;
    QueryCtx& operator=(const QueryCtx&) = delete;
    ~QueryCtx() { release_graphs(graphs); }
};

}  // namespace hdg

struct hdg_index {
    hdg_params params{};
    hdg::FilterSpec filter;
    bool built = false;
    hdg::HostIndex host;           // kept for save() and the debug/oracle handoff
    hdg::GridMeta grid;
    hdg::IndexDev dev{};
    hdg::DeviceBuffer arena;       // all index arrays
    hdg::DeviceBuffer map_buf;     // filter interval map
    // query contexts by stream (the last one used serves hdg_debug_fetch)
    std::map<void*, std::unique_ptr<hdg::QueryCtx>> ctxs;
    hdg::QueryCtx* last_ctx = nullptr;
    std::mutex ctx_mu;             // guards ctxs and last_ctx
    std::mutex stats_mu;           // guards the last-query stats and stage times
    int device = 0;
    // stage timing (break_down=1)
    std::vector<std::string> stage_names;
    std::vector<float> stage_ms;
    // last-query scalars (host copy)
    uint64_t last_q = 0, last_ncand = 0;
    uint64_t last_stats[10] = {0};
    float last_beta = 0.f;
    // learned per-query schedule: f32 master | Adam m | Adam v | gradient | bf16 weights
    hdg::DeviceBuffer mlp;
    bool mlp_ready = false;
    uint64_t mlp_step = 0;
    hdg_index() = default;
    hdg_index(const hdg_index&) = delete;
    hdg_index& operator=(const hdg_index&) = delete;
    ~hdg_index() = default;
};
