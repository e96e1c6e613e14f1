// extern "C" boundary of libhdgrid.  Every entry point catches hdg::Error (and any other
// exception) and turns it into an hdg_status plus hdg_last_error() text; nothing here
// exits the process (the reference calls exit() on CUDA errors,
// src/utils/debugging_utils.cuh:11-20).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>

#include "hdg_internal.h"

namespace hdg {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

void DeviceBuffer::reset() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

void DeviceBuffer::ensure(size_t b) {
    if (ptr && bytes >= b) return;
    reset();
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, b ? b : 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? HDG_ERR_OOM : HDG_ERR_CUDA,
             std::string("cudaMalloc of ") + std::to_string(b) + " bytes failed: " + cudaGetErrorString(e));
    }
    ptr = p;
    bytes = b;
}

template <typename F>
static hdg_status guarded(F&& f) {
    try {
        f();
        return HDG_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return HDG_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return HDG_ERR_INVALID_ARG;
    }
}

static void check_algorithm(const char* algorithm) {
    HDG_REQUIRE(algorithm, HDG_ERR_INVALID_ARG, "null algorithm");
    const std::string a = upper(algorithm);
    if (a == "SUPER-GRID") return;
    static const char* known[] = {"PQ", "PREFILTER", "SORTING", "PARAFILTER", "IVF-IVF_PQ",
                                  "GRID-IVF_PQ", "CAGRA-POST", "IVFPQ-POST"};
    for (const char* k : known)
        if (a == k)
            fail(HDG_ERR_UNSUPPORTED, std::string("algorithm '") + algorithm +
                                          "' is not implemented by this library (only super-grid)");
    fail(HDG_ERR_INVALID_ARG, std::string("Unknown index type: ") + algorithm);
}

static hdg_index* make_index(const std::string& conf, const std::string& filt) {
    std::unique_ptr<hdg_index> idx(new hdg_index());
    default_params(&idx->params);
    parse_hdgrid_conf(conf, &idx->params);
    parse_filter_conf(filt, &idx->filter);
    HDG_REQUIRE(idx->params.filter_dim == 1 || idx->params.filter_dim == 2, HDG_ERR_INVALID_ARG,
                "filter_dim must be 1 or 2");
    CK(cudaGetDevice(&idx->device));
    upload_filter(idx.get());
    return idx.release();
}

}  // namespace hdg

using namespace hdg;

extern "C" {

const char* hdg_last_error(void) { return g_last_error.c_str(); }
const char* hdg_version(void) { return "hdgrid-b200 0.1.0 (sm_100a)"; }

hdg_status hdg_create(const char* algorithm, const char* hdgrid_conf_path, const char* filter_conf_path,
                      hdg_index** out) {
    return guarded([&] {
        HDG_REQUIRE(out && hdgrid_conf_path, HDG_ERR_INVALID_ARG, "null argument");
        check_algorithm(algorithm);
        const std::string conf = read_text_file(hdgrid_conf_path);
        std::string fpath = filter_conf_path ? filter_conf_path : "";
        if (fpath.empty()) {  // default <path>/filter.conf (search-engine-auto-batch.cu:134-140)
            hdg_params p;
            default_params(&p);
            parse_hdgrid_conf(conf, &p);
            fpath = std::string(p.path) + "filter.conf";
        }
        *out = make_index(conf, read_text_file(fpath));
    });
}

hdg_status hdg_create_from_text(const char* algorithm, const char* conf, const char* filt, hdg_index** out) {
    return guarded([&] {
        HDG_REQUIRE(out && conf && filt, HDG_ERR_INVALID_ARG, "null argument");
        check_algorithm(algorithm);
        *out = make_index(conf, filt);
    });
}

hdg_status hdg_destroy(hdg_index* index) {
    return guarded([&] { delete index; });
}

hdg_status hdg_label_ranks(const float* labels, uint64_t n, uint32_t l, uint32_t* bits, float* thr,
                           uint32_t* n_thr, float* lab_min, float* lab_max) {
    return guarded([&] {
        HDG_REQUIRE(bits && l >= 1 && l <= (uint32_t)kMaxDims, HDG_ERR_INVALID_ARG, "bits missing or l outside 1..8");
        *bits = (uint32_t)rank_bits_for((int)l);
        if (!thr) return;
        HDG_REQUIRE(labels && n > 0 && n_thr && lab_min && lab_max, HDG_ERR_INVALID_ARG, "null argument or no rows");
        label_rank_thresholds(labels, n, (int)l, (int)*bits, thr, n_thr, lab_min, lab_max);
    });
}

hdg_status hdg_parse_config(const char* text, hdg_params* out) {
    return guarded([&] {
        HDG_REQUIRE(text && out, HDG_ERR_INVALID_ARG, "null argument");
        default_params(out);
        parse_hdgrid_conf(text, out);
    });
}

hdg_status hdg_parse_filter(const char* text, hdg_filter_spec* out) {
    static thread_local FilterSpec keep;
    return guarded([&] {
        HDG_REQUIRE(text && out, HDG_ERR_INVALID_ARG, "null argument");
        parse_filter_conf(text, &keep);
        std::memset(out, 0, sizeof(*out));
        out->l = keep.l;
        for (int i = 0; i < HDG_MAX_LABEL_DIMS; i++) {
            out->type[i] = keep.type[i];
            out->div_value[i] = keep.div_value[i];
            out->shift_val[2 * i] = keep.shift_val[2 * i];
            out->shift_val[2 * i + 1] = keep.shift_val[2 * i + 1];
        }
        out->n_map = (int32_t)keep.interval_map.size();
        out->interval_map = keep.interval_map.data();
    });
}

hdg_status hdg_get_params(const hdg_index* index, hdg_params* out) {
    return guarded([&] {
        HDG_REQUIRE(index && out, HDG_ERR_INVALID_ARG, "null argument");
        *out = index->params;
    });
}

hdg_status hdg_set_param(hdg_index* index, const char* key, uint64_t value) {
    return guarded([&] {
        HDG_REQUIRE(index && key, HDG_ERR_INVALID_ARG, "null argument");
        const std::string k = upper(key);
        hdg_params& p = index->params;
        uint64_t* f = nullptr;
        if (k == "N_LIST") f = &p.n_list;
        else if (k == "SUB_LISTS") f = &p.sub_lists;
        else if (k == "EXPS0") f = &p.exps0;
        else if (k == "TOPK") f = &p.topk;
        else if (k == "BREAK_DOWN") f = &p.break_down;
        else if (k == "IS_SPLIT") f = &p.is_split;
        else if (k == "N_SPLIT") f = &p.n_split;
        else if (k == "LUT_FP16") f = &p.lut_fp16;
        else if (k == "COARSE_BF16") f = &p.coarse_bf16;
        else if (k == "SCAN_CPT") f = &p.scan_cpt;
        else if (k == "SCAN_CHUNK") f = &p.scan_chunk;
        else if (k == "QUERY_GRAPH") f = &p.query_graph;
        else if (k == "LEARNED") f = &p.learned;
        else if (k == "PREFIX_ROWS") f = &p.prefix_rows;
        HDG_REQUIRE(f, HDG_ERR_INVALID_ARG, "not a search-time key: " + k);
        if (k == "SCAN_CHUNK")
            HDG_REQUIRE(value == 0 || (value >= 4096 && value <= 262144 && (value & (value - 1)) == 0),
                        HDG_ERR_INVALID_ARG, "SCAN_CHUNK must be 0 or a power of two in [4096, 262144]");
        *f = value;
        invalidate_graphs(index);  // captured graphs bake the old values in
    });
}

hdg_status hdg_build(hdg_index* index, const float* d_data, uint64_t n, uint32_t d, const float* d_labels,
                     uint32_t l, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(index, HDG_ERR_INVALID_ARG, "null index");
        build_index(index, d_data, n, d, d_labels, l, static_cast<cudaStream_t>(stream));
    });
}

hdg_status hdg_reserve(hdg_index* index, uint64_t max_queries) {
    return guarded([&] {
        HDG_REQUIRE(index, HDG_ERR_INVALID_ARG, "null index");
        reserve_workspace(index, max_queries);
    });
}

hdg_status hdg_query(hdg_index* index, const float* d_queries, uint64_t q, const float* d_query_labels,
                     uint32_t label_cols, const float* d_data, uint32_t k, float* d_dist, uint64_t* d_ids,
                     void* stream) {
    return guarded([&] {
        HDG_REQUIRE(index, HDG_ERR_INVALID_ARG, "null index");
        run_query(index, d_queries, q, d_query_labels, label_cols, d_data, k, d_dist, d_ids,
                  static_cast<cudaStream_t>(stream));
    });
}

hdg_status hdg_query_ex(hdg_index* index, const float* d_queries, uint64_t q, const float* d_query_labels,
                        uint32_t label_cols, const float* d_data, uint32_t k_max, const uint32_t* d_k,
                        const uint32_t* d_nprobe, const uint8_t* d_schedule, float* d_dist, uint64_t* d_ids,
                        void* stream) {
    return guarded([&] {
        HDG_REQUIRE(index, HDG_ERR_INVALID_ARG, "null index");
        run_query(index, d_queries, q, d_query_labels, label_cols, d_data, k_max, d_dist, d_ids,
                  static_cast<cudaStream_t>(stream), d_k, d_nprobe, d_schedule);
    });
}

hdg_status hdg_query_status(hdg_index* index) {
    if (!index) return HDG_ERR_INVALID_ARG;
    hdg_status st = HDG_OK;
    const hdg_status g = guarded([&] { st = finish_async_query(index); });
    return g != HDG_OK ? g : st;
}

hdg_status hdg_autotune(hdg_index* index, const float* d_queries, uint64_t q, const float* d_query_labels,
                        uint32_t label_cols, const float* d_data, uint32_t k, float* d_dist, uint64_t* d_ids,
                        void* stream, float* best_scan_ms) {
    return guarded([&] {
        HDG_REQUIRE(index, HDG_ERR_INVALID_ARG, "null index");
        autotune_query(index, d_queries, q, d_query_labels, label_cols, d_data, k, d_dist, d_ids,
                       static_cast<cudaStream_t>(stream), best_scan_ms);
    });
}

hdg_status hdg_query_features(hdg_index* index, const float* d_queries, uint64_t q, const float* d_query_labels,
                              uint32_t label_cols, const uint32_t* d_k, uint32_t k_max, float* d_features,
                              void* stream) {
    return guarded([&] {
        HDG_REQUIRE(index, HDG_ERR_INVALID_ARG, "null index");
        HDG_REQUIRE(k_max >= 1, HDG_ERR_INVALID_ARG, "k_max must be >= 1");
        query_features(index, d_queries, q, d_query_labels, label_cols, d_k, k_max, d_features,
                       static_cast<cudaStream_t>(stream));
    });
}

uint64_t hdg_mlp_param_count(void) { return (uint64_t)kMlpParams; }

hdg_status hdg_mlp_init(hdg_index* index, uint64_t seed) {
    return guarded([&] {
        HDG_REQUIRE(index, HDG_ERR_INVALID_ARG, "null index");
        mlp_init(index, seed);
    });
}

hdg_status hdg_mlp_set_weights(hdg_index* index, const float* host, uint64_t count) {
    return guarded([&] {
        HDG_REQUIRE(index && host, HDG_ERR_INVALID_ARG, "null argument");
        mlp_set(index, host, count);
    });
}

hdg_status hdg_mlp_get_weights(hdg_index* index, float* host, uint64_t count) {
    return guarded([&] {
        HDG_REQUIRE(index && host, HDG_ERR_INVALID_ARG, "null argument");
        mlp_get(index, host, count);
    });
}

hdg_status hdg_mlp_forward(hdg_index* index, const float* d_x, uint64_t n, float* d_z, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(index && d_x && d_z && n > 0, HDG_ERR_INVALID_ARG, "bad argument");
        mlp_forward(index, d_x, n, d_z, static_cast<cudaStream_t>(stream));
    });
}

hdg_status hdg_mlp_gradients(hdg_index* index, const float* d_x, const float* d_y, uint64_t n, float* d_grad,
                             double* loss, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(index && d_x && d_y && d_grad, HDG_ERR_INVALID_ARG, "null argument");
        const double l = mlp_gradients(index, d_x, d_y, n, d_grad, static_cast<cudaStream_t>(stream));
        if (loss) *loss = l;
    });
}

hdg_status hdg_mlp_train(hdg_index* index, const float* d_x, const float* d_y, uint64_t n, uint32_t epochs,
                         uint32_t batch, float lr, uint64_t seed, double* final_loss, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(index && d_x && d_y, HDG_ERR_INVALID_ARG, "null argument");
        const double l = mlp_train(index, d_x, d_y, n, epochs, batch, lr, seed, static_cast<cudaStream_t>(stream));
        if (final_loss) *final_loss = l;
    });
}

hdg_status hdg_merge_topk(const float* d_dist, const uint64_t* d_ids, uint64_t q, uint32_t k, uint32_t n_batches,
                          const uint64_t* d_offsets, float* d_out_dist, uint64_t* d_out_ids, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(d_dist && d_ids && d_offsets && d_out_dist && d_out_ids, HDG_ERR_INVALID_ARG, "null pointer");
        if (q == 0) return;
        merge_topk(d_dist, d_ids, q, k, n_batches, d_offsets, d_out_dist, d_out_ids,
                   static_cast<cudaStream_t>(stream));
    });
}

int hdg_last_query_stats(hdg_index* index, uint64_t* out, int cap) {
    if (!index || !out) return 0;
    guarded([&] { finish_async_query(index); });
    const int n = std::min(cap, 10);
    for (int i = 0; i < n; i++) out[i] = index->last_stats[i];
    return n;
}

int hdg_last_stage_times(const hdg_index* index, float* ms, const char** names, int cap) {
    if (!index) return 0;
    const int n = std::min<int>(cap, (int)index->stage_ms.size());
    for (int i = 0; i < n; i++) {
        if (ms) ms[i] = index->stage_ms[i];
        if (names) names[i] = index->stage_names[i].c_str();
    }
    return n;
}

hdg_status hdg_debug_fetch(const hdg_index* index, const char* name, void* host_dst, size_t bytes,
                           size_t* bytes_needed) {
    return guarded([&] {
        HDG_REQUIRE(index && name, HDG_ERR_INVALID_ARG, "null argument");
        const hdg::QueryCtx* cx = index->last_ctx;
        HDG_REQUIRE(cx, HDG_ERR_STATE, "no query has run on this index");
        const char* src = nullptr;
        size_t sz = 0;
        if (std::string(name) == "distances") {  // the ADC distance buffer (qoff gives the rows)
            src = static_cast<const char*>(cx->dist_buf.ptr);
            sz = cx->dist_buf.bytes;
        } else if (std::string(name) == "cand_pool") {  // selected candidates (sel_off gives the rows)
            src = static_cast<const char*>(cx->sel_buf.ptr);
            sz = cx->sel_buf.bytes;
        } else {
            auto it = cx->layout.find(name);
            HDG_REQUIRE(it != cx->layout.end(), HDG_ERR_INVALID_ARG,
                        std::string("no workspace buffer named ") + name);
            src = static_cast<const char*>(cx->work.ptr) + it->second.first;
            sz = it->second.second;
        }
        if (bytes_needed) *bytes_needed = sz;
        if (!host_dst) return;
        HDG_REQUIRE(bytes >= sz, HDG_ERR_INVALID_ARG, "destination too small");
        CK(cudaDeviceSynchronize());
        CK(cudaMemcpy(host_dst, src, sz, cudaMemcpyDeviceToHost));
    });
}

hdg_status hdg_get_info(const hdg_index* index, hdg_index_info* out) {
    return guarded([&] {
        HDG_REQUIRE(index && out, HDG_ERR_INVALID_ARG, "null argument");
        HDG_REQUIRE(index->built, HDG_ERR_STATE, "index not built");
        std::memset(out, 0, sizeof(*out));
        const HostIndex& H = index->host;
        out->n = H.n;
        out->d = H.d;
        out->l = H.l;
        out->M = H.M;
        out->M_pad = H.M_pad;
        out->n_lists = H.n_lists;
        out->clusters = H.C;
        out->tot_cells = H.grid.tot_cells;
        for (int i = 0; i < HDG_MAX_LABEL_DIMS; i++) {
            out->grid_dims[i] = H.grid.grid_dims[i];
            out->shuffle[i] = H.grid.shuffle[i];
            out->label_left[i] = H.grid.left[i];
            out->label_span[i] = H.grid.span[i];
        }
        out->morton_dims = H.grid.morton_dims;
        out->morton_max_bits = H.grid.morton_max_bits;
        out->morton_valid_map = H.grid.morton_valid_map;
        out->diff_dim = H.grid.diff_dim;
        out->device_bytes = index->arena.bytes;
        out->prefix_entries = index->host.prefix_off.empty() ? 0 : index->host.prefix_rows.size();
        out->rank_pack_bytes = index->dev.rankpack ? 4 : 0;
        out->rank_bits = index->dev.rank_bits;
    });
}

hdg_status hdg_save(const hdg_index* index, const char* path) {
    return guarded([&] {
        HDG_REQUIRE(index && path, HDG_ERR_INVALID_ARG, "null argument");
        save_index(index, path);
    });
}

hdg_status hdg_load(const char* path, hdg_index** out) {
    return guarded([&] {
        HDG_REQUIRE(path && out, HDG_ERR_INVALID_ARG, "null argument");
        *out = load_index(path);
    });
}

hdg_status hdg_pq_lut(const float* d_centers, const float* d_queries, uint64_t n_queries, uint32_t n_dim,
                      uint32_t pq_dim, uint32_t pq_len, uint32_t n_codes, float* d_lut, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(d_centers && d_queries && d_lut, HDG_ERR_INVALID_ARG, "null pointer");
        pq_lut(d_centers, d_queries, n_queries, n_dim, pq_dim, pq_len, n_codes, d_lut,
               static_cast<cudaStream_t>(stream));
    });
}

hdg_status hdg_pq_adc(const uint8_t* d_codebook, uint64_t tot_data, const float* d_lut, uint64_t n_queries,
                      uint32_t pq_dim, uint32_t n_codes, const uint64_t* d_indices, uint64_t n_cand,
                      float* d_dist, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(d_codebook && d_lut && d_dist, HDG_ERR_INVALID_ARG, "null pointer");
        pq_adc(d_codebook, tot_data, d_lut, n_queries, pq_dim, n_codes, d_indices, n_cand, d_dist,
               static_cast<cudaStream_t>(stream));
    });
}

hdg_status hdg_label_mask(const float* d_ranges, const float* d_labels, uint32_t l, uint64_t n_data,
                          uint64_t n_queries, const uint64_t* d_indices, uint64_t n_cand, int32_t* d_mask,
                          void* stream) {
    return guarded([&] {
        HDG_REQUIRE(d_ranges && d_labels && d_mask, HDG_ERR_INVALID_ARG, "null pointer");
        label_mask(d_ranges, d_labels, l, n_data, n_queries, d_indices, n_cand, d_mask,
                   static_cast<cudaStream_t>(stream));
    });
}

hdg_status hdg_recover_filters(const hdg_filter_spec* spec, const float* d_query_labels, uint64_t n_queries,
                               float* d_ranges, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(spec && d_query_labels && d_ranges, HDG_ERR_INVALID_ARG, "null pointer");
        HDG_REQUIRE(spec->l >= 1 && spec->l <= HDG_MAX_LABEL_DIMS, HDG_ERR_INVALID_ARG, "bad l");
        DeviceBuffer map;
        map.ensure(std::max<size_t>(16, (size_t)spec->n_map * 4));
        if (spec->n_map)
            CK(cudaMemcpy(map.ptr, spec->interval_map, (size_t)spec->n_map * 4, cudaMemcpyHostToDevice));
        FilterDev f{};
        f.l = spec->l;
        bool range = false;
        for (int i = 0; i < HDG_MAX_LABEL_DIMS; i++) {
            f.type[i] = spec->type[i];
            f.div_value[i] = spec->div_value[i] ? spec->div_value[i] : 1;
            f.shift_val[2 * i] = spec->shift_val[2 * i];
            f.shift_val[2 * i + 1] = spec->shift_val[2 * i + 1];
            if (i < spec->l && spec->type[i] == 3) range = true;
        }
        f.filter_dim = range ? 2 : 1;
        f.n_map = spec->n_map;
        f.map = static_cast<const float*>(map.ptr);
        recover_filters(f, d_query_labels, n_queries, d_ranges, static_cast<cudaStream_t>(stream));
        CK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    });
}

hdg_status hdg_bf16_gemm(const void* d_a, uint64_t rows, const void* d_b, uint64_t cols, uint32_t d, float* d_out,
                         uint64_t ldo, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(d_a && d_b && d_out && d > 0, HDG_ERR_INVALID_ARG, "bad argument");
        DeviceBuffer err;
        err.ensure(sizeof(int));
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        CK(cudaMemsetAsync(err.ptr, 0, sizeof(int), st));
        umma_dot(d_a, rows, d_b, cols, (int)d, d_out, ldo, static_cast<int*>(err.ptr), st);
        int h = 0;
        CK(cudaMemcpyAsync(&h, err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        HDG_REQUIRE(h == 0, HDG_ERR_TIMEOUT, "tensor-core wait expired in the coarse GEMM");
    });
}

hdg_status hdg_recover_filters_noalloc(const hdg_filter_spec* spec, const float* d_query_labels, uint64_t n_queries,
                                       float* d_ranges, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(spec && d_query_labels && d_ranges, HDG_ERR_INVALID_ARG, "null pointer");
        HDG_REQUIRE(spec->l >= 1 && spec->l <= HDG_MAX_LABEL_DIMS, HDG_ERR_INVALID_ARG, "bad l");
        HDG_REQUIRE(spec->n_map == 0 || spec->interval_map, HDG_ERR_INVALID_ARG, "null interval map");
        FilterDev f{};
        f.l = spec->l;
        bool range = false;
        for (int i = 0; i < HDG_MAX_LABEL_DIMS; i++) {
            f.type[i] = spec->type[i];
            f.div_value[i] = spec->div_value[i] ? spec->div_value[i] : 1;
            f.shift_val[2 * i] = spec->shift_val[2 * i];
            f.shift_val[2 * i + 1] = spec->shift_val[2 * i + 1];
            if (i < spec->l && spec->type[i] == 3) range = true;
        }
        f.filter_dim = range ? 2 : 1;
        f.n_map = spec->n_map;
        recover_filters_noalloc(f, spec->interval_map, d_query_labels, n_queries, d_ranges,
                                static_cast<cudaStream_t>(stream));
    });
}

hdg_status hdg_bruteforce_knn(const float* d_data, uint64_t n, uint32_t d, const float* d_labels, uint32_t l,
                              const float* d_queries, uint64_t q, const float* d_ranges, uint32_t k,
                              float* d_dist, uint64_t* d_ids, void* stream) {
    return guarded([&] {
        HDG_REQUIRE(d_data && d_labels && d_queries && d_ranges && d_dist && d_ids, HDG_ERR_INVALID_ARG,
                    "null pointer");
        bruteforce_knn(d_data, n, d, d_labels, l, d_queries, q, d_ranges, k, d_dist, d_ids,
                       static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
