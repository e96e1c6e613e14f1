// Versioned binary index file.  The reference has no index persistence (it rebuilds per
// run, src/search-engine/search-engine-auto-batch.cu:266-274); this format lets build and
// query run separately and lets the CPU oracle consume the exact index the GPU built.
//
// Layout (little-endian, fields written one by one, no struct padding):
//   "HDGB200I" u32 version=2 u32 0
//   params   24 x u64 (order of kParamOrder below), u32 path length + bytes
//   filter   i32 l, i32 type[8], f32 shift_val[16], i32 div_value[8], u32 n_map, f32 map[n_map]
//   sizes    u64 n, d, l, M, M_pad, pq_len, n_lists, C
//   grid     i32 l, i32 dims[8], i32 shuffle[8], u64 left[8], u64 span[8], u64 stride[8],
//            u64 tot_cells, i32 morton_dims, morton_max_bits, morton_valid_map, diff_dim
//   arrays   (u64 element count, raw elements) for: centers f32, sub_centers f32,
//            pq_centers f32, cluster_off u32, list_off u32, ids u32, prefix u32,
//            prefix_off u64, prefix_rows u64 (version 2; either the dense prefix array or the
//            compressed rows is non-empty), zcodes u64, codes u8 [n x M_pad], labels f32 [n x l]
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>

#include "hdg_internal.h"

namespace hdg {

static const char kMagic[8] = {'H', 'D', 'G', 'B', '2', '0', '0', 'I'};

static uint64_t* param_field(hdg_params& p, int i) {
    uint64_t* f[] = {&p.topk,       &p.filter_dim, &p.pq_dim,      &p.n_clusters,
                     &p.exps0,      &p.clusters,   &p.sub_clusters, &p.max_grids,
                     &p.n_list,     &p.sub_lists,  &p.n_split,     &p.label_mask,
                     &p.is_split,   &p.break_down, &p.enable_multi_gpu, &p.mem_bound,
                     &p.is_calc_mem_predictor_coeff, &p.lowest_query_batch, &p.data_width,
                     &p.index_width, &p.lut_fp16,  &p.coarse_bf16, &p.kmeans_iters, &p.seed};
    return f[i];
}
constexpr int kParams = 24;

struct Writer {
    std::ofstream f;
    explicit Writer(const std::string& path) : f(path, std::ios::binary) {
        if (!f) fail(HDG_ERR_IO, "cannot open " + path + " for writing");
    }
    template <typename T>
    void put(const T& v) {
        f.write(reinterpret_cast<const char*>(&v), sizeof(T));
    }
    template <typename T>
    void arr(const std::vector<T>& v) {
        put<uint64_t>(v.size());
        if (!v.empty()) f.write(reinterpret_cast<const char*>(v.data()), sizeof(T) * v.size());
    }
};

struct Reader {
    std::ifstream f;
    std::string path;
    explicit Reader(const std::string& p) : f(p, std::ios::binary), path(p) {
        if (!f) fail(HDG_ERR_IO, "cannot open " + p);
    }
    template <typename T>
    T get() {
        T v{};
        f.read(reinterpret_cast<char*>(&v), sizeof(T));
        if (!f) fail(HDG_ERR_IO, "truncated index file " + path);
        return v;
    }
    template <typename T>
    void any(std::vector<T>& v) {  // an array of any length (bounded by the file)
        const uint64_t n = get<uint64_t>();
        if (n > (1ull << 40)) fail(HDG_ERR_IO, "index file " + path + ": implausible array size");
        v.resize(n);
        if (n) f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
        if (!f) fail(HDG_ERR_IO, "truncated index file " + path);
    }
    template <typename T>
    void arr(std::vector<T>& v, uint64_t expect) {
        const uint64_t n = get<uint64_t>();
        if (n != expect) fail(HDG_ERR_IO, "index file " + path + ": array size mismatch");
        v.resize(n);
        if (n) f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
        if (!f) fail(HDG_ERR_IO, "truncated index file " + path);
    }
};

void save_index(const hdg_index* idx, const std::string& path) {
    HDG_REQUIRE(idx->built, HDG_ERR_STATE, "index not built");
    Writer w(path);
    w.f.write(kMagic, 8);
    w.put<uint32_t>(2);
    w.put<uint32_t>(0);
    hdg_params p = idx->params;
    for (int i = 0; i < kParams; i++) w.put<uint64_t>(*param_field(p, i));
    const std::string ps(p.path);
    w.put<uint32_t>((uint32_t)ps.size());
    w.f.write(ps.data(), ps.size());
    const FilterSpec& fs = idx->filter;
    w.put<int32_t>(fs.l);
    for (int i = 0; i < kMaxDims; i++) w.put<int32_t>(fs.type[i]);
    for (int i = 0; i < 2 * kMaxDims; i++) w.put<float>(fs.shift_val[i]);
    for (int i = 0; i < kMaxDims; i++) w.put<int32_t>(fs.div_value[i]);
    w.put<uint32_t>((uint32_t)fs.interval_map.size());
    for (float x : fs.interval_map) w.put<float>(x);
    const HostIndex& H = idx->host;
    for (uint64_t v : {H.n, H.d, H.l, H.M, H.M_pad, H.pq_len, H.n_lists, H.C}) w.put<uint64_t>(v);
    const GridMeta& g = H.grid;
    w.put<int32_t>(g.l);
    for (int i = 0; i < kMaxDims; i++) w.put<int32_t>(g.grid_dims[i]);
    for (int i = 0; i < kMaxDims; i++) w.put<int32_t>(g.shuffle[i]);
    for (int i = 0; i < kMaxDims; i++) w.put<uint64_t>(g.left[i]);
    for (int i = 0; i < kMaxDims; i++) w.put<uint64_t>(g.span[i]);
    for (int i = 0; i < kMaxDims; i++) w.put<uint64_t>(g.cell_stride[i]);
    w.put<uint64_t>(g.tot_cells);
    for (int v : {g.morton_dims, g.morton_max_bits, g.morton_valid_map, g.diff_dim}) w.put<int32_t>(v);
    w.arr(H.centers);
    w.arr(H.sub_centers);
    w.arr(H.pq_centers);
    w.arr(H.cluster_off);
    w.arr(H.list_off);
    w.arr(H.ids);
    w.arr(H.prefix);
    w.arr(H.prefix_off);
    w.arr(H.prefix_rows);
    w.arr(H.zcodes);
    w.arr(H.codes);
    w.arr(H.labels);
    if (!w.f) fail(HDG_ERR_IO, "write failed: " + path);
}

hdg_index* load_index(const std::string& path) {
    Reader r(path);
    char magic[8];
    r.f.read(magic, 8);
    if (!r.f || std::memcmp(magic, kMagic, 8) != 0) fail(HDG_ERR_IO, path + " is not an HDGrid index file");
    const uint32_t ver = r.get<uint32_t>();
    if (ver != 1 && ver != 2) fail(HDG_ERR_UNSUPPORTED, "unsupported index file version " + std::to_string(ver));
    r.get<uint32_t>();
    std::unique_ptr<hdg_index> idx(new hdg_index());
    default_params(&idx->params);
    for (int i = 0; i < kParams; i++) *param_field(idx->params, i) = r.get<uint64_t>();
    const uint32_t plen = r.get<uint32_t>();
    std::string ps(plen, '\0');
    if (plen) r.f.read(&ps[0], plen);
    std::snprintf(idx->params.path, sizeof(idx->params.path), "%s", ps.c_str());
    FilterSpec& fs = idx->filter;
    fs.l = r.get<int32_t>();
    for (int i = 0; i < kMaxDims; i++) fs.type[i] = r.get<int32_t>();
    for (int i = 0; i < 2 * kMaxDims; i++) fs.shift_val[i] = r.get<float>();
    for (int i = 0; i < kMaxDims; i++) fs.div_value[i] = r.get<int32_t>();
    const uint32_t nm = r.get<uint32_t>();
    fs.interval_map.resize(nm);
    for (uint32_t i = 0; i < nm; i++) fs.interval_map[i] = r.get<float>();
    HostIndex& H = idx->host;
    H.n = r.get<uint64_t>();
    H.d = r.get<uint64_t>();
    H.l = r.get<uint64_t>();
    H.M = r.get<uint64_t>();
    H.M_pad = r.get<uint64_t>();
    H.pq_len = r.get<uint64_t>();
    H.n_lists = r.get<uint64_t>();
    H.C = r.get<uint64_t>();
    GridMeta& g = H.grid;
    g.l = r.get<int32_t>();
    for (int i = 0; i < kMaxDims; i++) g.grid_dims[i] = r.get<int32_t>();
    for (int i = 0; i < kMaxDims; i++) g.shuffle[i] = r.get<int32_t>();
    for (int i = 0; i < kMaxDims; i++) g.left[i] = r.get<uint64_t>();
    for (int i = 0; i < kMaxDims; i++) g.span[i] = r.get<uint64_t>();
    for (int i = 0; i < kMaxDims; i++) g.cell_stride[i] = r.get<uint64_t>();
    g.tot_cells = r.get<uint64_t>();
    g.morton_dims = r.get<int32_t>();
    g.morton_max_bits = r.get<int32_t>();
    g.morton_valid_map = r.get<int32_t>();
    g.diff_dim = r.get<int32_t>();
    r.arr(H.centers, H.C * H.d);
    r.arr(H.sub_centers, H.n_lists * H.d);
    r.arr(H.pq_centers, H.M * kCodes * H.pq_len);
    r.arr(H.cluster_off, H.C + 1);
    r.arr(H.list_off, H.n_lists + 1);
    r.arr(H.ids, H.n);
    if (ver == 1) {
        r.arr(H.prefix, g.tot_cells * H.n_lists);
    } else {
        r.any(H.prefix);
        r.any(H.prefix_off);
        r.any(H.prefix_rows);
        const bool dense = H.prefix.size() == g.tot_cells * H.n_lists && H.prefix_off.empty();
        const uint64_t rows = g.grid_dims[g.diff_dim] ? g.tot_cells / (uint64_t)g.grid_dims[g.diff_dim] : 0;
        const bool packed = H.prefix.empty() && H.prefix_off.size() == rows * H.n_lists + 1 &&
                            H.prefix_off.back() == H.prefix_rows.size();
        if (!dense && !packed) fail(HDG_ERR_IO, "index file " + path + ": inconsistent prefix counts");
    }
    r.arr(H.zcodes, H.n);
    r.arr(H.codes, H.n * H.M_pad);
    r.arr(H.labels, H.n * H.l);
    CK(cudaGetDevice(&idx->device));
    upload_filter(idx.get());
    upload_index(idx.get(), 0);
    return idx.release();
}

}  // namespace hdg
