// search-engine: the reference's process entry point over libhdgrid.
//
//     search-engine <algorithm> <HDGrid.conf> [filter.conf]
//
// Same argv as src/auto-batch-search-main.cu:9-24 and the flow of auto_batch_search
// (src/search-engine/search-engine-auto-batch.cu:120-355):
//   * algorithm: "super-grid" (any case); other index types report UNSUPPORTED;
//   * the dataset directory is HDGrid.conf's PATH; filter.conf defaults to PATH/filter.conf;
//   * the directory holds `keys` and `dtypes` (one line per key) and, per key, the raw
//     row-major array `<key>` plus `<key>_size` (two int32: rows, cols), as
//     src/read_hfs5.py writes them (src/utils/io_utils.cu:3-28, 201-313).  train_vec /
//     train_label are the base set and its labels, test_vec / test_label the queries and
//     their filter labels (filter_dim columns per label dim), neighbors the int32 ground truth;
//   * with ENABLE_MULTI_GPU=1 every visible GPU holds a replica and takes an equal share of
//     the queries (uniformly_divide); otherwise GPU 0 answers all;
//   * when the base set is larger than MEM_BOUND bytes allow (d*4 + 64 bytes per point: the
//     vector plus codes, labels, Morton code, id and build scratch), it is split into data
//     batches: an index per batch answers every query and the per-batch top-k lists are
//     merged on the GPU with ids shifted by the batch start (the reference's data-batch split
//     and merge_intermediate_result, search-engine-auto-batch.cu:214-337, merge_res.cu:18-56);
//   * results go to res/distances_<gpu> (f32) and res/neighbors_<gpu> (u64), topk per query,
//     row-major, queries in order; then, when PATH/neighbors exists, the recall line.
// Labels stored as int32 / int64 / float64 are converted to f32 on load (the reference copies
// the raw bytes and reads them as f32, so it only works with f32 labels).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/hdgrid.h"

namespace {

struct Array {
    int32_t rows = 0, cols = 0;
    std::vector<float> f32;       // vectors and labels
    std::vector<int64_t> i64;     // neighbors
};

bool file_exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

std::vector<std::string> read_lines(const std::string& p) {
    std::ifstream f(p);
    if (!f) throw std::runtime_error("cannot open " + p);
    std::vector<std::string> out;
    std::string s;
    while (std::getline(f, s)) {
        while (!s.empty() && (s.back() == '\r' || s.back() == ' ')) s.pop_back();
        if (!s.empty()) out.push_back(s);
    }
    return out;
}

size_t dtype_size(const std::string& t) {
    static const std::map<std::string, size_t> m = {
        {"int32", 4}, {"float32", 4}, {"float", 4}, {"int64", 8}, {"float64", 8}, {"int8", 1},
        {"uint8", 1}, {"uint16", 2}, {"uint32", 4}, {"uint64", 8}, {"int", 4}, {"long", 8}};
    auto it = m.find(t);
    if (it == m.end()) throw std::runtime_error("data type not supported: " + t);
    return it->second;
}

Array load(const std::string& dir, const std::string& key, const std::string& type, bool as_int) {
    Array a;
    {
        std::ifstream f(dir + key + "_size", std::ios::binary);
        if (!f) throw std::runtime_error("cannot open " + dir + key + "_size");
        int32_t rc[2];
        f.read(reinterpret_cast<char*>(rc), sizeof(rc));
        if (!f) throw std::runtime_error("short read in " + dir + key + "_size");
        a.rows = rc[0];
        a.cols = rc[1];
    }
    const size_t n = (size_t)a.rows * (size_t)a.cols, es = dtype_size(type);
    std::vector<char> raw(n * es);
    std::ifstream f(dir + key, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + dir + key);
    f.read(raw.data(), (std::streamsize)raw.size());
    if ((size_t)f.gcount() != raw.size()) throw std::runtime_error("short read in " + dir + key);
    auto value = [&](size_t i) -> double {
        const char* p = raw.data() + i * es;
        if (type == "float32" || type == "float") { float v; std::memcpy(&v, p, 4); return v; }
        if (type == "float64") { double v; std::memcpy(&v, p, 8); return v; }
        if (type == "int32" || type == "int") { int32_t v; std::memcpy(&v, p, 4); return v; }
        if (type == "int64" || type == "long") { int64_t v; std::memcpy(&v, p, 8); return (double)v; }
        if (type == "uint32") { uint32_t v; std::memcpy(&v, p, 4); return v; }
        if (type == "uint64") { uint64_t v; std::memcpy(&v, p, 8); return (double)v; }
        if (type == "uint16") { uint16_t v; std::memcpy(&v, p, 2); return v; }
        if (type == "uint8") return (double)(uint8_t)p[0];
        return (double)(int8_t)p[0];
    };
    if (as_int) {
        a.i64.resize(n);
        for (size_t i = 0; i < n; i++) a.i64[i] = (int64_t)value(i);
    } else if (type == "float32" || type == "float") {
        a.f32.resize(n);
        std::memcpy(a.f32.data(), raw.data(), n * 4);
    } else {
        a.f32.resize(n);
        for (size_t i = 0; i < n; i++) a.f32[i] = (float)value(i);
    }
    return a;
}

void check(hdg_status s, const char* what) {
    if (s != HDG_OK) throw std::runtime_error(std::string(what) + ": " + hdg_last_error());
}

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

struct DeviceResult {
    std::vector<float> dist;
    std::vector<uint64_t> ids;
    double build_ms = 0, query_ms = 0;
    uint64_t data_batches = 0;
    std::string error;
};

uint64_t data_batch_rows(const hdg_params& P, uint64_t n, uint32_t d) {
    const uint64_t per_row = (uint64_t)d * 4 + 64;
    if (P.mem_bound == 0 || n * per_row <= P.mem_bound) return n;
    return std::max<uint64_t>(1, P.mem_bound / per_row);
}

// One GPU: for each data batch build an index, answer queries [q0, q0 + nq) in query
// batches, and merge the batch's top-k into the running results.
void run_device(int dev, const std::string& algo, const std::string& conf, const std::string& filt,
                const hdg_params& P, const Array& base, const Array& blab, const Array& qv, const Array& qlab,
                uint64_t q0, uint64_t nq, uint32_t topk, DeviceResult* out) {
    try {
        cuda_check(cudaSetDevice(dev), "cudaSetDevice");
        const uint64_t n = (uint64_t)base.rows;
        const uint32_t d = (uint32_t)base.cols, l = (uint32_t)blab.cols, lc = (uint32_t)qlab.cols;
        const uint64_t dbatch = data_batch_rows(P, n, d);
        const uint64_t batch = std::min<uint64_t>(std::max<uint64_t>(nq, 1), 50000);
        float *d_base = nullptr, *d_lab = nullptr, *d_q = nullptr, *d_ql = nullptr, *d_dist = nullptr;
        float *d_best_d = nullptr, *d_pair_d = nullptr;
        uint64_t *d_ids = nullptr, *d_best_i = nullptr, *d_pair_i = nullptr, *d_off = nullptr;
        const uint64_t nq1 = std::max<uint64_t>(nq, 1);
        cuda_check(cudaMalloc(&d_base, dbatch * d * 4), "cudaMalloc base");
        cuda_check(cudaMalloc(&d_lab, dbatch * l * 4), "cudaMalloc labels");
        cuda_check(cudaMalloc(&d_q, batch * d * 4), "cudaMalloc queries");
        cuda_check(cudaMalloc(&d_ql, batch * lc * 4), "cudaMalloc query labels");
        cuda_check(cudaMalloc(&d_dist, batch * topk * 4), "cudaMalloc distances");
        cuda_check(cudaMalloc(reinterpret_cast<void**>(&d_ids), batch * topk * 8), "cudaMalloc ids");
        cuda_check(cudaMalloc(&d_best_d, nq1 * topk * 4), "cudaMalloc results");
        cuda_check(cudaMalloc(reinterpret_cast<void**>(&d_best_i), nq1 * topk * 8), "cudaMalloc results");
        cuda_check(cudaMalloc(&d_pair_d, batch * topk * 2 * 4), "cudaMalloc merge");
        cuda_check(cudaMalloc(reinterpret_cast<void**>(&d_pair_i), batch * topk * 2 * 8), "cudaMalloc merge");
        cuda_check(cudaMalloc(reinterpret_cast<void**>(&d_off), 2 * 8), "cudaMalloc offsets");
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float ms = 0;
        for (uint64_t off = 0; off < n; off += dbatch) {
            const uint64_t nb = std::min(dbatch, n - off);
            hdg_index* idx = nullptr;
            check(hdg_create(algo.c_str(), conf.c_str(), filt.c_str(), &idx), "create");
            cuda_check(cudaMemcpy(d_base, base.f32.data() + off * d, nb * d * 4, cudaMemcpyHostToDevice), "copy base");
            cuda_check(cudaMemcpy(d_lab, blab.f32.data() + off * l, nb * l * 4, cudaMemcpyHostToDevice), "copy labels");
            cudaEventRecord(e0);
            check(hdg_build(idx, d_base, nb, d, d_lab, l, nullptr), "build");
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
            out->build_ms += ms;
            check(hdg_reserve(idx, batch), "reserve");
            const uint64_t offs[2] = {0, off};
            cuda_check(cudaMemcpy(d_off, offs, sizeof(offs), cudaMemcpyHostToDevice), "copy offsets");
            for (uint64_t a = 0; a < nq; a += batch) {
                const uint64_t m = std::min(nq, a + batch) - a;
                cuda_check(cudaMemcpy(d_q, qv.f32.data() + (q0 + a) * d, m * d * 4, cudaMemcpyHostToDevice),
                           "copy queries");
                cuda_check(cudaMemcpy(d_ql, qlab.f32.data() + (q0 + a) * lc, m * lc * 4, cudaMemcpyHostToDevice),
                           "copy query labels");
                cudaEventRecord(e0);
                check(hdg_query(idx, d_q, m, d_ql, lc, d_base, topk, d_dist, d_ids, nullptr), "query");
                float* bd = d_best_d + a * topk;
                uint64_t* bi = d_best_i + a * topk;
                if (off == 0) {
                    cuda_check(cudaMemcpyAsync(bd, d_dist, m * topk * 4, cudaMemcpyDeviceToDevice), "keep");
                    cuda_check(cudaMemcpyAsync(bi, d_ids, m * topk * 8, cudaMemcpyDeviceToDevice), "keep");
                } else {  // rows [running k | this batch's k], merged back into the running rows
                    const size_t kd = (size_t)topk * 4, ki = (size_t)topk * 8;
                    cuda_check(cudaMemcpy2DAsync(d_pair_d, 2 * kd, bd, kd, kd, m, cudaMemcpyDeviceToDevice), "pair");
                    cuda_check(cudaMemcpy2DAsync(d_pair_d + topk, 2 * kd, d_dist, kd, kd, m,
                                                 cudaMemcpyDeviceToDevice), "pair");
                    cuda_check(cudaMemcpy2DAsync(d_pair_i, 2 * ki, bi, ki, ki, m, cudaMemcpyDeviceToDevice), "pair");
                    cuda_check(cudaMemcpy2DAsync(d_pair_i + topk, 2 * ki, d_ids, ki, ki, m,
                                                 cudaMemcpyDeviceToDevice), "pair");
                    check(hdg_merge_topk(d_pair_d, d_pair_i, m, topk, 2, d_off, bd, bi, nullptr), "merge");
                }
                cudaEventRecord(e1);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms, e0, e1);
                out->query_ms += ms;
            }
            hdg_destroy(idx);
            out->data_batches++;
        }
        out->dist.resize(nq * topk);
        out->ids.resize(nq * topk);
        if (nq) {
            cuda_check(cudaMemcpy(out->dist.data(), d_best_d, nq * topk * 4, cudaMemcpyDeviceToHost), "copy d");
            cuda_check(cudaMemcpy(out->ids.data(), d_best_i, nq * topk * 8, cudaMemcpyDeviceToHost), "copy i");
        }
        for (void* p : {(void*)d_base, (void*)d_lab, (void*)d_q, (void*)d_ql, (void*)d_dist, (void*)d_ids,
                        (void*)d_best_d, (void*)d_best_i, (void*)d_pair_d, (void*)d_pair_i, (void*)d_off})
            cudaFree(p);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    } catch (const std::exception& ex) {
        out->error = ex.what();
    }
}

// recall = hits / valid ground-truth ids (verification.cuh:97-153 without the side file):
// per query the first topk ground-truth entries, negatives and repeats ignored.
double recall(const std::vector<uint64_t>& ids, uint64_t nq, uint32_t topk, const Array& gt) {
    uint64_t hits = 0, valid = 0;
    const uint32_t w = (uint32_t)gt.cols;
    for (uint64_t i = 0; i < nq && i < (uint64_t)gt.rows; i++) {
        std::unordered_set<int64_t> g;
        for (uint32_t j = 0; j < std::min(w, topk); j++) {
            const int64_t v = gt.i64[i * w + j];
            if (v >= 0) g.insert(v);
        }
        valid += g.size();
        std::unordered_set<uint64_t> seen;
        for (uint32_t j = 0; j < topk; j++) {
            const uint64_t v = ids[i * topk + j];
            if (v == ~0ull || !seen.insert(v).second) continue;
            hits += g.count((int64_t)v);
        }
    }
    return valid ? (double)hits / (double)valid : 0.0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3 || argc > 4) {
        std::fprintf(stderr, "Usage: %s <algorithm> <config_path> [filter_config_path]\n", argv[0]);
        return 1;
    }
    try {
        const std::string algo = argv[1], conf = argv[2];
        hdg_params P;
        {
            std::ifstream f(conf);
            if (!f) throw std::runtime_error("cannot open " + conf);
            std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
            check(hdg_parse_config(text.c_str(), &P), "HDGrid.conf");
        }
        const std::string dir = P.path;
        const std::string filt = argc == 4 ? std::string(argv[3]) : dir + "filter.conf";
        const auto keys = read_lines(dir + "keys");
        const auto types = read_lines(dir + "dtypes");
        if (types.size() < keys.size()) throw std::runtime_error("dtypes lists fewer entries than keys");
        std::map<std::string, std::string> type;
        for (size_t i = 0; i < keys.size(); i++) type[keys[i]] = types[i];
        for (const char* k : {"train_vec", "train_label", "test_vec", "test_label"})
            if (!type.count(k)) throw std::runtime_error(std::string("dataset key missing: ") + k);
        const Array base = load(dir, "train_vec", type["train_vec"], false);
        const Array blab = load(dir, "train_label", type["train_label"], false);
        const Array qv = load(dir, "test_vec", type["test_vec"], false);
        const Array qlab = load(dir, "test_label", type["test_label"], false);
        std::printf("add input dataset: train_vec %d x %d, test_vec %d x %d\n", base.rows, base.cols, qv.rows,
                    qv.cols);
        const uint32_t topk = (uint32_t)std::max<uint64_t>(1, P.topk);
        int n_dev = 1;
        if (P.enable_multi_gpu) cuda_check(cudaGetDeviceCount(&n_dev), "cudaGetDeviceCount");
        const uint64_t nq = (uint64_t)qv.rows;
        std::vector<DeviceResult> res(n_dev);
        std::vector<std::thread> workers;
        std::vector<uint64_t> q0(n_dev), qn(n_dev);
        for (int i = 0; i < n_dev; i++) {  // uniformly_divide: the first nq % n_dev GPUs take one more
            const uint64_t per = nq / n_dev, rem = nq % n_dev;
            qn[i] = per + ((uint64_t)i < rem ? 1 : 0);
            q0[i] = (uint64_t)i * per + std::min<uint64_t>(i, rem);
            workers.emplace_back(run_device, i, algo, conf, filt, std::cref(P), std::cref(base), std::cref(blab),
                                 std::cref(qv), std::cref(qlab), q0[i], qn[i], topk, &res[i]);
        }
        for (auto& w : workers) w.join();
        ::mkdir("res", 0755);
        std::vector<uint64_t> all_ids;
        for (int i = 0; i < n_dev; i++) {
            if (!res[i].error.empty()) throw std::runtime_error("device " + std::to_string(i) + ": " + res[i].error);
            std::ofstream fd("res/distances_" + std::to_string(i), std::ios::binary | std::ios::trunc);
            std::ofstream fi("res/neighbors_" + std::to_string(i), std::ios::binary | std::ios::trunc);
            fd.write(reinterpret_cast<const char*>(res[i].dist.data()), (std::streamsize)(res[i].dist.size() * 4));
            fi.write(reinterpret_cast<const char*>(res[i].ids.data()), (std::streamsize)(res[i].ids.size() * 8));
            if (!fd || !fi) throw std::runtime_error("Failed to flush query result!");
            std::printf("device: %d build time: %.3f ms, query time: %.3f ms (%llu queries, %.0f QPS, %llu data "
                        "batches)\n", i, res[i].build_ms, res[i].query_ms, (unsigned long long)qn[i],
                        res[i].query_ms > 0 ? qn[i] / (res[i].query_ms / 1e3) : 0.0,
                        (unsigned long long)res[i].data_batches);
            all_ids.insert(all_ids.end(), res[i].ids.begin(), res[i].ids.end());
        }
        if (type.count("neighbors") && file_exists(dir + "neighbors")) {
            const Array gt = load(dir, "neighbors", type["neighbors"], true);
            std::printf("final recall: %.6f\n", recall(all_ids, nq, topk, gt));
        }
        std::printf("search finish\n");
        return 0;
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "search-engine: %s\n", ex.what());
        return 2;
    }
}
