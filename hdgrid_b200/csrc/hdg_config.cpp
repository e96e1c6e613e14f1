// HDGrid.conf and filter.conf readers, byte-compatible with the reference's files.
//
// HDGrid.conf follows common_config::read_config (src/utils/config_utils.h:33-88):
// one `key = value` per line, the key upper-cased and trimmed, the value trimmed,
// optional double quotes stripped, unknown keys ignored.  Integer values are read
// with atoll.  The reference stores a non-integer value as float BITS into the
// uint64 field (config_utils.h:76-79); that is rejected here with a clear error.
//
// filter.conf follows filter_config::filter_config (config_utils.h:121-172):
// all whitespace is removed per line, `l=N` sizes the tables, `filterK:` opens a
// block whose `type=` line is followed by one parameter line
// (shift_val=[a,b] | interval_map=[...] | div_value=[v]); type 3 takes none.
#include <algorithm>
#include <cctype>
#include <fstream>
#include <sstream>

#include "hdg_common.h"

namespace hdg {

std::string upper(std::string s) {
    for (auto& c : s) c = static_cast<char>(::toupper(static_cast<unsigned char>(c)));
    return s;
}

static std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace(static_cast<unsigned char>(s[b]))) b++;
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) e--;
    return s.substr(b, e - b);
}

static bool is_integer(const std::string& s) {
    if (s.empty()) return false;
    size_t i = 0;
    if (s[0] == '+' || s[0] == '-') i++;
    for (; i < s.size(); i++)
        if (!std::isdigit(static_cast<unsigned char>(s[i]))) return false;
    return i > 0;
}

static std::string remove_spaces(const std::string& s) {
    std::string r;
    for (char c : s)
        if (!std::isspace(static_cast<unsigned char>(c))) r += c;
    return r;
}

template <typename T>
static std::vector<T> parse_array(std::string s) {
    std::vector<T> out;
    if (!s.empty() && s.front() == '[') s.erase(0, 1);
    if (!s.empty() && s.back() == ']') s.pop_back();
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        tok = trim(tok);
        if (tok.empty()) continue;
        try {
            out.push_back(static_cast<T>(std::stod(tok)));
        } catch (const std::exception&) {
            fail(HDG_ERR_INVALID_ARG, "filter.conf: bad number '" + tok + "'");
        }
    }
    return out;
}

std::string read_text_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) fail(HDG_ERR_IO, "unable to open configuration file: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

void default_params(hdg_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->topk = 100;
    p->filter_dim = 1;
    p->pq_dim = 32;
    p->n_clusters = 256;
    p->exps0 = 4;
    p->clusters = 8;
    p->sub_clusters = 8;
    p->max_grids = 1000000;
    p->n_list = 8;
    p->sub_lists = 64;
    p->n_split = 1;
    p->kmeans_iters = 20;
    p->seed = 1234;
    p->coarse_bf16 = 1;
}

void parse_hdgrid_conf(const std::string& text, hdg_params* p) {
    struct Key {
        const char* name;
        uint64_t* field;
    };
    const Key keys[] = {
        {"DATA_WIDTH", &p->data_width},
        {"INDEX_WIDTH", &p->index_width},
        {"TOPK", &p->topk},
        {"BREAK_DOWN", &p->break_down},
        {"ENABLE_MULTI_GPU", &p->enable_multi_gpu},
        {"MEM_BOUND", &p->mem_bound},
        {"IS_CALC_MEM_PREDICTOR_COEFF", &p->is_calc_mem_predictor_coeff},
        {"LOWEST_QUERY_BATCH", &p->lowest_query_batch},
        {"FILTER_DIM", &p->filter_dim},
        {"PQ_DIM", &p->pq_dim},
        {"N_CLUSTERS", &p->n_clusters},
        {"EXPS0", &p->exps0},
        {"CLUSTERS", &p->clusters},
        {"SUB_CLUSTERS", &p->sub_clusters},
        {"MAX_GRIDS", &p->max_grids},
        {"N_LIST", &p->n_list},
        {"SUB_LISTS", &p->sub_lists},
        {"N_SPLIT", &p->n_split},
        {"LABEL_MASK", &p->label_mask},
        {"IS_SPLIT", &p->is_split},
        {"LUT_FP16", &p->lut_fp16},
        {"COARSE_BF16", &p->coarse_bf16},
        {"KMEANS_ITERS", &p->kmeans_iters},
        {"SEED", &p->seed},
        {"SCAN_CPT", &p->scan_cpt},
        {"SCAN_CHUNK", &p->scan_chunk},
        {"QUERY_GRAPH", &p->query_graph},
        {"LEARNED", &p->learned},
        {"PREFIX_ROWS", &p->prefix_rows},
    };
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        size_t eq = line.find('=');
        std::string key = trim(upper(line.substr(0, eq)));
        std::string val = eq == std::string::npos ? line : trim(line.substr(eq + 1));
        size_t qs = val.find('"');
        bool quoted = false;
        if (qs != std::string::npos) {
            size_t qe = val.find('"', qs + 1);
            while (qe != std::string::npos && val.at(qe - 1) == '\\') {
                val.erase(qe - 1, 1);
                qe = val.find('"', qe);
            }
            if (qe != std::string::npos) {
                quoted = true;
                val = val.substr(qs + 1, qe - qs - 1);
            }
        }
        if (key == "PATH") {
            std::snprintf(p->path, sizeof(p->path), "%s", val.c_str());
            continue;
        }
        const Key* k = nullptr;
        for (const auto& kk : keys)
            if (key == kk.name) k = &kk;
        if (!k) continue;  // unknown key: logged and ignored by the reference
        if (quoted || !is_integer(val))
            fail(HDG_ERR_INVALID_ARG,
                 "HDGrid.conf: key " + key + " expects an integer, got '" + val + "'");
        *k->field = static_cast<uint64_t>(std::atoll(val.c_str()));
    }
}

void parse_filter_conf(const std::string& text, FilterSpec* f) {
    *f = FilterSpec();
    std::vector<std::vector<float>> maps;
    std::istringstream in(text);
    std::string line;
    bool have_l = false;
    auto check_index = [&](int i) {
        HDG_REQUIRE(have_l, HDG_ERR_INVALID_ARG, "filter.conf: filter block before l=");
        HDG_REQUIRE(i >= 0 && i < f->l, HDG_ERR_INVALID_ARG,
                    "filter.conf: filter index " + std::to_string(i) + " out of range");
    };
    while (std::getline(in, line)) {
        line = remove_spaces(line);
        if (line.empty() || line[0] == '#') continue;
        if (line.rfind("l=", 0) == 0) {
            int l = std::atoi(line.substr(2).c_str());
            HDG_REQUIRE(l >= 1 && l <= HDG_MAX_LABEL_DIMS, HDG_ERR_UNSUPPORTED,
                        "filter.conf: l must be in [1, 8]");
            f->l = l;
            maps.assign(l, {});
            have_l = true;
        } else if (line.rfind("filter", 0) == 0) {
            int idx = std::atoi(line.substr(6).c_str());
            check_index(idx);
            while (std::getline(in, line)) {
                line = remove_spaces(line);
                if (line.empty()) break;
                if (line.rfind("type=", 0) == 0) {
                    int t = std::atoi(line.substr(5).c_str());
                    HDG_REQUIRE(t >= 0 && t <= 3, HDG_ERR_INVALID_ARG,
                                "filter.conf: unknown filter type " + std::to_string(t));
                    f->type[idx] = t;
                    if (t == 3) break;
                } else if (line.rfind("shift_val=", 0) == 0) {
                    auto v = parse_array<float>(line.substr(10));
                    HDG_REQUIRE(v.size() >= 2, HDG_ERR_INVALID_ARG, "filter.conf: shift_val needs 2 values");
                    f->shift_val[2 * idx] = v[0];
                    f->shift_val[2 * idx + 1] = v[1];
                    break;
                } else if (line.rfind("interval_map=", 0) == 0) {
                    auto v = parse_array<int>(line.substr(13));
                    maps[idx].clear();
                    for (int x : v) maps[idx].push_back(static_cast<float>(x));
                    break;
                } else if (line.rfind("div_value=", 0) == 0) {
                    auto v = parse_array<int>(line.substr(10));
                    HDG_REQUIRE(!v.empty(), HDG_ERR_INVALID_ARG, "filter.conf: div_value needs a value");
                    f->div_value[idx] = v[0];
                    break;
                }
            }
        }
    }
    HDG_REQUIRE(have_l, HDG_ERR_INVALID_ARG, "filter.conf: missing l=");
    for (int i = 0; i < f->l; i++) {
        if (f->type[i] == 2)
            HDG_REQUIRE(f->div_value[i] != 0, HDG_ERR_INVALID_ARG, "filter.conf: div_value of 0");
        for (float x : maps[i]) f->interval_map.push_back(x);
    }
}

}  // namespace hdg
