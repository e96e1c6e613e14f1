// Shared host-side helpers of libhdgrid: status plumbing, the thread-local error
// message, CUDA error checks that return (never exit), and small math helpers.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hdgrid.h"

namespace hdg {

// Exception carrying an hdg_status; caught at the C ABI boundary and turned into a
// return code plus hdg_last_error() text.
struct Error : std::runtime_error {
    hdg_status status;
    Error(hdg_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

void set_last_error(const std::string& msg);

[[noreturn]] inline void fail(hdg_status s, const std::string& msg) { throw Error(s, msg); }

#define HDG_REQUIRE(cond, status, msg)                                   \
    do {                                                                 \
        if (!(cond)) ::hdg::fail((status), std::string(msg));            \
    } while (0)

inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }
inline uint32_t next_pow2(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Index/search parameters and filter configuration held by an index.
struct FilterSpec {
    int l = 0;
    int type[HDG_MAX_LABEL_DIMS] = {0};
    float shift_val[2 * HDG_MAX_LABEL_DIMS] = {0};
    int div_value[HDG_MAX_LABEL_DIMS] = {0};
    std::vector<float> interval_map;  // flat concatenation of every map filter's table
};

// HDGrid.conf parsing (config_utils.h:33-88 semantics; see hdg_config.cpp).
void default_params(hdg_params* p);
void parse_hdgrid_conf(const std::string& text, hdg_params* p);
void parse_filter_conf(const std::string& text, FilterSpec* f);
std::string read_text_file(const std::string& path);
std::string upper(std::string s);

}  // namespace hdg
