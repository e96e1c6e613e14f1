// HDGrid oracle -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ (OpenMP, no CUDA) restatement of the HDGrid "super-grid" filtered query path,
// used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to check results,
// never to produce them.
// Nothing in the product links or calls this library.
//
// Each function cites the reference file:line it restates (paths inside the HDGrid project).
// The reference itself cannot be compiled here (it needs RAFT/RMM fetched at configure time,
// CMakeLists.txt:17-35), so this restatement is pinned by the known-answer vectors of the
// reference's own kernel tests (src/verification/test_lut_build.cuh:41-60,
// test_compute_pq_dis.cuh:47-97, test_filter.cuh:17-57, test_select_element.cuh:62-106),
// committed under tests/golden/.  RAFT select_k tie order and RAFT k-means are not pinned
// by any reference test: ties here are broken by the lower candidate index.
//
// It consumes the binary index file written by libhdgrid's hdg_save (format documented in
// the product's hdg_io.cpp); it re-derives every integer stage (filter box, cell box,
// Morton codes, per-list filtered counts) from the labels instead of reading the product's
// intermediate results.
#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <numeric>
#include <random>
#include <string>
#include <vector>

namespace {

constexpr int kMaxDims = 8;
constexpr int kCodes = 256;

// ---- CUDA conversion semantics emulated on the host ------------------------------------
// A float->uint64 C cast on the GPU (cvt.rzi.u64.f32) saturates: values below 0 give 0,
// values >= 2^64 give UINT64_MAX, and NaN gives 2^63 (measured on B200 through the
// reference's own get_grid_id_device, tests/golden/reference_stages.json).  x86 casts differ,
// so the oracle spells it out.
uint64_t sat_f2u64(float x) {
    if (std::isnan(x)) return 1ull << 63;
    if (x <= 0.0f) return 0;
    if (x >= 18446744073709551616.0f) return ~0ull;
    return (uint64_t)x;
}

// get_grid_id_device (src/index/2-level_index/Super-Grid-IVF_PQ.cu:24-26):
// ((uint64_t)((x - l) * M)) / len, float arithmetic, result truncated to int.
int grid_id(float x, uint64_t left, uint64_t len, int M) {
    volatile float a = x - (float)left;  // volatile: keep the two f32 roundings separate
    volatile float b = a * (float)M;
    return (int)(uint32_t)(sat_f2u64(b) / len);
}

struct Grid {
    int l = 0;
    int dims[kMaxDims] = {0};
    int shuffle[kMaxDims] = {0};
    uint64_t left[kMaxDims] = {0}, span[kMaxDims] = {0}, stride[kMaxDims] = {0};
    uint64_t tot_cells = 0;
    int mdims = 0, max_bits = 0, valid_map = 0, diff_dim = 0;
};

struct Filter {
    int l = 0;
    int type[kMaxDims] = {0};
    float shift[2 * kMaxDims] = {0};
    int div[kMaxDims] = {0};
    std::vector<float> map;
};

// A C-style f32 -> s32 cast as the GPU executes it (cvt.rzi.s32.f32): truncation, NaN -> 0,
// saturating at INT_MIN / INT_MAX.  An x86 cast of an out-of-range value gives INT_MIN instead.
static int cuda_f2i(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT_MAX;
    if (x <= -2147483648.0f) return INT_MIN;
    return (int)x;
}

// denormalize_labels_kernel (src/core/preprocessing.cu:3-32) for one query row.
void recover_row(const Filter& f, const float* row, float* out) {
    for (int i = 0; i < f.l; i++) {
        float lo, hi;
        switch (f.type[i]) {
            case 0: {  // max(float, 1e-7) promotes to double (:14-15)
                const double sl = std::max((double)f.shift[2 * i], 1e-7);
                const double sr = std::max((double)f.shift[2 * i + 1], 1e-7);
                lo = (float)((double)row[i] - sl);
                hi = (float)((double)row[i] + sr);
                break;
            }
            case 1: {  // label - 1 indexes the flat interval table (:18-20)
                volatile float t = row[i] - 1.0f;
                const int v = cuda_f2i(t);
                if (v >= 0 && 2 * (int64_t)v + 1 < (int64_t)f.map.size()) {
                    lo = f.map[2 * v];
                    hi = f.map[2 * v + 1];
                } else {  // out of the table: undefined in the reference; empty here
                    lo = FLT_MAX;
                    hi = -FLT_MAX;
                }
                break;
            }
            case 2: {  // integer division, upper bound FLT_MAX (:22-25)
                const int v = cuda_f2i(row[i]);
                const int dv = f.div[i] ? f.div[i] : 1;
                // INT_MIN / -1 is the one quotient that overflows: kept as INT_MIN (as the kernels do)
                lo = (float)((v == INT_MIN && dv == -1) ? v : v / dv);
                hi = FLT_MAX;
                break;
            }
            default:  // type 3: explicit [lo, hi] pair per dim (:27-28)
                lo = row[2 * i];
                hi = row[2 * i + 1];
        }
        out[2 * i] = lo;
        out[2 * i + 1] = hi;
    }
}

// get_filter_grid_ranges_kernel (Super-Grid-IVF_PQ.cu:930-961), shuffled dim order.
void cell_box(const Grid& g, const float* box, int* cells) {
    for (int i = 0; i < g.l; i++) {
        const int d = g.shuffle[i];
        const uint64_t blo = sat_f2u64(box[2 * d]), bhi = sat_f2u64(box[2 * d + 1]);
        const float l = (float)std::max(blo, g.left[i]);
        const float r = (float)std::min(bhi, g.left[i] + g.span[i]);
        const int gl = grid_id(l, g.left[i], g.span[i], g.dims[i]);
        const int gr = grid_id(r, g.left[i], g.span[i], g.dims[i]);
        int hi = std::min(gr, g.dims[i] - 1);
        int lo = std::min(hi, gl);
        if (hi < 0) hi = 0;  // int truncation below zero: out-of-bounds in the reference
        if (lo < 0) lo = 0;
        cells[2 * i] = lo;
        cells[2 * i + 1] = hi;
    }
}

// morton_encode (src/core/zorder.cu:3-15).
uint64_t morton(const int* c, int dims, int max_bits, int valid_map) {
    uint64_t code = 0;
    for (int b = 0; b < max_bits; ++b)
        for (int i = 0; i < dims; ++i) {
            if (!((valid_map >> i) & 1)) continue;
            code = (code << 1) | (uint64_t)((c[i] >> (max_bits - 1 - b)) & 1);
        }
    return code;
}

// Inverse of morton(): coords of every dim (masked dims 0), zorder.cu:17-34.
void unmorton(uint64_t code, int* c, int dims, int max_bits, int valid_map) {
    int active = 0;
    for (int i = 0; i < dims; i++) active += (valid_map >> i) & 1;
    for (int i = 0; i < dims; i++) c[i] = 0;
    for (int b = 0; b < max_bits; b++) {
        int j = 0;
        for (int i = 0; i < dims; i++) {
            if (!((valid_map >> i) & 1)) continue;
            const int shift = (max_bits - 1 - b) * active + (active - 1 - j);
            c[i] |= (int)((code >> shift) & 1) << (max_bits - 1 - b);
            j++;
        }
    }
}

bool in_cell_box(const int* c, const int* box, int dims) {
    for (int i = 0; i < dims; i++)
        if (c[i] < box[2 * i] || c[i] > box[2 * i + 1]) return false;
    return true;
}

// bit s (0 = most significant of max_bits) of v
inline int bit_at(int v, int s, int max_bits) { return (v >> (max_bits - 1 - s)) & 1; }

// getNextZValueBaseline (zorder.cu:83-243): the code the reference jumps to from cur.
bool next_in_box(uint64_t cur, const int* box, int dims, int max_bits, int valid_map, uint64_t* next) {
    const uint64_t nisp = cur + 1;
    int c[kMaxDims];
    unmorton(nisp, c, dims, max_bits, valid_map);
    if (in_cell_box(c, box, dims)) {
        *next = nisp;
        return true;
    }
    std::vector<int> act;  // active (unmasked) dims in order
    for (int i = 0; i < dims; i++)
        if ((valid_map >> i) & 1) act.push_back(i);
    const int A = (int)act.size();
    int flag[kMaxDims] = {0}, step[kMaxDims], smin[kMaxDims], smax[kMaxDims];
    for (int i : act) {
        step[i] = smin[i] = smax[i] = max_bits;
        const int lo = box[2 * i], hi = box[2 * i + 1];
        for (int s = 0; s < max_bits; s++) {
            const int cb = bit_at(c[i], s, max_bits), lb = bit_at(lo, s, max_bits);
            if (cb != lb) {
                if (cb < lb) {
                    flag[i] = -1;
                    step[i] = s;
                }
                break;
            }
        }
        if (flag[i] == 0)
            for (int s = 0; s < max_bits; s++) {
                const int cb = bit_at(c[i], s, max_bits), hb = bit_at(hi, s, max_bits);
                if (cb != hb) {
                    if (cb > hb) {
                        flag[i] = 1;
                        step[i] = s;
                    }
                    break;
                }
            }
        if (flag[i] != -1)
            for (int s = 0; s < max_bits; s++)
                if (bit_at(c[i], s, max_bits) > bit_at(lo, s, max_bits)) {
                    smin[i] = s;
                    break;
                }
        if (flag[i] != 1)
            for (int s = 0; s < max_bits; s++)
                if (bit_at(c[i], s, max_bits) < bit_at(hi, s, max_bits)) {
                    smax[i] = s;
                    break;
                }
    }
    // bit position (LSB = 0) of active dim j at step s
    auto pos = [&](int s, int j) { return (max_bits - 1 - s) * A + (A - 1 - j); };
    int change = 0;
    for (int j = 0; j < A; j++)
        if (step[act[j]] < max_bits) change = std::max(change, pos(step[act[j]], j));
    int d = act[A - 1 - change % A];
    if (flag[d] == 1) {
        int found = -1;
        for (int bp = change + 1; bp < max_bits * A; bp++) {
            const int j = A - 1 - bp % A;
            if (bp <= pos(smax[act[j]], j) && ((nisp >> bp) & 1) == 0) {
                found = bp;
                break;
            }
        }
        if (found < 0) return false;
        change = found;
        d = act[A - 1 - change % A];
        smin[d] = max_bits - 1 - change / A;
        flag[d] = 0;
    }
    const int blocks = change / A;
    for (int j = 0; j < A; j++) {
        const int i = act[j];
        if (flag[i] < 0) {
            c[i] = box[2 * i];
            continue;
        }
        const int k = blocks + (i > d ? 1 : 0);
        const uint64_t m = (1ull << k) - 1;
        const uint64_t src = change <= pos(smin[i], j) ? 0 : (uint64_t)(int64_t)box[2 * i];
        c[i] = (int)(((uint64_t)(int64_t)c[i] & ~m) | (src & m));
    }
    *next = morton(c, dims, max_bits, valid_map) | (1ull << change);
    return true;
}

// Cell coords of one point (get_grid_ids_kernel, Super-Grid-IVF_PQ.cu:28-52).
void point_cell(const Grid& g, const float* lab, int* coords) {
    for (int i = 0; i < g.l; i++) {
        int c = grid_id(lab[g.shuffle[i]], g.left[i], g.span[i], g.dims[i]);
        c = std::min(c, g.dims[i] - 1);
        coords[i] = std::max(c, 0);
    }
}

// compute_l2_distances_kernel_shared (src/core/refine.cu:36-75) for d <= 512: each thread
// holds one rounded squared difference, thread 0 sums them in dimension order.
float ref_l2(const float* a, const float* b, int d) {
    float s = 0.f;
    for (int i = 0; i < d; i++) {
        volatile float t = a[i] - b[i];
        volatile float sq = t * t;
        s = s + sq;
    }
    return s;
}

struct Index {
    uint64_t params[24] = {0};
    Filter f;
    uint64_t n = 0, d = 0, l = 0, M = 0, M_pad = 0, pq_len = 0, L = 0, C = 0;
    Grid g;
    std::vector<float> centers, sub_centers, pq_centers, labels;
    std::vector<uint32_t> cluster_off, list_off, ids, prefix;
    // compressed prefix rows (file version 2, prefix empty): per (grid row t, list j) the change
    // points (z << 32 | count) of the inclusive prefix along the diff dim
    std::vector<uint64_t> prefix_off, prefix_rows;
    std::vector<uint64_t> zcodes;
    // inclusive prefix count of list j at flat cell `flat` from either stored form
    uint32_t prefix_at(uint64_t flat, uint64_t j) const {
        if (prefix_off.empty()) return prefix[flat * L + j];
        const uint64_t Dd = (uint64_t)g.dims[g.diff_dim];
        const uint64_t r = (flat / Dd) * L + j, z = flat % Dd;
        const uint64_t* b = prefix_rows.data() + prefix_off[r];
        const uint64_t* e = prefix_rows.data() + prefix_off[r + 1];
        // query_compressed_sum_device (Super-Grid-IVF_PQ.cu:648-691): the last change point <= z
        const uint64_t* it = std::upper_bound(b, e, z, [](uint64_t key, uint64_t v) { return key < (v >> 32); });
        return it == b ? 0u : (uint32_t)it[-1];
    }
    std::vector<uint8_t> codes;
    uint64_t topk() const { return params[0]; }
    uint64_t filter_dim() const { return params[1]; }
    uint64_t exps0() const { return params[4]; }
    uint64_t n_list() const { return params[8]; }
    uint64_t sub_lists() const { return params[9]; }
    uint64_t lut_fp16() const { return params[20]; }
    uint64_t n_split() const { return params[10]; }
    uint64_t is_split() const { return params[12]; }
};

template <typename T>
bool rd(std::ifstream& f, T& v) {
    f.read(reinterpret_cast<char*>(&v), sizeof(T));
    return (bool)f;
}
template <typename T>
bool rdv(std::ifstream& f, std::vector<T>& v) {
    uint64_t n;
    if (!rd(f, n)) return false;
    v.resize(n);
    if (n) f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
    return (bool)f;
}

std::string g_err;

}  // namespace

extern "C" {

const char* ora_last_error() { return g_err.c_str(); }

// ---- known-answer-test level functions -------------------------------------------------

// build_pq_lut_kernel (src/index/product-quantization.cu:4-35); CPU twin compute_lut_cpu
// (src/verification/ground_truth.cuh:58-137).  The reference's `ans += (c-q)*(c-q)` is
// contracted into an FMA by nvcc's default -fmad=true; the oracle uses fmaf likewise.
void ora_pq_lut(const float* centers, const float* queries, uint64_t nq, uint32_t n_dim, uint32_t pq_dim,
                uint32_t pq_len, uint32_t n_codes, float* lut) {
    for (uint64_t q = 0; q < nq; q++)
        for (uint32_t m = 0; m < pq_dim; m++)
            for (uint32_t c = 0; c < n_codes; c++) {
                float s = 0.f;
                for (uint32_t t = 0; t < pq_len && m * pq_len + t < n_dim; t++) {
                    const float df = centers[((uint64_t)m * n_codes + c) * pq_len + t] - queries[q * n_dim + m * pq_len + t];
                    s = std::fmaf(df, df, s);
                }
                lut[(q * pq_dim + m) * n_codes + c] = s;
            }
}

// compute_batched_L2_distance_kernel (product-quantization.cu:37-77), codes column-major.
void ora_pq_adc(const uint8_t* codebook, uint64_t tot_data, const float* lut, uint64_t nq, uint32_t pq_dim,
                uint32_t n_codes, const uint64_t* indices, uint64_t n_cand, float* dist) {
    for (uint64_t q = 0; q < nq; q++)
        for (uint64_t j = 0; j < n_cand; j++) {
            const uint64_t idx = indices ? indices[q * n_cand + j] : j;
            if (idx >= tot_data) {
                dist[q * n_cand + j] = FLT_MAX;
                continue;
            }
            float s = 0.f;
            for (uint32_t m = 0; m < pq_dim; m++) s += lut[(q * pq_dim + m) * n_codes + codebook[m * tot_data + idx]];
            dist[q * n_cand + j] = s;
        }
}

// label_matrix_by_filter_indices_kernel (src/core/filter.cu:30-64).
void ora_label_mask(const float* ranges, const float* labels, uint32_t l, uint64_t n_data, uint64_t nq,
                    const uint64_t* indices, uint64_t n_cand, int32_t* mask) {
    for (uint64_t q = 0; q < nq; q++)
        for (uint64_t j = 0; j < n_cand; j++) {
            const uint64_t idx = indices ? indices[q * n_cand + j] : j;
            int ok = idx < n_data;
            for (uint32_t i = 0; ok && i < l; i++) {
                const float v = labels[idx * l + i];
                if (v < ranges[q * 2 * l + 2 * i] || v > ranges[q * 2 * l + 2 * i + 1]) ok = 0;
            }
            mask[q * n_cand + j] = ok;
        }
}

// select_elements_kernel / select_elements_row_kernel (src/core/mat_operators.cuh:151-186):
// row gather (out[x][y][:] = in[idx[x][y]][:]) and element gather (out[x][y] = in[x][idx[x][y]]).
void ora_select_elements(const float* in, uint64_t n_row_i, uint64_t n_dim_i, const uint64_t* idx,
                         uint64_t n_row_o, uint64_t n_dim_o, int select_row, float invalid, float* out) {
    for (uint64_t x = 0; x < n_row_o; x++)
        for (uint64_t y = 0; y < n_dim_o; y++) {
            const uint64_t id = idx[x * n_dim_o + y];
            if (select_row) {
                for (uint64_t z = 0; z < n_dim_i; z++)
                    out[(x * n_dim_o + y) * n_dim_i + z] =
                        id < n_row_i ? in[id * n_dim_i + z] : std::sqrt(invalid / (float)n_dim_i);
            } else {
                out[x * n_dim_o + y] = id < n_dim_i ? in[x * n_dim_i + id] : invalid;
            }
        }
}

// recovery_filters for a batch; type/shift/div/map as in filter.conf.
void ora_recover_filters(int l, const int* type, const float* shift, const int* div, const float* map, int n_map,
                         int filter_dim, const float* qlabels, uint64_t nq, float* out) {
    Filter f;
    f.l = l;
    for (int i = 0; i < l; i++) {
        f.type[i] = type[i];
        f.div[i] = div[i];
        f.shift[2 * i] = shift[2 * i];
        f.shift[2 * i + 1] = shift[2 * i + 1];
    }
    f.map.assign(map, map + n_map);
    for (uint64_t q = 0; q < nq; q++) recover_row(f, qlabels + q * l * filter_dim, out + q * 2 * l);
}

uint64_t ora_morton_encode(const int* coords, int dims, int max_bits, int valid_map) {
    return morton(coords, dims, max_bits, valid_map);
}

int ora_grid_id(float x, uint64_t left, uint64_t len, int M) { return grid_id(x, left, len, M); }

// get_filter_grid_ranges_kernel (Super-Grid-IVF_PQ.cu:930-961) for n boxes [n x 2l] f32 against
// a grid given in shuffled order (dims, shuffle, left, span); cells [n x 2l] i32.
void ora_cell_boxes(const float* boxes, uint64_t n, int l, const int* dims, const int* shuffle, const uint64_t* left,
                    const uint64_t* span, int32_t* cells) {
    Grid g;
    g.l = l;
    for (int i = 0; i < l; i++) {
        g.dims[i] = dims[i];
        g.shuffle[i] = shuffle[i];
        g.left[i] = left[i];
        g.span[i] = span[i];
    }
    for (uint64_t r = 0; r < n; r++) cell_box(g, boxes + r * 2 * l, cells + r * 2 * l);
}

// getNextZValueBaseline (zorder.cu:83-244) for n (code, cell box [2 * dims]) pairs: next[i] and
// ok[i] (0 where the reference returns false).
void ora_next_in_box(const uint64_t* cur, const int32_t* boxes, uint64_t n, int dims, int max_bits, int valid_map,
                     uint64_t* next, int32_t* ok) {
    for (uint64_t r = 0; r < n; r++) {
        uint64_t nx = 0;
        ok[r] = next_in_box(cur[r], boxes + r * 2 * dims, dims, max_bits, valid_map, &nx) ? 1 : 0;
        next[r] = ok[r] ? nx : 0;
    }
}

// calc_grid_shape (Super-Grid-IVF_PQ.cu:305-412).  Outputs dims/shuffle/left/span in shuffled
// order plus max_bits and valid_map.  A zero span is raised to 1 (division by zero upstream).
int ora_grid_shape(const float* mins, const float* maxs, int l, uint64_t max_grids, uint64_t label_mask, int* dims,
                   int* shuffle, uint64_t* left, uint64_t* span, int* max_bits, int* valid_map) {
    const uint8_t lm = (uint8_t)(~(uint8_t)label_mask);
    int cnt = 0;
    for (int i = 0; i < l; i++) cnt += (lm >> i) & 1;
    std::vector<std::pair<uint64_t, int>> sp(l);
    for (int i = 0; i < l; i++) {
        // `ceil(global_max[i]) - floor(global_min[i])` (:326) on float elements: the float
        // overloads, so the difference is rounded to f32 (a span above 2^24 with an odd
        // exact difference loses its last bit) before the uint64 conversion
        volatile float mx = std::ceil(maxs[i]);
        volatile float mn = std::floor(mins[i]);
        volatile float diff = mx - mn;
        uint64_t s = (uint64_t)diff;
        sp[i] = {s ? s : 1, i};
    }
    int main_grids = (int)std::floor(std::sqrt((double)max_grids));
    std::sort(sp.begin(), sp.end());
    if (l == 1) main_grids = (int)std::min<uint64_t>(max_grids, sp[0].first);
    int remain = 1, remain_cnt = cnt - 1, last_valid = l - 1;
    if (l > 1) remain = (int)(max_grids / (uint64_t)main_grids);
    uint8_t mm = 0xff;
    for (int i = 0; i < l; i++) {
        const int id = sp[i].second;
        const uint64_t len = sp[i].first;
        if ((lm >> id) & 1) {
            if (remain_cnt == 0) {
                last_valid = i;
                continue;
            }
            const uint64_t root = (uint64_t)std::floor(std::pow((double)main_grids, 1.0 / (double)(float)(cnt - 1)));
            int dl = (int)std::min<uint64_t>((uint64_t)remain, std::min<uint64_t>(len, root));
            if (remain_cnt == 1) dl = (int)std::min<uint64_t>((uint64_t)remain, len);
            remain_cnt--;
            if (dl < 1) return -1;
            dims[i] = dl;
            remain /= dl;
        } else {
            mm &= (uint8_t)~(1 << i);
            dims[i] = 1;
        }
    }
    dims[last_valid] = main_grids;
    int mx = 0;
    for (int i = 0; i < l; i++) {
        shuffle[i] = sp[i].second;
        span[i] = sp[i].first;
        left[i] = (uint64_t)std::floor((double)mins[sp[i].second]);
        mx = std::max(mx, dims[i]);
    }
    *max_bits = (int)std::ceil(std::log2((double)mx + 1));
    *valid_map = mm & (uint8_t)((1u << l) - 1);
    return 0;
}

// ---- filtered brute force (the correctness oracle) -------------------------------------
// brute_forece_vector_search (src/verification/ground_truth.cuh:165-232) generalised to the
// filter.conf box: exact distances in FP64, f32 label predicate, smallest k by (distance, id).
void ora_bruteforce_f64(const float* data, uint64_t n, uint32_t d, const float* labels, uint32_t l,
                        const float* queries, uint64_t q, const float* ranges, uint32_t k, double* out_dist,
                        uint64_t* out_ids, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t qi = 0; qi < (int64_t)q; qi++) {
        std::vector<std::pair<double, uint64_t>> best;
        best.reserve(k + 1);
        const float* box = ranges + qi * 2 * l;
        const float* qv = queries + qi * d;
        for (uint64_t i = 0; i < n; i++) {
            bool ok = true;
            for (uint32_t c = 0; c < l && ok; c++) {
                const float v = labels[i * l + c];
                if (v < box[2 * c] || v > box[2 * c + 1]) ok = false;
            }
            if (!ok) continue;
            double s = 0.0;
            const float* x = data + i * d;
            for (uint32_t j = 0; j < d; j++) {
                const double df = (double)qv[j] - (double)x[j];
                s += df * df;
            }
            const std::pair<double, uint64_t> e{s, i};
            if (best.size() < k) {
                best.push_back(e);
                std::push_heap(best.begin(), best.end());
            } else if (e < best.front()) {
                std::pop_heap(best.begin(), best.end());
                best.back() = e;
                std::push_heap(best.begin(), best.end());
            }
        }
        std::sort_heap(best.begin(), best.end());
        for (uint32_t j = 0; j < k; j++) {
            out_dist[qi * k + j] = j < best.size() ? best[j].first : INFINITY;
            out_ids[qi * k + j] = j < best.size() ? best[j].second : ~0ull;
        }
    }
}

// ---- the index file and the reference query schedule ------------------------------------

void* ora_open(const char* path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        g_err = std::string("cannot open ") + path;
        return nullptr;
    }
    char magic[8];
    f.read(magic, 8);
    uint32_t ver, pad;
    if (!f || std::memcmp(magic, "HDGB200I", 8) != 0 || !rd(f, ver) || (ver != 1 && ver != 2) || !rd(f, pad)) {
        g_err = "bad index file header";
        return nullptr;
    }
    Index* ix = new Index();
    bool ok = true;
    for (auto& p : ix->params) ok = ok && rd(f, p);
    uint32_t plen = 0;
    ok = ok && rd(f, plen);
    f.seekg(plen, std::ios::cur);
    ok = ok && rd(f, ix->f.l);
    for (int i = 0; i < kMaxDims; i++) ok = ok && rd(f, ix->f.type[i]);
    for (int i = 0; i < 2 * kMaxDims; i++) ok = ok && rd(f, ix->f.shift[i]);
    for (int i = 0; i < kMaxDims; i++) ok = ok && rd(f, ix->f.div[i]);
    uint32_t nm = 0;
    ok = ok && rd(f, nm);
    ix->f.map.resize(nm);
    for (uint32_t i = 0; i < nm; i++) ok = ok && rd(f, ix->f.map[i]);
    for (uint64_t* v : {&ix->n, &ix->d, &ix->l, &ix->M, &ix->M_pad, &ix->pq_len, &ix->L, &ix->C}) ok = ok && rd(f, *v);
    Grid& g = ix->g;
    ok = ok && rd(f, g.l);
    for (int i = 0; i < kMaxDims; i++) ok = ok && rd(f, g.dims[i]);
    for (int i = 0; i < kMaxDims; i++) ok = ok && rd(f, g.shuffle[i]);
    for (int i = 0; i < kMaxDims; i++) ok = ok && rd(f, g.left[i]);
    for (int i = 0; i < kMaxDims; i++) ok = ok && rd(f, g.span[i]);
    for (int i = 0; i < kMaxDims; i++) ok = ok && rd(f, g.stride[i]);
    ok = ok && rd(f, g.tot_cells) && rd(f, g.mdims) && rd(f, g.max_bits) && rd(f, g.valid_map) && rd(f, g.diff_dim);
    ok = ok && rdv(f, ix->centers) && rdv(f, ix->sub_centers) && rdv(f, ix->pq_centers) && rdv(f, ix->cluster_off) &&
         rdv(f, ix->list_off) && rdv(f, ix->ids) && rdv(f, ix->prefix) &&
         (ver == 1 || (rdv(f, ix->prefix_off) && rdv(f, ix->prefix_rows))) && rdv(f, ix->zcodes) &&
         rdv(f, ix->codes) && rdv(f, ix->labels);
    if (!ok) {
        g_err = "truncated index file";
        delete ix;
        return nullptr;
    }
    return ix;
}

void ora_close(void* h) { delete static_cast<Index*>(h); }

// Geometry accessors for tests: [n, d, l, M, M_pad, L, C, tot_cells, max_bits, valid_map,
// topk, filter_dim, exps0, n_list, sub_lists].
void ora_info(void* h, uint64_t* out) {
    const Index& ix = *static_cast<Index*>(h);
    const uint64_t v[] = {ix.n, ix.d, ix.l, ix.M, ix.M_pad, ix.L, ix.C, ix.g.tot_cells,
                          (uint64_t)ix.g.max_bits, (uint64_t)ix.g.valid_map, ix.topk(), ix.filter_dim(),
                          ix.exps0(), std::max<uint64_t>(1, ix.n_list()), std::max<uint64_t>(1, ix.sub_lists()),
                          ix.is_split(), ix.is_split() ? std::max<uint64_t>(1, ix.n_split()) : 1};
    std::memcpy(out, v, sizeof(v));
}

void ora_grid(void* h, int* dims, int* shuffle, uint64_t* left, uint64_t* span) {
    const Index& ix = *static_cast<Index*>(h);
    for (int i = 0; i < ix.g.l; i++) {
        dims[i] = ix.g.dims[i];
        shuffle[i] = ix.g.shuffle[i];
        left[i] = ix.g.left[i];
        span[i] = ix.g.span[i];
    }
}

// Checks the stored pool layout against the labels: Morton code of every point recomputed
// from its labels (== stored zcodes), Z-order sorted inside each list, prefix counts equal
// to a direct per-cell count.  Returns the number of mismatches (0 = bit-exact).
uint64_t ora_check_layout(void* h) {
    const Index& ix = *static_cast<Index*>(h);
    const Grid& g = ix.g;
    uint64_t bad = 0;
    // the stored grid against calc_grid_shape re-derived here from the stored labels' extremes
    // (calculate_batch_min_max, Super-Grid-IVF_PQ.cu:308-310)
    if (ix.n && ix.l) {
        std::vector<float> mn(ix.l, FLT_MAX), mx(ix.l, -FLT_MAX);
        for (uint64_t p = 0; p < ix.n; p++)
            for (uint64_t i = 0; i < ix.l; i++) {
                mn[i] = std::min(mn[i], ix.labels[p * ix.l + i]);
                mx[i] = std::max(mx[i], ix.labels[p * ix.l + i]);
            }
        int dims[kMaxDims], sh[kMaxDims], mb = 0, vm = 0;
        uint64_t left[kMaxDims], span[kMaxDims];
        if (ora_grid_shape(mn.data(), mx.data(), (int)ix.l, ix.params[7], ix.params[11], dims, sh, left, span, &mb,
                           &vm) != 0)
            bad++;
        else {
            for (uint64_t i = 0; i < ix.l; i++)
                bad += (dims[i] != g.dims[i]) + (sh[i] != g.shuffle[i]) + (left[i] != g.left[i]) +
                       (span[i] != g.span[i]);
            bad += (mb != g.max_bits) + (vm != g.valid_map);
        }
    }
    std::vector<uint32_t> dense(g.tot_cells * ix.L, 0);
    for (uint64_t j = 0; j < ix.L; j++)
        for (uint32_t p = ix.list_off[j]; p < ix.list_off[j + 1]; p++) {
            int c[kMaxDims];
            point_cell(g, &ix.labels[(uint64_t)p * ix.l], c);
            if (morton(c, g.mdims, g.max_bits, g.valid_map) != ix.zcodes[p]) bad++;
            if (p > ix.list_off[j] && (ix.zcodes[p - 1] > ix.zcodes[p] ||
                                       (ix.zcodes[p - 1] == ix.zcodes[p] && ix.ids[p - 1] > ix.ids[p])))
                bad++;
            uint64_t flat = 0;
            for (int i = 0; i < g.l; i++) flat += (uint64_t)c[i] * g.stride[i];
            dense[flat * ix.L + j]++;
        }
    // inclusive multi-dim scan (HOPS::multi_dim_scan, src/core/HOPS.cu:3-74)
    for (int a = 0; a < g.l; a++) {
        const uint64_t inner = g.stride[a], len = (uint64_t)g.dims[a];
        const uint64_t outer = g.tot_cells / (inner * len);
        for (uint64_t o = 0; o < outer; o++)
            for (uint64_t in = 0; in < inner; in++)
                for (uint64_t j = 0; j < ix.L; j++) {
                    uint32_t s = 0;
                    for (uint64_t x = 0; x < len; x++) {
                        uint32_t& v = dense[((o * len + x) * inner + in) * ix.L + j];
                        s += v;
                        v = s;
                    }
                }
    }
    // the stored counts, dense or compressed, against this dense recount at every cell and list
    for (uint64_t c = 0; c < g.tot_cells; c++)
        for (uint64_t j = 0; j < ix.L; j++)
            if (dense[c * ix.L + j] != ix.prefix_at(c, j)) bad++;
    return bad;
}

// Trace of one batch (any pointer may be NULL).  Sizes: box [q*2l] f32, cells [q*2l] i32,
// zrange [q*2] u64, list_counts [q*L] u32, probe_clusters [q*n_list] u32, probe_lists
// [q*sub_lists] u32, range_start / range_len [q*sub_lists] u32, scalars [4]:
// (n_cand, beta as double bits, coarse total, real total).
struct OraTrace {
    float* box;
    int32_t* cells;
    uint64_t* zrange;
    uint32_t* list_counts;
    uint32_t* probe_clusters;
    uint32_t* probe_lists;
    uint32_t* range_start;
    uint32_t* range_len;
    double* scalars;
};

// super_grid::index::query (Super-Grid-IVF_PQ.cu:985-1249) on the CPU.
// Outputs dist [q x k] f32 and ids [q x k] u64 (ascending; +inf / UINT64_MAX when empty).
// Optional per-query arrays (NULL = uniform), the semantics of hdg_query_ex: qk result
// count clamped to [1, k] (rows keep stride k); qps probed sub-lists clamped to
// [1, sub_lists]; qsched 1 = label predicate during the ADC pass, budget exps0*k_q, exact
// re-rank without a second predicate.  These have no reference counterpart; with all three
// NULL this is the reference's query.  adc_mode bit 0: the scan's lane-rotated ADC order
// (below); bit 1: per-list counts from the index's prefix counts, as the reference counts
// (otherwise a direct count of the points in the cell box, the independent check).
int ora_query_ex(void* h, const float* queries, uint64_t q, const float* qlabels, uint32_t label_cols,
                 const float* data, uint32_t k, const uint32_t* qk, const uint32_t* qps, const uint8_t* qsched,
                 float* out_dist, uint64_t* out_ids, OraTrace* tr, int threads, int adc_mode) {
    const Index& ix = *static_cast<Index*>(h);
    const Grid& g = ix.g;
    const int l = (int)ix.l, d = (int)ix.d, M = (int)ix.M;
    const uint64_t L = ix.L, C = ix.C;
    const int Pc = (int)std::max<uint64_t>(1, ix.n_list()), Ps = (int)std::max<uint64_t>(1, ix.sub_lists());
    const uint64_t exps0 = ix.exps0();
    const int mode = exps0 <= 1 ? 0 : (l > 1 ? 1 : 2);  // pre-filter / post-filter / l==1
    const bool split = ix.is_split() != 0;
    const int ns = split ? (int)std::max<uint64_t>(1, ix.n_split()) : 1;
    const int R = Ps * ns;  // candidate ranges per query
    if (threads > 0) omp_set_num_threads(threads);
    struct QState {
        float box[2 * kMaxDims];
        std::vector<uint32_t> start, len;
        uint64_t cand = 0, exact = 0;
    };
    std::vector<QState> st(q);
    // ---- phase 1: box, cells, counts, probes, Morton ranges -----------------------------
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t qi = 0; qi < (int64_t)q; qi++) {
        QState& s = st[qi];
        recover_row(ix.f, qlabels + qi * label_cols, s.box);
        int cells[2 * kMaxDims];
        cell_box(g, s.box, cells);
        int lo[kMaxDims], hi[kMaxDims];
        for (int i = 0; i < l; i++) {
            lo[i] = cells[2 * i];
            hi[i] = cells[2 * i + 1];
        }
        const uint64_t zlo = morton(lo, g.mdims, g.max_bits, g.valid_map);
        const uint64_t zhi = morton(hi, g.mdims, g.max_bits, g.valid_map);
        // per-list filtered counts: a direct count of the list's points whose cell lies in
        // the cell box over the unmasked dims -- equal to the reference's 2^d-corner
        // inclusion-exclusion over its compressed prefix sums (:648-765).
        std::vector<uint32_t> lc(L, 0);
        if (adc_mode & 2) {
            // the reference's own count (get_prefix_sum_device, :693-724): inclusion-exclusion
            // over the 2^d corners of the cell box, read from the index's inclusive per-list
            // prefix counts (a lower corner below cell 0 contributes nothing)
            int dv = 0;
            for (int i = 0; i < l; i++) dv += (g.valid_map >> i) & 1;
            std::vector<long long> acc(L, 0);
            for (int mask = 0; mask < (1 << dv); mask++) {
                int sign = 1, vi = 0;
                bool zero = false;
                uint64_t flat = 0;
                for (int i = 0; i < l; i++) {
                    int c = 0;
                    if ((g.valid_map >> i) & 1) {
                        if ((mask >> vi) & 1) {
                            c = lo[i] - 1;
                            sign = -sign;
                            if (c < 0) zero = true;
                        } else {
                            c = hi[i];
                        }
                        vi++;
                    }
                    flat += (uint64_t)(c < 0 ? 0 : c) * g.stride[i];
                }
                if (zero) continue;
                for (uint64_t j = 0; j < L; j++) acc[j] += sign * (long long)ix.prefix_at(flat, j);
            }
            for (uint64_t j = 0; j < L; j++) lc[j] = (uint32_t)acc[j];
        } else {
            for (uint64_t j = 0; j < L; j++) {
                uint32_t cnt = 0;
                for (uint32_t p = ix.list_off[j]; p < ix.list_off[j + 1]; p++) {
                    int c[kMaxDims];
                    point_cell(g, &ix.labels[(uint64_t)p * l], c);
                    bool in = true;
                    for (int i = 0; i < l && in; i++)
                        if (((g.valid_map >> i) & 1) && (c[i] < lo[i] || c[i] > hi[i])) in = false;
                    cnt += in;
                }
                lc[j] = cnt;
            }
        }
        // coarse: exact L2 to clusters with a non-zero count, sorted (::refine, :1034-1042)
        std::vector<std::pair<float, uint32_t>> cl;
        for (uint64_t c = 0; c < C; c++) {
            uint64_t sum = 0;
            for (uint32_t j = ix.cluster_off[c]; j < ix.cluster_off[c + 1]; j++) sum += lc[j];
            if (sum) cl.push_back({ref_l2(queries + qi * d, &ix.centers[c * d], d), (uint32_t)c});
        }
        std::sort(cl.begin(), cl.end());
        const int npc = std::min<int>(Pc, (int)cl.size());
        // lists of the chosen clusters with a non-zero count (select_sub_clusters, :849-901)
        std::vector<std::pair<float, uint32_t>> sl;
        for (int i = 0; i < npc; i++) {
            const uint32_t c = cl[i].second;
            for (uint32_t j = ix.cluster_off[c]; j < ix.cluster_off[c + 1]; j++)
                if (lc[j]) sl.push_back({ref_l2(queries + qi * d, &ix.sub_centers[(uint64_t)j * d], d), j});
        }
        std::sort(sl.begin(), sl.end());
        const int psq = qps ? std::max(1, std::min(Ps, (int)qps[qi])) : Ps;
        const int nps = std::min<int>(psq, (int)sl.size());
        // the chosen lists in list-id (= pool) order; RAFT select_k returns them unsorted
        std::sort(sl.begin(), sl.begin() + nps, [](const auto& a, const auto& b) { return a.second < b.second; });
        s.start.assign((size_t)R, split ? 0xffffffffu : 0u);
        s.len.assign((size_t)R, 0);
        for (int i = 0; i < nps; i++) {
            const uint32_t j = sl[i].second;
            const uint64_t* zb = &ix.zcodes[ix.list_off[j]];
            const uint64_t* ze = &ix.zcodes[ix.list_off[j + 1]];
            // get_query_end_points_no_split_kernel (zorder.cu:656-685)
            const uint32_t a = (uint32_t)(std::lower_bound(zb, ze, zlo) - zb);
            const uint32_t b = (uint32_t)(std::lower_bound(zb, ze, zhi + 1) - zb);
            s.exact += lc[j];
            if (!split) {
                s.start[i] = ix.list_off[j] + a;
                s.len[i] = b - a;
                s.cand += b - a;
                continue;
            }
            // is_split: near-equal parts (get_query_end_points_kernel, zorder.cu:596-654), each
            // start moved by up to three next-in-box jumps, the part dropped when a jump fails or
            // passes its last code (zorder_range_query_kernel, :474-594, indexing this query's
            // probed list rather than candidates[c] of :500)
            const uint32_t n = b - a;
            const uint32_t parts = std::min<uint32_t>(n, (uint32_t)ns);
            for (uint32_t sp = 0; sp < parts; sp++) {
                const uint32_t qn = n / parts, rem = n % parts;
                uint32_t lo = ix.list_off[j] + a + sp * qn + std::min(sp, rem);
                const uint32_t hi = lo + qn + (sp < rem ? 1 : 0);
                const uint64_t* z = ix.zcodes.data();
                const uint64_t zmax = z[hi - 1];
                uint64_t cur = z[lo];
                bool ok = true;
                for (int jump = 0; jump < 3; jump++) {
                    const uint32_t at = (uint32_t)(std::lower_bound(z + lo, z + hi, cur) - z);
                    if (at >= hi) break;
                    lo = at;
                    int c[kMaxDims];
                    unmorton(z[at], c, g.mdims, g.max_bits, g.valid_map);
                    if (in_cell_box(c, cells, g.mdims)) break;
                    uint64_t nz = 0;
                    if (!next_in_box(z[at], cells, g.mdims, g.max_bits, g.valid_map, &nz) || nz >= zmax) {
                        ok = false;
                        break;
                    }
                    cur = nz;
                }
                s.start[(size_t)i * ns + sp] = lo;
                s.len[(size_t)i * ns + sp] = ok ? hi - lo : 0;
                s.cand += ok ? hi - lo : 0;
            }
        }
        if (tr) {
            if (tr->box) std::memcpy(tr->box + qi * 2 * l, s.box, sizeof(float) * 2 * l);
            if (tr->cells) std::memcpy(tr->cells + qi * 2 * l, cells, sizeof(int) * 2 * l);
            if (tr->zrange) {
                tr->zrange[qi * 2] = zlo;
                tr->zrange[qi * 2 + 1] = zhi;
            }
            if (tr->list_counts) std::memcpy(tr->list_counts + qi * L, lc.data(), sizeof(uint32_t) * L);
            if (tr->probe_clusters)
                for (int i = 0; i < Pc; i++) tr->probe_clusters[qi * Pc + i] = i < npc ? cl[i].second : 0xffffffffu;
            for (int i = 0; i < Ps; i++)
                if (tr->probe_lists) tr->probe_lists[qi * Ps + i] = i < nps ? sl[i].second : 0xffffffffu;
            for (int r = 0; r < R; r++) {
                if (tr->range_start) tr->range_start[qi * R + r] = s.start[r];
                if (tr->range_len) tr->range_len[qi * R + r] = s.len[r];
            }
        }
    }
    // ---- candidate budget (post-filter: beta over the batch, :1198-1222) -----------------
    uint64_t K = k;
    double beta = 0.0;
    uint64_t coarse = 0, real = 0, max_row = 0;
    for (uint64_t qi = 0; qi < q; qi++) {
        coarse += st[qi].cand;
        real += st[qi].exact;
        max_row = std::max(max_row, st[qi].cand);
    }
    if (mode == 1) {
        if (real == 0) {
            K = max_row;
            beta = INFINITY;
        } else {
            const float b = (float)coarse / (float)real;
            beta = b;
            const float want = (float)(exps0 * (uint64_t)k) * b;
            const uint64_t nc = want >= 1.8e19f ? ~0ull : (uint64_t)want;
            K = std::min(nc, max_row);
        }
    } else if (mode == 2) {
        K = exps0 * k;
    }
    // the same budget for a query's schedule; the batch's k, not the query's own: the reference
    // has one topk per batch, so a mixed-k batch runs as a batch of the call's k whose rows are
    // cut to each query's k
    auto budget = [&](bool sched1) -> uint64_t {
        if (mode == 2 || sched1) return exps0 * (uint64_t)k;
        if (real == 0) return max_row;
        const float want = (float)(exps0 * (uint64_t)k) * (float)beta;
        return std::min<uint64_t>(want >= 1.8e19f ? ~0ull : (uint64_t)want, max_row);
    };
    if (tr && tr->scalars) {
        tr->scalars[0] = (double)K;
        tr->scalars[1] = beta;
        tr->scalars[2] = (double)coarse;
        tr->scalars[3] = (double)real;
    }
    // ---- phase 2: LUT, ADC, predicate, re-rank -------------------------------------------
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t qi = 0; qi < (int64_t)q; qi++) {
        const QState& s = st[qi];
        const float* qv = queries + qi * d;
        std::vector<float> lut((size_t)M * kCodes);
        for (int m = 0; m < M; m++)
            for (int c = 0; c < kCodes; c++) {
                float acc = 0.f;
                for (uint64_t t = 0; t < ix.pq_len; t++) {
                    const float df = ix.pq_centers[((uint64_t)m * kCodes + c) * ix.pq_len + t] - qv[m * ix.pq_len + t];
                    acc = std::fmaf(df, df, acc);
                }
                // LUT_FP16=1: entries stored in binary16 (round to nearest even), summed in f32
                lut[(size_t)m * kCodes + c] = ix.lut_fp16() ? (float)(_Float16)acc : acc;
            }
        auto pred = [&](uint32_t pool) {
            for (int i = 0; i < l; i++) {
                const float v = ix.labels[(uint64_t)pool * l + i];
                if (v < s.box[2 * i] || v > s.box[2 * i + 1]) return false;
            }
            return true;
        };
        // adc_mode 0: subspace order 0..M-1 (compute_batched_L2_distance_kernel :69-72).
        // adc_mode 1 (test mode): the order of the GPU scan's bank-rotated LUT, where the
        // candidate at position e of the query sums each group of 32 subspaces starting at
        // subspace (e mod 32) and wrapping, alternate steps into two partial sums that are
        // added last -- used to check that scan bit for bit.
        auto adc = [&](uint32_t pool, uint32_t pos) {
            float sum = 0.f;
            const uint8_t* cp = &ix.codes[(uint64_t)pool * ix.M_pad];
            if (adc_mode & 1) {
                // even steps and odd steps in two running sums, added at the end
                const int lane = (int)(pos & 31);
                float s1 = 0.f;
                for (int g0 = 0; g0 < M; g0 += 32)
                    for (int st = 0; st < 32; st++) {
                        const int m = g0 + ((lane + st) & 31);
                        if (st & 1)
                            s1 += lut[(size_t)m * kCodes + cp[m]];
                        else
                            sum += lut[(size_t)m * kCodes + cp[m]];
                    }
                sum += s1;
            } else {
                for (int m = 0; m < M; m++) sum += lut[(size_t)m * kCodes + cp[m]];
            }
            return sum;
        };
        const uint32_t kq = qk ? std::max(1u, std::min(qk[qi], k)) : k;
        const bool sched1 = mode != 0 && qsched && qsched[qi] == 1;
        const bool pre = mode == 0 || sched1;
        std::vector<std::pair<float, uint32_t>> cand;
        uint32_t pos = 0;
        for (int r = 0; r < R; r++)
            for (uint32_t p = s.start[r]; p < s.start[r] + s.len[r]; p++, pos++) {
                if (pre && !pred(p)) continue;  // query_prefilter (prefiltering.cu:36-51)
                cand.push_back({adc(p, pos), p});
            }
        // the smallest (distance, pool row) pairs; pairs are unique, so a selection gives the
        // same set a full sort would
        if (mode == 0) {
            const size_t nk = std::min<size_t>(cand.size(), kq);
            std::partial_sort(cand.begin(), cand.begin() + nk, cand.end());
            for (uint32_t j = 0; j < k; j++) {
                out_dist[qi * k + j] = j < std::min<size_t>(cand.size(), kq) ? cand[j].first : INFINITY;
                out_ids[qi * k + j] = j < std::min<size_t>(cand.size(), kq) ? ix.ids[cand[j].second] : ~0ull;
            }
            continue;
        }
        const uint64_t Kq = qsched ? budget(sched1) : K;
        if (cand.size() > Kq) {
            std::nth_element(cand.begin(), cand.begin() + Kq, cand.end());
            cand.resize(Kq);
        }
        std::vector<std::pair<float, uint32_t>> fin;
        for (const auto& c : cand) {
            if (mode == 1 && !sched1 && !pred(c.second)) continue;  // post-filter predicate (:1227-1236)
            const uint32_t id = ix.ids[c.second];
            fin.push_back({ref_l2(qv, data + (uint64_t)id * d, d), id});
        }
        std::sort(fin.begin(), fin.end());
        for (uint32_t j = 0; j < k; j++) {
            out_dist[qi * k + j] = j < std::min<size_t>(fin.size(), kq) ? fin[j].first : INFINITY;
            out_ids[qi * k + j] = j < std::min<size_t>(fin.size(), kq) ? fin[j].second : ~0ull;
        }
    }
    return 0;
}

int ora_query(void* h, const float* queries, uint64_t q, const float* qlabels, uint32_t label_cols,
              const float* data, uint32_t k, float* out_dist, uint64_t* out_ids, OraTrace* tr, int threads,
              int adc_mode) {
    return ora_query_ex(h, queries, q, qlabels, label_cols, data, k, nullptr, nullptr, nullptr, out_dist, out_ids,
                        tr, threads, adc_mode);
}

}  // extern "C"
