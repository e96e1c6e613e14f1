/*
 * hdgrid.h -- C ABI of the B200-native HDGrid ("super-grid") filtered ANN index.
 *
 * Every entry point is plain C: opaque handles, raw pointers, sizes and a status code.
 * Pointers named d_* are DEVICE pointers owned by the caller (the index never frees
 * them).  Streams are passed as `void*` holding a cudaStream_t (NULL = legacy stream).
 *
 * Reference interfaces replaced (paths inside the HDGrid project):
 *   hdg_create*      config_factory::create + index_factory::create
 *                    (src/index/index-factory.cuh:10-87), HDGrid.conf reader
 *                    (src/utils/config_utils.h:33-88), filter.conf reader (:121-172)
 *   hdg_build        super_grid::index::build (src/index/2-level_index/Super-Grid-IVF_PQ.cu:420-646)
 *                    through index_base_t::build (src/core/interfaces.cuh:30)
 *   hdg_query        super_grid::index::query (Super-Grid-IVF_PQ.cu:985-1249)
 *                    through index_base_t::query (src/core/interfaces.cuh:31)
 *   hdg_pq_lut       build_pq_lut_kernel (src/index/product-quantization.cu:4-35)
 *   hdg_pq_adc       compute_batched_L2_distance_kernel (product-quantization.cu:37-77)
 *   hdg_label_mask   label_matrix_by_filter_indices_kernel (src/core/filter.cu:30-64)
 *   hdg_recover_filters  recovery_filters / denormalize_labels_kernel (src/core/preprocessing.cu:3-32,206-230)
 *   hdg_bruteforce_knn   brute_forece_vector_search (src/verification/ground_truth.cuh:165-232),
 *                    generalised to the filter.conf predicate
 *   hdg_save/hdg_load    no counterpart: the reference rebuilds the index every run
 *                    (src/search-engine/search-engine-auto-batch.cu:266-274)
 */
#ifndef HDGRID_H_
#define HDGRID_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference exits the process on any CUDA error
 * (src/utils/debugging_utils.cuh:11-20); every entry point here returns instead. */
typedef enum hdg_status {
    HDG_OK = 0,
    HDG_ERR_INVALID_ARG = 1,
    HDG_ERR_IO = 2,
    HDG_ERR_CUDA = 3,
    HDG_ERR_OOM = 4,
    HDG_ERR_TIMEOUT = 5,
    HDG_ERR_UNSUPPORTED = 6,
    HDG_ERR_STATE = 7
} hdg_status;

typedef struct hdg_index hdg_index;

#define HDG_MAX_LABEL_DIMS 8

/* Index and search parameters: the union of the HDGrid.conf keys read by
 * common_config (config_utils.h:97-108), pq::config_t (product-quantization.cuh:33-35)
 * and super_grid::config_t (Super-Grid-IVF_PQ.cuh:47-54), plus the B200 precision switches. */
typedef struct hdg_params {
    uint64_t topk;          /* TOPK */
    uint64_t filter_dim;    /* FILTER_DIM: label columns per label dim in the query labels (1 or 2) */
    uint64_t pq_dim;        /* PQ_DIM: number of PQ subspaces M */
    uint64_t n_clusters;    /* N_CLUSTERS: PQ codebook size (only 256 is supported) */
    uint64_t exps0;         /* EXPS0: refine ratio; <=1 selects the pre-filter schedule */
    uint64_t clusters;      /* CLUSTERS: coarse clusters C */
    uint64_t sub_clusters;  /* SUB_CLUSTERS: inverted lists per cluster S (C*S lists in total) */
    uint64_t max_grids;     /* MAX_GRIDS: label-grid cell budget */
    uint64_t n_list;        /* N_LIST: coarse clusters probed per query */
    uint64_t sub_lists;     /* SUB_LISTS: inverted lists probed per query */
    uint64_t n_split;       /* N_SPLIT: Morton sub-ranges per probed list when is_split=1 */
    uint64_t label_mask;    /* LABEL_MASK: bit i set = label dim i left out of the grid */
    uint64_t is_split;      /* IS_SPLIT */
    uint64_t break_down;    /* BREAK_DOWN: per-stage timing log */
    uint64_t enable_multi_gpu, mem_bound, is_calc_mem_predictor_coeff, lowest_query_batch;
    uint64_t data_width, index_width;  /* accepted and ignored, as in the reference */
    char path[512];         /* PATH: dataset directory */
    /* B200 precision / schedule switches (not HDGrid.conf keys of the reference; the
     * conf reader accepts them under the same names in upper case). */
    uint64_t lut_fp16;      /* LUT_FP16: store the PQ LUT in FP16 (FP32 accumulation) */
    uint64_t coarse_bf16;   /* COARSE_BF16: coarse assignment as a BF16 tensor-core GEMM */
    uint64_t kmeans_iters;  /* KMEANS_ITERS: Lloyd iterations of the index build (default 20) */
    uint64_t seed;          /* SEED: build RNG seed (default 1234) */
    uint64_t scan_cpt;      /* SCAN_CPT: ADC scan candidates per thread (1, 2 or 4; 0 = default) */
    uint64_t scan_chunk;    /* SCAN_CHUNK: candidates per scan work item (power of two in
                             * [4096, 262144]; 0 = 32768) -- the list/query split of the scan */
    uint64_t query_graph;   /* QUERY_GRAPH: 1 = hdg_query replays a captured CUDA graph per
                             * (pointers, q, k); status of a replay via hdg_query_status */
    uint64_t learned;       /* LEARNED: 1 = per-query lists to probe and predicate-first flag
                             * from the index's trained MLP (hdg_mlp_*); 0 = plain schedule */
    uint64_t prefix_rows;   /* PREFIX_ROWS: per-list prefix counts as compressed rows (the
                             * reference's compress_HOPS_data form): 1 = always, 2 = never (dense
                             * cells x lists array), 0 = rows when the dense array would pass 2 GiB */
} hdg_params;

/* filter.conf contents (config_utils.h:112-172).  interval_map is the flat
 * concatenation of every map filter's table, exactly as the reference uploads it
 * (preprocessing.cu:145-150). */
typedef struct hdg_filter_spec {
    int32_t l;
    int32_t type[HDG_MAX_LABEL_DIMS];
    float shift_val[2 * HDG_MAX_LABEL_DIMS];
    int32_t div_value[HDG_MAX_LABEL_DIMS];
    int32_t n_map;
    const float* interval_map; /* host pointer, n_map floats; copied by the callee */
} hdg_filter_spec;

/* ---- lifetime ---------------------------------------------------------------- */

/* algorithm: "super-grid" (case-insensitive, so the README's "Super-Grid" works too).
 * Other algorithm names of the reference return HDG_ERR_UNSUPPORTED. */
hdg_status hdg_create(const char* algorithm, const char* hdgrid_conf_path,
                      const char* filter_conf_path, hdg_index** out);
/* Same, with the two files' contents passed as strings. */
hdg_status hdg_create_from_text(const char* algorithm, const char* hdgrid_conf_text,
                                const char* filter_conf_text, hdg_index** out);
hdg_status hdg_destroy(hdg_index* index);

/* Parse an HDGrid.conf / filter.conf text without creating an index. */
hdg_status hdg_parse_config(const char* hdgrid_conf_text, hdg_params* out);
/* interval_map of *out points into storage owned by the library until the next call. */
hdg_status hdg_parse_filter(const char* filter_conf_text, hdg_filter_spec* out);
hdg_status hdg_get_params(const hdg_index* index, hdg_params* out);
/* Change a search-time key of a built index without rebuilding (no counterpart in the
 * reference, whose parameters are fixed per run): N_LIST, SUB_LISTS, EXPS0, TOPK,
 * BREAK_DOWN, IS_SPLIT, N_SPLIT, LUT_FP16, COARSE_BF16 (case-insensitive).  Build-time keys
 * return HDG_ERR_INVALID_ARG. */
hdg_status hdg_set_param(hdg_index* index, const char* key, uint64_t value);

/* ---- build / query --------------------------------------------------------------- */

/* d_data [n x d] f32 row-major, d_labels [n x l] f32 row-major (l = filter.conf's l). */
hdg_status hdg_build(hdg_index* index, const float* d_data, uint64_t n, uint32_t d,
                     const float* d_labels, uint32_t l, void* stream);

/* Pre-size the query workspace of calls on the NULL stream for batches of up to
 * max_queries, so that later hdg_query calls on such batches allocate nothing (calls on
 * another stream size their own workspace on their first call).  Queries on different
 * streams use different workspaces and may run concurrently from different host threads;
 * calls on one stream run one after another. */
hdg_status hdg_reserve(hdg_index* index, uint64_t max_queries);

/* d_queries [q x d] f32; d_query_labels [q x label_cols] f32 with label_cols = l*filter_dim;
 * d_data is the base set [n x d] (used by the exact re-rank, as query_input_t::dataset).
 * Outputs d_dist [q x k] f32 (ascending) and d_ids [q x k] u64.  Slots without a
 * result hold id UINT64_MAX and distance +inf. */
hdg_status hdg_query(hdg_index* index, const float* d_queries, uint64_t q,
                     const float* d_query_labels, uint32_t label_cols, const float* d_data,
                     uint32_t k, float* d_dist, uint64_t* d_ids, void* stream);

/* hdg_query with per-query parameters, each an optional device array of q entries (NULL =
 * the uniform value).  No reference counterpart: super_grid::index::query
 * (Super-Grid-IVF_PQ.cu:985-1249) takes one k and one probe count for the whole batch.
 *   d_k        result count of each query, clamped to [1, k_max]; rows keep stride k_max and
 *              the slots past a query's k hold id UINT64_MAX and distance +inf.  The candidate
 *              budgets are those of a k_max batch (the reference has one topk per batch, so a
 *              mixed-k batch is a k_max batch whose rows are cut to each query's k);
 *   d_nprobe   sub-lists probed per query, clamped to [1, sub_lists];
 *   d_schedule 0 = the index's schedule (Super-Grid-IVF_PQ.cu:1151-1241), 1 = predicate-first
 *              scan (label test fused into the ADC pass) with a budget of exps0*k_max and an
 *              exact re-rank -- the schedule of the reference's batch-split branch
 *              (:1165-1171); needs exps0 > 1. */
hdg_status hdg_query_ex(hdg_index* index, const float* d_queries, uint64_t q,
                        const float* d_query_labels, uint32_t label_cols, const float* d_data,
                        uint32_t k_max, const uint32_t* d_k, const uint32_t* d_nprobe,
                        const uint8_t* d_schedule, float* d_dist, uint64_t* d_ids, void* stream);

/* ---- learned per-query schedule (no reference counterpart) ------------------------------
 * A BF16 MLP, 48 features -> 128 -> 128 -> 2 (ReLU), whose outputs are z0 = log2(lists to
 * probe) and z1 = logit of the predicate-first flag.  With LEARNED=1 and a model loaded,
 * hdg_query / hdg_query_ex (without their own n_probe / schedule arrays) take each query's
 * probe count round(2^z0) clamped to [1, sub_lists] and schedule (z1 > 0) from it; it
 * replaces the batch-wide n_list / sub_lists of super_grid::index::query
 * (Super-Grid-IVF_PQ.cu:1034-1042, 849-901) per query.  Weights are one f32 vector:
 * W1 [128 x 48], b1 [128], W2 [128 x 128], b2 [128], W3 [2 x 128], b3 [2]. */

/* The 48 features of each query ([q x 48] f32 device output); d_k may be NULL (k_max). */
hdg_status hdg_query_features(hdg_index* index, const float* d_queries, uint64_t q,
                              const float* d_query_labels, uint32_t label_cols, const uint32_t* d_k,
                              uint32_t k_max, float* d_features, void* stream);
uint64_t hdg_mlp_param_count(void);
hdg_status hdg_mlp_init(hdg_index* index, uint64_t seed);  /* He-uniform weights, zero biases */
hdg_status hdg_mlp_set_weights(hdg_index* index, const float* host, uint64_t count);
hdg_status hdg_mlp_get_weights(hdg_index* index, float* host, uint64_t count);
/* d_z [n x 2] = network outputs for d_x [n x 48] (device pointers). */
hdg_status hdg_mlp_forward(hdg_index* index, const float* d_x, uint64_t n, float* d_z, void* stream);
/* Gradient of the mean loss (z0 - y0)^2 + BCE(sigmoid(z1), y1) over the n rows, w.r.t. all
 * parameters, into d_grad [hdg_mlp_param_count()] (device); loss (may be NULL) gets the loss. */
hdg_status hdg_mlp_gradients(hdg_index* index, const float* d_x, const float* d_y, uint64_t n,
                             float* d_grad, double* loss, void* stream);
/* Adam (beta 0.9 / 0.999) over shuffled mini-batches of the n rows for the given epochs;
 * final_loss (may be NULL) gets the last epoch's mean batch loss. */
hdg_status hdg_mlp_train(hdg_index* index, const float* d_x, const float* d_y, uint64_t n,
                         uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                         double* final_loss, void* stream);

/* Scalars of the last hdg_query: out[0] queries, [1] candidate budget n_cand as the
 * reference computes it (Super-Grid-IVF_PQ.cu:1222), [2] budget used (the same value: no
 * cap), [3] sum of Morton candidate-range sizes, [4] sum of exact filtered counts of the
 * probed lists, [5] largest per-query candidate count, [6] beta as float bits, [7] schedule
 * (0 pre-filter, 1 post-filter, 2 single label dim), [8] kernels launched, [9] queries
 * dropped by a captured graph's buffer capacity.  Returns entries written (<= 10). */
int hdg_last_query_stats(hdg_index* index, uint64_t* out, int cap);

/* With QUERY_GRAPH=1 hdg_query returns once the captured graph is enqueued; this waits for
 * the last replay and returns its device status: HDG_OK, HDG_ERR_TIMEOUT (a tensor-core
 * wait of the coarse GEMM expired) or HDG_ERR_OOM (the batch had more candidates than the
 * distance buffer sized at capture -- 1.25x the first batch of the shape -- and the
 * queries past it returned no results).  HDG_OK when no replay is pending.  No reference
 * counterpart: the reference synchronises after every stage. */
hdg_status hdg_query_status(hdg_index* index);

/* The project autotuner: runs the batch through the plain path once per scan variant --
 * threads x candidates-per-thread (SCAN_CPT 1, 2, 4) and work-item size (SCAN_CHUNK 8192 ..
 * 65536 candidates, the split of the scan between lists and queries) -- and keeps the
 * fastest scan in the index's parameters.  Outputs as hdg_query; best_scan_ms (may be
 * NULL) receives the chosen variant's scan time.  Replaces the reference's memory
 * predictor (search-engine/search-engine-auto-batch.cu:178-190, 381-430, 431-490), which
 * picks batch sizes instead. */
hdg_status hdg_autotune(hdg_index* index, const float* d_queries, uint64_t q,
                        const float* d_query_labels, uint32_t label_cols, const float* d_data,
                        uint32_t k, float* d_dist, uint64_t* d_ids, void* stream,
                        float* best_scan_ms);

/* Per-stage device timings (ms) of the last hdg_query when break_down=1; returns the
 * number of stages written (<= cap) and their names via names (may be NULL). */
int hdg_last_stage_times(const hdg_index* index, float* ms, const char** names, int cap);

/* Copy a named intermediate buffer of the last query to host memory (parity tests).
 * Names: "box", "cells", "zrange", "list_counts", "cluster_counts", "probe_clusters",
 * "probe_lists", "range_start", "range_len", "cand_count", "budget", "sel_off", "scalars",
 * "qoff", "qstat", "labels_read" (candidates of the predicate pass whose labels were read),
 * "ranks_read" (candidates of the predicate pass whose packed label ranks were read),
 * "rank_box" (per query: the label-rank box and its inner box, four words), "refine_rows"
 * (rows the re-rank computed exactly), "refine_labels_read" (selected entries whose labels
 * the re-rank read), "distances" (the f32 ADC distance of every scanned candidate, query rows
 * at the "qoff" offsets) and "cand_pool" (each query's selected candidates, rows at the
 * "sel_off" offsets, "cand_count" of them; a predicate-first query whose budget takes all its
 * survivors keeps them, as pool rows, in its "distances" row instead). */
hdg_status hdg_debug_fetch(const hdg_index* index, const char* name, void* host_dst,
                           size_t bytes, size_t* bytes_needed);

/* Index geometry: n_lists, C, M, l, grid dims, Morton bits, ... (host copy). */
typedef struct hdg_index_info {
    uint64_t n, d, l, M, M_pad, n_lists, clusters;
    uint64_t tot_cells;
    int32_t grid_dims[HDG_MAX_LABEL_DIMS];
    int32_t shuffle[HDG_MAX_LABEL_DIMS];
    uint64_t label_left[HDG_MAX_LABEL_DIMS];
    uint64_t label_span[HDG_MAX_LABEL_DIMS];
    int32_t morton_dims, morton_max_bits, morton_valid_map, diff_dim;
    uint64_t device_bytes;
    uint64_t prefix_entries;  /* change points of the compressed prefix rows; 0 = dense form */
    uint64_t rank_pack_bytes; /* bytes per point of the packed label ranks that the predicate pass
                               * reads before the labels (4; 0 = not kept) */
    uint64_t rank_bits;       /* bits per label dim of a packed rank (2^bits - 1 thresholds at most) */
} hdg_index_info;
hdg_status hdg_get_info(const hdg_index* index, hdg_index_info* out);

/* ---- persistence ------------------------------------------------------------------ */

hdg_status hdg_save(const hdg_index* index, const char* path);
hdg_status hdg_load(const char* path, hdg_index** out);

/* ---- kernel-level entry points (the reference's kernels, same data layouts) -------- */

/* LUT[q][m][c] = sum_t (centers[m][c][t] - queries[q][m*pq_len+t])^2 ; f32. */
hdg_status hdg_pq_lut(const float* d_centers, const float* d_queries, uint64_t n_queries,
                      uint32_t n_dim, uint32_t pq_dim, uint32_t pq_len, uint32_t n_codes,
                      float* d_lut, void* stream);
/* dist[q][j] = sum_m lut[q][m][codebook[m*tot_data + idx]], idx = indices[q*n_cand+j]
 * (or j when d_indices is NULL); idx >= tot_data gives FLT_MAX.  Column-major codes. */
hdg_status hdg_pq_adc(const uint8_t* d_codebook, uint64_t tot_data, const float* d_lut,
                      uint64_t n_queries, uint32_t pq_dim, uint32_t n_codes,
                      const uint64_t* d_indices, uint64_t n_cand, float* d_dist, void* stream);
/* mask[q][j] = AND_i (ranges[q][2i] <= labels[idx][i] <= ranges[q][2i+1]); idx >= n_data gives 0. */
hdg_status hdg_label_mask(const float* d_ranges, const float* d_labels, uint32_t l,
                          uint64_t n_data, uint64_t n_queries, const uint64_t* d_indices,
                          uint64_t n_cand, int32_t* d_mask, void* stream);
/* filters [q x 2l] f32 from the query labels and a filter spec. */
hdg_status hdg_recover_filters(const hdg_filter_spec* spec, const float* d_query_labels,
                               uint64_t n_queries, float* d_ranges, void* stream);
/* out[r][c] = sum_k a[r][k] * b[c][k] for bf16 a [rows x d] and b [cols x d] (row-major,
 * d % 8 == 0), FP32 accumulation on the tcgen05 tensor cores; out has row stride ldo.
 * The query-by-centroid contraction of the coarse assignment (the dot products inside
 * ::refine, src/core/refine.cu:36-75, before its select_k).  Returns HDG_ERR_TIMEOUT if a
 * tensor-core wait expired. */
hdg_status hdg_bf16_gemm(const void* d_a, uint64_t rows, const void* d_b, uint64_t cols, uint32_t d,
                         float* d_out, uint64_t ldo, void* stream);

/* Allocation-free variant of hdg_recover_filters -- no counterpart in the reference.
 * For callers that must not allocate device memory while they run: a host application
 * whose own allocator owns the GPU's memory, or a serving loop that cannot afford the
 * device-wide synchronisation cudaMalloc / cudaFree may cause.  hdg_recover_filters keeps
 * a per-call device copy of the filter's interval-map table; this variant keeps it in a
 * fixed scratch array of HDG_NOALLOC_MAP_MAX floats inside the library (present on every
 * GPU that loads the library until the process exits) and allocates nothing.  The caller
 * still passes the labels and the output.  Maps longer than HDG_NOALLOC_MAP_MAX entries
 * return HDG_ERR_INVALID_ARG.  The first call on a device looks up the scratch array's
 * device address (make that device current, and make that first call before any stream
 * capture).  All calls share the one array: calls whose work overlaps on the GPU (other
 * streams, other threads) race on it and must be serialised by the caller.  The map is
 * copied from spec->interval_map on `stream` (stream-ordered): that host memory must stay
 * valid and unchanged until the call's stream work has completed.  The looked-up address
 * is kept per device ordinal for the life of the process; it does not survive a
 * cudaDeviceReset (or a primary-context reset) of that device. */
#define HDG_NOALLOC_MAP_MAX 65536
hdg_status hdg_recover_filters_noalloc(const hdg_filter_spec* spec, const float* d_query_labels,
                                       uint64_t n_queries, float* d_ranges, void* stream);

/* Exact filtered kNN in FP32: distances of every base vector whose labels pass the
 * per-query box d_ranges [q x 2l]; k smallest, ascending, ties by lower id. */
hdg_status hdg_bruteforce_knn(const float* d_data, uint64_t n, uint32_t d,
                              const float* d_labels, uint32_t l, const float* d_queries,
                              uint64_t q, const float* d_ranges, uint32_t k,
                              float* d_dist, uint64_t* d_ids, void* stream);

/* Merge of per-data-batch results, replacing merge_intermediate_result
 * (src/core/merge_res.cu:18-56): row r of d_dist / d_ids [q x (k * n_batches)] holds
 * n_batches blocks of k results, block b from an index built on base rows starting at
 * d_offsets[b] (device array); ids are shifted by that offset (UINT64_MAX stays invalid) and
 * the k smallest (distance, id) of the row are written ascending to d_out_dist / d_out_ids
 * [q x k].  k * n_batches <= 8192. */
hdg_status hdg_merge_topk(const float* d_dist, const uint64_t* d_ids, uint64_t q, uint32_t k,
                          uint32_t n_batches, const uint64_t* d_offsets, float* d_out_dist,
                          uint64_t* d_out_ids, void* stream);

/* ---- label ranks (no reference counterpart) -----------------------------------------------
 * The predicate pass and the re-rank test a point's packed label ranks before its labels: per
 * label dim, up to 2^bits - 1 ascending thresholds, a label's rank being the number of them at
 * or below it (bits = min(12, (32 - l) / l)).  The build derives them from the base set's
 * labels with this function.  labels: host [n x l] f32, row-major.  *bits receives the bits
 * per dim; with thr non-NULL, thr receives [l x (2^bits - 1)] thresholds (row i: the first
 * n_thr[i] entries, strictly ascending) -- the distinct values of a strided sample of at most
 * 262,144 rows when they fit, else the sample's quantiles -- and lab_min / lab_max each dim's
 * smallest and largest label over every row.  NaN labels are left out.  1 <= l <= 8. */
hdg_status hdg_label_ranks(const float* labels, uint64_t n, uint32_t l, uint32_t* bits, float* thr,
                           uint32_t* n_thr, float* lab_min, float* lab_max);

/* Thread-local message of the last failing call. */
const char* hdg_last_error(void);
const char* hdg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* HDGRID_H_ */
