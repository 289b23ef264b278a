/*
 * C ABI of libnsparse_b200.so: the nsparse Index API for foreign-function
 * callers (ctypes, cgo, JNI, N-API). Plain pointers and sizes only; no call
 * throws across the boundary. Every function returns an nsp_status_t; on
 * failure nsp_last_error() holds the message for the calling thread.
 *
 * Status codes map to the reference's exception types, which its SWIG layer
 * turns into Python exceptions (nsparse/python/swignsparse.swig:47-59):
 *   NSP_ERR_INVALID_ARGUMENT  std::invalid_argument -> ValueError
 *   NSP_ERR_OUT_OF_RANGE      std::out_of_range     -> IndexError
 *   NSP_ERR_NO_MEMORY         std::bad_alloc        -> MemoryError
 *   NSP_ERR_RUNTIME           std::runtime_error    -> RuntimeError
 *                             (CUDA failures included)
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the reference project).
 */
#ifndef NSPARSE_C_H
#define NSPARSE_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NSP_OK = 0,
    NSP_ERR_INVALID_ARGUMENT = 1,
    NSP_ERR_RUNTIME = 2,
    NSP_ERR_OUT_OF_RANGE = 3,
    NSP_ERR_NO_MEMORY = 4
} nsp_status_t;

typedef struct nsp_index nsp_index_t;           /* nsparse::Index* (owned) */
typedef struct nsp_id_selector nsp_id_selector_t; /* nsparse::IDSelector* (owned) */
typedef struct nsp_search_params nsp_search_params_t; /* nsparse::SearchParameters* (owned) */

/* Message of the calling thread's last failure ("" if none). */
const char* nsp_last_error(void);

/* ---- index lifecycle -------------------------------------------------- */

/* index_factory (nsparse/index_factory.h:16, index_factory.cpp:63-153).
 * Caller owns *out; release with nsp_index_free. */
nsp_status_t nsp_index_factory(int dim, const char* description, nsp_index_t** out);

/* delete Index* (SWIG %newobject ownership, swignsparse.swig:178-189). */
nsp_status_t nsp_index_free(nsp_index_t* index);

/* Index::add (nsparse/index.h:34-35): n rows of CSR, int32 indptr[n+1],
 * uint16 indices and float32 values of indptr[n] entries. */
nsp_status_t nsp_index_add(nsp_index_t* index, int32_t n, const int32_t* indptr,
                           const uint16_t* indices, const float* values);

/* Index::add_with_ids (nsparse/index.h:52-54; IDMapIndex, id_map_index.cpp:70-80). */
nsp_status_t nsp_index_add_with_ids(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                    const uint16_t* indices, const float* values,
                                    const int32_t* ids);

/* Extension with no counterpart in the reference (whose ids are 32 bits):
 * IDMapIndex::add_with_ids with 64-bit external ids. Other index types raise
 * as add_with_ids does. */
nsp_status_t nsp_index_add_with_ids64(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                      const uint16_t* indices, const float* values,
                                      const int64_t* ids);

/* Index::build (nsparse/index.h:36). SEISMIC indexes build on the GPU. */
nsp_status_t nsp_index_build(nsp_index_t* index);

/* Index::search (nsparse/index.h:37-40, index.cpp:32-49; SWIG search_c /
 * search_with_params, swignsparse.swig:149-163). distances/labels are
 * caller-owned n*k arrays, row-major, padded with (-1.0, -1). params may be
 * NULL. Host buffers; the copies to and from the GPU happen inside. */
nsp_status_t nsp_index_search(nsp_index_t* index, int32_t n, const int32_t* indptr,
                              const uint16_t* indices, const float* values, int k,
                              float* distances, int32_t* labels,
                              const nsp_search_params_t* params);

/* Extension with no counterpart in the reference: nsp_index_search with
 * 64-bit labels, for an IDMapIndex whose external ids need them (its
 * nsp_index_search raises NSP_ERR_INVALID_ARGUMENT once one does). Other
 * index types return their 32-bit labels widened. */
nsp_status_t nsp_index_search64(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                const uint16_t* indices, const float* values, int k,
                                float* distances, int64_t* labels,
                                const nsp_search_params_t* params);

/* Index::num_vectors (nsparse/index.h:45-48). */
nsp_status_t nsp_index_num_vectors(const nsp_index_t* index, int64_t* out);

/* Index::get_dimension (nsparse/index.h:43). */
nsp_status_t nsp_index_dimension(const nsp_index_t* index, int32_t* out);

/* Index::id (nsparse/index.h:33): four characters, not NUL-terminated. */
nsp_status_t nsp_index_fourcc(const nsp_index_t* index, char out[4]);

/* Index::read_csr (nsparse/index.h:56-58, index.cpp:63-142). residency:
 * 0 in-memory: the interchange CSR layout; 1 mmap: for a seismic index the
 * native layout (MmapIndex::read_csr, mmap_index.h:24-36, 72-131; the engine
 * copies it to the GPU), rejected by a quantized index
 * (seismic_scalar_quantized_index.cpp:149-157), the interchange layout for
 * the other index types. */
nsp_status_t nsp_index_read_csr(nsp_index_t* index, const char* path, int residency);

/* csr_layout::convert (nsparse/utils/csr_layout.h:62-65, csr_layout.cpp:69-156):
 * rewrites an interchange CSR file in the native layout. */
nsp_status_t nsp_csr_convert(const char* interchange_path, const char* native_path);

/* write_index / read_index (nsparse/io/index_io.h:29-32). io_flags: 1 =
 * kUseMmap (accepted). The file layout is the reference's. */
nsp_status_t nsp_write_index(nsp_index_t* index, const char* path);
nsp_status_t nsp_read_index(const char* path, int io_flags, nsp_index_t** out);

/* ---- id selectors (nsparse/id_selector.h:22-86) ------------------------ */

nsp_status_t nsp_id_selector_set_new(size_t n, const int32_t* ids, nsp_id_selector_t** out);
nsp_status_t nsp_id_selector_array_new(size_t n, const int32_t* ids, nsp_id_selector_t** out);
/* NotIDSelector borrows `inner`, which must outlive it (as in the reference). */
nsp_status_t nsp_id_selector_not_new(nsp_id_selector_t* inner, nsp_id_selector_t** out);
/* Extension with no counterpart in the reference: a ready-made membership
 * bitmap over ids [0, n_bits), bit d of word d/64; the bits are copied. */
nsp_status_t nsp_id_selector_bitmap_new(int64_t n_bits, const uint64_t* bits,
                                        nsp_id_selector_t** out);
/* Extension with no counterpart in the reference: a set of 64-bit ids (an
 * IDMapIndex's wide external ids). */
nsp_status_t nsp_id_selector_set64_new(size_t n, const int64_t* ids, nsp_id_selector_t** out);
nsp_status_t nsp_id_selector_is_member(const nsp_id_selector_t* sel, int32_t id, int* out);
nsp_status_t nsp_id_selector_free(nsp_id_selector_t* sel);

/* ---- search parameters ------------------------------------------------- */

/* SearchParameters (nsparse/index.h:21-28). */
nsp_status_t nsp_search_params_new(nsp_search_params_t** out);
/* SeismicSearchParameters(cut, heap_factor) (nsparse/seismic_index.h:26-32). */
nsp_status_t nsp_seismic_search_params_new(int cut, float heap_factor,
                                           nsp_search_params_t** out);
/* SeismicSQSearchParameters(vmin, vmax, cut, heap_factor)
 * (nsparse/seismic_scalar_quantized_index.h:27-33). */
nsp_status_t nsp_seismic_sq_search_params_new(float vmin, float vmax, int cut,
                                              float heap_factor, nsp_search_params_t** out);
/* SearchParameters::set_id_selector (borrowed; NULL clears). */
nsp_status_t nsp_search_params_set_id_selector(nsp_search_params_t* params,
                                               nsp_id_selector_t* sel);
/* Extension: plain = 1 runs one kernel launch per query instead of one
 * batched launch; warps_per_block (1-32; the warp-per-query variants 0-1 use
 * at most 8) = 0 lets the engine choose. */
nsp_status_t nsp_search_params_set_engine(nsp_search_params_t* params, int plain,
                                          int warps_per_block);
/* Extension: SEISMIC kernel variant (-1 engine's choice, 0 one warp per query
 * with direct row loads, 1 the same with rows staged in shared memory by bulk
 * copy, 2-5 one CTA per query with 1, 2, 4 or 8 lanes per scored doc) and its
 * tuning value: variant 1's buffer size in bytes, variants 2-5's candidate
 * docs per batch (0 = default). Results do not depend on either. */
nsp_status_t nsp_search_params_set_kernel(nsp_search_params_t* params, int variant,
                                          int tuning);
/* Extension: CTAs per query of SEISMIC variants 2-5 (0 engine's choice, 1 one
 * CTA, 2/4/8 a thread-block cluster: the CTAs score each batch of the query's
 * candidates together, for lower latency per query). Results do not depend on
 * it. */
nsp_status_t nsp_search_params_set_split(nsp_search_params_t* params, int ctas_per_query);
/* Extension: count_unique != 0 makes a batched SEISMIC search (kernel variants
 * 2-5) a counting pass: slower, same results, and its stats also count each
 * scored doc's row once per query, as the reference's visited set does
 * (nsp_search_stats_t.unique_*). */
nsp_status_t nsp_search_params_set_count_unique(nsp_search_params_t* params, int count_unique);
nsp_status_t nsp_search_params_free(nsp_search_params_t* params);

/* ---- engine extensions -------------------------------------------------- */

typedef struct {
    uint64_t docs_scored;
    uint64_t blocks_visited;
    uint64_t bytes;        /* algorithmic bytes the search kernels read */
    uint64_t lists_probed;
    float kernel_ms;       /* device time of the search kernels */
    int32_t launches;
    uint64_t row_bytes;    /* the rows' share of `bytes` (rows as often as scored) */
    uint64_t unique_docs;  /* counting pass only: docs counted once per query */
    uint64_t unique_row_bytes;  /* counting pass only: their rows' bytes */
} nsp_search_stats_t;

/* Counters of the calling thread's last nsp_index_search. */
nsp_status_t nsp_last_search_stats(nsp_search_stats_t* out);

/* SEISMIC search with queries and results already in device memory (no host
 * copies): d_indptr/d_indices/d_values describe n canonical query rows (terms
 * ascending and unique within a row), max_row_nnz bounds the row length.
 * d_distances/d_labels receive n*k results. Runs on `cuda_stream`
 * (cudaStream_t, NULL = the thread's engine stream) and returns once the work
 * is enqueued. Extension with no counterpart in the reference. */
nsp_status_t nsp_index_search_device(nsp_index_t* index, int32_t n, const int32_t* d_indptr,
                                     const uint16_t* d_indices, const float* d_values,
                                     int32_t max_row_nnz, int k, float* d_distances,
                                     int32_t* d_labels, const nsp_search_params_t* params,
                                     void* cuda_stream);

/* SEISMIC search that allocates nothing. No counterpart in the reference.
 *
 * For callers that cannot allocate device memory per call: an engine
 * embedded in a host whose allocator accounts for every device byte against
 * a fixed budget, or a latency-critical loop that cannot afford
 * cudaMalloc/cudaFree, which can synchronize the device. Same arguments,
 * kernel and results as nsp_index_search_device (the default one-CTA-per-query
 * kernel, the index's autotuned launch shape, the knobs of `params`), plus:
 *   - `nnz`: the number of query entries, d_indptr[n]. The call reads and
 *     (quantized index) encodes exactly nnz values; a row that ends past nnz
 *     is treated like a row longer than max_row_nnz (below).
 *   - `d_status` (device int32, may be NULL): set to 0 by the call and to 3
 *     by the kernel when a row is longer than max_row_nnz or ends past nnz;
 *     such rows return padding. Read it after synchronizing the stream.
 * The search's scratch (work counter, counters, encoded query codes,
 * block-score rows, visiting orders) lives in a fixed device array of
 * NSP_NOALLOC_SCRATCH_BYTES that every GPU loading the library reserves until
 * exit; no cudaMalloc, cudaFree or allocating library routine is called. The
 * grid is capped to the CTAs whose scratch fits the array.
 *   - `cuda_stream` NULL is the legacy default stream.
 *   - The first call on a device looks up that array's device address (set-up
 *     once per device); make that first call before any stream capture.
 *   - The index must already be resident on the GPU (one ordinary search or a
 *     build followed by a search does that); otherwise the call is rejected.
 *   - Rejected with NSP_ERR_INVALID_ARGUMENT: an id selector, plain mode, or a
 *     batch whose codes (2*nnz bytes) or the block-score rows of one CTA (4
 *     bytes per block of the largest posting list, per warp) do not fit the
 *     array.
 *   - All calls share the array and it keeps the last call's contents: calls
 *     that overlap on the GPU (other streams, other host threads) race; order
 *     them on one stream. */
#define NSP_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
nsp_status_t nsp_index_search_device_noalloc(nsp_index_t* index, int32_t n,
                                             const int32_t* d_indptr, const uint16_t* d_indices,
                                             const float* d_values, int32_t nnz,
                                             int32_t max_row_nnz, int k, float* d_distances,
                                             int32_t* d_labels, const nsp_search_params_t* params,
                                             void* cuda_stream, int32_t* d_status);

/* Kernel autotuner. Times each one-CTA-per-query launch shape of the SEISMIC
 * search (lanes per doc, candidate docs per batch, warps per CTA) on the n
 * sample queries with the given parameters, then the CTAs per query (1, 2, 4,
 * 8) of one-query launches on up to 16 of them searched alone, and keeps the
 * fastest for this index: later searches whose parameters leave the kernel to
 * the engine (variant -1) use it. Results do not depend on the choice. Writes
 * the choice to the out pointers (any may be NULL). Extension with no
 * counterpart in the reference. */
nsp_status_t nsp_index_autotune(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                const uint16_t* indices, const float* values, int k,
                                const nsp_search_params_t* params, int* variant, int* batch_docs,
                                int* warps_per_block, float* kernel_ms, int* ctas_per_query);

/* ---- CUDA-graph search steps (extension with no counterpart in the
 * reference; each step returns what nsp_index_search_device returns for the
 * same rows) -------------------------------------------------------------
 *
 * A batched SEISMIC search step of `n` query rows, captured once as a CUDA
 * graph and replayed per batch: the counter resets, the query encode of a
 * quantized index and the persistent search kernel become one graph launch,
 * with the kernel's scratch owned by the graph (no allocation per step).
 * Parameters (k, cut, heap factor, kernel, an id selector's doc set) are
 * fixed at capture; `nnz_cap` bounds the query entries of a step and
 * `max_row_nnz` one row's. The index must stay alive and unchanged: after an
 * add, build or read the step is refused (NSP_ERR_RUNTIME); capture anew.
 * IDMapIndex and selectors with at most k ids (the exact-match path) are
 * rejected. One step of a graph is in flight at a time. */
typedef struct nsp_search_graph nsp_search_graph_t;
/* Device buffers of a step: n+1 row offsets, nnz_cap terms and values
 * (rows canonical: terms ascending and unique), n*k results. */
typedef struct {
    int32_t* indptr;
    uint16_t* indices;
    float* values;
    float* distances;
    int32_t* labels;
} nsp_graph_buffers_t;
/* `device_buffers`: the caller's buffers (kept alive by the caller), or NULL
 * for buffers the graph allocates (all rows empty until written). */
nsp_status_t nsp_search_graph_new(nsp_index_t* index, int32_t n, int32_t nnz_cap,
                                  int32_t max_row_nnz, int k, const nsp_search_params_t* params,
                                  const nsp_graph_buffers_t* device_buffers,
                                  nsp_search_graph_t** out);
nsp_status_t nsp_search_graph_free(nsp_search_graph_t* graph);
nsp_status_t nsp_search_graph_buffers(const nsp_search_graph_t* graph, nsp_graph_buffers_t* out);
/* Replays the step on `cuda_stream` (NULL = the graph's own stream), after
 * the work queued there (e.g. the copies that wrote the rows); returns. */
nsp_status_t nsp_search_graph_launch(nsp_search_graph_t* graph, void* cuda_stream);
/* Waits for `cuda_stream` (NULL = the graph's own stream); reports a kernel
 * error of the step and makes its counters the thread's last search stats. */
nsp_status_t nsp_search_graph_sync(nsp_search_graph_t* graph, void* cuda_stream);
/* Host rows in, host results out (n <= the graph's rows; rows in any order
 * of terms, as nsp_index_search takes them): copies through pinned staging,
 * one graph launch, waits. */
nsp_status_t nsp_search_graph_search(nsp_search_graph_t* graph, int32_t n, const int32_t* indptr,
                                     const uint16_t* indices, const float* values,
                                     float* distances, int32_t* labels);

/* ---- serving loop (extension with no counterpart in the reference) ------
 * Single-query requests, each with its own k and an optional doc filter, are
 * batched continuously: `slots` worker threads (one CUDA stream each) take
 * whatever requests are waiting when they are free -- those sharing the
 * oldest request's k, cut and heap factor, up to max_batch, within the
 * scratch budget -- and run them as one launch, so batches overlap on the GPU.
 * A request's result equals a search of that query alone. The index (a
 * seismic index, or an IDMapIndex over one) must outlive the server and stay
 * unchanged while it runs. */
typedef struct nsp_server nsp_server_t;
typedef struct {
    int32_t max_batch;             /* queries per launch (0: 4096) */
    int32_t slots;                 /* launches in flight (0: 3) */
    int64_t scratch_budget_bytes;  /* request bytes in flight (0: 256 MiB) */
} nsp_server_config_t;
nsp_status_t nsp_server_new(nsp_index_t* index, const nsp_server_config_t* config,
                            nsp_server_t** out);
nsp_status_t nsp_server_free(nsp_server_t* server);
/* A doc filter: bitmap over internal doc ids (bit d of word d/64), at least
 * (n_docs + 64) / 64 words, copied to the device once. */
nsp_status_t nsp_server_add_filter(nsp_server_t* server, const uint64_t* bits, int64_t words,
                                   int32_t* filter_id);
/* 64-bit labels: result labels become ids[internal doc id]. */
nsp_status_t nsp_server_set_external_ids(nsp_server_t* server, const int64_t* ids, int64_t n);
/* filter_id -1: no filter. */
nsp_status_t nsp_server_submit(nsp_server_t* server, int32_t nnz, const uint16_t* terms,
                               const float* values, int k, int cut, float heap_factor,
                               int32_t filter_id, int64_t* ticket);
/* Blocks until the request is done; writes k results and the latency. */
nsp_status_t nsp_server_wait(nsp_server_t* server, int64_t ticket, float* distances,
                             int64_t* labels, double* latency_us);
/* Trace replay: request i (row i of the CSR batch, k_per[i], filter_per[i]
 * or none when filter_per is NULL) is submitted arrival_us[i] microseconds
 * after the call starts; returns when all are done, with k_stride results
 * per request (padded with -1.0 / -1) and each latency from its scheduled
 * arrival to its completion. */
nsp_status_t nsp_server_replay(nsp_server_t* server, int32_t n, const int32_t* indptr,
                               const uint16_t* indices, const float* values, const int32_t* k_per,
                               const int32_t* filter_per, const double* arrival_us, int cut,
                               float heap_factor, int k_stride, float* distances, int64_t* labels,
                               double* latency_us);
/* batches, requests, largest batch, most request bytes in flight. */
nsp_status_t nsp_server_stats(nsp_server_t* server, int64_t* out4);

/* Number of CUDA devices visible and the name of the current one. */
nsp_status_t nsp_device_info(int32_t* n_devices, char* name, size_t name_len);

#ifdef __cplusplus
}
#endif

#endif /* NSPARSE_C_H */
