// C ABI over the nsparse C++ API (include/nsparse_c.h). Exceptions are caught
// here and mapped to status codes; the message is kept per thread.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>

#include "engine.h"
#include "index_state.h"
#include "serve.h"
#include "nsparse/brutal_index.h"
#include "nsparse/id_map_index.h"
#include "nsparse/index_factory.h"
#include "nsparse/inverted_index.h"
#include "nsparse/io/index_io.h"
#include "nsparse/seismic_index.h"
#include "nsparse/seismic_scalar_quantized_index.h"
#include "nsparse/utils/csr_layout.h"
#include "nsparse_c.h"

using namespace nsparse;

namespace {

thread_local std::string g_error;

template <class F>
nsp_status_t guarded(F&& f) {
    try {
        g_error.clear();
        f();
        return NSP_OK;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        return NSP_ERR_INVALID_ARGUMENT;
    } catch (const std::out_of_range& e) {
        g_error = e.what();
        return NSP_ERR_OUT_OF_RANGE;
    } catch (const std::bad_alloc& e) {
        g_error = e.what();
        return NSP_ERR_NO_MEMORY;
    } catch (const std::exception& e) {
        g_error = e.what();
        return NSP_ERR_RUNTIME;
    } catch (...) {
        g_error = "unknown error";
        return NSP_ERR_RUNTIME;
    }
}

Index* as_index(nsp_index_t* p) {
    if (p == nullptr) throw std::invalid_argument("unexpected nullptr");
    return reinterpret_cast<Index*>(p);
}
const Index* as_index(const nsp_index_t* p) {
    if (p == nullptr) throw std::invalid_argument("unexpected nullptr");
    return reinterpret_cast<const Index*>(p);
}
IDSelector* as_sel(nsp_id_selector_t* p) { return reinterpret_cast<IDSelector*>(p); }
SearchParameters* as_params(const nsp_search_params_t* p) {
    return reinterpret_cast<SearchParameters*>(const_cast<nsp_search_params_t*>(p));
}
template <class T>
void check_out(T** out) {
    if (out == nullptr) throw std::invalid_argument("unexpected nullptr");
}

}  // namespace

namespace nsp {
// Lets entry points defined in other files report through nsp_last_error.
void set_last_error(const char* msg) { g_error = msg; }
}  // namespace nsp

extern "C" {

const char* nsp_last_error(void) { return g_error.c_str(); }

nsp_status_t nsp_index_factory(int dim, const char* description, nsp_index_t** out) {
    return guarded([&] {
        check_out(out);
        *out = reinterpret_cast<nsp_index_t*>(index_factory(dim, description));
    });
}

nsp_status_t nsp_index_free(nsp_index_t* index) {
    return guarded([&] { delete reinterpret_cast<Index*>(index); });
}

nsp_status_t nsp_index_add(nsp_index_t* index, int32_t n, const int32_t* indptr,
                           const uint16_t* indices, const float* values) {
    return guarded([&] { as_index(index)->add(n, indptr, indices, values); });
}

nsp_status_t nsp_index_add_with_ids(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                    const uint16_t* indices, const float* values,
                                    const int32_t* ids) {
    return guarded([&] { as_index(index)->add_with_ids(n, indptr, indices, values, ids); });
}

nsp_status_t nsp_index_add_with_ids64(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                      const uint16_t* indices, const float* values,
                                      const int64_t* ids) {
    return guarded([&] {
        Index* idx = as_index(index);
        if (auto* m = dynamic_cast<IDMapIndex*>(idx)) {
            m->add_with_ids64(n, indptr, indices, values, ids);
            return;
        }
        // the base's behaviour for an index without an id map
        if (n > 0 && ids == nullptr) throw std::invalid_argument("unexpected nullptr");
        std::vector<idx_t> narrow(ids, ids + (n > 0 ? n : 0));
        idx->add_with_ids(n, indptr, indices, values, narrow.data());
    });
}

nsp_status_t nsp_index_build(nsp_index_t* index) {
    return guarded([&] { as_index(index)->build(); });
}

nsp_status_t nsp_index_search(nsp_index_t* index, int32_t n, const int32_t* indptr,
                              const uint16_t* indices, const float* values, int k,
                              float* distances, int32_t* labels,
                              const nsp_search_params_t* params) {
    return guarded([&] {
        as_index(index)->search(n, indptr, indices, values, k, distances, labels,
                                as_params(params));
    });
}

nsp_status_t nsp_index_search64(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                const uint16_t* indices, const float* values, int k,
                                float* distances, int64_t* labels,
                                const nsp_search_params_t* params) {
    return guarded([&] {
        Index* idx = as_index(index);
        if (auto* m = dynamic_cast<IDMapIndex*>(idx)) {
            m->search64(n, indptr, indices, values, k, distances, labels, as_params(params));
            return;
        }
        if (labels == nullptr) throw std::invalid_argument("unexpected nullptr");
        std::vector<idx_t> narrow(n > 0 && k > 0 ? static_cast<size_t>(n) * k : 0);
        idx->search(n, indptr, indices, values, k, distances, narrow.empty() ? nullptr : narrow.data(),
                    as_params(params));
        for (size_t i = 0; i < narrow.size(); ++i) labels[i] = narrow[i];
    });
}

nsp_status_t nsp_index_num_vectors(const nsp_index_t* index, int64_t* out) {
    return guarded([&] {
        check_out(&out);
        *out = static_cast<int64_t>(as_index(index)->num_vectors());
    });
}

nsp_status_t nsp_index_dimension(const nsp_index_t* index, int32_t* out) {
    return guarded([&] {
        check_out(&out);
        *out = as_index(index)->get_dimension();
    });
}

nsp_status_t nsp_index_fourcc(const nsp_index_t* index, char out[4]) {
    return guarded([&] {
        if (out == nullptr) throw std::invalid_argument("unexpected nullptr");
        const auto id = as_index(index)->id();
        std::memcpy(out, id.data(), 4);
    });
}

nsp_status_t nsp_index_read_csr(nsp_index_t* index, const char* path, int residency) {
    return guarded([&] {
        as_index(index)->read_csr(path, residency == 1 ? Residency::kMmap : Residency::kInMemory);
    });
}

nsp_status_t nsp_csr_convert(const char* interchange_path, const char* native_path) {
    return guarded([&] {
        if (interchange_path == nullptr || native_path == nullptr)
            throw std::invalid_argument("unexpected nullptr");
        nsparse::csr_layout::convert(interchange_path, native_path);
    });
}

nsp_status_t nsp_write_index(nsp_index_t* index, const char* path) {
    return guarded([&] { write_index(as_index(index), path); });
}

nsp_status_t nsp_read_index(const char* path, int io_flags, nsp_index_t** out) {
    return guarded([&] {
        check_out(out);
        *out = reinterpret_cast<nsp_index_t*>(read_index(path, io_flags));
    });
}

nsp_status_t nsp_id_selector_set_new(size_t n, const int32_t* ids, nsp_id_selector_t** out) {
    return guarded([&] {
        check_out(out);
        if (n > 0 && ids == nullptr) throw std::invalid_argument("unexpected nullptr");
        *out = reinterpret_cast<nsp_id_selector_t*>(new SetIDSelector(n, ids));
    });
}

nsp_status_t nsp_id_selector_set64_new(size_t n, const int64_t* ids, nsp_id_selector_t** out) {
    return guarded([&] {
        check_out(out);
        if (n > 0 && ids == nullptr) throw std::invalid_argument("unexpected nullptr");
        *out = reinterpret_cast<nsp_id_selector_t*>(new SetIDSelector64(n, ids));
    });
}

nsp_status_t nsp_id_selector_array_new(size_t n, const int32_t* ids, nsp_id_selector_t** out) {
    return guarded([&] {
        check_out(out);
        if (n > 0 && ids == nullptr) throw std::invalid_argument("unexpected nullptr");
        *out = reinterpret_cast<nsp_id_selector_t*>(new ArrayIDSelector(n, ids));
    });
}

nsp_status_t nsp_id_selector_not_new(nsp_id_selector_t* inner, nsp_id_selector_t** out) {
    return guarded([&] {
        check_out(out);
        if (inner == nullptr) throw std::invalid_argument("unexpected nullptr");
        *out = reinterpret_cast<nsp_id_selector_t*>(new NotIDSelector(as_sel(inner)));
    });
}

nsp_status_t nsp_id_selector_bitmap_new(int64_t n_bits, const uint64_t* bits,
                                        nsp_id_selector_t** out) {
    return guarded([&] {
        check_out(out);
        *out = reinterpret_cast<nsp_id_selector_t*>(new BitmapIDSelector(n_bits, bits));
    });
}

nsp_status_t nsp_id_selector_is_member(const nsp_id_selector_t* sel, int32_t id, int* out) {
    return guarded([&] {
        if (sel == nullptr || out == nullptr) throw std::invalid_argument("unexpected nullptr");
        *out = reinterpret_cast<const IDSelector*>(sel)->is_member(id) ? 1 : 0;
    });
}

nsp_status_t nsp_id_selector_free(nsp_id_selector_t* sel) {
    return guarded([&] { delete as_sel(sel); });
}

nsp_status_t nsp_search_params_new(nsp_search_params_t** out) {
    return guarded([&] {
        check_out(out);
        *out = reinterpret_cast<nsp_search_params_t*>(new SearchParameters());
    });
}

nsp_status_t nsp_seismic_search_params_new(int cut, float heap_factor,
                                           nsp_search_params_t** out) {
    return guarded([&] {
        check_out(out);
        *out = reinterpret_cast<nsp_search_params_t*>(new SeismicSearchParameters(cut, heap_factor));
    });
}

nsp_status_t nsp_seismic_sq_search_params_new(float vmin, float vmax, int cut,
                                              float heap_factor, nsp_search_params_t** out) {
    return guarded([&] {
        check_out(out);
        *out = reinterpret_cast<nsp_search_params_t*>(
            new SeismicSQSearchParameters(vmin, vmax, cut, heap_factor));
    });
}

nsp_status_t nsp_search_params_set_id_selector(nsp_search_params_t* params,
                                               nsp_id_selector_t* sel) {
    return guarded([&] {
        if (params == nullptr) throw std::invalid_argument("unexpected nullptr");
        as_params(params)->set_id_selector(as_sel(sel));
    });
}

nsp_status_t nsp_search_params_set_engine(nsp_search_params_t* params, int plain,
                                          int warps_per_block) {
    return guarded([&] {
        if (params == nullptr) throw std::invalid_argument("unexpected nullptr");
        as_params(params)->engine.plain = plain != 0;
        if (warps_per_block < 0 || warps_per_block > 32)
            throw std::invalid_argument("warps_per_block must be in [0, 32]");
        as_params(params)->engine.warps_per_block = warps_per_block;
    });
}

nsp_status_t nsp_search_params_set_kernel(nsp_search_params_t* params, int variant,
                                          int tuning) {
    return guarded([&] {
        if (params == nullptr) throw std::invalid_argument("unexpected nullptr");
        if (variant < -1 || variant > 5) throw std::invalid_argument("variant must be in [-1, 5]");
        auto& e = as_params(params)->engine;
        e.variant = variant;
        e.stage_bytes = 0;
        e.batch_docs = 0;
        if (variant >= 2) {
            if (tuning < 0 || tuning > 8192)
                throw std::invalid_argument("batch_docs must be in [0, 8192]");
            e.batch_docs = tuning;
        } else {
            if (tuning < 0 || tuning > (96 << 10))
                throw std::invalid_argument("stage_bytes must be in [0, 98304]");
            e.stage_bytes = tuning;
        }
    });
}

nsp_status_t nsp_search_params_set_split(nsp_search_params_t* params, int ctas_per_query) {
    return guarded([&] {
        if (params == nullptr) throw std::invalid_argument("unexpected nullptr");
        if (ctas_per_query != 0 && ctas_per_query != 1 && ctas_per_query != 2 &&
            ctas_per_query != 4 && ctas_per_query != 8)
            throw std::invalid_argument("ctas_per_query must be 0, 1, 2, 4 or 8");
        as_params(params)->engine.ctas_per_query = ctas_per_query;
    });
}

nsp_status_t nsp_search_params_set_count_unique(nsp_search_params_t* params, int count_unique) {
    return guarded([&] {
        if (params == nullptr) throw std::invalid_argument("unexpected nullptr");
        as_params(params)->engine.count_unique = count_unique != 0;
    });
}

nsp_status_t nsp_search_params_free(nsp_search_params_t* params) {
    return guarded([&] { delete as_params(params); });
}

nsp_status_t nsp_last_search_stats(nsp_search_stats_t* out) {
    return guarded([&] {
        if (out == nullptr) throw std::invalid_argument("unexpected nullptr");
        const SearchStats& s = last_search_stats();
        out->docs_scored = s.docs_scored;
        out->blocks_visited = s.blocks_visited;
        out->bytes = s.bytes;
        out->lists_probed = s.lists_probed;
        out->kernel_ms = s.kernel_ms;
        out->launches = s.launches;
        out->row_bytes = s.row_bytes;
        out->unique_docs = s.unique_docs;
        out->unique_row_bytes = s.unique_row_bytes;
    });
}

nsp_status_t nsp_index_search_device(nsp_index_t* index, int32_t n, const int32_t* d_indptr,
                                     const uint16_t* d_indices, const float* d_values,
                                     int32_t max_row_nnz, int k, float* d_distances,
                                     int32_t* d_labels, const nsp_search_params_t* params,
                                     void* cuda_stream) {
    return guarded([&] {
        detail::search_device(as_index(index), n, d_indptr, d_indices, d_values, max_row_nnz, k,
                              d_distances, d_labels, as_params(params),
                              static_cast<cudaStream_t>(cuda_stream));
    });
}

nsp_status_t nsp_index_autotune(nsp_index_t* index, int32_t n, const int32_t* indptr,
                                const uint16_t* indices, const float* values, int k,
                                const nsp_search_params_t* params, int* variant, int* batch_docs,
                                int* warps_per_block, float* kernel_ms, int* ctas_per_query) {
    return guarded([&] {
        if (index == nullptr) throw std::invalid_argument("unexpected nullptr");
        const nsp::KernelChoice c = detail::seismic_autotune(
            as_index(index), n, indptr, indices, values, k, as_params(params));
        if (variant != nullptr) *variant = c.variant;
        if (batch_docs != nullptr) *batch_docs = c.batch_docs;
        if (warps_per_block != nullptr) *warps_per_block = c.warps_per_block;
        if (kernel_ms != nullptr) *kernel_ms = c.kernel_ms;
        if (ctas_per_query != nullptr) *ctas_per_query = c.split;
    });
}

struct nsp_search_graph {
    std::unique_ptr<nsparse::detail::IndexSearchGraph> g;
};

nsp_status_t nsp_search_graph_new(nsp_index_t* index, int32_t n, int32_t nnz_cap,
                                  int32_t max_row_nnz, int k, const nsp_search_params_t* params,
                                  const nsp_graph_buffers_t* device_buffers,
                                  nsp_search_graph_t** out) {
    return guarded([&] {
        if (index == nullptr || out == nullptr) throw std::invalid_argument("unexpected nullptr");
        nsp::GraphBuffers b;
        if (device_buffers != nullptr) {
            b.indptr = device_buffers->indptr;
            b.indices = device_buffers->indices;
            b.values = device_buffers->values;
            b.distances = device_buffers->distances;
            b.labels = device_buffers->labels;
        }
        auto h = std::make_unique<nsp_search_graph>();
        h->g = std::make_unique<detail::IndexSearchGraph>(as_index(index), n, nnz_cap,
                                                          max_row_nnz, k, as_params(params),
                                                          device_buffers != nullptr ? &b : nullptr);
        *out = h.release();
    });
}

nsp_status_t nsp_search_graph_free(nsp_search_graph_t* graph) {
    return guarded([&] { delete graph; });
}

nsp_status_t nsp_search_graph_buffers(const nsp_search_graph_t* graph, nsp_graph_buffers_t* out) {
    return guarded([&] {
        if (graph == nullptr || out == nullptr) throw std::invalid_argument("unexpected nullptr");
        const nsp::GraphBuffers& b = graph->g->buffers();
        out->indptr = b.indptr;
        out->indices = b.indices;
        out->values = b.values;
        out->distances = b.distances;
        out->labels = b.labels;
    });
}

nsp_status_t nsp_search_graph_launch(nsp_search_graph_t* graph, void* cuda_stream) {
    return guarded([&] {
        if (graph == nullptr) throw std::invalid_argument("unexpected nullptr");
        graph->g->launch(static_cast<cudaStream_t>(cuda_stream));
    });
}

nsp_status_t nsp_search_graph_sync(nsp_search_graph_t* graph, void* cuda_stream) {
    return guarded([&] {
        if (graph == nullptr) throw std::invalid_argument("unexpected nullptr");
        graph->g->sync(static_cast<cudaStream_t>(cuda_stream));
    });
}

nsp_status_t nsp_search_graph_search(nsp_search_graph_t* graph, int32_t n, const int32_t* indptr,
                                     const uint16_t* indices, const float* values,
                                     float* distances, int32_t* labels) {
    return guarded([&] {
        if (graph == nullptr) throw std::invalid_argument("unexpected nullptr");
        graph->g->search(n, indptr, indices, values, distances, labels);
    });
}

struct nsp_server {
    std::unique_ptr<nsparse::detail::Server> s;
};

namespace {
nsparse::detail::Server& as_server(nsp_server_t* p) {
    if (p == nullptr || !p->s) throw std::invalid_argument("unexpected nullptr");
    return *p->s;
}
}  // namespace

nsp_status_t nsp_server_new(nsp_index_t* index, const nsp_server_config_t* config,
                            nsp_server_t** out) {
    return guarded([&] {
        if (index == nullptr || out == nullptr) throw std::invalid_argument("unexpected nullptr");
        detail::ServerConfig c;
        if (config != nullptr) {
            if (config->max_batch < 0 || config->slots < 0 || config->scratch_budget_bytes < 0)
                throw std::invalid_argument("server limits must not be negative");
            if (config->max_batch > 0) c.max_batch = config->max_batch;
            if (config->slots > 0) c.slots = config->slots;
            if (config->scratch_budget_bytes > 0) c.scratch_budget = config->scratch_budget_bytes;
        }
        auto h = std::make_unique<nsp_server>();
        h->s = std::make_unique<detail::Server>(as_index(index), c);
        *out = h.release();
    });
}

nsp_status_t nsp_server_free(nsp_server_t* server) {
    return guarded([&] { delete server; });
}

nsp_status_t nsp_server_add_filter(nsp_server_t* server, const uint64_t* bits, int64_t words,
                                   int32_t* filter_id) {
    return guarded([&] {
        const int id = as_server(server).add_filter(bits, words);
        if (filter_id != nullptr) *filter_id = id;
    });
}

nsp_status_t nsp_server_set_external_ids(nsp_server_t* server, const int64_t* ids, int64_t n) {
    return guarded([&] { as_server(server).set_external_ids(ids, n); });
}

nsp_status_t nsp_server_submit(nsp_server_t* server, int32_t nnz, const uint16_t* terms,
                               const float* values, int k, int cut, float heap_factor,
                               int32_t filter_id, int64_t* ticket) {
    return guarded([&] {
        if (ticket == nullptr) throw std::invalid_argument("unexpected nullptr");
        *ticket = as_server(server).submit(nnz, terms, values, k, cut, heap_factor, filter_id);
    });
}

nsp_status_t nsp_server_wait(nsp_server_t* server, int64_t ticket, float* distances,
                             int64_t* labels, double* latency_us) {
    return guarded([&] { as_server(server).wait(ticket, distances, labels, latency_us); });
}

nsp_status_t nsp_server_replay(nsp_server_t* server, int32_t n, const int32_t* indptr,
                               const uint16_t* indices, const float* values, const int32_t* k_per,
                               const int32_t* filter_per, const double* arrival_us, int cut,
                               float heap_factor, int k_stride, float* distances, int64_t* labels,
                               double* latency_us) {
    return guarded([&] {
        as_server(server).replay(n, indptr, indices, values, k_per, filter_per, arrival_us, cut,
                                 heap_factor, k_stride, distances, labels, latency_us);
    });
}

nsp_status_t nsp_server_stats(nsp_server_t* server, int64_t* out4) {
    return guarded([&] {
        if (out4 == nullptr) throw std::invalid_argument("unexpected nullptr");
        const detail::ServerStats st = as_server(server).stats();
        out4[0] = st.batches;
        out4[1] = st.requests;
        out4[2] = st.max_batch;
        out4[3] = st.max_in_flight_bytes;
    });
}

nsp_status_t nsp_device_info(int32_t* n_devices, char* name, size_t name_len) {
    return guarded([&] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
        if (n_devices != nullptr) *n_devices = n;
        if (name != nullptr && name_len > 0) {
            name[0] = '\0';
            if (n > 0) {
                int dev = 0;
                cudaGetDevice(&dev);
                cudaDeviceProp prop{};
                if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
                    std::strncpy(name, prop.name, name_len - 1);
                    name[name_len - 1] = '\0';
                }
            }
        }
    });
}

}  // extern "C"
