// Test infrastructure (the checker, never the product): extern "C" entry points
// over the reference library's own C++ classes, compiled from the reference's
// unmodified sources by oracle/Makefile into oracle/_ref/. Python tests and the
// CPU-baseline leg of bench.py drive it through ctypes. Every function catches
// what the reference throws and reports it through ref_last_error().
//
// What each entry point exercises in the reference (paths inside its project):
//   ref_index_factory / ref_add / ref_build / ref_search   index_factory.cpp:63-153,
//       index.h:30-68, index.cpp:32-49 (public search that copies into D/L)
//   ref_write_index / ref_read_index                        io/index_io.cpp:166-190
//   ref_kmeans_train                                        cluster/random_kmeans.cpp:65-78
//   ref_map_docs_to_clusters                                cluster/kmeans_utils.cpp:162-195
//   ref_summarize                                           cluster/inverted_list_clusters.cpp:215-228
//   ref_prune_and_keep                                      invlists/inverted_lists.cpp:110-132
//   ref_top_k_tokens_*                                      utils/vector_process.h:18-30
//   ref_sq_*                                                utils/scalar_quantizer.h:52-101
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "nsparse/cluster/inverted_list_clusters.h"
#include "nsparse/cluster/kmeans_utils.h"
#include "nsparse/cluster/random_kmeans.h"
#include "nsparse/id_selector.h"
#include "nsparse/index.h"
#include "nsparse/index_factory.h"
#include "nsparse/invlists/inverted_lists.h"
#include "nsparse/io/buffered_io.h"
#include "nsparse/io/index_io.h"
#include "nsparse/seismic_index.h"
#include "nsparse/seismic_scalar_quantized_index.h"
#include "nsparse/sparse_vectors.h"
#include "nsparse/utils/csr_layout.h"
#include "nsparse/utils/scalar_quantizer.h"
#include "nsparse/utils/vector_process.h"

namespace {
thread_local std::string g_err;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return 1;
    } catch (const std::out_of_range& e) {
        g_err = e.what();
        return 3;
    } catch (const std::bad_alloc& e) {
        g_err = e.what();
        return 4;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 2;
    }
}

nsparse::SparseVectors make_vectors(int dim, int esz, int32_t n,
                                    const int32_t* indptr,
                                    const uint16_t* indices,
                                    const uint8_t* value_bytes) {
    nsparse::SparseVectors v({.element_size = static_cast<size_t>(esz),
                              .dimension = static_cast<size_t>(dim)});
    const size_t nnz = static_cast<size_t>(indptr[n]);
    v.add_vectors(indptr, static_cast<size_t>(n) + 1, indices, nnz, value_bytes,
                  nnz * static_cast<size_t>(esz));
    return v;
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_set_threads(int n) { omp_set_num_threads(n); }

int ref_max_threads() { return omp_get_max_threads(); }

void* ref_index_factory(int dim, const char* desc) {
    nsparse::Index* out = nullptr;
    if (guarded([&] { out = nsparse::index_factory(dim, desc); }) != 0) {
        return nullptr;
    }
    return out;
}

// index_factory's outcome as a status (0 ok, else the guarded() code) and,
// on success, the index's fourcc in out4.
int ref_factory_status(int dim, const char* desc, char* out4) {
    return guarded([&] {
        std::unique_ptr<nsparse::Index> idx(nsparse::index_factory(dim, desc));
        const auto id = idx->id();
        std::memcpy(out4, id.data(), 4);
    });
}

void ref_index_free(void* h) { delete static_cast<nsparse::Index*>(h); }

int ref_add(void* h, int32_t n, const int32_t* indptr, const uint16_t* indices,
            const float* values) {
    return guarded(
        [&] { static_cast<nsparse::Index*>(h)->add(n, indptr, indices, values); });
}

int ref_add_with_ids(void* h, int32_t n, const int32_t* indptr,
                     const uint16_t* indices, const float* values,
                     const int32_t* ids) {
    return guarded([&] {
        static_cast<nsparse::Index*>(h)->add_with_ids(n, indptr, indices,
                                                      values, ids);
    });
}

int ref_build(void* h) {
    return guarded([&] { static_cast<nsparse::Index*>(h)->build(); });
}

int64_t ref_num_vectors(void* h) {
    return static_cast<int64_t>(static_cast<nsparse::Index*>(h)->num_vectors());
}

// param_kind: 0 none, 1 SearchParameters, 2 SeismicSearchParameters,
// 3 SeismicSQSearchParameters. sel_kind: 0 none, 1 SetIDSelector,
// 2 ArrayIDSelector, 3 NotIDSelector(SetIDSelector).
int ref_search(void* h, int32_t n, const int32_t* indptr, const uint16_t* indices,
               const float* values, int k, float* distances, int32_t* labels,
               int param_kind, int cut, float heap_factor, float vmin, float vmax,
               int sel_kind, int64_t n_sel, const int32_t* sel_ids) {
    return guarded([&] {
        std::unique_ptr<nsparse::SearchParameters> params;
        if (param_kind == 1) {
            params = std::make_unique<nsparse::SearchParameters>();
        } else if (param_kind == 2) {
            params = std::make_unique<nsparse::SeismicSearchParameters>(
                cut, heap_factor);
        } else if (param_kind == 3) {
            params = std::make_unique<nsparse::SeismicSQSearchParameters>(
                vmin, vmax, cut, heap_factor);
        }
        std::unique_ptr<nsparse::IDSelector> inner;
        std::unique_ptr<nsparse::IDSelector> outer;
        if (sel_kind == 1 || sel_kind == 3) {
            inner = std::make_unique<nsparse::SetIDSelector>(
                static_cast<size_t>(n_sel), sel_ids);
        } else if (sel_kind == 2) {
            inner = std::make_unique<nsparse::ArrayIDSelector>(
                static_cast<size_t>(n_sel), sel_ids);
        }
        nsparse::IDSelector* sel = inner.get();
        if (sel_kind == 3) {
            outer = std::make_unique<nsparse::NotIDSelector>(inner.get());
            sel = outer.get();
        }
        if (sel != nullptr) {
            if (!params) {
                params = std::make_unique<nsparse::SearchParameters>();
            }
            params->set_id_selector(sel);
        }
        static_cast<nsparse::Index*>(h)->search(n, indptr, indices, values, k,
                                                distances, labels, params.get());
    });
}

int ref_write_index(void* h, const char* path) {
    return guarded([&] {
        nsparse::write_index(static_cast<nsparse::Index*>(h),
                             const_cast<char*>(path));
    });
}

// Index::read_csr with a residency: 0 in-memory, 1 mmap.
int ref_read_csr(void* h, const char* path, int residency) {
    return guarded([&] {
        static_cast<nsparse::Index*>(h)->read_csr(
            path, residency == 1 ? nsparse::Residency::kMmap : nsparse::Residency::kInMemory);
    });
}

// csr_layout::convert: interchange CSR file -> native (.mcsr) file.
int ref_csr_convert(const char* interchange_path, const char* native_path) {
    return guarded([&] { nsparse::csr_layout::convert(interchange_path, native_path); });
}

void* ref_read_index(const char* path, int io_flags) {
    nsparse::Index* out = nullptr;
    if (guarded([&] {
            out = nsparse::read_index(const_cast<char*>(path), io_flags);
        }) != 0) {
        return nullptr;
    }
    return out;
}

// Clusters a posting list with the reference's own k-means. Writes the flat
// clusters (centroid first, then members) and their offsets.
int ref_kmeans_train(int dim, int esz, int32_t n_docs, const int32_t* indptr,
                     const uint16_t* indices, const uint8_t* value_bytes,
                     const int32_t* doc_ids, int32_t n_ids, int n_clusters,
                     uint32_t seed, int32_t* out_docs, int32_t* out_offsets,
                     int32_t* out_n_clusters) {
    return guarded([&] {
        auto v = make_vectors(dim, esz, n_docs, indptr, indices, value_bytes);
        std::vector<int32_t> ids(doc_ids, doc_ids + n_ids);
        auto clusters = nsparse::detail::RandomKMeans::train(
            &v, ids, static_cast<size_t>(n_clusters), seed);
        int32_t pos = 0;
        out_offsets[0] = 0;
        for (size_t c = 0; c < clusters.size(); ++c) {
            for (int32_t d : clusters[c]) out_docs[pos++] = d;
            out_offsets[c + 1] = pos;
        }
        *out_n_clusters = static_cast<int32_t>(clusters.size());
    });
}

// Assigns `doc_ids` to the given centroids with the reference's assigner.
int ref_map_docs_to_clusters(int dim, int esz, int32_t n_docs,
                             const int32_t* indptr, const uint16_t* indices,
                             const uint8_t* value_bytes, const int32_t* doc_ids,
                             int32_t n_ids, const int32_t* centroids,
                             int n_clusters, int32_t* out_docs,
                             int32_t* out_offsets) {
    return guarded([&] {
        auto v = make_vectors(dim, esz, n_docs, indptr, indices, value_bytes);
        std::vector<int32_t> ids(doc_ids, doc_ids + n_ids);
        std::vector<std::vector<int32_t>> clusters(n_clusters);
        for (int c = 0; c < n_clusters; ++c) clusters[c].push_back(centroids[c]);
        nsparse::detail::map_docs_to_clusters(&v, ids, clusters);
        int32_t pos = 0;
        out_offsets[0] = 0;
        for (int c = 0; c < n_clusters; ++c) {
            for (int32_t d : clusters[c]) out_docs[pos++] = d;
            out_offsets[c + 1] = pos;
        }
    });
}

// Summarizes given clusters with the reference and returns the serialized
// InvertedListClusters (docs, offsets, CSC summaries) in `out`. Returns the
// byte count, or -1 on error / -2 when `cap` is too small.
int64_t ref_summarize(int dim, int esz, int32_t n_docs, const int32_t* indptr,
                      const uint16_t* indices, const uint8_t* value_bytes,
                      const int32_t* cl_docs, const int32_t* cl_offsets,
                      int n_clusters, float alpha, uint8_t* out, int64_t cap) {
    int64_t written = -1;
    int rc = guarded([&] {
        auto v = make_vectors(dim, esz, n_docs, indptr, indices, value_bytes);
        std::vector<std::vector<int32_t>> clusters(n_clusters);
        for (int c = 0; c < n_clusters; ++c) {
            clusters[c].assign(cl_docs + cl_offsets[c], cl_docs + cl_offsets[c + 1]);
        }
        nsparse::InvertedListClusters ilc(clusters);
        ilc.summarize(&v, alpha);
        nsparse::BufferedIOWriter w;
        ilc.serialize(&w);
        const auto& bytes = w.data();
        if (static_cast<int64_t>(bytes.size()) > cap) {
            written = -2;
            return;
        }
        std::memcpy(out, bytes.data(), bytes.size());
        written = static_cast<int64_t>(bytes.size());
    });
    return rc == 0 ? written : -1;
}

// λ truncation of one posting list (doc ids + raw value bytes at `esz`).
int ref_prune_and_keep(int esz, int32_t n, const int32_t* doc_ids,
                       const uint8_t* value_bytes, int32_t lambda,
                       int32_t* out_ids, int32_t* out_n) {
    return guarded([&] {
        nsparse::InvertedList list(static_cast<size_t>(esz));
        list.add_entries(static_cast<size_t>(n), doc_ids, value_bytes);
        auto kept = list.prune_and_keep_doc_ids(static_cast<size_t>(lambda));
        std::memcpy(out_ids, kept.data(), kept.size() * sizeof(int32_t));
        *out_n = static_cast<int32_t>(kept.size());
    });
}

int ref_top_k_tokens_f32(const uint16_t* idx, const float* w, int size, int k,
                         uint16_t* out, int32_t* out_n) {
    return guarded([&] {
        auto r = nsparse::detail::top_k_tokens<float>(idx, w, size, k);
        std::memcpy(out, r.data(), r.size() * sizeof(uint16_t));
        *out_n = static_cast<int32_t>(r.size());
    });
}

int ref_top_k_tokens_u8(const uint16_t* idx, const uint8_t* w, int size, int k,
                        uint16_t* out, int32_t* out_n) {
    return guarded([&] {
        auto r = nsparse::detail::top_k_tokens<uint8_t>(idx, w, size, k);
        std::memcpy(out, r.data(), r.size() * sizeof(uint16_t));
        *out_n = static_cast<int32_t>(r.size());
    });
}

int ref_sq_encode(int qtype, float vmin, float vmax, const float* vals,
                  uint8_t* codes, int64_t n) {
    return guarded([&] {
        nsparse::ScalarQuantizer sq(qtype == 16 ? nsparse::QuantizerType::QT_16bit
                                                : nsparse::QuantizerType::QT_8bit,
                                    vmin, vmax);
        sq.encode(vals, codes, static_cast<size_t>(n));
    });
}

float ref_sq_decode_dot(int qtype, float vmin, float vmax, float score,
                        float qvmin, float qvmax) {
    nsparse::ScalarQuantizer sq(qtype == 16 ? nsparse::QuantizerType::QT_16bit
                                            : nsparse::QuantizerType::QT_8bit,
                                vmin, vmax);
    nsparse::ScalarQuantizer qsq(sq.get_quantizer_type(), qvmin, qvmax);
    return sq.decode_dot_product(score, qsq);
}

}  // extern "C"
