// Internal state behind the nsparse index classes: the host copy of the
// forward index (kept for persistence and rebuilds), its device image, and
// the SEISMIC lists on host and device.
#ifndef NSP_INDEX_STATE_H
#define NSP_INDEX_STATE_H

#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include "engine.h"
#include "nsparse/id_selector.h"
#include "nsparse/index.h"
#include "nsparse/seismic_index.h"

namespace nsparse {
namespace detail {

struct ForwardState {
    ForwardState(int dim, int esz) {
        host.dim = dim;
        host.esz = esz;
    }
    nsp::HostCsr host;
    nsp::ForwardDevice dev;
    nsp::PostingsDevice post;  // exact search's term-at-a-time postings
    bool dirty = true;
    mutable std::mutex mu;
    void append(idx_t n, const idx_t* indptr, const term_t* indices, const uint8_t* value_bytes);
    void ensure_device();
    // ensure_device, then the postings of the device rows (rebuilt after
    // every upload).
    const nsp::PostingsDevice* ensure_postings();
    // Every stored term < dim. The largest term is kept and extended over
    // appended elements only (a replaced host array is scanned afresh), so a
    // search does not rescan the whole index.
    bool terms_in_range(int dim) const;
    mutable const uint16_t* scanned_at = nullptr;
    mutable size_t scanned_len = 0;
    mutable int max_term = -1;
};

struct SeismicState {
    SeismicState(int dim, int esz) : vectors(dim, esz) { lists.esz = esz; }
    ForwardState vectors;
    nsp::SeismicHost lists;          // host copy, valid when host_valid
    std::vector<uint8_t> list_esz;   // element width each list declares on disk
    nsp::SeismicDevice lists_dev;
    bool host_valid = false;
    bool dev_valid = false;
    nsp::KernelChoice tuned;         // set by autotune; used when the caller leaves the choice
    std::mutex mu;
    // Uploads the host lists if the device copy is stale.
    void ensure_lists();
    // Host copy of the lists (downloaded after a device build).
    const nsp::SeismicHost& host_lists();
};

// SEISMIC build on the device (seismic_build.cu).
void seismic_build(SeismicState& st, int dim, const SeismicClusterParameters& params);

std::vector<uint64_t> selector_bitmap(const IDSelector* sel, int64_t n_docs);

// The SEISMIC state behind `index` (an IDMapIndex's delegate too) and the
// kernel arguments `params` ask for, SQ query encoding included; throws
// std::invalid_argument for other index types.
SeismicState* resolve_seismic(Index* index, SearchParameters* params, int k,
                              nsp::SeismicSearchArgs& a);

// The autotuner's launch shape, where the caller left the choice to the engine.
void apply_tuned(const SeismicState& st, nsp::SeismicSearchArgs& a, int64_t n_queries);

// Times every one-CTA-per-query launch shape (lanes per doc x batch x warps)
// on a sample of queries and keeps the fastest for later searches that leave
// the kernel to the engine (seismic indexes, also through an IDMapIndex).
nsp::KernelChoice seismic_autotune(Index* index, idx_t n, const idx_t* indptr,
                                   const term_t* indices, const float* values, int k,
                                   SearchParameters* params);

// SEISMIC search over device-resident queries and results (nsparse_c.h,
// nsp_index_search_device). Enqueues on `s` and returns.
void search_device(Index* index, int32_t n, const int32_t* d_indptr, const uint16_t* d_idx,
                   const float* d_val, int32_t max_nnz, int k, float* d_out, int32_t* d_lab,
                   SearchParameters* params, cudaStream_t s);

// One batched search step of a seismic index captured as a CUDA graph
// (nsparse_c.h, nsp_search_graph_*). It refuses to run once the index's
// device arrays were replaced (add, build, read) since the capture.
class IndexSearchGraph {
public:
    IndexSearchGraph(Index* index, int32_t n, int32_t nnz_cap, int32_t max_nnz, int k,
                     SearchParameters* params, const nsp::GraphBuffers* bind);
    const nsp::GraphBuffers& buffers() const { return g_->buffers(); }
    nsp::SearchGraph& graph() { return *g_; }
    // Replays the step on `s` (null: the graph's own stream) and returns.
    void launch(cudaStream_t s);
    // Waits for `s` (null: the graph's own stream), raises a kernel error,
    // records the step's counters as the thread's last search stats.
    void sync(cudaStream_t s);
    // Host queries in, host results out (at most the graph's rows).
    void search(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                float* distances, idx_t* labels);

private:
    void ensure_current() const;
    SeismicState* st_ = nullptr;
    int dim_ = 0;
    uint64_t fwd_gen_ = 0, ix_gen_ = 0;
    std::unique_ptr<nsp::SearchGraph> g_;
};

}  // namespace detail
}  // namespace nsparse

#endif  // NSP_INDEX_STATE_H
