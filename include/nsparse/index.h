// The Index interface (reference: nsparse/index.h:21-68). Search runs on the
// GPU; `distances` and `labels` are caller-owned n*k arrays, row-major, padded
// with (-1.0, -1) where fewer than k results exist.
#ifndef NSPARSE_B200_INDEX_H
#define NSPARSE_B200_INDEX_H

#include <array>
#include <cstddef>
#include <cstdint>

#include "nsparse/id_selector.h"
#include "nsparse/types.h"

namespace nsparse {

// Engine knobs with no counterpart in the reference. `plain` runs one kernel
// launch per query (the per-query baseline); the default batches every query
// of a call into one persistent launch. warps_per_block = 0 lets the engine
// choose.
struct EngineOptions {
    bool plain = false;
    int warps_per_block = 0;
    // SEISMIC kernel variant: -1 lets the engine choose, 0 one warp per query
    // loading doc rows straight from HBM, 1 the same with rows staged in
    // shared memory by bulk copy (stage_bytes per buffer, 0 = default), 2-5
    // one CTA per query with 1, 2, 4 or 8 lanes per scored doc, in batches of
    // batch_docs candidate docs (0 = default). Results are identical.
    int variant = -1;
    int stage_bytes = 0;
    int batch_docs = 0;
    // CTAs per query for variants 2-5: 0 lets the engine choose, 1 one CTA,
    // 2, 4 or 8 a thread-block cluster whose CTAs score each query's batches
    // together (lower latency per query; identical results).
    int ctas_per_query = 0;
    // Batched SEISMIC search on variants 2-5 only: a slower counting pass
    // that also counts each scored doc's row once per query, as the
    // reference's visited set does (SearchStats::unique_*); results are the
    // same.
    bool count_unique = false;
};

struct SearchParameters {
    virtual ~SearchParameters() = default;
    const IDSelector* get_id_selector() const { return id_selector; }
    void set_id_selector(IDSelector* selector) { id_selector = selector; }
    EngineOptions engine;

private:
    IDSelector* id_selector = nullptr;
};

// Work counters and device time of the calling thread's last search.
struct SearchStats {
    uint64_t docs_scored = 0;
    uint64_t blocks_visited = 0;
    uint64_t bytes = 0;          // bytes the kernels read, rows as often as scored
    uint64_t lists_probed = 0;
    float kernel_ms = 0.0f;
    int launches = 0;
    uint64_t row_bytes = 0;      // the rows' share of `bytes`
    // Counting pass (EngineOptions::count_unique) only: docs and row bytes
    // counted once per query. The reference's algorithmic bytes are then
    // bytes - row_bytes + unique_row_bytes (SEISMIC scores a doc met again in
    // a later list again; the reference skips it).
    uint64_t unique_docs = 0;
    uint64_t unique_row_bytes = 0;
};
const SearchStats& last_search_stats();

class Index {
public:
    explicit Index(int dim = 0);
    virtual ~Index() = default;
    virtual std::array<char, 4> id() const = 0;
    virtual void add(idx_t n, const idx_t* indptr, const term_t* indices,
                     const float* values) = 0;
    virtual void build();
    virtual void search(idx_t n, const idx_t* indptr, const term_t* indices,
                        const float* values, int k, float* distances, idx_t* labels,
                        SearchParameters* search_parameters = nullptr);

    int get_dimension() const { return dimension_; }
    virtual size_t num_vectors() const = 0;
    virtual void add_with_ids(idx_t n, const idx_t* indptr, const term_t* indices,
                              const float* values, const idx_t* ids);

    // File layout: int64 header (rows, cols, nnz), then int64 indptr
    // (rows + 1 entries), int32 indices and float32 values (nnz each).
    virtual void read_csr(const char* file_path, Residency residency = Residency::kInMemory);

protected:
    // Called by search() after argument validation.
    virtual void search_impl(idx_t n, const idx_t* indptr, const term_t* indices,
                             const float* values, int k, float* distances, idx_t* labels,
                             SearchParameters* search_parameters) = 0;
    int dimension_;
};

}  // namespace nsparse

#endif
