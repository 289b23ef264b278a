// The nsparse C++ API (include/nsparse/*.h) over the GPU engine. Argument
// checks, error types and padding follow the reference (nsparse/index.cpp,
// brutal_index.cpp, inverted_index.cpp, seismic_index.cpp,
// seismic_scalar_quantized_index.cpp, id_map_index.cpp, index_factory.cpp);
// every score is computed by the kernels in search_*.cu.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "csr_layout_read.h"
#include "index_state.h"
#include "nsparse/brutal_index.h"
#include "nsparse/id_map_index.h"
#include "nsparse/index.h"
#include "nsparse/index_factory.h"
#include "nsparse/inverted_index.h"
#include "nsparse/seismic_index.h"
#include "nsparse/seismic_scalar_quantized_index.h"

namespace nsparse {

// ------------------------------------------------------------- helpers --

namespace {

void throw_if_not_positive(long long v, const char* msg = "value must be positive") {
    if (v <= 0) throw std::invalid_argument(msg);
}

template <class... P>
void throw_if_any_null(P... ptrs) {
    if (((ptrs == nullptr) || ...)) throw std::invalid_argument("unexpected nullptr");
}

thread_local SearchStats g_last_stats;

void record_stats(const nsp::SearchStats& s) {
    g_last_stats.docs_scored = s.docs_scored;
    g_last_stats.blocks_visited = s.blocks_visited;
    g_last_stats.bytes = s.bytes;
    g_last_stats.lists_probed = s.lists_probed;
    g_last_stats.kernel_ms = s.kernel_ms;
    g_last_stats.launches = s.launches;
    g_last_stats.row_bytes = s.row_bytes;
    g_last_stats.unique_docs = s.unique_docs;
    g_last_stats.unique_row_bytes = s.unique_row_bytes;
}

void fill_padding(idx_t n, int k, float* d, idx_t* l) {
    const size_t cnt = static_cast<size_t>(n) * k;
    std::fill(d, d + cnt, -1.0F);
    std::fill(l, l + cnt, detail::INVALID_IDX);
}

inline void set_bit(uint64_t* bits, int64_t d) { bits[d >> 6] |= uint64_t{1} << (d & 63); }

// Query quantizer arguments of a SEISMIC search.
nsp::SeismicSearchArgs seismic_args(const SearchParameters* p, int k) {
    nsp::SeismicSearchArgs a;
    a.k = k;
    const auto* sp = dynamic_cast<const SeismicSearchParameters*>(p);
    // Parameters without cut / heap factor fall back to the defaults
    // (seismic_index.cpp:161-168).
    SeismicSearchParameters defaults;
    if (sp == nullptr) sp = &defaults;
    if (sp->cut <= 0) throw std::invalid_argument("value must be positive");
    a.cut = sp->cut;
    a.heap_factor = sp->heap_factor;
    if (p != nullptr) {
        a.plain = p->engine.plain;
        a.warps_per_block = p->engine.warps_per_block;
        a.variant = p->engine.variant;
        a.stage_bytes = p->engine.stage_bytes;
        a.batch_docs = p->engine.batch_docs;
        a.cluster = p->engine.ctas_per_query;
        a.count_unique = p->engine.count_unique;
    }
    return a;
}

}  // namespace

const SearchStats& last_search_stats() { return g_last_stats; }

// ----------------------------------------------------------- selectors --

void IDSelector::fill_bitmap(uint64_t* bits, int64_t n_docs) const {
    for (int64_t d = 0; d < n_docs; ++d)
        if (is_member(static_cast<idx_t>(d))) set_bit(bits, d);
}

void IDSelectorEnumerable::fill_bitmap(uint64_t* bits, int64_t n_docs) const {
    for (idx_t d : ids())
        if (d >= 0 && d < n_docs) set_bit(bits, d);
}

void NotIDSelector::fill_bitmap(uint64_t* bits, int64_t n_docs) const {
    const int64_t words = (n_docs + 63) / 64;
    std::vector<uint64_t> inner(static_cast<size_t>(words), 0);
    delegate_->fill_bitmap(inner.data(), n_docs);
    for (int64_t w = 0; w < words; ++w) bits[w] = ~inner[w];
    if (n_docs % 64 != 0) bits[words - 1] &= (uint64_t{1} << (n_docs % 64)) - 1;
}

BitmapIDSelector::BitmapIDSelector(int64_t n_bits, const uint64_t* bits) : n_bits_(n_bits) {
    if (n_bits < 0) throw std::invalid_argument("bitmap size must not be negative");
    if (n_bits > 0 && bits == nullptr) throw std::invalid_argument("unexpected nullptr");
    bits_.assign(bits, bits + (n_bits + 63) / 64);
}

bool BitmapIDSelector::is_member(idx_t id) const {
    return id >= 0 && id < n_bits_ && ((bits_[id >> 6] >> (id & 63)) & 1U);
}

void BitmapIDSelector::fill_bitmap(uint64_t* bits, int64_t n_docs) const {
    const int64_t m = std::min(n_docs, n_bits_);
    const int64_t full = m / 64;
    for (int64_t w = 0; w < full; ++w) bits[w] |= bits_[w];
    for (int64_t d = full * 64; d < m; ++d)
        if (is_member(static_cast<idx_t>(d))) set_bit(bits, d);
}

namespace detail {

std::vector<uint64_t> selector_bitmap(const IDSelector* sel, int64_t n_docs) {
    std::vector<uint64_t> bits(static_cast<size_t>((n_docs + 64) / 64), 0);
    sel->fill_bitmap(bits.data(), n_docs);
    return bits;
}

// Selectors IDMapIndex hands its delegate (reference: id_map_index.h:20-73).
// is_member and ids() translate between internal and external ids.
class IDSelectorWithIDMap : public IDSelector {
public:
    IDSelectorWithIDMap(const IDSelector* d, const std::vector<int64_t>& map,
                        const std::unordered_map<int64_t, idx_t>& ext)
        : delegate_(d), map_(map), ext_(ext) {}
    bool is_member(idx_t id) const override { return delegate_->is_member64(map_[id]); }
    void fill_bitmap(uint64_t* bits, int64_t n_docs) const override {
        // NOT(enumerable): everything but the mapped ids of the inner set.
        if (const auto* nots = dynamic_cast<const NotIDSelector*>(delegate_)) {
            if (const auto* en = dynamic_cast<const IDSelectorEnumerable*>(nots->delegate())) {
                const int64_t words = (n_docs + 63) / 64;
                for (int64_t w = 0; w < words; ++w) bits[w] = ~uint64_t{0};
                if (n_docs % 64 != 0) bits[words - 1] = (uint64_t{1} << (n_docs % 64)) - 1;
                for (int64_t e : en->ids64()) {
                    auto it = ext_.find(e);
                    if (it != ext_.end() && it->second < n_docs)
                        bits[it->second >> 6] &= ~(uint64_t{1} << (it->second & 63));
                }
                return;
            }
        }
        const int64_t m = std::min<int64_t>(n_docs, static_cast<int64_t>(map_.size()));
        for (int64_t d = 0; d < m; ++d)
            if (delegate_->is_member64(map_[d])) set_bit(bits, d);
    }

private:
    const IDSelector* delegate_;
    const std::vector<int64_t>& map_;
    const std::unordered_map<int64_t, idx_t>& ext_;
};

// id_map_index.h:42-75: an enumerable external selector enumerates the
// internal ids of its members.
class IDSelectorEnumerableWithIDMap : public IDSelectorEnumerable {
public:
    IDSelectorEnumerableWithIDMap(const IDSelectorEnumerable* d, const std::vector<int64_t>& map,
                                  const std::unordered_map<int64_t, idx_t>& ext)
        : delegate_(d), map_(map), ext_(ext) {}
    bool is_member(idx_t id) const override { return delegate_->is_member64(map_[id]); }
    std::vector<idx_t> ids() const override {
        std::vector<idx_t> out;
        for (int64_t e : delegate_->ids64()) {
            auto it = ext_.find(e);
            if (it != ext_.end()) out.push_back(it->second);
        }
        return out;
    }
    // The external selector's size, as the reference reports it
    // (id_map_index.h:56): it decides the exact-match shortcut.
    size_t size() const override { return delegate_->size(); }

private:
    const IDSelectorEnumerable* delegate_;
    const std::vector<int64_t>& map_;
    const std::unordered_map<int64_t, idx_t>& ext_;
};

// ---------------------------------------------------------- state types --

void ForwardState::append(idx_t n, const idx_t* indptr, const term_t* indices,
                          const uint8_t* value_bytes) {
    std::lock_guard<std::mutex> g(mu);
    host.append(n, indptr, indices, value_bytes);
    dirty = true;
}

void ForwardState::ensure_device() {
    std::lock_guard<std::mutex> g(mu);
    if (dirty) {
        dev.upload(host);
        dirty = false;
    }
}

const nsp::PostingsDevice* ForwardState::ensure_postings() {
    std::lock_guard<std::mutex> g(mu);
    if (dirty) {
        dev.upload(host);
        dirty = false;
    }
    if (post.generation() != dev.generation()) post.build(dev, nsp::exact_taat_chunk_docs());
    return &post;
}

bool ForwardState::terms_in_range(int dim) const {
    std::lock_guard<std::mutex> g(mu);
    const std::vector<uint16_t>& ix = host.indices;
    if (ix.data() != scanned_at || ix.size() < scanned_len) {
        scanned_len = 0;
        max_term = -1;
    }
    for (size_t i = scanned_len; i < ix.size(); ++i) max_term = std::max<int>(max_term, ix[i]);
    scanned_at = ix.data();
    scanned_len = ix.size();
    return max_term < dim;
}

}  // namespace detail

// ------------------------------------------------------------ Index base --

Index::Index(int dim) : dimension_(dim) {}

void Index::build() { throw std::runtime_error("not implemented"); }

void Index::search(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                   int k, float* distances, idx_t* labels, SearchParameters* search_parameters) {
    throw_if_not_positive(n);
    throw_if_not_positive(k);
    throw_if_any_null(indptr, indices, values, labels, distances);
    search_impl(n, indptr, indices, values, k, distances, labels, search_parameters);
}

void Index::add_with_ids(idx_t, const idx_t*, const term_t*, const float*, const idx_t*) {
    throw std::runtime_error("add_with_ids not implemented in Index");
}

// Interchange CSR file (reference: index.cpp:63-142).
void Index::read_csr(const char* file_path, Residency) {
    if (file_path == nullptr) throw std::invalid_argument("file_path must not be null");
    if (!std::filesystem::exists(file_path))
        throw std::invalid_argument(std::string("CSR file does not exist: ") + file_path);
    std::ifstream file(file_path, std::ios::binary);
    if (!file.is_open()) throw std::runtime_error(std::string("Cannot open CSR file: ") + file_path);
    auto read_or_throw = [&](void* dest, size_t bytes) {
        file.read(static_cast<char*>(dest), static_cast<std::streamsize>(bytes));
        if (!file) throw std::runtime_error(std::string("Truncated CSR file: ") + file_path);
    };
    std::array<int64_t, 3> header{};
    read_or_throw(header.data(), sizeof(header));
    const int64_t rows = header[0], cols = header[1], nnz = header[2];
    if (rows <= 0 || cols <= 0 || nnz < 0)
        throw std::invalid_argument(std::string("Invalid CSR header in: ") + file_path);
    if (rows > std::numeric_limits<idx_t>::max() || nnz > std::numeric_limits<idx_t>::max())
        throw std::invalid_argument(std::string("CSR file too large for ") +
                                    "32-bit offsets: " + file_path);
    if (cols > dimension_)
        throw std::invalid_argument(std::string("CSR column count exceeds index dimension: ") +
                                    file_path);
    const uint64_t expect = 24 + 8 * static_cast<uint64_t>(rows + 1) + 8 * static_cast<uint64_t>(nnz);
    if (std::filesystem::file_size(file_path) != expect)
        throw std::invalid_argument(std::string("CSR file is not in the interchange layout: ") +
                                    file_path);
    std::vector<int64_t> fip(static_cast<size_t>(rows) + 1);
    read_or_throw(fip.data(), fip.size() * 8);
    if (fip.front() != 0 || fip.back() != nnz)
        throw std::invalid_argument(std::string("Inconsistent CSR indptr in: ") + file_path);
    std::vector<idx_t> ip(fip.begin(), fip.end());
    std::vector<int32_t> fidx(static_cast<size_t>(nnz));
    read_or_throw(fidx.data(), fidx.size() * 4);
    for (int32_t t : fidx)
        if (t < 0 || t >= cols || t > std::numeric_limits<term_t>::max())
            throw std::invalid_argument(std::string("CSR term out of range in: ") + file_path);
    std::vector<term_t> idx(fidx.begin(), fidx.end());
    std::vector<float> vals(static_cast<size_t>(nnz));
    read_or_throw(vals.data(), vals.size() * 4);
    add(static_cast<idx_t>(rows), ip.data(), idx.data(), vals.data());
}

// ------------------------------------------------------------- Brutal ----

BrutalIndex::BrutalIndex(int dim) : Index(dim), fwd_(new detail::ForwardState(dim, 4)) {}
BrutalIndex::~BrutalIndex() = default;

void BrutalIndex::add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) {
    throw_if_not_positive(n);
    throw_if_any_null(indptr, indices, values);
    fwd_->append(n, indptr, indices, reinterpret_cast<const uint8_t*>(values));
}

size_t BrutalIndex::num_vectors() const { return static_cast<size_t>(fwd_->host.n()); }

// brutal_index.cpp:45-96. The selector is ignored, as in the reference.
void BrutalIndex::search_impl(idx_t n, const idx_t* indptr, const term_t* indices,
                              const float* values, int k, float* distances, idx_t* labels,
                              SearchParameters*) {
    if (fwd_->host.n() == 0) return fill_padding(n, k, distances, labels);
    if (!fwd_->terms_in_range(dimension_)) throw std::invalid_argument("term_id out of range");
    const nsp::PostingsDevice* post = fwd_->ensure_postings();
    const nsp::QueryBatch q = nsp::canonicalize(n, indptr, indices, values, dimension_);
    nsp::SearchStats st;
    nsp::exact_search(fwd_->dev, post, q, k, 0, nullptr, distances, labels, &st);
    record_stats(st);
}

// ----------------------------------------------------------- Inverted ----

InvertedIndex::InvertedIndex(int dim) : Index(dim), fwd_(new detail::ForwardState(dim, 4)) {}
InvertedIndex::~InvertedIndex() = default;

void InvertedIndex::add(idx_t n, const idx_t* indptr, const term_t* indices,
                        const float* values) {
    throw_if_not_positive(n);
    throw_if_any_null(indptr, indices, values);
    fwd_->append(n, indptr, indices, reinterpret_cast<const uint8_t*>(values));
}

// inverted_index.cpp:236-252: a term >= dimension has no posting list. The
// device postings of the exact search are built here, as the reference
// builds its posting lists here.
void InvertedIndex::build() {
    if (!fwd_->terms_in_range(dimension_)) throw std::invalid_argument("term_id out of range");
    fwd_->ensure_postings();
    built_ = true;
}

size_t InvertedIndex::num_vectors() const { return static_cast<size_t>(fwd_->host.n()); }

void InvertedIndex::search_impl(idx_t n, const idx_t* indptr, const term_t* indices,
                                const float* values, int k, float* distances, idx_t* labels,
                                SearchParameters* params) {
    if (!built_ || fwd_->host.n() == 0) return fill_padding(n, k, distances, labels);
    const nsp::PostingsDevice* post = fwd_->ensure_postings();
    const nsp::QueryBatch q = nsp::canonicalize(n, indptr, indices, values, dimension_);
    const IDSelector* sel = params == nullptr ? nullptr : params->get_id_selector();
    std::vector<uint64_t> bits;
    if (sel != nullptr) bits = detail::selector_bitmap(sel, fwd_->host.n());
    nsp::SearchStats st;
    nsp::exact_search(fwd_->dev, post, q, k, 1, sel != nullptr ? &bits : nullptr, distances, labels,
                      &st);
    record_stats(st);
}

// ------------------------------------------------------ SEISMIC common ---

namespace detail {

// should_run_exact_match (seismic_common.h:117-128).
const IDSelectorEnumerable* exact_match_selector(const IDSelector* sel, int k) {
    if (sel == nullptr) return nullptr;
    const auto* en = dynamic_cast<const IDSelectorEnumerable*>(sel);
    if (en == nullptr) return nullptr;
    return en->size() <= static_cast<size_t>(k) ? en : nullptr;
}

// The autotuner's launch shape, where the caller left the choice to the engine.
// The tuned variant applies to every launch. The tuned batch and warps were
// chosen among 4- and 8-warp CTAs on a large batch, so they apply only where
// the planner itself would fill every SM with several CTAs (more than two
// queries per SM, not the one-query plain path); smaller launches keep the
// planner's wider CTAs, which finish a lone query sooner.
void apply_tuned(const SeismicState& st, nsp::SeismicSearchArgs& a, int64_t n_queries) {
    if (a.variant >= 0 || st.tuned.variant < 0) return;
    a.variant = st.tuned.variant;
    if (a.cluster == 0 && st.tuned.split > 0) {
        // the split measured fastest for a lone query, where the engine's
        // rule would give a launch this small a cluster at all
        const int rule = nsp::auto_cluster(
            a.plain ? 1 : static_cast<int>(std::min<int64_t>(n_queries, 1 << 30)));
        a.cluster = std::min(rule, st.tuned.split);
    }
    if (a.plain || n_queries <= 2 * static_cast<int64_t>(nsp::device_sm_count())) return;
    if (a.batch_docs == 0) a.batch_docs = st.tuned.batch_docs;
    if (a.warps_per_block == 0) a.warps_per_block = st.tuned.warps_per_block;
}

void seismic_search_common(SeismicState& st, int dim, idx_t n, const idx_t* indptr,
                           const term_t* indices, const float* values, int k, float* distances,
                           idx_t* labels, SearchParameters* params, nsp::SeismicSearchArgs args) {
    if (st.vectors.host.n() == 0) return fill_padding(n, k, distances, labels);
    apply_tuned(st, args, n);
    st.vectors.ensure_device();
    const nsp::QueryBatch q = nsp::canonicalize(n, indptr, indices, values, dim);
    const IDSelector* sel = params == nullptr ? nullptr : params->get_id_selector();
    if (const auto* en = exact_match_selector(sel, k)) {
        // ExactMatcher (exact_matcher.h:23-58): the selector's ids, ascending.
        std::vector<idx_t> ids = en->ordered_ids();
        nsp::exact_list_search(st.vectors.dev, q, args, ids, distances, labels);
        g_last_stats = SearchStats{};
        return;
    }
    st.ensure_lists();
    std::vector<uint64_t> bits;
    if (sel != nullptr) bits = selector_bitmap(sel, st.vectors.host.n());
    nsp::SearchStats s;
    nsp::seismic_search(st.vectors.dev, st.lists_dev, q, args, sel != nullptr ? &bits : nullptr,
                        distances, labels, &s);
    record_stats(s);
}

}  // namespace detail

// ------------------------------------------------------------- SEISMIC ---

SeismicIndex::SeismicIndex(int dim)
    : SeismicIndex(dim, SeismicClusterParameters{-1, -1, 0.4F}) {}

SeismicIndex::SeismicIndex(int dim, SeismicClusterParameters parameter)
    : Index(dim), cluster_parameter_(parameter), st_(new detail::SeismicState(dim, 4)) {}

SeismicIndex::~SeismicIndex() = default;

void SeismicIndex::add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) {
    throw_if_not_positive(n);
    throw_if_any_null(indptr, indices, values);
    st_->vectors.append(n, indptr, indices, reinterpret_cast<const uint8_t*>(values));
}

size_t SeismicIndex::num_vectors() const { return static_cast<size_t>(st_->vectors.host.n()); }

void SeismicIndex::read_csr(const char* file_path, Residency residency) {
    if (residency == Residency::kInMemory) return Index::read_csr(file_path, residency);
    if (residency != Residency::kMmap) throw std::invalid_argument("invalid residency");
    if (file_path == nullptr) throw std::invalid_argument("file_path must not be null");
    if (st_->vectors.host.n() > 0) throw std::runtime_error("mmap index already has vectors");
    const detail::NativeCsr c = detail::read_native_csr(file_path, dimension_);
    st_->vectors.append(c.rows, c.indptr.data(), c.indices.data(),
                        reinterpret_cast<const uint8_t*>(c.values.data()));
}

void SeismicIndex::build() {
    detail::seismic_build(*st_, dimension_, cluster_parameter_);
}

void SeismicIndex::search_impl(idx_t n, const idx_t* indptr, const term_t* indices,
                               const float* values, int k, float* distances, idx_t* labels,
                               SearchParameters* params) {
    detail::seismic_search_common(*st_, dimension_, n, indptr, indices, values, k, distances,
                                  labels, params, seismic_args(params, k));
}

// ---------------------------------------------------------- SEISMIC-SQ ---

ScalarQuantizer::ScalarQuantizer(QuantizerType qtype, float vmin, float vmax)
    : qtype_(qtype), vmin_(vmin), vmax_(vmax) {
    if (!std::isfinite(vmin) || !std::isfinite(vmax))
        throw std::invalid_argument("vmin and vmax must be finite");
    if (vmax <= vmin) throw std::invalid_argument("vmax must be greater than vmin");
}

float ScalarQuantizer::encode_scale() const {
    const float kmax = qtype_ == QuantizerType::QT_8bit ? 255.0F : 65535.0F;
    return kmax / (vmax_ - vmin_);
}

// scalar_quantizer.h:97-101 (8-bit) and 108-112 (16-bit). Each value is
// encoded on its own, so large inputs are split over host threads (a corpus
// of 1.24B values took seconds on one).
void ScalarQuantizer::encode(const float* vals, uint8_t* codes, size_t n) const {
    const float kmax = qtype_ == QuantizerType::QT_8bit ? 255.0F : 65535.0F;
    const float scale = encode_scale();
    auto range = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
            float scaled = (vals[i] - vmin_) * scale;
            scaled = std::max(0.0F, std::min(kmax, scaled));
            const long r = std::lround(scaled);
            if (qtype_ == QuantizerType::QT_8bit)
                codes[i] = static_cast<uint8_t>(r);
            else
                reinterpret_cast<uint16_t*>(codes)[i] = static_cast<uint16_t>(r);
        }
    };
    constexpr size_t kPerThread = size_t{1} << 22;
    const size_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t nth = std::min(hw, (n + kPerThread - 1) / kPerThread);
    if (nth <= 1) return range(0, n);
    std::vector<std::thread> pool;
    const size_t step = (n + nth - 1) / nth;
    for (size_t t = 1; t < nth; ++t)
        pool.emplace_back(range, std::min(n, t * step), std::min(n, (t + 1) * step));
    range(0, std::min(n, step));
    for (auto& th : pool) th.join();
}

void ScalarQuantizer::decode(const uint8_t* codes, float* vals, size_t n) const {
    const float kmax = qtype_ == QuantizerType::QT_8bit ? 255.0F : 65535.0F;
    for (size_t i = 0; i < n; ++i) {
        const float c = qtype_ == QuantizerType::QT_8bit
                            ? static_cast<float>(codes[i])
                            : static_cast<float>(reinterpret_cast<const uint16_t*>(codes)[i]);
        vals[i] = vmin_ + (c * (vmax_ - vmin_) / kmax);
    }
}

// scalar_quantizer.h:85-93 (vmin is not used, as in the reference).
float ScalarQuantizer::decode_scale(const ScalarQuantizer& query_sq) const {
    const float ingest_range = vmax_ - vmin_;
    const float query_range = query_sq.get_max() - query_sq.get_min();
    const float max_q = qtype_ == QuantizerType::QT_8bit ? 255.0F : 65535.0F;
    return (ingest_range * query_range) / (max_q * max_q);
}

SeismicScalarQuantizedIndex::SeismicScalarQuantizedIndex(int dim)
    : Index(dim),
      cluster_parameter_{-1, -1, 0.4F},
      st_(new detail::SeismicState(dim, 1)) {}

SeismicScalarQuantizedIndex::SeismicScalarQuantizedIndex(QuantizerType quantizer_type,
                                                         float vmin, float vmax,
                                                         SeismicClusterParameters parameter,
                                                         int dim)
    : Index(dim),
      sq_(quantizer_type, vmin, vmax),
      cluster_parameter_(parameter),
      st_(new detail::SeismicState(dim, static_cast<int>(sq_.bytes_per_value()))) {}

SeismicScalarQuantizedIndex::~SeismicScalarQuantizedIndex() = default;

void SeismicScalarQuantizedIndex::add(idx_t n, const idx_t* indptr, const term_t* indices,
                                      const float* values) {
    throw_if_not_positive(n);
    throw_if_any_null(indptr, indices, values);
    const size_t nnz = static_cast<size_t>(indptr[n] - indptr[0]);
    std::vector<uint8_t> codes(nnz * sq_.bytes_per_value());
    sq_.encode(values + indptr[0], codes.data(), nnz);
    // rebase so the codes array starts at element 0
    std::vector<idx_t> ip(indptr, indptr + n + 1);
    for (auto& v : ip) v -= indptr[0];
    st_->vectors.append(n, ip.data(), indices + indptr[0], codes.data());
}

size_t SeismicScalarQuantizedIndex::num_vectors() const {
    return static_cast<size_t>(st_->vectors.host.n());
}

void SeismicScalarQuantizedIndex::read_csr(const char* file_path, Residency residency) {
    if (residency == Residency::kMmap)
        throw std::invalid_argument(
            "mmap residency is not available for a quantized index: a mapped CSR is borrowed as "
            "float, and this index searches over codes");
    Index::read_csr(file_path, residency);
}

void SeismicScalarQuantizedIndex::build() {
    detail::seismic_build(*st_, dimension_, cluster_parameter_);
}

// seismic_scalar_quantized_index.cpp:182-191.
ScalarQuantizer SeismicScalarQuantizedIndex::query_quantizer(const SearchParameters* p) const {
    const auto* sqp = dynamic_cast<const SeismicSQSearchParameters*>(p);
    if (sqp == nullptr) return sq_;
    return ScalarQuantizer(sq_.get_quantizer_type(), sqp->vmin, sqp->vmax);
}

void SeismicScalarQuantizedIndex::search_impl(idx_t n, const idx_t* indptr,
                                              const term_t* indices, const float* values, int k,
                                              float* distances, idx_t* labels,
                                              SearchParameters* params) {
    const ScalarQuantizer qsq = query_quantizer(params);
    nsp::SeismicSearchArgs a = seismic_args(params, k);
    a.qbits = sq_.bits();
    a.q_vmin = qsq.get_min();
    a.q_scale = qsq.encode_scale();
    a.decode_scale = sq_.decode_scale(qsq);
    detail::seismic_search_common(*st_, dimension_, n, indptr, indices, values, k, distances,
                                  labels, params, a);
}

// ------------------------------------------------------ device-resident --

namespace detail {

void search_device(Index* index, int32_t n, const int32_t* d_indptr, const uint16_t* d_idx,
                   const float* d_val, int32_t max_nnz, int k, float* d_out, int32_t* d_lab,
                   SearchParameters* params, cudaStream_t s) {
    throw_if_not_positive(n);
    throw_if_not_positive(k);
    throw_if_any_null(d_indptr, d_idx, d_val, d_out, d_lab);
    SeismicState* st = nullptr;
    nsp::SeismicSearchArgs a = seismic_args(params, k);
    if (auto* si = dynamic_cast<SeismicIndex*>(index)) {
        st = si->state();
    } else if (auto* qi = dynamic_cast<SeismicScalarQuantizedIndex*>(index)) {
        st = qi->state();
        const auto* sqp = dynamic_cast<const SeismicSQSearchParameters*>(params);
        const ScalarQuantizer& isq = qi->get_scalar_quantizer();
        const ScalarQuantizer qsq =
            sqp == nullptr ? isq : ScalarQuantizer(isq.get_quantizer_type(), sqp->vmin, sqp->vmax);
        a.qbits = isq.bits();
        a.q_vmin = qsq.get_min();
        a.q_scale = qsq.encode_scale();
        a.decode_scale = isq.decode_scale(qsq);
    } else {
        throw std::invalid_argument("device-resident search supports seismic indexes");
    }
    if (st->vectors.host.n() == 0) throw std::runtime_error("index is empty");
    if (max_nnz < 0) throw std::invalid_argument("max_row_nnz must not be negative");
    apply_tuned(*st, a, n);
    const IDSelector* sel = params == nullptr ? nullptr : params->get_id_selector();
    if (exact_match_selector(sel, k) != nullptr)
        throw std::invalid_argument("device-resident search does not take the exact-match path");
    st->vectors.ensure_device();
    st->ensure_lists();
    nsp::Workspace& ws = nsp::Workspace::get();
    if (s == nullptr) s = ws.stream();
    const void* vals = d_val;
    if (a.qbits != 0) {
        int32_t last = 0;
        nsp::cuda_check(cudaMemcpyAsync(&last, d_indptr + n, sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, s), "D2H");
        nsp::cuda_check(cudaStreamSynchronize(s), "sync");
        void* codes = ws.dev(nsp::Workspace::kQCode, static_cast<size_t>(last) * 2 + 16);
        nsp::cuda_check(nsp::launch_sq_encode(d_val, codes, last, a.qbits, a.q_vmin, a.q_scale, s),
                        "query encode");
        vals = codes;
    }
    const uint64_t* d_sel = nullptr;
    if (sel != nullptr) {
        const std::vector<uint64_t> bits = selector_bitmap(sel, st->vectors.host.n());
        auto* d = static_cast<uint64_t*>(ws.dev(nsp::Workspace::kSel, bits.size() * 8));
        nsp::cuda_check(cudaMemcpyAsync(d, bits.data(), bits.size() * 8, cudaMemcpyHostToDevice, s),
                        "H2D selector");
        nsp::cuda_check(cudaStreamSynchronize(s), "sync");
        d_sel = d;
    }
    nsp::seismic_search_device(st->vectors.dev, st->lists_dev, n, d_indptr, d_idx, vals, max_nnz,
                               a, d_sel, d_out, d_lab, s, nullptr);
}

IndexSearchGraph::IndexSearchGraph(Index* index, int32_t n, int32_t nnz_cap, int32_t max_nnz,
                                   int k, SearchParameters* params,
                                   const nsp::GraphBuffers* bind) {
    throw_if_not_positive(n);
    throw_if_not_positive(k);
    if (nnz_cap < 0 || max_nnz < 0) throw std::invalid_argument("nnz must not be negative");
    if (dynamic_cast<IDMapIndex*>(index) != nullptr)
        throw std::invalid_argument("a search graph runs on a seismic index, not an IDMapIndex");
    nsp::SeismicSearchArgs a;
    st_ = resolve_seismic(index, params, k, a);
    dim_ = index->get_dimension();
    if (st_->vectors.host.n() == 0) throw std::runtime_error("index is empty");
    apply_tuned(*st_, a, n);
    const IDSelector* sel = params == nullptr ? nullptr : params->get_id_selector();
    if (exact_match_selector(sel, k) != nullptr)
        throw std::invalid_argument("a search graph does not take the exact-match path");
    st_->vectors.ensure_device();
    st_->ensure_lists();
    std::vector<uint64_t> bits;
    if (sel != nullptr) bits = selector_bitmap(sel, st_->vectors.host.n());
    fwd_gen_ = st_->vectors.dev.generation();
    ix_gen_ = st_->lists_dev.generation();
    g_ = std::make_unique<nsp::SearchGraph>(st_->vectors.dev, st_->lists_dev, a, n, nnz_cap,
                                            max_nnz, sel != nullptr ? &bits : nullptr, bind);
}

void IndexSearchGraph::ensure_current() const {
    if (st_->vectors.dirty || st_->vectors.dev.generation() != fwd_gen_ ||
        st_->lists_dev.generation() != ix_gen_)
        throw std::runtime_error(
            "the index changed since the search graph was captured; capture a new one");
}

void IndexSearchGraph::launch(cudaStream_t s) {
    ensure_current();
    g_->launch(s == nullptr ? g_->stream() : s);
}

void IndexSearchGraph::sync(cudaStream_t s) {
    nsp::SearchStats st;
    g_->check(s == nullptr ? g_->stream() : s, &st);
    record_stats(st);
}

void IndexSearchGraph::search(idx_t n, const idx_t* indptr, const term_t* indices,
                              const float* values, float* distances, idx_t* labels) {
    throw_if_not_positive(n);
    throw_if_any_null(indptr, indices, values, distances, labels);
    ensure_current();
    const nsp::QueryBatch q = nsp::canonicalize(n, indptr, indices, values, dim_);
    nsp::SearchStats st;
    g_->search_host(q, distances, labels, &st);
    record_stats(st);
}

SeismicState* resolve_seismic(Index* index, SearchParameters* params, int k,
                              nsp::SeismicSearchArgs& a) {
    if (auto* im = dynamic_cast<IDMapIndex*>(index)) index = im->delegate();
    a = seismic_args(params, k);
    if (auto* si = dynamic_cast<SeismicIndex*>(index)) return si->state();
    if (auto* qi = dynamic_cast<SeismicScalarQuantizedIndex*>(index)) {
        const auto* sqp = dynamic_cast<const SeismicSQSearchParameters*>(params);
        const ScalarQuantizer& isq = qi->get_scalar_quantizer();
        const ScalarQuantizer qsq =
            sqp == nullptr ? isq : ScalarQuantizer(isq.get_quantizer_type(), sqp->vmin, sqp->vmax);
        a.qbits = isq.bits();
        a.q_vmin = qsq.get_min();
        a.q_scale = qsq.encode_scale();
        a.decode_scale = isq.decode_scale(qsq);
        return qi->state();
    }
    throw std::invalid_argument("this operation applies to seismic indexes");
}

nsp::KernelChoice seismic_autotune(Index* index, idx_t n, const idx_t* indptr,
                                   const term_t* indices, const float* values, int k,
                                   SearchParameters* params) {
    throw_if_not_positive(n);
    throw_if_not_positive(k);
    throw_if_any_null(indptr, indices, values);
    nsp::SeismicSearchArgs a;
    SeismicState* st = resolve_seismic(index, params, k, a);
    if (auto* im = dynamic_cast<IDMapIndex*>(index)) index = im->delegate();
    if (st->vectors.host.n() == 0) throw std::runtime_error("index is empty");
    st->vectors.ensure_device();
    st->ensure_lists();
    const nsp::QueryBatch q = nsp::canonicalize(n, indptr, indices, values, index->get_dimension());
    std::vector<float> d(static_cast<size_t>(n) * k);
    std::vector<idx_t> l(static_cast<size_t>(n) * k);
    nsp::KernelChoice best;
    for (int variant = 2; variant <= 5; ++variant) {
        for (int batch : {256, 512, 640, 1024}) {
            for (int warps : {4, 8}) {
                nsp::SeismicSearchArgs t = a;
                t.variant = variant;
                t.batch_docs = batch;
                t.warps_per_block = warps;
                t.plain = false;
                float ms = 0.0f;
                for (int rep = 0; rep < 2; ++rep) {  // the first run warms caches
                    nsp::SearchStats s;
                    nsp::seismic_search(st->vectors.dev, st->lists_dev, q, t, nullptr, d.data(),
                                        l.data(), &s);
                    ms = s.kernel_ms;
                }
                if (best.variant < 0 || ms < best.kernel_ms) {
                    best.variant = variant;
                    best.batch_docs = batch;
                    best.warps_per_block = warps;
                    best.kernel_ms = ms;
                }
            }
        }
    }
    // CTAs per query for one-query launches (the latency of a lone query):
    // the fastest of 1, 2, 4, 8 over up to 16 of the sample's queries, each
    // searched alone with the chosen lanes per doc
    const int n1 = std::min<int>(n, 16);
    float best_ms = 0.0f;
    for (int split : {1, 2, 4, 8}) {
        nsp::SeismicSearchArgs t = a;
        t.variant = best.variant;
        t.plain = true;
        t.cluster = split;
        float total = 0.0f;
        for (int rep = 0; rep < 2; ++rep) {  // the first pass warms caches
            total = 0.0f;
            for (int i = 0; i < n1; ++i) {
                nsp::QueryBatch one;
                one.n = 1;
                one.indptr = {0, q.ip[i + 1] - q.ip[i]};
                one.idx.assign(q.ix + q.ip[i], q.ix + q.ip[i + 1]);
                one.val.assign(q.vv + q.ip[i], q.vv + q.ip[i + 1]);
                one.max_nnz = one.indptr[1];
                one.ip = one.indptr.data();
                one.ix = one.idx.data();
                one.vv = one.val.data();
                nsp::SearchStats s;
                nsp::seismic_search(st->vectors.dev, st->lists_dev, one, t, nullptr, d.data(),
                                    l.data(), &s);
                total += s.kernel_ms;
            }
        }
        if (best.split == 0 || total < best_ms) {
            best.split = split;
            best_ms = total;
        }
    }
    std::lock_guard<std::mutex> g(st->mu);
    st->tuned = best;
    return best;
}

}  // namespace detail

// ------------------------------------------------------------- IDMap -----

// The base keeps dimension 0, as the reference's constructor leaves it
// (id_map_index.cpp:27); files record it in the IDMP header.
IDMapIndex::IDMapIndex(Index* delegate) : Index(0), delegate_(delegate) {}

void IDMapIndex::add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) {
    delegate_->add(n, indptr, indices, values);
}

void IDMapIndex::build() { delegate_->build(); }

size_t IDMapIndex::num_vectors() const { return delegate_ == nullptr ? 0 : delegate_->num_vectors(); }

// id_map_index.cpp:70-80.
void IDMapIndex::add_with_ids(idx_t n, const idx_t* indptr, const term_t* indices,
                              const float* values, const idx_t* ids) {
    const size_t old = delegate_->num_vectors();
    delegate_->add(n, indptr, indices, values);
    std::vector<int64_t> wide(ids, ids + (n > 0 ? n : 0));
    map_ids(old, n, wide.data());
}

void IDMapIndex::add_with_ids64(idx_t n, const idx_t* indptr, const term_t* indices,
                                const float* values, const int64_t* ids) {
    if (n > 0 && ids == nullptr) throw std::invalid_argument("unexpected nullptr");
    const size_t old = delegate_->num_vectors();
    delegate_->add(n, indptr, indices, values);
    map_ids(old, n, ids);
}

void IDMapIndex::map_ids(size_t first, idx_t n, const int64_t* ids) {
    internal_to_external_.resize(first + (n > 0 ? n : 0));
    for (idx_t i = 0; i < n; ++i) {
        internal_to_external_[first + i] = ids[i];
        external_to_internal_[ids[i]] = static_cast<idx_t>(first + i);
        wide_ = wide_ || ids[i] < INT32_MIN || ids[i] > INT32_MAX;
    }
}

// id_map_index.cpp:29-60. The caller's selector is restored on return (the
// reference leaves the translated one in place).
void IDMapIndex::search_internal(idx_t n, const idx_t* indptr, const term_t* indices,
                                 const float* values, int k, float* distances, idx_t* labels,
                                 SearchParameters* params) {
    std::unique_ptr<IDSelector> wrapped;
    IDSelector* original = nullptr;
    if (params != nullptr && params->get_id_selector() != nullptr) {
        original = const_cast<IDSelector*>(params->get_id_selector());
        if (const auto* en = dynamic_cast<const IDSelectorEnumerable*>(original)) {
            wrapped.reset(new detail::IDSelectorEnumerableWithIDMap(en, internal_to_external_,
                                                                    external_to_internal_));
        } else {
            wrapped.reset(new detail::IDSelectorWithIDMap(original, internal_to_external_,
                                                          external_to_internal_));
        }
        params->set_id_selector(wrapped.get());
    }
    try {
        delegate_->search(n, indptr, indices, values, k, distances, labels, params);
    } catch (...) {
        if (original != nullptr) params->set_id_selector(original);
        throw;
    }
    if (original != nullptr) params->set_id_selector(original);
}

void IDMapIndex::search(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                        int k, float* distances, idx_t* labels, SearchParameters* params) {
    if (wide_)
        throw std::invalid_argument(
            "external ids need 64 bits: search with search64 (32-bit labels cannot hold them)");
    search_internal(n, indptr, indices, values, k, distances, labels, params);
    const size_t cnt = static_cast<size_t>(n) * k;
    for (size_t i = 0; i < cnt; ++i) {
        if (labels[i] >= 0) labels[i] = static_cast<idx_t>(internal_to_external_[labels[i]]);
    }
}

void IDMapIndex::search64(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                          int k, float* distances, int64_t* labels, SearchParameters* params) {
    if (labels == nullptr) throw std::invalid_argument("unexpected nullptr");
    if (n <= 0 || k <= 0) {
        // the delegate raises the reference's argument errors
        search_internal(n, indptr, indices, values, k, distances, nullptr, params);
        return;
    }
    std::vector<idx_t> internal(static_cast<size_t>(n) * k);
    search_internal(n, indptr, indices, values, k, distances, internal.data(), params);
    for (size_t i = 0; i < internal.size(); ++i)
        labels[i] = internal[i] >= 0 ? internal_to_external_[internal[i]] : -1;
}

// ------------------------------------------------------------ factory ----

namespace {
std::vector<std::string> split(const std::string& s, char d) {
    std::vector<std::string> out;
    size_t start = 0, end = s.find(d);
    while (end != std::string::npos) {
        out.push_back(s.substr(start, end - start));
        start = end + 1;
        end = s.find(d, start);
    }
    out.push_back(s.substr(start));
    return out;
}
std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\n\r");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\n\r");
    return s.substr(a, b - a + 1);
}
}  // namespace

// index_factory.cpp:63-153: same grammar and defaults (lambda=10, beta=5,
// alpha=0.5, seed=-1; seismic_sq quantizer=8bit, vmin=0, vmax=1).
Index* index_factory(int dimension, const char* description) {
    if (description == nullptr || std::strlen(description) == 0)
        throw std::invalid_argument("Description cannot be null or empty");
    const std::string desc(description);
    const auto segments = split(desc, ',');
    const std::string type = trim(segments[0]);
    std::vector<std::pair<std::string, std::string>> params;
    if (segments.size() > 1) {
        for (const auto& tok : split(segments[1], '|')) {
            const auto kv = split(tok, '=');
            if (kv.size() == 2) params.emplace_back(trim(kv[0]), trim(kv[1]));
        }
    }
    auto get = [&](const std::string& key, const std::string& def) {
        for (const auto& [k, v] : params)
            if (k == key) return v;
        return def;
    };
    if (type == "brutal") return new BrutalIndex(dimension);
    if (type == "inverted") return new InvertedIndex(dimension);
    if (type == "seismic") {
        SeismicClusterParameters p{std::stoi(get("lambda", "10")), std::stoi(get("beta", "5")),
                                   std::stof(get("alpha", "0.5"))};
        p.seed = std::stoi(get("seed", std::to_string(kRandomSeed)));
        return new SeismicIndex(dimension, p);
    }
    if (type == "seismic_sq") {
        const std::string qs = get("quantizer", "8bit");
        const QuantizerType qt = qs == "16bit" ? QuantizerType::QT_16bit : QuantizerType::QT_8bit;
        const float vmin = std::stof(get("vmin", "0.0"));
        const float vmax = std::stof(get("vmax", "1.0"));
        SeismicClusterParameters p{std::stoi(get("lambda", "10")), std::stoi(get("beta", "5")),
                                   std::stof(get("alpha", "0.5"))};
        p.seed = std::stoi(get("seed", std::to_string(kRandomSeed)));
        return new SeismicScalarQuantizedIndex(qt, vmin, vmax, p, dimension);
    }
    if (type == "idmap") {
        if (segments.size() < 2) throw std::invalid_argument("idmap requires a delegate index type");
        std::string dd;
        for (size_t i = 1; i < segments.size(); ++i) {
            if (i > 1) dd += ",";
            dd += segments[i];
        }
        return new IDMapIndex(index_factory(dimension, dd.c_str()));
    }
    throw std::invalid_argument("Unknown index type: " + type);
}

}  // namespace nsparse
