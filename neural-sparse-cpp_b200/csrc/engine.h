// Host-side engine internals: device buffers, per-thread streams and scratch,
// the device-resident forward index and SEISMIC lists, and the search drivers
// that launch the kernels of search_*.cu. Internal to libnsparse_b200.so.
#ifndef NSP_ENGINE_H
#define NSP_ENGINE_H

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "nsp_device.h"

namespace nsp {

// Throws std::runtime_error("CUDA error in <what>: <name>") on failure.
void cuda_check(cudaError_t e, const char* what);

int device_sm_count();

// Owning device array (cudaMalloc / cudaFree).
template <class T>
class DevArray {
public:
    DevArray() = default;
    explicit DevArray(size_t n) { resize(n); }
    ~DevArray() { reset(); }
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    DevArray(DevArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DevArray& operator=(DevArray&& o) noexcept {
        if (this != &o) {
            reset();
            p_ = o.p_;
            n_ = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void resize(size_t n) {
        reset();
        if (n > 0) {
            void* p = nullptr;
            cuda_check(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
            p_ = static_cast<T*>(p);
            n_ = n;
        }
    }
    void reset() {
        if (p_ != nullptr) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    void upload(const T* h, size_t n, cudaStream_t s) {
        if (n_ < n) resize(n);
        if (n > 0)
            cuda_check(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s), "H2D");
    }
    void download(T* h, size_t n, cudaStream_t s) const {
        if (n > 0)
            cuda_check(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s), "D2H");
    }
    // Capacity for at least n elements, contents not kept; never shrinks.
    void grow(size_t n) {
        if (n_ < n) resize(n + n / 8);
    }
    T* data() { return p_; }
    const T* data() const { return p_; }
    size_t size() const { return n_; }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

// Device scratch by slot, grow-only: the per-thread Workspace, or the
// buffers a captured search graph owns.
class Scratch {
public:
    virtual void* dev(int slot, size_t bytes) = 0;

protected:
    ~Scratch() = default;
};

// Per-thread stream plus grow-only device and pinned scratch, so concurrent
// searches from several host threads never share buffers (the reference's
// per-thread scratch, seismic_index.cpp:197-201).
class Workspace : public Scratch {
public:
    enum Slot : int {
        kQIndptr, kQIdx, kQVal, kQCode, kOutD, kOutL, kSel, kBScore, kCounter, kStats,
        kCandD, kCandL, kHeapD, kHeapL, kQValG, kIds, kErr, kOrder, kSortKeys, kVisit, kQOrder,
        kNumSlots
    };
    static Workspace& get();
    cudaStream_t stream() const { return stream_; }
    void* dev(int s, size_t bytes) override;
    void* pinned(Slot s, size_t bytes);
    ~Workspace();

private:
    Workspace();
    cudaStream_t stream_ = nullptr;
    int device_ = 0;
    void* dptr_[kNumSlots] = {};
    size_t dcap_[kNumSlots] = {};
    void* hptr_[kNumSlots] = {};
    size_t hcap_[kNumSlots] = {};
};

// Host CSR in the reference's SparseVectors layout (sparse_vectors.h:23-111):
// int32 row offsets, uint16 terms, values as raw bytes of width esz.
struct HostCsr {
    int dim = 0;
    int esz = 4;
    std::vector<int32_t> indptr{0};
    std::vector<uint16_t> indices;
    std::vector<uint8_t> values;

    int64_t n() const { return static_cast<int64_t>(indptr.size()) - 1; }
    int64_t nnz() const { return indptr.back(); }
    // SparseVectors::add_vectors (sparse_vectors.cpp:92-126): append and rebase.
    void append(int32_t n, const int32_t* ip, const uint16_t* idx, const uint8_t* vals);
};

class ForwardDevice {
public:
    // Builds the padded layout (nsp_device.h) and uploads it.
    void upload(const HostCsr& h);
    FwdView view() const;
    bool empty() const { return n_docs_ == 0; }
    int32_t n_docs() const { return n_docs_; }
    int esz() const { return esz_; }
    size_t device_bytes() const;
    // Changes with every upload (row offsets move).
    uint64_t generation() const { return generation_; }

private:
    uint64_t generation_ = 0;
    int32_t n_docs_ = 0;
    int dim_ = 0;
    int esz_ = 4;
    DevArray<uint2> rowinfo_;
    DevArray<uint16_t> idx_;
    DevArray<uint8_t> val_;
};

// Doc-ascending postings of an fp32 forward index for the exact search's
// term-at-a-time path (nsp_device.h, PostingsView), built on the device from
// the resident rows. Usable only when every row holds strictly ascending
// terms: then a doc's products, applied term by term, arrive in row order.
class PostingsDevice {
public:
    // (Re)builds from `fwd` for doc chunks of `chunk_docs`.
    void build(const ForwardDevice& fwd, int chunk_docs);
    bool usable() const { return usable_; }
    uint64_t generation() const { return generation_; }  // of the forward index it mirrors
    PostingsView view() const;
    size_t device_bytes() const;

private:
    uint64_t generation_ = 0;
    bool usable_ = false;
    int32_t n_chunks_ = 0;
    int32_t chunk_docs_ = 0;
    DevArray<int32_t> doc_;
    DevArray<float> val_;
    DevArray<int32_t> chunk_at_;
};

// SEISMIC lists flattened over terms, in host memory (the reference's
// InvertedListClusters fields per list, cluster/inverted_list_clusters.h:75-84).
struct SeismicHost {
    int esz = 4;
    std::vector<int64_t> lbp{0};     // blocks per list (prefix)
    std::vector<int64_t> bdp{0};     // docs per block (prefix)
    std::vector<int32_t> docs;
    std::vector<int64_t> ltp{0};     // summary columns per list (prefix)
    std::vector<uint16_t> sterm;     // column term, ascending within a list
    std::vector<int64_t> srun{0};    // entries per column (prefix)
    std::vector<uint16_t> sblk;      // block id local to the list
    std::vector<uint8_t> sval;       // value bytes, width esz
    int32_t n_lists() const { return static_cast<int32_t>(lbp.size()) - 1; }
};

class SeismicDevice {
public:
    void upload(const SeismicHost& h, int dim);
    // Takes lists built on the device: the offset arrays come from the host,
    // the per-posting and per-entry arrays are moved in (their capacity may
    // exceed what the offsets use).
    void adopt(const std::vector<int64_t>& lbp, const std::vector<int64_t>& bdp,
               const std::vector<int64_t>& ltp, int esz, int dim, DevArray<int32_t>&& docs,
               DevArray<uint16_t>&& sterm, DevArray<int64_t>&& srun, DevArray<uint16_t>&& sblk,
               DevArray<uint8_t>&& sval);
    void download(SeismicHost& h) const;
    SeismicView view() const;
    bool empty() const { return n_lists_ == 0; }
    int32_t max_blocks() const { return max_blocks_; }
    size_t device_bytes() const;
    // Copies each posting's forward-row info {start/16, length} next to its
    // doc id (drow), so a block's candidates are read contiguously instead of
    // through one random row-info load each; redone when `fwd` was
    // re-uploaded since.
    void bind_rows(const ForwardDevice& fwd, cudaStream_t s);

private:
    friend struct SeismicBuilder;
    int32_t n_lists_ = 0;
    int32_t words_ = 0;
    int32_t max_blocks_ = 0;
    int esz_ = 4;
    DevArray<int64_t> lbp_, bdp_, ltp_, srun_;
    DevArray<uint16_t> sterm_;
    DevArray<int32_t> docs_;
    DevArray<uint2> lmeta_;
    DevArray<uint16_t> sblk_;
    DevArray<uint8_t> sval_;
    DevArray<uint2> drow_;
    uint64_t drow_gen_ = 0;  // generation of the forward index drow_ reflects
    uint64_t generation_ = 0;

public:
    // Changes whenever a device array of the lists is replaced.
    uint64_t generation() const { return generation_; }
};

// A host query batch in canonical form (terms ascending and unique per row;
// a repeated term keeps its last value, as the reference's dense scatter
// does, sparse_vectors.cpp:157-177).
struct QueryBatch {
    int32_t n = 0;
    std::vector<int32_t> indptr;
    std::vector<uint16_t> idx;
    std::vector<float> val;
    int32_t max_nnz = 0;
    const int32_t* ip = nullptr;     // points at the caller's arrays when
    const uint16_t* ix = nullptr;    // they are canonical already
    const float* vv = nullptr;
};
QueryBatch canonicalize(int32_t n, const int32_t* indptr, const uint16_t* idx, const float* val,
                        int dim);

struct SearchStats {
    unsigned long long docs_scored = 0;
    unsigned long long blocks_visited = 0;
    unsigned long long bytes = 0;
    unsigned long long lists_probed = 0;
    float kernel_ms = 0.0f;
    int launches = 0;
    unsigned long long row_bytes = 0;         // rows' share of `bytes`
    unsigned long long unique_docs = 0;       // counting pass only
    unsigned long long unique_row_bytes = 0;  // counting pass only
};

// A SEISMIC kernel launch shape chosen by the autotuner (variant < 0: none).
struct KernelChoice {
    int variant = -1;
    int batch_docs = 0;
    int warps_per_block = 0;
    float kernel_ms = 0.0f;  // on the tuning sample
    int split = 0;           // CTAs per query of one-query launches (0: the engine's rule)
};

// CTAs per query the engine gives a launch of `n_queries` queries: the most
// of 1, 2, 4, 8 that still gives every query its own SMs (n * c <= SM count),
// so a launch of few queries spreads each over a thread-block cluster; large
// launches keep one CTA per query.
int auto_cluster(int n_queries);

struct SeismicSearchArgs {
    int k = 10;
    int cut = 10;
    float heap_factor = 1.0f;
    int qbits = 0;            // 0: fp32 index; 8/16: quantized index
    float q_vmin = 0.0f;      // query quantizer
    float q_scale = 0.0f;     // kMax / (vmax - vmin) of the query quantizer
    float decode_scale = 0.0f;
    bool plain = false;       // one query per launch
    int warps_per_block = 0;  // 0 = autotuned
    int variant = -1;         // -1 auto, 0 direct row loads, 1 bulk-copy staged rows,
                              // 2-5 one CTA per query with 1, 2, 4, 8 lanes per doc
    int stage_bytes = 0;      // staged: bytes per stage buffer (0 = default)
    int batch_docs = 0;       // variants 2-5: candidate docs per batch (0 = default)
    int cluster = 0;          // variants 2-5: CTAs per query (0 = engine's choice, 1, 2, 4, 8)
    // variants 2-5: one device doc bitmap per query (a null entry admits every
    // doc), in device memory; replaces the launch-wide selector
    const uint64_t* const* d_sel_q = nullptr;
    int max_ctas = 0;         // cap on the persistent grid's CTAs (0: none)
    // variants 2-5, batched: count each scored doc's row once per query, as
    // the reference's visited set does (a slower counting pass: one stamp per
    // doc per CTA, on a grid of one CTA per SM)
    bool count_unique = false;
    int32_t nnz_cap = -1;     // entries the query arrays hold (negative: not checked)
    // variants 2-5: per query, set to 1 once its results are written (see
    // seismic_search_start), or nullptr
    int32_t* d_done = nullptr;
};

// Device scratch a batched (not plain) run_seismic of `n` queries with `args`
// asks for: `fixed` bytes whatever the grid, plus `per_cta` for each of the
// `ctas` CTAs of its grid (a whole number of `cluster`-CTA clusters).
struct SeismicScratchNeed {
    size_t fixed = 0;
    size_t per_cta = 0;
    int ctas = 0;
    int cluster = 1;
};
SeismicScratchNeed seismic_scratch_need(const ForwardDevice& fwd, const SeismicDevice& ix,
                                        int32_t n, int32_t max_nnz, const SeismicSearchArgs& args);

// Host queries in; results written by the kernel straight to `out_d` /
// `out_l` (addresses the device can write and the host can read: mapped
// pinned memory), done[i] set to 1 after query i's -- so a caller can take
// each query's results as it finishes. Returns once the launch is queued on
// this thread's stream; seismic_search_wait() then waits for it and raises
// the kernel's errors. Batched one-CTA-per-query kernels only.
void seismic_search_start(const ForwardDevice& fwd, const SeismicDevice& ix, const QueryBatch& q,
                          const SeismicSearchArgs& args, float* out_d, int32_t* out_l,
                          int32_t* done);
void seismic_search_wait();

// Host buffers in, host buffers out (the reference-facing path).
void seismic_search(const ForwardDevice& fwd, const SeismicDevice& ix, const QueryBatch& q,
                    const SeismicSearchArgs& args, const std::vector<uint64_t>* sel_bits,
                    float* out_d, int32_t* out_l, SearchStats* stats);

// `post` (may be null): the forward index's postings; the term-at-a-time
// kernel runs when they are usable and k <= kTaatMaxK, else the tile kernel.
void exact_search(const ForwardDevice& fwd, const PostingsDevice* post, const QueryBatch& q, int k,
                  int mode, const std::vector<uint64_t>* sel_bits, float* out_d, int32_t* out_l,
                  SearchStats* stats);

void exact_list_search(const ForwardDevice& fwd, const QueryBatch& q, const SeismicSearchArgs& args,
                       const std::vector<int32_t>& ids, float* out_d, int32_t* out_l);

// Enqueues one SEISMIC search on `s`, its scratch drawn from `scratch`. With
// `stats` null nothing on the host waits for the device (so the call can be
// captured into a CUDA graph); else it waits and fills the kernel's time and
// counters.
void run_seismic(const ForwardDevice& fwd, const SeismicDevice& ix, int32_t n,
                 const int32_t* d_indptr, const uint16_t* d_idx, const void* d_vals, int32_t qcap,
                 const SeismicSearchArgs& args, const uint64_t* d_sel, float* d_out,
                 int32_t* d_lab, cudaStream_t s, Scratch& scratch, SearchStats* stats);

// Grows the calling thread's workspace to what seismic_search of `n`
// queries of up to `max_nnz` terms with `args` asks for, so a later search
// within those bounds allocates nothing (growing a buffer frees the old one,
// and cudaFree waits for the whole device).
void reserve_seismic_scratch(const ForwardDevice& fwd, const SeismicDevice& ix, int32_t n,
                             int32_t max_nnz, const SeismicSearchArgs& args);

// Device-resident variant: queries, outputs and stream owned by the caller.
void seismic_search_device(const ForwardDevice& fwd, const SeismicDevice& ix, int32_t n,
                           const int32_t* d_indptr, const uint16_t* d_idx, const void* d_val,
                           int32_t max_nnz, const SeismicSearchArgs& args, const uint64_t* d_sel,
                           float* d_out, int32_t* d_lab, cudaStream_t s, SearchStats* stats);

// Device buffers of a captured search step: the queries in CSR form (`n`
// rows, room for `nnz_cap` entries; rows with terms ascending and unique) and
// the results (n x k, row-major).
struct GraphBuffers {
    int32_t* indptr = nullptr;
    uint16_t* indices = nullptr;
    float* values = nullptr;
    float* distances = nullptr;
    int32_t* labels = nullptr;
};

// One batched SEISMIC search step captured once as a CUDA graph and replayed
// for every batch: the resets of the step's counters, the query encode of a
// quantized index and the persistent search kernel run as one graph launch on
// buffers fixed at capture. The scratch belongs to the graph, so replays need
// no allocation and no host synchronisation. One step of a graph is in flight
// at a time (its launches are ordered on the stream they are given).
class SearchGraph {
public:
    // `bind`: the caller's device buffers for queries and results (kept alive
    // by the caller), or null for buffers the graph allocates. `sel_bits`: a
    // doc bitmap every query of every step is filtered by, or null.
    SearchGraph(const ForwardDevice& fwd, const SeismicDevice& ix, const SeismicSearchArgs& args,
                int32_t n, int32_t nnz_cap, int32_t qcap, const std::vector<uint64_t>* sel_bits,
                const GraphBuffers* bind);
    ~SearchGraph();
    SearchGraph(const SearchGraph&) = delete;
    SearchGraph& operator=(const SearchGraph&) = delete;

    const GraphBuffers& buffers() const { return buf_; }
    int32_t n() const { return n_; }
    int32_t nnz_cap() const { return nnz_cap_; }
    int32_t qcap() const { return qcap_; }
    int k() const { return args_.k; }
    cudaStream_t stream() const { return stream_; }
    // Replays the step on `s`, after the work already queued there.
    void launch(cudaStream_t s);
    // Waits for `s` and raises if the kernel flagged an error (as the
    // ordinary search does); `stats` (optional) gets the step's counters.
    void check(cudaStream_t s, SearchStats* stats = nullptr);
    // Host queries in (canonical, at most n rows), host results out: staged
    // copies and one graph launch on the graph's own stream.
    void search_host(const QueryBatch& q, float* out_d, int32_t* out_l,
                     SearchStats* stats = nullptr);

private:
    struct Owned;
    void enqueue(cudaStream_t s);
    const ForwardDevice& fwd_;
    const SeismicDevice& ix_;
    SeismicSearchArgs args_;
    int32_t n_, nnz_cap_, qcap_;
    GraphBuffers buf_;
    std::unique_ptr<Owned> own_;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t done_ = nullptr;  // recorded after each launch
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
};

}  // namespace nsp

#endif  // NSP_ENGINE_H
