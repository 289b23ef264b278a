// A batched SEISMIC search step captured as a CUDA graph (engine.h,
// SearchGraph). The step the engine otherwise issues call by call -- the
// memsets of the kernel's counters and error flag, the work-stealing counter
// reset, the query encode of a quantized index and the persistent search
// kernel -- is recorded once into a graph over buffers fixed at capture and
// then replayed with one cudaGraphLaunch per batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

#include "engine.h"
#include "nsp_device.h"

namespace nsp {

namespace {

// The graph's own scratch. It grows only before capture (the warm-up step
// sizes it); a request to grow while frozen would mean the captured step
// differs from the warm-up one and is an error, not an allocation.
class GraphScratch final : public Scratch {
public:
    void* dev(int slot, size_t bytes) override {
        if (slot < 0 || slot >= Workspace::kNumSlots) throw std::logic_error("bad scratch slot");
        if (bytes == 0) bytes = 16;
        DevArray<uint8_t>& a = slots_[slot];
        if (a.size() < bytes) {
            if (frozen_) throw std::logic_error("search graph scratch grew after capture");
            a.resize(bytes);
        }
        return a.data();
    }
    void freeze() { frozen_ = true; }

private:
    DevArray<uint8_t> slots_[Workspace::kNumSlots];
    bool frozen_ = false;
};

void raise_kernel_error(int32_t h) {
    if (h == 1) throw std::runtime_error("search kernel gave up waiting for a bulk copy");
    if (h == 2) throw std::runtime_error("search kernel had no buffer to sort a list's blocks");
    if (h == 3) throw std::invalid_argument("a query row is longer than max_nnz");
    if (h != 0) throw std::runtime_error("search kernel reported an error");
}

}  // namespace

struct SearchGraph::Owned {
    GraphScratch scratch;
    DevArray<int32_t> indptr;
    DevArray<uint16_t> indices;
    DevArray<float> values;
    DevArray<float> distances;
    DevArray<int32_t> labels;
    DevArray<uint8_t> codes;   // encoded query values (quantized index)
    DevArray<uint64_t> sel;    // the step's doc bitmap
    // pinned staging of the host path
    int32_t* h_indptr = nullptr;
    uint16_t* h_idx = nullptr;
    float* h_val = nullptr;
    float* h_d = nullptr;
    int32_t* h_l = nullptr;
    int32_t* h_err = nullptr;
    ~Owned() {
        for (void* p : {static_cast<void*>(h_indptr), static_cast<void*>(h_idx),
                        static_cast<void*>(h_val), static_cast<void*>(h_d),
                        static_cast<void*>(h_l), static_cast<void*>(h_err)})
            if (p != nullptr) cudaFreeHost(p);
    }
};

SearchGraph::SearchGraph(const ForwardDevice& fwd, const SeismicDevice& ix,
                         const SeismicSearchArgs& args, int32_t n, int32_t nnz_cap, int32_t qcap,
                         const std::vector<uint64_t>* sel_bits, const GraphBuffers* bind)
    : fwd_(fwd), ix_(ix), args_(args), n_(n), nnz_cap_(nnz_cap), qcap_(std::max(qcap, 1)),
      own_(new Owned()) {
    if (n <= 0) throw std::invalid_argument("a search graph needs at least one query row");
    if (nnz_cap < 0) throw std::invalid_argument("nnz capacity must not be negative");
    if (args.plain) throw std::invalid_argument("a search graph runs the batched launch only");
    if (args.d_sel_q != nullptr)
        throw std::invalid_argument("a search graph takes one selector for the whole step");
    if (fwd.empty()) throw std::invalid_argument("index is empty");
    const size_t cnt = static_cast<size_t>(n) * args.k;
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    try {
        cuda_check(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "event");
        if (bind != nullptr) {
            if (bind->indptr == nullptr || bind->indices == nullptr || bind->values == nullptr ||
                bind->distances == nullptr || bind->labels == nullptr)
                throw std::invalid_argument("unexpected nullptr");
            buf_ = *bind;
        } else {
            Owned& o = *own_;
            o.indptr.resize(static_cast<size_t>(n) + 1);
            o.indices.resize(static_cast<size_t>(nnz_cap) + 8);
            o.values.resize(static_cast<size_t>(nnz_cap) + 4);
            o.distances.resize(cnt);
            o.labels.resize(cnt);
            // every row starts empty: a replay before any queries are
            // written returns padding
            cuda_check(cudaMemsetAsync(o.indptr.data(), 0, (n + 1) * sizeof(int32_t), stream_),
                       "memset");
            cuda_check(cudaMemsetAsync(o.indices.data(), 0, o.indices.size() * 2, stream_),
                       "memset");
            cuda_check(cudaMemsetAsync(o.values.data(), 0, o.values.size() * 4, stream_), "memset");
            buf_.indptr = o.indptr.data();
            buf_.indices = o.indices.data();
            buf_.values = o.values.data();
            buf_.distances = o.distances.data();
            buf_.labels = o.labels.data();
        }
        if (args_.qbits != 0) {
            own_->codes.resize(static_cast<size_t>(nnz_cap) * 2 + 16);
            cuda_check(cudaMemsetAsync(own_->codes.data(), 0, own_->codes.size(), stream_),
                       "memset");
        }
        if (sel_bits != nullptr) {
            own_->sel.resize(std::max<size_t>(sel_bits->size(), 1));
            cuda_check(cudaMemcpyAsync(own_->sel.data(), sel_bits->data(),
                                       sel_bits->size() * sizeof(uint64_t), cudaMemcpyHostToDevice,
                                       stream_),
                       "H2D selector");
        }
        // A caller's buffers may hold anything yet; the warm-up step reads
        // the graph's own (all-empty) rows instead when the caller bound
        // buffers, by running on a private empty batch.
        DevArray<int32_t> empty_rows;
        GraphBuffers keep = buf_;
        if (bind != nullptr) {
            empty_rows.resize(static_cast<size_t>(n) + 1);
            cuda_check(cudaMemsetAsync(empty_rows.data(), 0, (n + 1) * sizeof(int32_t), stream_),
                       "memset");
            buf_.indptr = empty_rows.data();
        }
        // warm-up: sizes the scratch, sets the kernels' attributes
        enqueue(stream_);
        check(stream_);
        buf_ = keep;
        own_->scratch.freeze();

        // relaxed: the launchers query device attributes and set the
        // kernels' shared-memory limit, which are not stream work
        cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed),
                   "begin capture");
        try {
            enqueue(stream_);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream_, &g);
            if (g != nullptr) cudaGraphDestroy(g);
            throw;
        }
        cuda_check(cudaStreamEndCapture(stream_, &graph_), "end capture");
        cuda_check(cudaGraphInstantiate(&exec_, graph_, 0), "graph instantiate");

        Owned& o = *own_;
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&o.h_indptr), (n + 1) * sizeof(int32_t),
                                 cudaHostAllocDefault),
                   "cudaHostAlloc");
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&o.h_idx),
                                 std::max<size_t>(nnz_cap, 1) * sizeof(uint16_t),
                                 cudaHostAllocDefault),
                   "cudaHostAlloc");
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&o.h_val),
                                 std::max<size_t>(nnz_cap, 1) * sizeof(float),
                                 cudaHostAllocDefault),
                   "cudaHostAlloc");
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&o.h_d), cnt * sizeof(float),
                                 cudaHostAllocDefault),
                   "cudaHostAlloc");
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&o.h_l), cnt * sizeof(int32_t),
                                 cudaHostAllocDefault),
                   "cudaHostAlloc");
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&o.h_err), 64, cudaHostAllocDefault),
                   "cudaHostAlloc");
    } catch (...) {
        if (exec_ != nullptr) cudaGraphExecDestroy(exec_);
        if (graph_ != nullptr) cudaGraphDestroy(graph_);
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
        if (done_ != nullptr) cudaEventDestroy(done_);
        throw;
    }
}

SearchGraph::~SearchGraph() {
    // The graph's buffers are freed after this; wait for the last step
    // launched, on whichever stream it went.
    cudaEventSynchronize(done_);
    cudaStreamSynchronize(stream_);
    cudaGraphExecDestroy(exec_);
    cudaGraphDestroy(graph_);
    cudaStreamDestroy(stream_);
    cudaEventDestroy(done_);
}

void SearchGraph::enqueue(cudaStream_t s) {
    const void* vals = buf_.values;
    if (args_.qbits != 0) {
        // the whole capacity is encoded: the graph cannot know a step's nnz,
        // and entries past it are never read
        cuda_check(launch_sq_encode(buf_.values, own_->codes.data(), nnz_cap_, args_.qbits,
                                    args_.q_vmin, args_.q_scale, s),
                   "query encode");
        vals = own_->codes.data();
    }
    run_seismic(fwd_, ix_, n_, buf_.indptr, buf_.indices, vals, qcap_, args_,
                own_->sel.size() > 0 ? own_->sel.data() : nullptr, buf_.distances, buf_.labels, s,
                own_->scratch, nullptr);
}

void SearchGraph::launch(cudaStream_t s) {
    cuda_check(cudaGraphLaunch(exec_, s), "graph launch");
    cuda_check(cudaEventRecord(done_, s), "event");
}

void SearchGraph::check(cudaStream_t s, SearchStats* stats) {
    auto* err = static_cast<int32_t*>(own_->scratch.dev(Workspace::kErr, sizeof(int32_t)));
    int32_t h = 0;
    int32_t* dst = own_->h_err != nullptr ? own_->h_err : &h;
    cuda_check(cudaMemcpyAsync(dst, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "D2H");
    unsigned long long c[kStatCount] = {};
    if (stats != nullptr) {
        auto* st = own_->scratch.dev(Workspace::kStats, kStatCount * sizeof(unsigned long long));
        cuda_check(cudaMemcpyAsync(c, st, sizeof(c), cudaMemcpyDeviceToHost, s), "D2H stats");
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
    h = *dst;
    if (stats != nullptr) {
        *stats = SearchStats{};
        stats->docs_scored = c[kStatDocsScored];
        stats->blocks_visited = c[kStatBlocksVisited];
        stats->bytes = c[kStatBytes];
        stats->lists_probed = c[kStatListsProbed];
        stats->launches = 1;
    }
    raise_kernel_error(h);
}

void SearchGraph::search_host(const QueryBatch& q, float* out_d, int32_t* out_l,
                              SearchStats* stats) {
    if (q.n > n_)
        throw std::invalid_argument("batch of " + std::to_string(q.n) +
                                    " queries exceeds the graph's " + std::to_string(n_) + " rows");
    const int32_t base = q.ip[0];
    const int64_t nnz = static_cast<int64_t>(q.ip[q.n]) - base;
    if (nnz > nnz_cap_)
        throw std::invalid_argument("batch of " + std::to_string(nnz) +
                                    " query entries exceeds the graph's capacity of " +
                                    std::to_string(nnz_cap_));
    if (q.max_nnz > qcap_) throw std::invalid_argument("a query row is longer than max_nnz");
    Owned& o = *own_;
    for (int32_t i = 0; i <= q.n; ++i) o.h_indptr[i] = q.ip[i] - base;
    for (int32_t i = q.n + 1; i <= n_; ++i) o.h_indptr[i] = static_cast<int32_t>(nnz);
    std::memcpy(o.h_idx, q.ix + base, nnz * sizeof(uint16_t));
    std::memcpy(o.h_val, q.vv + base, nnz * sizeof(float));
    cudaStream_t s = stream_;
    cuda_check(cudaMemcpyAsync(buf_.indptr, o.h_indptr, (n_ + 1) * sizeof(int32_t),
                               cudaMemcpyHostToDevice, s),
               "H2D queries");
    cuda_check(cudaMemcpyAsync(buf_.indices, o.h_idx, nnz * sizeof(uint16_t),
                               cudaMemcpyHostToDevice, s),
               "H2D queries");
    cuda_check(cudaMemcpyAsync(buf_.values, o.h_val, nnz * sizeof(float), cudaMemcpyHostToDevice,
                               s),
               "H2D queries");
    launch(s);
    const size_t cnt = static_cast<size_t>(q.n) * args_.k;
    cuda_check(cudaMemcpyAsync(o.h_d, buf_.distances, cnt * sizeof(float), cudaMemcpyDeviceToHost,
                               s),
               "D2H");
    cuda_check(cudaMemcpyAsync(o.h_l, buf_.labels, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost,
                               s),
               "D2H");
    check(s, stats);
    std::memcpy(out_d, o.h_d, cnt * sizeof(float));
    std::memcpy(out_l, o.h_l, cnt * sizeof(int32_t));
}

}  // namespace nsp
