// Serving loop over a SEISMIC index (an extension with no counterpart in the
// reference, which searches batches a caller has already formed).
//
// Requests (one query each, with its own k and optional doc filter) arrive
// one at a time. `slots` worker threads each own a CUDA stream and its
// scratch (the engine's per-thread workspace). A worker that is free takes
// the oldest waiting request and every waiting request with the same k, cut
// and heap factor, up to `max_batch` and as far as the scratch budget allows,
// and runs them as one launch of the one-CTA-per-query kernel; while it runs,
// requests that arrive meanwhile are taken by the next free worker, so
// batches overlap on the GPU (continuous batching, no fixed batching window).
// Each request's result is exactly what a search of that query alone returns:
// the kernel treats every query on its own, with its own heap. A request
// completes as soon as its own query's results are written: the kernel
// writes them, with a done flag per query, into the worker's mapped host
// memory, and the worker polls the flags while the launch runs.
#include "serve.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <stdexcept>
#include <thread>

#include "engine.h"
#include "index_state.h"
#include "nsparse/id_map_index.h"

namespace nsparse {
namespace detail {

namespace {

using Clock = std::chrono::steady_clock;

// Bounds the workers reserve scratch for up front (larger requests still run;
// their batches grow the scratch once).
constexpr int kReserveK = 100;
constexpr int kReserveNnz = 256;

// Page-locked host memory the device writes into (cudaHostAllocMapped): a
// worker's results and per-query done flags, read by the host while the
// launch still runs.
template <class T>
struct Mapped {
    T* h = nullptr;  // host address
    T* d = nullptr;  // the device's address of the same memory
    size_t n = 0;
    Mapped() = default;
    Mapped(const Mapped&) = delete;
    Mapped& operator=(const Mapped&) = delete;
    ~Mapped() {
        if (h != nullptr) cudaFreeHost(h);
    }
    // Room for `want` elements; only between launches (the old memory goes).
    void grow(size_t want) {
        if (want <= n) return;
        if (h != nullptr) cudaFreeHost(h);
        h = nullptr;
        d = nullptr;
        n = 0;
        void* p = nullptr;
        nsp::cuda_check(cudaHostAlloc(&p, want * sizeof(T), cudaHostAllocMapped), "cudaHostAlloc");
        h = static_cast<T*>(p);
        void* dp = nullptr;
        nsp::cuda_check(cudaHostGetDevicePointer(&dp, p, 0), "cudaHostGetDevicePointer");
        d = static_cast<T*>(dp);
        n = want;
    }
};

int64_t request_bytes(const ServerRequest& r) {
    // query terms and values, results, one selector pointer
    return static_cast<int64_t>(r.terms.size()) * 6 + 4 + static_cast<int64_t>(r.k) * 8 + 8;
}

}  // namespace

Server::Server(Index* index, const ServerConfig& cfg) : index_(index), cfg_(cfg) {
    if (index == nullptr) throw std::invalid_argument("unexpected nullptr");
    if (cfg_.max_batch <= 0 || cfg_.slots <= 0 || cfg_.scratch_budget <= 0)
        throw std::invalid_argument("server limits must be positive");
    nsp::SeismicSearchArgs a;
    st_ = resolve_seismic(index, nullptr, 10, a);
    if (auto* im = dynamic_cast<IDMapIndex*>(index)) id_map_ = &im->internal_to_external();
    nsp::cuda_check(cudaGetDevice(&device_), "cudaGetDevice");
    dim_ = index_dimension();
    if (st_->vectors.host.n() == 0) throw std::runtime_error("index is empty");
    st_->vectors.ensure_device();
    st_->ensure_lists();
    for (int i = 0; i < cfg_.slots; ++i) workers_.emplace_back([this] { worker(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : workers_) t.join();
    for (void* p : filters_) cudaFree(p);
}

int Server::index_dimension() const {
    if (auto* im = dynamic_cast<IDMapIndex*>(index_)) return im->delegate()->get_dimension();
    return index_->get_dimension();
}

int Server::add_filter(const uint64_t* bits, int64_t words) {
    if (bits == nullptr) throw std::invalid_argument("unexpected nullptr");
    const int64_t need = (static_cast<int64_t>(st_->vectors.host.n()) + 64) / 64;
    if (words < need) throw std::invalid_argument("filter bitmap shorter than the index's docs");
    void* d = nullptr;
    nsp::cuda_check(cudaMalloc(&d, static_cast<size_t>(need) * 8), "cudaMalloc filter");
    nsp::cuda_check(cudaMemcpy(d, bits, static_cast<size_t>(need) * 8, cudaMemcpyHostToDevice),
                    "H2D filter");
    std::lock_guard<std::mutex> g(mu_);
    filters_.push_back(d);
    return static_cast<int>(filters_.size()) - 1;
}

void Server::set_external_ids(const int64_t* ids, int64_t n) {
    if (ids == nullptr) throw std::invalid_argument("unexpected nullptr");
    if (n != static_cast<int64_t>(st_->vectors.host.n()))
        throw std::invalid_argument("one external id per indexed doc is needed");
    std::lock_guard<std::mutex> g(mu_);
    ext_ids_.assign(ids, ids + n);
}

std::shared_ptr<ServerRequest> Server::make_request(int32_t nnz, const uint16_t* terms,
                                                    const float* values, int k, int cut, float hf,
                                                    int filter) const {
    if (nnz < 0 || (nnz > 0 && (terms == nullptr || values == nullptr)))
        throw std::invalid_argument("bad query row");
    if (k <= 0 || cut <= 0) throw std::invalid_argument("value must be positive");
    const int32_t ip[2] = {0, nnz};
    const nsp::QueryBatch q = nsp::canonicalize(1, ip, terms, values, dim_);
    auto r = std::make_shared<ServerRequest>();
    r->terms.assign(q.ix + q.ip[0], q.ix + q.ip[1]);
    r->values.assign(q.vv + q.ip[0], q.vv + q.ip[1]);
    r->k = k;
    r->cut = cut;
    r->hf = hf;
    r->filter = filter;
    return r;
}

int64_t Server::submit(int32_t nnz, const uint16_t* terms, const float* values, int k, int cut,
                       float hf, int filter) {
    auto r = make_request(nnz, terms, values, k, cut, hf, filter);
    std::lock_guard<std::mutex> g(mu_);
    if (filter >= static_cast<int>(filters_.size())) throw std::invalid_argument("unknown filter id");
    r->ticket = next_ticket_++;
    r->t_arrive = Clock::now();
    live_[r->ticket] = r;
    enqueue(r);
    return r->ticket;
}

void Server::wait(int64_t ticket, float* distances, int64_t* labels, double* latency_us) {
    std::shared_ptr<ServerRequest> r;
    {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = live_.find(ticket);
        if (it == live_.end()) throw std::invalid_argument("unknown ticket");
        r = it->second;
        cv_done_.wait(lk, [&] { return r->done; });
        live_.erase(it);
    }
    if (!r->error.empty()) throw std::runtime_error(r->error);
    if (distances != nullptr) std::copy(r->d.begin(), r->d.end(), distances);
    if (labels != nullptr) std::copy(r->l.begin(), r->l.end(), labels);
    if (latency_us != nullptr)
        *latency_us = std::chrono::duration<double, std::micro>(r->t_done - r->t_arrive).count();
}

void Server::replay(int32_t n, const int32_t* indptr, const uint16_t* indices, const float* values,
                    const int32_t* k_per, const int32_t* filter_per, const double* arrival_us,
                    int cut, float hf, int k_stride, float* distances, int64_t* labels,
                    double* latency_us) {
    if (n <= 0) throw std::invalid_argument("value must be positive");
    if (indptr == nullptr || indices == nullptr || values == nullptr || k_per == nullptr ||
        arrival_us == nullptr || distances == nullptr || labels == nullptr)
        throw std::invalid_argument("unexpected nullptr");
    std::vector<std::shared_ptr<ServerRequest>> reqs(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i) {
        if (k_per[i] > k_stride) throw std::invalid_argument("k above the output stride");
        reqs[i] = make_request(indptr[i + 1] - indptr[i], indices + indptr[i], values + indptr[i],
                               k_per[i], cut, hf, filter_per == nullptr ? -1 : filter_per[i]);
    }
    {
        std::lock_guard<std::mutex> g(mu_);
        for (const auto& r : reqs)
            if (r->filter >= static_cast<int>(filters_.size()))
                throw std::invalid_argument("unknown filter id");
    }
    const Clock::time_point t0 = Clock::now();
    for (int32_t i = 0; i < n; ++i) {
        const Clock::time_point at =
            t0 + std::chrono::duration_cast<Clock::duration>(
                     std::chrono::duration<double, std::micro>(arrival_us[i]));
        for (;;) {
            const Clock::time_point now = Clock::now();
            if (now >= at) break;
            if (at - now > std::chrono::microseconds(200))
                std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        std::lock_guard<std::mutex> g(mu_);
        reqs[i]->ticket = next_ticket_++;
        reqs[i]->t_arrive = at;  // latency counts from the scheduled arrival
        enqueue(reqs[i]);
    }
    {
        // requests finish roughly in order: the scan resumes where it stopped
        size_t j = 0;
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] {
            while (j < reqs.size() && reqs[j]->done) ++j;
            return j == reqs.size();
        });
    }
    for (int32_t i = 0; i < n; ++i) {
        const ServerRequest& r = *reqs[i];
        if (!r.error.empty()) throw std::runtime_error(r.error);
        float* d = distances + static_cast<size_t>(i) * k_stride;
        int64_t* l = labels + static_cast<size_t>(i) * k_stride;
        for (int j = 0; j < k_stride; ++j) {
            d[j] = j < r.k ? r.d[j] : -1.0f;
            l[j] = j < r.k ? r.l[j] : -1;
        }
        if (latency_us != nullptr)
            latency_us[i] =
                std::chrono::duration<double, std::micro>(r.t_done - r.t_arrive).count();
    }
}

// Requests wait in one queue per (k, cut, heap factor): a launch serves one
// such combination, and taking a batch never scans other requests.
void Server::enqueue(const std::shared_ptr<ServerRequest>& r) {
    uint32_t hf_bits = 0;
    std::memcpy(&hf_bits, &r->hf, sizeof(hf_bits));
    const QueueKey key{r->k, r->cut, hf_bits};
    pending_[key].push_back(r);
    ++n_pending_;
    cv_work_.notify_one();
}

ServerStats Server::stats() const {
    std::lock_guard<std::mutex> g(mu_);
    return stats_;
}

void Server::worker() {
    if (cudaSetDevice(device_) != cudaSuccess) return;
    nsp::DevArray<const uint64_t*> d_sel;  // this worker's per-query selector table
    // the kernel writes each query's results and its done flag here, so a
    // request completes when its own query does, not when the launch's
    // slowest query does
    Mapped<float> md;
    Mapped<int32_t> ml, mdone;
    try {
        md.grow(static_cast<size_t>(cfg_.max_batch) * kReserveK);
        ml.grow(static_cast<size_t>(cfg_.max_batch) * kReserveK);
        mdone.grow(static_cast<size_t>(cfg_.max_batch));
        // Scratch for every batch size up to max_batch (rows up to kReserveNnz
        // terms, k up to kReserveK) before the first request: a buffer grown
        // mid-stream frees the old one, and that cudaFree waits for every
        // worker's work on the device.
        d_sel.resize(static_cast<size_t>(cfg_.max_batch));
        const int sms = nsp::device_sm_count();
        for (int k : {10, kReserveK}) {
            SeismicSearchParameters params(10, 1.0f);
            nsp::SeismicSearchArgs a;
            resolve_seismic(index_, &params, k, a);
            for (int n : {1, sms / 2, sms, 2 * sms, 2 * sms + 1, 4 * sms, cfg_.max_batch}) {
                if (n < 1 || n > cfg_.max_batch) continue;
                nsp::SeismicSearchArgs t = a;
                apply_tuned(*st_, t, n);
                if (t.variant >= 0 && t.variant < 2) t.variant = -1;
                nsp::reserve_seismic_scratch(st_->vectors.dev, st_->lists_dev, n, kReserveNnz, t);
            }
        }
    } catch (const std::exception&) {
        // a failed reservation only means later batches grow their scratch
    }
    for (;;) {
        std::vector<std::shared_ptr<ServerRequest>> batch;
        std::vector<const uint64_t*> sel;
        int64_t est = 0;
        int64_t others = 0;  // queries other workers have on the GPU
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_work_.wait(lk, [&] {
                return stop_ || (n_pending_ > 0 && in_use_ < cfg_.scratch_budget);
            });
            if (n_pending_ == 0) {
                if (stop_) return;
                continue;
            }
            // the queue (one per k, cut, heap factor) whose head waited longest
            auto q = pending_.end();
            for (auto it = pending_.begin(); it != pending_.end(); ++it)
                if (!it->second.empty() &&
                    (q == pending_.end() ||
                     it->second.front()->t_arrive < q->second.front()->t_arrive))
                    q = it;
            auto& dq = q->second;
            while (!dq.empty() && static_cast<int>(batch.size()) < cfg_.max_batch) {
                const int64_t e = request_bytes(*dq.front());
                if (!batch.empty() && in_use_ + est + e > cfg_.scratch_budget) break;
                est += e;
                batch.push_back(dq.front());
                dq.pop_front();
            }
            n_pending_ -= static_cast<int64_t>(batch.size());
            in_use_ += est;
            others = in_flight_queries_;
            in_flight_queries_ += static_cast<int64_t>(batch.size());
            sel.assign(batch.size(), nullptr);
            for (size_t i = 0; i < batch.size(); ++i)
                if (batch[i]->filter >= 0)
                    sel[i] = static_cast<const uint64_t*>(filters_[batch[i]->filter]);
            ++stats_.batches;
            stats_.requests += static_cast<int64_t>(batch.size());
            stats_.max_batch = std::max<int64_t>(stats_.max_batch, batch.size());
            stats_.max_in_flight_bytes = std::max(stats_.max_in_flight_bytes, in_use_);
        }
        std::string error;
        const int n = static_cast<int>(batch.size());
        const int k = batch[0]->k;
        std::vector<char> fin(static_cast<size_t>(n), 0);
        int left = n;
        // requests whose results are in the mapped buffers: done, under the lock
        auto complete = [&](const std::vector<int>& ready) {
            std::lock_guard<std::mutex> g(mu_);
            const Clock::time_point now = Clock::now();
            for (const int i : ready) {
                ServerRequest& r = *batch[i];
                r.d.assign(md.h + static_cast<size_t>(i) * k, md.h + static_cast<size_t>(i + 1) * k);
                r.l.resize(static_cast<size_t>(k));
                for (int j = 0; j < k; ++j) {
                    const int32_t v = ml.h[static_cast<size_t>(i) * k + j];
                    int64_t out = v;
                    if (v >= 0 && !ext_ids_.empty())
                        out = ext_ids_[v];
                    else if (v >= 0 && id_map_ != nullptr)
                        out = (*id_map_)[v];
                    r.l[j] = out;
                }
                r.t_done = now;
                r.done = true;
            }
        };
        try {
            nsp::QueryBatch q;
            q.n = n;
            q.indptr.assign(1, 0);
            for (const auto& r : batch) {
                q.idx.insert(q.idx.end(), r->terms.begin(), r->terms.end());
                q.val.insert(q.val.end(), r->values.begin(), r->values.end());
                q.indptr.push_back(static_cast<int32_t>(q.idx.size()));
                q.max_nnz = std::max<int32_t>(q.max_nnz, static_cast<int32_t>(r->terms.size()));
            }
            q.ip = q.indptr.data();
            q.ix = q.idx.data();
            q.vv = q.val.data();
            SeismicSearchParameters params(batch[0]->cut, batch[0]->hf);
            nsp::SeismicSearchArgs a;
            resolve_seismic(index_, &params, k, a);
            // CTAs per query by the queries on the GPU at once, this batch's
            // and the other workers': a cluster per query only while the SMs
            // would otherwise idle (capped by the autotuner's split)
            a.cluster = std::min(
                nsp::auto_cluster(static_cast<int>(std::min<int64_t>(others + n, 1 << 30))),
                st_->tuned.split > 0 ? st_->tuned.split : 8);
            apply_tuned(*st_, a, static_cast<int64_t>(batch.size()));
            if (a.variant >= 0 && a.variant < 2) a.variant = -1;  // needs one CTA per query
            const bool any =
                std::any_of(sel.begin(), sel.end(), [](const uint64_t* p) { return p != nullptr; });
            if (any) {
                if (d_sel.size() < sel.size()) d_sel.resize(sel.size() * 2);
                d_sel.upload(sel.data(), sel.size(), nsp::Workspace::get().stream());
                a.d_sel_q = d_sel.data();
            }
            md.grow(static_cast<size_t>(n) * k);
            ml.grow(static_cast<size_t>(n) * k);
            mdone.grow(static_cast<size_t>(n));
            std::memset(mdone.h, 0, static_cast<size_t>(n) * sizeof(int32_t));
            nsp::seismic_search_start(st_->vectors.dev, st_->lists_dev, q, a, md.d, ml.d,
                                      mdone.d);
            // each request completes when its query's flag is up; once the
            // launch has ended, one more sweep finds the last flags
            const cudaStream_t s = nsp::Workspace::get().stream();
            const volatile int32_t* flags = mdone.h;
            std::vector<int> ready;
            bool ended = false;
            for (;;) {
                ready.clear();
                for (int i = 0; i < n; ++i)
                    if (!fin[i] && flags[i] != 0) ready.push_back(i);
                if (!ready.empty()) {
                    std::atomic_thread_fence(std::memory_order_acquire);
                    complete(ready);
                    cv_done_.notify_all();
                    for (const int i : ready) fin[i] = 1;
                    left -= static_cast<int>(ready.size());
                }
                if (left == 0 || ended) break;
                ended = cudaStreamQuery(s) != cudaErrorNotReady;
                if (!ended) std::this_thread::yield();
            }
            nsp::seismic_search_wait();  // raises the launch's errors
            if (left > 0) throw std::runtime_error("a search launch ended without some results");
        } catch (const std::exception& e) {
            error = e.what();
            // nothing of this batch may still run when the mapped buffers
            // are reused (or regrown) for the next one
            cudaStreamSynchronize(nsp::Workspace::get().stream());
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            const Clock::time_point now = Clock::now();
            for (int i = 0; i < n; ++i) {
                if (fin[i]) continue;
                ServerRequest& r = *batch[i];
                r.error = error;
                r.d.assign(static_cast<size_t>(k), -1.0f);
                r.l.assign(static_cast<size_t>(k), -1);
                r.t_done = now;
                r.done = true;
            }
            in_use_ -= est;
            in_flight_queries_ -= n;
        }
        cv_done_.notify_all();
        cv_work_.notify_all();
    }
}

}  // namespace detail
}  // namespace nsparse
