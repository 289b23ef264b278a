// Serving loop over a SEISMIC index (serve.cpp): continuous batching of
// single-query requests onto several CUDA streams.
#ifndef NSP_SERVE_H
#define NSP_SERVE_H

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "nsparse/index.h"

namespace nsparse {
namespace detail {

struct SeismicState;

struct ServerConfig {
    int max_batch = 4096;                   // queries per launch
    int slots = 3;                          // launches in flight (one stream each)
    int64_t scratch_budget = 256ll << 20;   // bytes of request data in flight
};

struct ServerStats {
    int64_t batches = 0;
    int64_t requests = 0;
    int64_t max_batch = 0;
    int64_t max_in_flight_bytes = 0;
};

struct ServerRequest {
    int64_t ticket = -1;
    std::vector<uint16_t> terms;  // canonical: ascending, unique
    std::vector<float> values;
    int k = 10;
    int cut = 10;
    float hf = 1.0f;
    int filter = -1;  // registered filter id, -1: none
    std::chrono::steady_clock::time_point t_arrive, t_done;
    bool done = false;
    std::string error;
    std::vector<float> d;
    std::vector<int64_t> l;
};

class Server {
public:
    // `index` (a seismic index, possibly inside an IDMapIndex) must outlive
    // the server and must not be modified while it runs.
    Server(Index* index, const ServerConfig& cfg);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // A doc filter (bitmap over internal doc ids), uploaded once; requests
    // name it by the returned id.
    int add_filter(const uint64_t* bits, int64_t words);
    // Labels become ids[internal id] (e.g. 64-bit external ids).
    void set_external_ids(const int64_t* ids, int64_t n);

    int64_t submit(int32_t nnz, const uint16_t* terms, const float* values, int k, int cut,
                   float hf, int filter);
    void wait(int64_t ticket, float* distances, int64_t* labels, double* latency_us);
    // Submits request i at arrival_us[i] after the call starts, waits for all,
    // and writes results (k_stride per request, padded) and latencies.
    void replay(int32_t n, const int32_t* indptr, const uint16_t* indices, const float* values,
                const int32_t* k_per, const int32_t* filter_per, const double* arrival_us, int cut,
                float hf, int k_stride, float* distances, int64_t* labels, double* latency_us);
    ServerStats stats() const;

private:
    std::shared_ptr<ServerRequest> make_request(int32_t nnz, const uint16_t* terms,
                                                const float* values, int k, int cut, float hf,
                                                int filter) const;
    int index_dimension() const;
    void worker();
    void enqueue(const std::shared_ptr<ServerRequest>& r);  // under mu_

    struct QueueKey {
        int k;
        int cut;
        uint32_t hf_bits;
        bool operator<(const QueueKey& o) const {
            return std::tie(k, cut, hf_bits) < std::tie(o.k, o.cut, o.hf_bits);
        }
    };

    Index* index_;
    ServerConfig cfg_;
    SeismicState* st_ = nullptr;
    const std::vector<int64_t>* id_map_ = nullptr;
    int dim_ = 0;
    int device_ = 0;
    std::vector<int64_t> ext_ids_;
    std::vector<void*> filters_;

    mutable std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::map<QueueKey, std::deque<std::shared_ptr<ServerRequest>>> pending_;
    int64_t n_pending_ = 0;
    std::unordered_map<int64_t, std::shared_ptr<ServerRequest>> live_;
    int64_t next_ticket_ = 0;
    int64_t in_use_ = 0;
    int64_t in_flight_queries_ = 0;  // queries of the launches running now
    bool stop_ = false;
    ServerStats stats_;
    std::vector<std::thread> workers_;
};

}  // namespace detail
}  // namespace nsparse

#endif  // NSP_SERVE_H
