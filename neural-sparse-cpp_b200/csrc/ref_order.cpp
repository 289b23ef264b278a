// Compiled as C++20: std::ranges::sort is the call the reference makes.
#include "ref_order.h"

#include <algorithm>
#include <thread>
#include <utility>

namespace nsp {

void reference_kept_order(const HostCsr& h, const std::vector<int64_t>& post,
                          const std::vector<int32_t>& lists, int64_t cap,
                          std::vector<int32_t>& out) {
    const int n_terms = h.dim;
    std::vector<int32_t> slot(static_cast<size_t>(std::max(n_terms, 1)), -1);
    for (size_t j = 0; j < lists.size(); ++j) slot[lists[j]] = static_cast<int32_t>(j);
    using Pair = std::pair<float, int32_t>;
    const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const float* val = reinterpret_cast<const float*>(h.values.data());
    const int64_t n_docs = h.n();
    // (value, doc) pairs per list in doc order, as the reference's posting
    // lists hold them (inverted_lists.cpp:159-180): each thread collects a
    // contiguous doc range, and the ranges are joined in order
    std::vector<std::vector<std::vector<Pair>>> part(nth, std::vector<std::vector<Pair>>(lists.size()));
    {
        std::vector<std::thread> pool;
        for (unsigned w = 0; w < nth; ++w)
            pool.emplace_back([&, w] {
                const int64_t d0 = n_docs * w / nth, d1 = n_docs * (w + 1) / nth;
                auto& mine = part[w];
                for (int64_t d = d0; d < d1; ++d)
                    for (int64_t e = h.indptr[d]; e < h.indptr[d + 1]; ++e) {
                        const uint16_t t = h.indices[e];
                        const int32_t j = t < n_terms ? slot[t] : -1;
                        if (j >= 0) mine[j].emplace_back(val[e], static_cast<int32_t>(d));
                    }
            });
        for (auto& th : pool) th.join();
    }
    out.assign(lists.size() * static_cast<size_t>(cap), -1);
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < nth; ++w)
        pool.emplace_back([&, w] {
            std::vector<Pair> v;
            for (size_t j = w; j < lists.size(); j += nth) {
                v.clear();
                v.reserve(static_cast<size_t>(post[lists[j] + 1] - post[lists[j]]));
                for (unsigned r = 0; r < nth; ++r) {
                    v.insert(v.end(), part[r][j].begin(), part[r][j].end());
                    std::vector<Pair>().swap(part[r][j]);
                }
                std::ranges::sort(v, [](const auto& a, const auto& b) { return a.first > b.first; });
                const int64_t n = std::min<int64_t>(cap, static_cast<int64_t>(v.size()));
                for (int64_t i = 0; i < n; ++i) out[j * cap + i] = v[i].second;
            }
        });
    for (auto& th : pool) th.join();
}

std::vector<uint16_t> reference_summary_kept(const HostCsr& h, const int32_t* docs, size_t n_docs,
                                             float alpha) {
    const float* val = reinterpret_cast<const float*>(h.values.data());
    std::vector<float> acc(static_cast<size_t>(std::max(h.dim, 1)), 0.0F);
    std::vector<uint8_t> seen(static_cast<size_t>(std::max(h.dim, 1)), 0);
    std::vector<uint16_t> touched;
    float sum = 0.0F;
    for (size_t i = 0; i < n_docs; ++i) {
        const int32_t d = docs[i];
        for (int64_t e = h.indptr[d]; e < h.indptr[d + 1]; ++e) {
            const uint16_t t = h.indices[e];
            const float v = val[e];
            if (!seen[t]) {
                seen[t] = 1;
                const float first = std::max(0.0F, v);
                acc[t] = first;
                touched.push_back(t);
                sum += first;
            } else if (v > acc[t]) {
                sum += v - acc[t];
                acc[t] = v;
            }
        }
    }
    std::vector<std::pair<uint16_t, float>> pairs;
    pairs.reserve(touched.size());
    for (const uint16_t t : touched) pairs.emplace_back(t, acc[t]);
    std::ranges::sort(pairs, [](const auto& a, const auto& b) { return a.second > b.second; });
    float addup = 0.0F;
    for (size_t j = 0; j < pairs.size(); ++j) {
        addup += pairs[j].second;
        if (addup / sum >= alpha) {
            pairs.erase(pairs.begin() + static_cast<std::ptrdiff_t>(j) + 1, pairs.end());
            break;
        }
    }
    std::vector<uint16_t> kept;
    kept.reserve(pairs.size());
    for (const auto& pr : pairs) kept.push_back(pr.first);
    return kept;
}

}  // namespace nsp
