// Device helpers shared by the SEISMIC search kernels: value widening and the
// warp-cooperative top-k insert.
#ifndef NSP_SEARCH_COMMON_CUH
#define NSP_SEARCH_COMMON_CUH

#include <cuda_runtime.h>

#include <cstdint>

#include "ref_ranking.cuh"

namespace nsp {
namespace detail_search {

constexpr unsigned kFull = 0xffffffffu;

template <typename V>
struct ValT;
template <>
struct ValT<float> {
    __device__ static float f(float v) { return v; }
};
template <>
struct ValT<uint8_t> {
    __device__ static float f(uint8_t v) { return static_cast<float>(v); }
};
template <>
struct ValT<uint16_t> {
    __device__ static float f(uint16_t v) { return static_cast<float>(v); }
};

// A query entry's weight as the reference's TopKHolder sees it (a float).
template <typename V>
struct QueryWeight {
    const V* q;
    __host__ __device__ float operator()(uint16_t i) const { return static_cast<float>(q[i]); }
};

// The query's top-k holder in shared memory: the reference's TopKHolder
// (utils/ranker.h:34-138), a binary heap with the smallest score on top
// (hs[0], hid[0]), restated in ref_ranking.cuh. A full holder rejects
// score <= its top; otherwise a full holder pops, then pushes. A doc already
// held is not offered twice (the reference never offers a doc twice: its
// visited set; a doc offered again here scored at most the top when it was
// dropped or rejected, and the top only grows). All lanes of the warp call
// with the same arguments; lane 0 moves the entries.
__device__ __forceinline__ void heap_offer(float s, int32_t d, float* hs, int32_t* hid,
                                           int& n, int k, int lane) {
    if (n >= k && s <= hs[0]) return;
    bool found = false;
    for (int i = lane; i < n; i += 32) found |= (hid[i] == d);
    if (__any_sync(kFull, found)) return;
    if (lane == 0) {
        int m = n;
        ranking::topk_add(ranking::TopK{hs, hid}, m, k, s, d);
    }
    __syncwarp();
    n = n < k ? n + 1 : k;
}

// The holder's smallest score (valid when it holds k entries).
__device__ __forceinline__ float heap_top(const float* hs) { return hs[0]; }

// Results as TopKHolder::top_k_items_descending gives them (ranker.h:
// 113-127), padded with (-1.0, -1) to k (seismic_index.cpp:270-273); scores
// times `scale` when it is not 0 (SQ decode,
// seismic_scalar_quantized_index.cpp:345-355). Empties the holder. Lane 0
// pops; all lanes pad.
__device__ __forceinline__ void heap_emit(float* hs, int32_t* hid, int n, int k, float scale,
                                          float* od, int32_t* ol, int lane) {
    if (lane == 0) {
        int m = n;
        const ranking::TopK h{hs, hid};
        for (int i = n - 1; i >= 0; --i) {
            const float s = hs[0];
            od[i] = scale != 0.0f ? __fmul_rn(s, scale) : s;
            ol[i] = hid[0];
            ranking::topk_pop(h, m);
        }
    }
    for (int i = n + lane; i < k; i += 32) {
        od[i] = -1.0f;
        ol[i] = -1;
    }
    __syncwarp();
}

}  // namespace detail_search
}  // namespace nsp

#endif  // NSP_SEARCH_COMMON_CUH
