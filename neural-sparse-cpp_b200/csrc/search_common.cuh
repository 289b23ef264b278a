// Device helpers shared by the SEISMIC search kernels: value widening and the
// warp-cooperative top-k insert.
#ifndef NSP_SEARCH_COMMON_CUH
#define NSP_SEARCH_COMMON_CUH

#include <cuda_runtime.h>

#include <cstdint>

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

// Sorted (score desc, id asc) array of size n <= k in shared memory. A full
// heap rejects score <= its minimum (utils/ranker.h:58-60) and otherwise drops
// its worst entry (ranker.h:67-71). A doc already present is not inserted
// twice. All lanes of the warp call with the same arguments.
__device__ __forceinline__ void heap_offer(float s, int32_t d, float* hs, int32_t* hid,
                                           int& n, int k, int lane) {
    if (n == k && !(s > hs[k - 1])) return;
    bool found = false;
    for (int i = lane; i < n; i += 32) found |= (hid[i] == d);
    if (__any_sync(kFull, found)) return;
    int cnt = 0;
    for (int i = lane; i < n; i += 32) {
        const float a = hs[i];
        cnt += (a > s || (a == s && hid[i] < d)) ? 1 : 0;
    }
    const int pos = static_cast<int>(__reduce_add_sync(kFull, static_cast<unsigned>(cnt)));
    const int newn = n < k ? n + 1 : k;
    for (int hi = newn - 1; hi > pos; hi -= 32) {
        const int j = hi - lane;
        const bool act = j > pos;
        float tv = 0.0f;
        int32_t ti = 0;
        if (act) {
            tv = hs[j - 1];
            ti = hid[j - 1];
        }
        __syncwarp();
        if (act) {
            hs[j] = tv;
            hid[j] = ti;
        }
        __syncwarp();
    }
    if (lane == 0) {
        hs[pos] = s;
        hid[pos] = d;
    }
    __syncwarp();
    n = newn;
}

}  // namespace detail_search
}  // namespace nsp

#endif  // NSP_SEARCH_COMMON_CUH
