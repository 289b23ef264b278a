// Three-pass device scan: per-tile sums, a single-CTA scan of the tile sums,
// then a per-tile scan that adds its tile's offset. Tiles are 4096 elements
// (1024 threads x 4 items).
#include "scan.h"

#include <cuda_runtime.h>

#include "engine.h"

namespace nsp {
namespace {

constexpr int kThreads = 1024;
constexpr int kItems = 4;
constexpr int kTile = kThreads * kItems;

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ int64_t block_excl_scan(int64_t v, int64_t* total) {
    __shared__ int64_t warp_tot[32];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    int64_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        int64_t w = lane < nw ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) warp_tot[lane] = w;
    }
    __syncthreads();
    const int64_t before = wid > 0 ? warp_tot[wid - 1] : 0;
    *total = warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + incl - v;
}

__global__ void __launch_bounds__(kThreads) tile_sums_kernel(const int64_t* in, int64_t n,
                                                             int64_t* sums) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kItems;
    int64_t v = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i)
        if (base + i < n) v += in[base + i];
    int64_t total = 0;
    block_excl_scan(v, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads) scan_sums_kernel(int64_t* sums, int64_t n) {
    int64_t carry = 0;
    for (int64_t base = 0; base < n; base += kThreads) {
        const int64_t i = base + threadIdx.x;
        const int64_t v = i < n ? sums[i] : 0;
        int64_t total = 0;
        const int64_t ex = block_excl_scan(v, &total);
        if (i < n) sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void __launch_bounds__(kThreads) tile_scan_kernel(const int64_t* in, int64_t* out,
                                                             int64_t n, const int64_t* sums) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kItems;
    int64_t v[kItems];
    int64_t local = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
        local += v[i];
    }
    int64_t total = 0;
    int64_t run = block_excl_scan(local, &total) + sums[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

}  // namespace

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    const int64_t tiles = (n + kTile - 1) / kTile;
    DevArray<int64_t> sums(static_cast<size_t>(tiles));
    tile_sums_kernel<<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(in, n, sums.data());
    cuda_check(cudaGetLastError(), "tile_sums_kernel");
    scan_sums_kernel<<<1, kThreads, 0, s>>>(sums.data(), tiles);
    cuda_check(cudaGetLastError(), "scan_sums_kernel");
    tile_scan_kernel<<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(in, out, n, sums.data());
    cuda_check(cudaGetLastError(), "tile_scan_kernel");
    cuda_check(cudaStreamSynchronize(s), "scan sync");
}

}  // namespace nsp
