// Doc-ascending postings of an fp32 forward index, built on the device for
// the exact search's term-at-a-time kernel (search_exact.cu).
//
// The reference's InvertedIndex keeps per-term posting lists in doc order
// (invlists/inverted_lists.cpp:159-180, built from the forward index by
// inverted_index.cpp:236-252). Here they come from the resident padded rows
// in five device steps: row lengths (and a check that every row's terms are
// strictly ascending), an exclusive scan, a doc-major compaction of (term,
// value | doc) pairs, a stable radix sort by term -- which keeps each term's
// postings in doc order --, and the per-(term, doc chunk) start table.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "engine.h"
#include "scan.h"

namespace nsp {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// off[d] = row d's length; *unsorted = 1 if some row's terms are not
// strictly ascending. One warp per row.
__global__ void row_lens_kernel(FwdView f, int64_t* off, int* unsorted) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t d = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
         d < f.n_docs; d += warps) {
        const uint2 ri = f.rowinfo[d];
        const int len = static_cast<int>(ri.y);
        const uint16_t* ip = f.idx + static_cast<size_t>(ri.x) * kRowAlign;
        bool bad = false;
        for (int e = lane + 1; e < len; e += 32) bad |= ip[e] <= ip[e - 1];
        if (__any_sync(kFull, bad) && lane == 0) atomicOr(unsorted, 1);
        if (lane == 0) off[d] = len;
    }
}

// keys[off[d] + e] = term, vals[off[d] + e] = value bits << 32 | doc, in
// doc-major order.
__global__ void compact_kernel(FwdView f, const int64_t* off, uint16_t* keys,
                               unsigned long long* vals) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const float* fv = static_cast<const float*>(f.val);
    for (int64_t d = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
         d < f.n_docs; d += warps) {
        const uint2 ri = f.rowinfo[d];
        const int len = static_cast<int>(ri.y);
        const size_t src = static_cast<size_t>(ri.x) * kRowAlign;
        const int64_t dst = off[d];
        for (int e = lane; e < len; e += 32) {
            keys[dst + e] = f.idx[src + e];
            vals[dst + e] = (static_cast<unsigned long long>(__float_as_uint(fv[src + e])) << 32) |
                            static_cast<uint32_t>(d);
        }
    }
}

// tstart[t] = first position of term t in the sorted keys, t = 0..dim.
__global__ void term_start_kernel(const uint16_t* keys, int64_t nnz, int dim, int32_t* tstart) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > dim) return;
    int64_t lo = 0, hi = nnz;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (static_cast<int>(keys[mid]) < t) lo = mid + 1;
        else hi = mid;
    }
    tstart[t] = static_cast<int32_t>(lo);
}

__global__ void unpack_kernel(const unsigned long long* v, int64_t nnz, int32_t* doc, float* val) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < nnz;
         j += stride) {
        const unsigned long long x = v[j];
        doc[j] = static_cast<int32_t>(static_cast<uint32_t>(x));
        val[j] = __uint_as_float(static_cast<uint32_t>(x >> 32));
    }
}

// chunk_at[t * (nc + 1) + c] = first posting of term t with doc >= c * C.
__global__ void chunk_at_kernel(const int32_t* tstart, const int32_t* doc, int dim, int nc, int C,
                                int32_t* chunk_at) {
    const int64_t total = static_cast<int64_t>(dim) * (nc + 1);
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += stride) {
        const int t = static_cast<int>(i / (nc + 1));
        const int c = static_cast<int>(i - static_cast<int64_t>(t) * (nc + 1));
        int32_t lo = tstart[t];
        int32_t hi = tstart[t + 1];
        if (c < nc) {
            const int64_t bound = static_cast<int64_t>(c) * C;
            while (lo < hi) {
                const int32_t mid = lo + ((hi - lo) >> 1);
                if (doc[mid] < bound) lo = mid + 1;
                else hi = mid;
            }
        } else {
            lo = hi;
        }
        chunk_at[i] = lo;
    }
}

int grid_for(int64_t work, int per_block) {
    const int64_t g = (work + per_block - 1) / per_block;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32)));
}

}  // namespace

void PostingsDevice::build(const ForwardDevice& fwd, int chunk_docs) {
    cudaStream_t s = Workspace::get().stream();
    generation_ = fwd.generation();
    usable_ = false;
    doc_.reset();
    val_.reset();
    chunk_at_.reset();
    n_chunks_ = 0;
    chunk_docs_ = chunk_docs;
    if (fwd.empty() || fwd.esz() != 4 || chunk_docs <= 0) return;
    const FwdView f = fwd.view();
    const int32_t n = f.n_docs;

    DevArray<int64_t> off(static_cast<size_t>(n) + 1);
    DevArray<int> flag(1);
    cuda_check(cudaMemsetAsync(flag.data(), 0, sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(off.data() + n, 0, sizeof(int64_t), s), "memset");
    row_lens_kernel<<<grid_for(static_cast<int64_t>(n) * 32, 256), 256, 0, s>>>(f, off.data(),
                                                                                flag.data());
    cuda_check(cudaGetLastError(), "row_lens_kernel");
    exclusive_scan_i64(off.data(), off.data(), static_cast<int64_t>(n) + 1, s);
    int64_t nnz = 0;
    int unsorted = 0;
    cuda_check(cudaMemcpyAsync(&nnz, off.data() + n, sizeof(nnz), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(&unsorted, flag.data(), sizeof(int), cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (unsorted != 0 || nnz >= INT_MAX) return;  // the tile kernel serves this index

    n_chunks_ = (n + chunk_docs - 1) / chunk_docs;
    const int dim = f.dim;
    DevArray<int32_t> tstart(static_cast<size_t>(dim) + 1);
    doc_.resize(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    val_.resize(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    if (nnz > 0) {
        DevArray<uint16_t> k_in(static_cast<size_t>(nnz)), k_out(static_cast<size_t>(nnz));
        DevArray<unsigned long long> v_in(static_cast<size_t>(nnz)), v_out(static_cast<size_t>(nnz));
        compact_kernel<<<grid_for(static_cast<int64_t>(n) * 32, 256), 256, 0, s>>>(
            f, off.data(), k_in.data(), v_in.data());
        cuda_check(cudaGetLastError(), "compact_kernel");
        size_t tmp_bytes = 0;
        cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, k_in.data(), k_out.data(),
                                                   v_in.data(), v_out.data(), static_cast<int>(nnz),
                                                   0, 16, s),
                   "radix sort size");
        DevArray<unsigned char> tmp(std::max<size_t>(tmp_bytes, 1));
        cuda_check(cub::DeviceRadixSort::SortPairs(tmp.data(), tmp_bytes, k_in.data(), k_out.data(),
                                                   v_in.data(), v_out.data(), static_cast<int>(nnz),
                                                   0, 16, s),
                   "radix sort");
        term_start_kernel<<<(dim + 1 + 255) / 256, 256, 0, s>>>(k_out.data(), nnz, dim,
                                                                tstart.data());
        cuda_check(cudaGetLastError(), "term_start_kernel");
        unpack_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(v_out.data(), nnz, doc_.data(),
                                                         val_.data());
        cuda_check(cudaGetLastError(), "unpack_kernel");
        // the temporaries are freed when this scope ends: wait for their users
        cuda_check(cudaStreamSynchronize(s), "sync");
    } else {
        cuda_check(cudaMemsetAsync(tstart.data(), 0, (static_cast<size_t>(dim) + 1) * 4, s),
                   "memset");
    }
    chunk_at_.resize(static_cast<size_t>(dim) * (n_chunks_ + 1));
    chunk_at_kernel<<<grid_for(static_cast<int64_t>(dim) * (n_chunks_ + 1), 256), 256, 0, s>>>(
        tstart.data(), doc_.data(), dim, n_chunks_, chunk_docs, chunk_at_.data());
    cuda_check(cudaGetLastError(), "chunk_at_kernel");
    cuda_check(cudaStreamSynchronize(s), "sync");
    usable_ = true;
}

PostingsView PostingsDevice::view() const {
    PostingsView v;
    v.n_chunks = n_chunks_;
    v.chunk_docs = chunk_docs_;
    v.doc = doc_.data();
    v.val = val_.data();
    v.chunk_at = chunk_at_.data();
    return v;
}

size_t PostingsDevice::device_bytes() const {
    return doc_.size() * 4 + val_.size() * 4 + chunk_at_.size() * 4;
}

}  // namespace nsp
