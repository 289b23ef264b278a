// SEISMIC index build on the device (the reference's
// build_inverted_lists_clusters, seismic_common.h:146-184).
//
//  1. postings      one warp per document scatters its (term, doc, value)
//                   entries into per-term lists (warp-aggregated atomics);
//                   a segmented sort orders each list: by value descending,
//                   then doc ascending, when it exceeds the posting cap lambda
//                   (invlists/inverted_lists.cpp:110-132), else by doc
//                   (the order build_inverted_lists produces, :159-180).
//  2. centroids     drawn on the host with std::mt19937 and
//                   std::uniform_int_distribution<> seeded base_seed + list,
//                   the reference's own draw (cluster/random_kmeans.cpp:28-51);
//                   it depends only on list lengths, so only those come back.
//  3. assignment    one CTA per list: the centroids' terms are indexed term
//                   major in scratch, one warp per document accumulates its
//                   similarity to every centroid in the document's term order
//                   (cluster/kmeans_utils.cpp:131-145; fp32 products and sums
//                   rounded separately, int64 for codes) and takes the strict
//                   argmax, lowest index on ties (:147-156).
//  4. blocks        a stable segmented sort puts each centroid first and its
//                   members after it in list order.
//  5. summaries     per block: entries sorted by term (stable), a per-term
//                   running max gives each entry's increment of the block's
//                   mass, summed in the reference's entry order
//                   (cluster/inverted_list_clusters.cpp:72-124); the maxima
//                   are sorted by value descending (term ascending on ties)
//                   and cut where the running mass reaches alpha (:37-65),
//                   then transposed term-major per list (:230-293).
//                   uint8 codes take a fused path (section 5'): per block in
//                   shared memory, the maxima in a hash or per-term table,
//                   the integer mass and the cut from a histogram of the
//                   maxima, no sort of the entries.
// The lists come back to the host for persistence and are uploaded in the
// search layout.
#include <cub/device/device_segmented_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <random>
#include <utility>
#include <string>
#include <stdexcept>
#include <thread>
#include <vector>

#include "engine.h"
#include "index_state.h"
#include "ref_order.h"
#include "scan.h"

namespace nsparse {
namespace detail {
namespace {

using nsp::cuda_check;
using nsp::DevArray;

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------- parameters ------

// seismic_common.h:130-144
int calc_lambda(int lambda, size_t n_vectors) {
    if (lambda == -1)
        return std::max(static_cast<int>(0.0005F * static_cast<float>(n_vectors)), 160);
    return lambda;
}

int calc_beta(int beta, int lambda) {
    if (beta == -1) return static_cast<int>(static_cast<float>(lambda) * 0.1F);
    return beta;
}

// random_kmeans.cpp:53-63 with the caller's int beta converted to size_t.
size_t clusters_for(size_t n_docs, int beta) {
    size_t nc = static_cast<size_t>(static_cast<long long>(beta));  // wraps like the reference
    if (beta == 0) nc = static_cast<size_t>(std::sqrt(n_docs));
    nc = nc > n_docs ? n_docs : nc;
    return std::max<size_t>(1, nc);
}

// Positions (into the list's kept order) of the centroids of one list:
// random_kmeans.cpp:28-51, applied to positions instead of ids.
void draw_positions(size_t n, size_t nc, uint32_t seed, std::vector<int32_t>& perm,
                    int32_t* out) {
    perm.resize(n);
    for (size_t i = 0; i < n; ++i) perm[i] = static_cast<int32_t>(i);
    std::mt19937 gen(seed);
    for (size_t i = 0; i < nc; ++i) {
        std::uniform_int_distribution<> distrib(0, static_cast<int>(n - i - 1));
        const size_t r = static_cast<size_t>(distrib(gen));
        out[i] = perm[r];
        std::swap(perm[r], perm[n - 1 - i]);
    }
}

// ------------------------------------------------------------- keys ------

// Order-preserving map of a value to uint32 (ascending value = ascending key).
__device__ __forceinline__ uint32_t orderable(float v) {
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

template <int ESZ>
__device__ __forceinline__ float value_at(const uint8_t* val, int64_t i) {
    if constexpr (ESZ == 4) return reinterpret_cast<const float*>(val)[i];
    if constexpr (ESZ == 2) return static_cast<float>(reinterpret_cast<const uint16_t*>(val)[i]);
    return static_cast<float>(val[i]);
}

// ------------------------------------------------------------ 1. postings --

__global__ void post_count_kernel(nsp::FwdView f, unsigned long long* cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t d = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
         d < f.n_docs; d += warps) {
        const uint2 ri = f.rowinfo[d];
        const uint16_t* ip = f.idx + static_cast<size_t>(ri.x) * nsp::kRowAlign;
        for (uint32_t e0 = 0; e0 < ri.y; e0 += 32) {
            const uint32_t e = e0 + lane;
            const bool valid = e < ri.y;
            const uint32_t t = valid ? ip[e] : 0xffffffffu;
            const unsigned peers = __match_any_sync(kFull, t);
            if (valid && (__ffs(peers) - 1) == lane) atomicAdd(cnt + t, __popc(peers));
        }
    }
}

// Writes each entry's sort key into its list: (~value << 32 | doc) when the
// list is over the cap, doc otherwise.
template <int ESZ>
__global__ void post_scatter_kernel(nsp::FwdView f, const int64_t* post_ptr,
                                    unsigned long long* cursor, int64_t cap,
                                    uint64_t* keys) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const uint8_t* vals = static_cast<const uint8_t*>(f.val);
    for (int64_t d = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
         d < f.n_docs; d += warps) {
        const uint2 ri = f.rowinfo[d];
        const int64_t base = static_cast<int64_t>(ri.x) * nsp::kRowAlign;
        for (uint32_t e0 = 0; e0 < ri.y; e0 += 32) {
            const uint32_t e = e0 + lane;
            const bool valid = e < ri.y;
            const uint32_t t = valid ? f.idx[base + e] : 0xffffffffu;
            const unsigned peers = __match_any_sync(kFull, t);
            const int leader = __ffs(peers) - 1;
            unsigned long long start = 0;
            if (valid && leader == lane) start = atomicAdd(cursor + t, __popc(peers));
            start = __shfl_sync(kFull, start, leader);
            if (valid) {
                const int rank = __popc(peers & ((1u << lane) - 1u));
                const int64_t len = post_ptr[t + 1] - post_ptr[t];
                const uint64_t key =
                    (cap > 0 && len > cap)
                        ? (static_cast<uint64_t>(~orderable(value_at<ESZ>(vals, base + e))) << 32) |
                              static_cast<uint32_t>(d)
                        : static_cast<uint64_t>(static_cast<uint32_t>(d));
                keys[post_ptr[t] + static_cast<int64_t>(start) + rank] = key;
            }
        }
    }
}

__global__ void kept_copy_kernel(const uint64_t* keys, const int64_t* post_ptr,
                                 const int64_t* kept_ptr, int32_t n_lists, int32_t* kept) {
    for (int32_t t = blockIdx.x; t < n_lists; t += gridDim.x) {
        const int64_t n = kept_ptr[t + 1] - kept_ptr[t];
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
            kept[kept_ptr[t] + i] = static_cast<int32_t>(keys[post_ptr[t] + i] & 0xffffffffu);
    }
}

// Flags a truncated list (len > cap) whose first cap + 1 sorted keys hold two
// equal values: its kept order (and, with a tie across the cut, its kept set)
// is what the reference's unstable sort leaves, which the host reproduces.
__global__ void tie_flag_kernel(const uint64_t* keys, const int64_t* post_ptr, int32_t n_lists,
                                int64_t cap, uint8_t* flag) {
    for (int32_t t = blockIdx.x; t < n_lists; t += gridDim.x) {
        const int64_t len = post_ptr[t + 1] - post_ptr[t];
        if (cap <= 0 || len <= cap) {
            if (threadIdx.x == 0) flag[t] = 0;
            continue;
        }
        const uint64_t* k = keys + post_ptr[t];
        int tie = 0;
        for (int64_t i = threadIdx.x + 1; i <= cap; i += blockDim.x)
            tie |= (k[i] >> 32) == (k[i - 1] >> 32);
        tie = __syncthreads_or(tie);
        if (threadIdx.x == 0) flag[t] = static_cast<uint8_t>(tie);
    }
}

// ---------------------------------------------------------- 3. assignment --

struct AssignArgs {
    nsp::FwdView f;
    int32_t n_lists;
    const int64_t* kept_ptr;
    const int32_t* kept;
    const int64_t* cptr;
    const int32_t* cpos;
    uint32_t* out_key;      // per kept position: cluster * 2 + (centroid ? 0 : 1)
    int32_t* work;          // list counter
    // per-CTA scratch
    int32_t* tcnt;          // [dim] per CTA, zero between lists
    int32_t* tstart;        // [dim] per CTA
    int32_t* tcur;          // [dim] per CTA
    int2* trun;             // [dim] per CTA: (start, count) of the term's centroid
                            // entries, count zero between lists
    int32_t* touched;       // [max centroid entries] per CTA
    uint16_t* ccl;          // [max centroid entries] per CTA
    uint8_t* cw;            // [max centroid entries * esz] per CTA
    uint8_t* is_centroid;   // [max kept] per CTA
    void* sims;             // per warp [max nc] (float or int64)
    int64_t max_centroid_entries;
    int64_t max_kept;
    int32_t max_nc;
    int32_t sims_in_smem;  // 1: the similarity rows are in dynamic shared memory
};

// Similarity accumulators: fp32 for fp32 values; int for uint8 codes (at
// most 400 products of two codes below 2^16 each, exact), int64 for uint16.
template <int ESZ>
using assign_acc_t = typename std::conditional<
    ESZ == 4, float, typename std::conditional<ESZ == 1, int, long long>::type>::type;

// One centroid entry of a term's run: the centroid and its value.
template <int ESZ>
__device__ __forceinline__ void centroid_entry(const uint16_t* ccl, const uint8_t* cw, int32_t k,
                                               int32_t& c, assign_acc_t<ESZ>& w) {
    c = ccl[k];
    if constexpr (ESZ == 4) w = reinterpret_cast<const float*>(cw)[k];
    else if constexpr (ESZ == 2) w = reinterpret_cast<const uint16_t*>(cw)[k];
    else w = cw[k];
}

template <int ESZ>
__device__ __forceinline__ void add_product(assign_acc_t<ESZ>* sims, int32_t c,
                                            assign_acc_t<ESZ> dv, assign_acc_t<ESZ> w) {
    if constexpr (ESZ == 4) sims[c] = __fadd_rn(sims[c], __fmul_rn(dv, w));
    else sims[c] += dv * w;
}

template <int ESZ>
__global__ void __launch_bounds__(1024) assign_kernel(AssignArgs a) {
    using acc_t = assign_acc_t<ESZ>;
    // centroid entries of one term in flight per lane: a term's run is
    // loaded kChunks * 32 entries at a time, the next hit term's first
    // chunk while the current one is applied
    constexpr int kChunks = 4;
    __shared__ int32_t s_list;
    __shared__ int32_t s_touched;
    __shared__ int32_t s_total;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int dim = a.f.dim;
    int32_t* tcnt = a.tcnt + static_cast<size_t>(blockIdx.x) * dim;
    int32_t* tstart = a.tstart + static_cast<size_t>(blockIdx.x) * dim;
    int32_t* tcur = a.tcur + static_cast<size_t>(blockIdx.x) * dim;
    int2* trun = a.trun + static_cast<size_t>(blockIdx.x) * dim;
    int32_t* touched = a.touched + static_cast<size_t>(blockIdx.x) * a.max_centroid_entries;
    uint16_t* ccl = a.ccl + static_cast<size_t>(blockIdx.x) * a.max_centroid_entries;
    uint8_t* cw = a.cw + static_cast<size_t>(blockIdx.x) * a.max_centroid_entries * ESZ;
    uint8_t* isc = a.is_centroid + static_cast<size_t>(blockIdx.x) * a.max_kept;
    // each warp's row of similarities: shared memory when the launch gave
    // room for it (the read-modify-writes of one doc are serial), else global
    extern __shared__ __align__(16) unsigned char dyn[];
    acc_t* sims = a.sims_in_smem ? reinterpret_cast<acc_t*>(dyn) + static_cast<size_t>(warp) * a.max_nc
                                 : static_cast<acc_t*>(a.sims) +
                                       static_cast<size_t>(blockIdx.x * wpb + warp) * a.max_nc;
    const uint8_t* fval = static_cast<const uint8_t*>(a.f.val);

    for (;;) {
        if (threadIdx.x == 0) s_list = atomicAdd(a.work, 1);
        __syncthreads();
        const int32_t t = s_list;
        __syncthreads();
        if (t >= a.n_lists) break;
        const int64_t kb = a.kept_ptr[t];
        const int32_t n = static_cast<int32_t>(a.kept_ptr[t + 1] - kb);
        const int32_t nc = static_cast<int32_t>(a.cptr[t + 1] - a.cptr[t]);
        if (n == 0) continue;
        const int32_t* cp = a.cpos + a.cptr[t];
        for (int32_t i = threadIdx.x; i < n; i += blockDim.x) isc[i] = 0;
        if (threadIdx.x == 0) {
            s_touched = 0;
            s_total = 0;
        }
        __syncthreads();
        for (int32_t c = threadIdx.x; c < nc; c += blockDim.x) isc[cp[c]] = 1;
        // index the centroid entries by term: count, ranges, scatter
        for (int32_t c = warp; c < nc; c += wpb) {
            const int32_t doc = a.kept[kb + cp[c]];
            const uint2 ri = a.f.rowinfo[doc];
            const uint16_t* ip = a.f.idx + static_cast<size_t>(ri.x) * nsp::kRowAlign;
            for (uint32_t e = lane; e < ri.y; e += 32) {
                const int32_t term = ip[e];
                if (atomicAdd(tcnt + term, 1) == 0) touched[atomicAdd(&s_touched, 1)] = term;
            }
        }
        __syncthreads();
        const int32_t nt = s_touched;
        for (int32_t i = threadIdx.x; i < nt; i += blockDim.x) {
            const int32_t term = touched[i];
            const int32_t cnt = tcnt[term];
            const int32_t st = atomicAdd(&s_total, cnt);
            tstart[term] = st;
            tcur[term] = 0;
            trun[term] = make_int2(st, cnt);
        }
        __syncthreads();
        for (int32_t c = warp; c < nc; c += wpb) {
            const int32_t doc = a.kept[kb + cp[c]];
            const uint2 ri = a.f.rowinfo[doc];
            const int64_t rb = static_cast<int64_t>(ri.x) * nsp::kRowAlign;
            for (uint32_t e = lane; e < ri.y; e += 32) {
                const int32_t term = a.f.idx[rb + e];
                const int32_t pos = tstart[term] + atomicAdd(tcur + term, 1);
                ccl[pos] = static_cast<uint16_t>(c);
                for (int b = 0; b < ESZ; ++b) cw[static_cast<size_t>(pos) * ESZ + b] = fval[(rb + e) * ESZ + b];
            }
        }
        __syncthreads();
        // assign every non-centroid doc, one warp per doc
        for (int32_t p = warp; p < n; p += wpb) {
            if (isc[p]) {
                // centroid: its own cluster, placed first
                if (lane == 0) {
                    int32_t c = 0;
                    while (cp[c] != p) ++c;
                    a.out_key[kb + p] = static_cast<uint32_t>(c) * 2u;
                }
                continue;
            }
            const int32_t doc = a.kept[kb + p];
            for (int32_t c = lane; c < nc; c += 32) sims[c] = 0;
            __syncwarp();
            const uint2 ri = a.f.rowinfo[doc];
            const int64_t rb = static_cast<int64_t>(ri.x) * nsp::kRowAlign;
            for (uint32_t e0 = 0; e0 < ri.y; e0 += 32) {
                const uint32_t e = e0 + lane;
                int2 run = make_int2(0, 0);
                acc_t v = 0;
                if (e < ri.y) {
                    run = trun[a.f.idx[rb + e]];
                    if constexpr (ESZ == 4) v = reinterpret_cast<const float*>(fval)[rb + e];
                    else if constexpr (ESZ == 2) v = reinterpret_cast<const uint16_t*>(fval)[rb + e];
                    else v = fval[rb + e];
                }
                // doc terms in order (kmeans_utils.cpp:134-145); a term's
                // centroids are distinct, so its products commute, and the
                // warp barrier between terms keeps each similarity's sum in
                // doc-term order
                unsigned m = __ballot_sync(kFull, run.y > 0);
                int32_t nc_[kChunks];
                acc_t nw[kChunks];
                int32_t s0 = 0, cnt = 0;
                acc_t dv = 0;
                if (m) {
                    const int src = __ffs(m) - 1;
                    s0 = __shfl_sync(kFull, run.x, src);
                    cnt = __shfl_sync(kFull, run.y, src);
                    dv = __shfl_sync(kFull, v, src);
#pragma unroll
                    for (int j = 0; j < kChunks; ++j) {
                        const int32_t k = j * 32 + lane;
                        nc_[j] = -1;
                        if (k < cnt) centroid_entry<ESZ>(ccl, cw, s0 + k, nc_[j], nw[j]);
                    }
                }
                while (m) {
                    m &= m - 1;
                    int32_t cc[kChunks];
                    acc_t cwv[kChunks];
#pragma unroll
                    for (int j = 0; j < kChunks; ++j) {
                        cc[j] = nc_[j];
                        cwv[j] = nw[j];
                    }
                    const int32_t cs0 = s0, ccnt = cnt;
                    const acc_t cdv = dv;
                    if (m) {
                        const int src = __ffs(m) - 1;
                        s0 = __shfl_sync(kFull, run.x, src);
                        cnt = __shfl_sync(kFull, run.y, src);
                        dv = __shfl_sync(kFull, v, src);
#pragma unroll
                        for (int j = 0; j < kChunks; ++j) {
                            const int32_t k = j * 32 + lane;
                            nc_[j] = -1;
                            if (k < cnt) centroid_entry<ESZ>(ccl, cw, s0 + k, nc_[j], nw[j]);
                        }
                    }
#pragma unroll
                    for (int j = 0; j < kChunks; ++j)
                        if (cc[j] >= 0) add_product<ESZ>(sims, cc[j], cdv, cwv[j]);
                    for (int32_t k0 = kChunks * 32; k0 < ccnt; k0 += kChunks * 32) {
#pragma unroll
                        for (int j = 0; j < kChunks; ++j) {
                            const int32_t k = k0 + j * 32 + lane;
                            cc[j] = -1;
                            if (k < ccnt) centroid_entry<ESZ>(ccl, cw, cs0 + k, cc[j], cwv[j]);
                        }
#pragma unroll
                        for (int j = 0; j < kChunks; ++j)
                            if (cc[j] >= 0) add_product<ESZ>(sims, cc[j], cdv, cwv[j]);
                    }
                    __syncwarp();
                }
            }
            // strict >, ascending: ties go to the lowest cluster (kmeans_utils.cpp:147-156)
            acc_t best = 0;
            int32_t bi = -1;
            for (int32_t c = lane; c < nc; c += 32) {
                const acc_t s = sims[c];
                if (bi < 0 || s > best) {
                    best = s;
                    bi = c;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const acc_t s2 = __shfl_xor_sync(kFull, best, o);
                const int32_t i2 = __shfl_xor_sync(kFull, bi, o);
                if (i2 >= 0 && (bi < 0 || s2 > best || (s2 == best && i2 < bi))) {
                    best = s2;
                    bi = i2;
                }
            }
            if (lane == 0) a.out_key[kb + p] = static_cast<uint32_t>(bi) * 2u + 1u;
            __syncwarp();
        }
        __syncthreads();
        for (int32_t i = threadIdx.x; i < nt; i += blockDim.x) {
            tcnt[touched[i]] = 0;
            trun[touched[i]] = make_int2(0, 0);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ 5. summaries --

// Entries of a batch of blocks: for block b (global id), its docs' rows in
// block order. term -> ekey, value -> eval, original index -> eidx.
template <int ESZ>
__global__ void entries_kernel(nsp::FwdView f, const int32_t* docs, const int64_t* bdp,
                               int64_t b0, int64_t nb, const int64_t* doc_eoff, int64_t e_base,
                               uint16_t* ekey, uint32_t* eidx, float* eval) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const int64_t d0 = bdp[b0], d1 = bdp[b0 + nb];
    const uint8_t* vals = static_cast<const uint8_t*>(f.val);
    for (int64_t j = d0 + ((blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5); j < d1;
         j += warps) {
        const int32_t doc = docs[j];
        const uint2 ri = f.rowinfo[doc];
        const int64_t rb = static_cast<int64_t>(ri.x) * nsp::kRowAlign;
        const int64_t out = doc_eoff[j - d0] - e_base;
        for (uint32_t e = lane; e < ri.y; e += 32) {
            ekey[out + e] = f.idx[rb + e];
            eidx[out + e] = static_cast<uint32_t>(out + e);
            eval[out + e] = value_at<ESZ>(vals, rb + e);
        }
    }
}

// One thread per (block, term) run of the term-sorted entries: the running max
// gives each entry's increment of the block mass (inverted_list_clusters.cpp:
// 96-114); the run's final max becomes a candidate summary pair.
// uint8 codes: a block's mass is a sum of integer increments below 2^24, so
// every order of the float additions gives the same value -- the sum of its
// terms' maxima. Each run adds its max to the block's integer mass instead
// of writing per-entry increments for the ordered sum.
template <int ESZ>
__global__ void runs_kernel(const uint16_t* skey, const uint32_t* sidx, const float* eval,
                            const int32_t* run_start, int64_t n_runs, int64_t n_entries,
                            const int32_t* entry_block, float* delta, uint8_t* has_delta,
                            uint64_t* pkey, int32_t* pblock, uint32_t* mass_u) {
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n_runs;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t s = run_start[r];
        const int64_t e = r + 1 < n_runs ? run_start[r + 1] : n_entries;
        float acc = 0.0f;
        if constexpr (ESZ == 1) {
            for (int64_t i = s; i < e; ++i) acc = fmaxf(acc, eval[sidx[i]]);
            atomicAdd(mass_u + entry_block[sidx[s]], static_cast<uint32_t>(acc));
        } else {
        for (int64_t i = s; i < e; ++i) {
            const uint32_t oi = sidx[i];
            const float v = eval[oi];
            if (i == s) {
                // first touch: max(T(0), v)
                acc = v > 0.0f ? v : 0.0f;
                delta[oi] = acc;
                has_delta[oi] = 1;
            } else if (v > acc) {
                if constexpr (ESZ == 4) delta[oi] = __fsub_rn(v, acc);
                else delta[oi] = static_cast<float>(static_cast<int>(v) - static_cast<int>(acc));
                has_delta[oi] = 1;
                acc = v;
            } else {
                has_delta[oi] = 0;
            }
        }
        }
        const uint32_t term = skey[s];
        // sort key for the alpha cut: value descending, term ascending
        pkey[r] = (static_cast<uint64_t>(~orderable(acc)) << 16) | term;
        pblock[r] = entry_block[sidx[s]];
    }
}

__device__ __forceinline__ float unorderable(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(b);
}

// alpha cut (inverted_list_clusters.cpp:43-51): one thread per block walks its
// pairs by value descending, summing until addup / sum >= alpha.
__global__ void cut_kernel(const uint64_t* pkey_sorted, const int64_t* pair_off, int64_t nb,
                           const float* mass, float alpha, int32_t* keep) {
    for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b < nb;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t s = pair_off[b], e = pair_off[b + 1];
        float addup = 0.0f;
        int32_t k = static_cast<int32_t>(e - s);
        for (int64_t i = s; i < e; ++i) {
            const float v = unorderable(~static_cast<uint32_t>(pkey_sorted[i] >> 16));
            addup = __fadd_rn(addup, v);
            if (__fdiv_rn(addup, mass[b]) >= alpha) {
                k = static_cast<int32_t>(i - s + 1);
                break;
            }
        }
        keep[b] = k;
    }
}

// Blocks whose alpha cut falls inside a run of equal maxima: which of them
// the reference keeps is its unstable sort's choice (settled on the host).
__global__ void cut_tie_kernel(const uint64_t* pkey_sorted, const int64_t* pair_off, int64_t nb,
                               const int32_t* keep, uint8_t* tie) {
    for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b < nb;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t s = pair_off[b], n = pair_off[b + 1] - s;
        const int64_t k = keep[b];
        tie[b] = (k > 0 && k < n &&
                  (pkey_sorted[s + k - 1] >> 16) == (pkey_sorted[s + k] >> 16)) ? 1 : 0;
    }
}

template <class K, class V>
void segmented_sort_pairs(const K* kin, K* kout, const V* vin, V* vout, int64_t n,
                          int64_t segs, const int32_t* off, cudaStream_t s, bool stable,
                          DevArray<uint8_t>* pool = nullptr) {
    if (n == 0 || segs == 0) return;
    if (n > INT32_MAX || segs > INT32_MAX) throw std::invalid_argument("build batch too large");
    size_t tmp = 0;
    if (stable)
        cuda_check(cub::DeviceSegmentedSort::StableSortPairs(nullptr, tmp, kin, kout, vin, vout,
                                                             static_cast<int>(n), static_cast<int>(segs),
                                                             off, off + 1, s), "cub sort");
    else
        cuda_check(cub::DeviceSegmentedSort::SortPairs(nullptr, tmp, kin, kout, vin, vout,
                                                       static_cast<int>(n), static_cast<int>(segs),
                                                       off, off + 1, s), "cub sort");
    DevArray<uint8_t> own;
    DevArray<uint8_t>& t = pool != nullptr ? *pool : own;
    t.grow(tmp + 16);
    if (stable)
        cuda_check(cub::DeviceSegmentedSort::StableSortPairs(t.data(), tmp, kin, kout, vin, vout,
                                                             static_cast<int>(n), static_cast<int>(segs),
                                                             off, off + 1, s), "cub sort");
    else
        cuda_check(cub::DeviceSegmentedSort::SortPairs(t.data(), tmp, kin, kout, vin, vout,
                                                       static_cast<int>(n), static_cast<int>(segs),
                                                       off, off + 1, s), "cub sort");
    if (pool == nullptr) cuda_check(cudaStreamSynchronize(s), "sort sync");
}

template <class K>
void segmented_sort_keys(const K* kin, K* kout, int64_t n, int64_t segs, const int32_t* off,
                         cudaStream_t s, DevArray<uint8_t>* pool = nullptr) {
    if (n == 0 || segs == 0) return;
    if (n > INT32_MAX || segs > INT32_MAX) throw std::invalid_argument("build batch too large");
    size_t tmp = 0;
    cuda_check(cub::DeviceSegmentedSort::SortKeys(nullptr, tmp, kin, kout, static_cast<int>(n),
                                                  static_cast<int>(segs), off, off + 1, s),
               "cub sort");
    DevArray<uint8_t> own;
    DevArray<uint8_t>& t = pool != nullptr ? *pool : own;
    t.grow(tmp + 16);
    cuda_check(cub::DeviceSegmentedSort::SortKeys(t.data(), tmp, kin, kout, static_cast<int>(n),
                                                  static_cast<int>(segs), off, off + 1, s),
               "cub sort");
    if (pool == nullptr) cuda_check(cudaStreamSynchronize(s), "sort sync");
}

template <class T>
std::vector<T> to_host(const DevArray<T>& d, size_t n, cudaStream_t s) {
    std::vector<T> h(n);
    d.download(h.data(), n, s);
    cuda_check(cudaStreamSynchronize(s), "D2H");
    return h;
}

template <class T>
void to_dev(DevArray<T>& d, const std::vector<T>& h, cudaStream_t s) {
    d.upload(h.data(), h.size(), s);
}

std::vector<int32_t> to_i32_offsets(const std::vector<int64_t>& v) {
    std::vector<int32_t> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        if (v[i] > INT32_MAX) throw std::invalid_argument("build batch too large");
        o[i] = static_cast<int32_t>(v[i]);
    }
    return o;
}

__global__ void fill_block_kernel(const int32_t* boff, int64_t nb, int32_t* entry_block) {
    for (int64_t b = blockIdx.x; b < nb; b += gridDim.x)
        for (int64_t i = boff[b] + threadIdx.x; i < boff[b + 1]; i += blockDim.x)
            entry_block[i] = static_cast<int32_t>(b);
}

// 1 where a (block, term) run starts in the term-sorted entries.
__global__ void run_flag_kernel(const uint16_t* skey, const int32_t* entry_block, int64_t ne,
                                int64_t* flag) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < ne;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        flag[i] = (i == 0 || entry_block[i] != entry_block[i - 1] || skey[i] != skey[i - 1]) ? 1 : 0;
}

__global__ void run_compact_kernel(const int64_t* flag, const int64_t* pos, int64_t ne,
                                   int32_t* run_start) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < ne;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (flag[i]) run_start[pos[i]] = static_cast<int32_t>(i);
}

// The run index at each block's first entry (n_runs for a block past the
// last entry); empty blocks are fixed up on the host.
__global__ void block_first_run_kernel(const int64_t* pos, const int32_t* boff, int64_t nb,
                                       int64_t ne, int64_t n_runs, int64_t* first_run) {
    for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b < nb;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x)
        first_run[b] = boff[b] < ne ? pos[boff[b]] : n_runs;
}

__global__ void mass_from_int_kernel(const uint32_t* mass_u, int64_t nb, float* mass) {
    for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b < nb;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x)
        mass[b] = static_cast<float>(mass_u[b]);
}

__global__ void mass_kernel(const float* delta, const uint8_t* has_delta, const int32_t* boff,
                            int64_t nb, float* mass) {
    for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b < nb;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        float sum = 0.0f;
        for (int64_t i = boff[b]; i < boff[b + 1]; ++i)
            if (has_delta[i]) sum = __fadd_rn(sum, delta[i]);
        mass[b] = sum;
    }
}

// Kept pairs of each block, keyed (term << 16 | block within its list) for
// the per-list term-major transpose.
__global__ void kept_pairs_kernel(const uint64_t* pkey_sorted, const int64_t* pair_off,
                                  const int32_t* keep, const int64_t* kept_off,
                                  const uint16_t* block_local, int64_t nb, uint32_t* tkey,
                                  float* tval) {
    for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        for (int32_t i = threadIdx.x; i < keep[b]; i += blockDim.x) {
            const uint64_t k = pkey_sorted[pair_off[b] + i];
            const uint32_t term = static_cast<uint32_t>(k & 0xffffu);
            tkey[kept_off[b] + i] = (term << 16) | block_local[b];
            tval[kept_off[b] + i] = unorderable(~static_cast<uint32_t>(k >> 16));
        }
    }
}

// Per kept summary pair (sorted by (term, block) within each list): its block
// id, its value as the index stores it, and a flag where a new term starts.
template <int ESZ>
__global__ void columns_kernel(const uint32_t* key, const float* val, int64_t n, uint16_t* blk,
                               uint8_t* out_val, int64_t* flag) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        blk[i] = static_cast<uint16_t>(key[i] & 0xffffu);
        const float v = val[i];
        if constexpr (ESZ == 4) {
            reinterpret_cast<float*>(out_val)[i] = v;
        } else if constexpr (ESZ == 2) {
            reinterpret_cast<uint16_t*>(out_val)[i] = static_cast<uint16_t>(v);
        } else {
            out_val[i] = static_cast<uint8_t>(v);
        }
        flag[i] = (i == 0 || (key[i] >> 16) != (key[i - 1] >> 16)) ? 1 : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) flag[n] = 0;
}

// A list's first pair always starts a column (its term may equal the last
// term of the list before).
__global__ void list_start_kernel(const int32_t* list_off, int32_t nl, int64_t n, int64_t* flag) {
    const int32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < nl && list_off[l] < list_off[l + 1] && list_off[l] < n) flag[list_off[l]] = 1;
}

__global__ void column_compact_kernel(const uint32_t* key, const int64_t* flag, const int64_t* pos,
                                      int64_t n, uint16_t* term, int64_t* start) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (flag[i]) {
            term[pos[i]] = static_cast<uint16_t>(key[i] >> 16);
            start[pos[i]] = i;
        }
    }
}

// Columns before each list boundary.
__global__ void list_cols_kernel(const int32_t* list_off, int32_t nl, const int64_t* pos,
                                 int64_t* cols) {
    const int32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l <= nl) cols[l] = pos[list_off[l]];
}

// Time per step of the summary pipeline, summed over batches, on stderr when
// NSP_VERBOSE=1 (the engine's one debug switch; it synchronizes each step).
struct StepTimes {
    bool on = false;
    cudaStream_t s = nullptr;
    std::chrono::steady_clock::time_point t;
    std::vector<std::pair<std::string, double>> acc;
    void start(cudaStream_t st) {
        const char* v = std::getenv("NSP_VERBOSE");
        on = v != nullptr && v[0] == '1';
        s = st;
        acc.clear();
        t = std::chrono::steady_clock::now();
    }
    void mark(const char* name) {
        if (!on) return;
        cudaStreamSynchronize(s);
        const auto now = std::chrono::steady_clock::now();
        const double dt = std::chrono::duration<double>(now - t).count();
        t = now;
        for (auto& a : acc)
            if (a.first == name) {
                a.second += dt;
                return;
            }
        acc.emplace_back(name, dt);
    }
    void print() const {
        if (!on) return;
        for (const auto& a : acc)
            std::fprintf(stderr, "[nsparse build]   %-14s %8.3f s\n", a.first.c_str(), a.second);
    }
};
thread_local StepTimes g_steps;

// Summary columns of all lists built so far, in device memory: the index's
// final arrays, handed to the device image without a round trip through
// host memory (the host copy is made only if it is asked for, e.g. to write
// the index file).
struct DevColumns {
    DevArray<uint16_t> sterm, sblk;
    DevArray<int64_t> srun;
    DevArray<uint8_t> sval;
    size_t n_cols = 0;     // sterm used; srun holds n_cols + 1 boundaries
    size_t n_entries = 0;  // sblk used; sval holds n_entries * esz bytes
};

// Appends n elements at src (device) after the first `used` of dst, growing
// dst geometrically.
template <class T>
void dev_append(DevArray<T>& dst, size_t used, const T* src, size_t n, cudaStream_t s) {
    if (used + n > dst.size()) {
        DevArray<T> bigger(std::max(dst.size() * 2, used + n));
        if (used > 0)
            cuda_check(cudaMemcpyAsync(bigger.data(), dst.data(), used * sizeof(T),
                                       cudaMemcpyDeviceToDevice, s),
                       "D2D");
        cuda_check(cudaStreamSynchronize(s), "sync");
        dst = std::move(bigger);
    }
    if (n > 0)
        cuda_check(cudaMemcpyAsync(dst.data() + used, src, n * sizeof(T), cudaMemcpyDeviceToDevice,
                                   s),
                   "D2D");
}

// Column boundaries of a batch: column c > 0 starts where column c-1 ends;
// the last ends after the batch's n_kept entries; all offset by `ebase`.
__global__ void column_bounds_kernel(const int64_t* start, int64_t n_cols, int64_t ebase,
                                     int64_t n_kept, int64_t* srun_tail) {
    for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < n_cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x)
        srun_tail[c] = ebase + (c + 1 < n_cols ? start[c + 1] : n_kept);
}

// Device buffers of the summary pipeline, kept across batches of lists (they
// only grow), so a batch allocates and frees nothing.
// ------------------------------------------- 5'. uint8 summaries, fused --
// With uint8 codes a block's summary needs no ordered arithmetic: its mass is
// the integer sum of its terms' maxima (below 2^24, so every float sum of
// them is exact), and the alpha cut over the maxima sorted by (value desc,
// term asc) follows from a 256-bin histogram of the maxima: the level at
// which the running sum first reaches alpha * mass, and how many of that
// level's terms -- the smallest term ids -- are kept. Each block is summed up
// in shared memory without sorting its entries: blocks of up to
// kSumHashEntries entries by a CTA of kSumHashThreads threads over a hash
// table of (term, max), larger blocks by a CTA with a per-term table. A
// count pass gives each block's kept pairs, a write pass writes them (in no
// particular order: the per-list transpose sorts them by term and block).

constexpr int kSumSlotsLog = 12;
constexpr int kSumSlots = 1 << kSumSlotsLog;  // hash slots per CTA
constexpr int kSumHashEntries = 3072;         // <= 3/4 of the slots: probes stay short
constexpr int kSumHashThreads = 128;
constexpr int kSumDenseThreads = 512;
constexpr int kSumTieScratch = 512;           // tied terms ranked in shared memory

struct SumU8Args {
    nsp::FwdView f;
    const int32_t* docs;  // every block's docs, block after block
    const int64_t* bdp;   // [n_blocks + 1]
    const int64_t* ids;   // the blocks this launch sums up (global ids), ascending
    int64_t n_ids;
    float alpha;
    int32_t* keep;        // count pass: kept pairs per block (global id)
    // write pass: block b's pairs go to kept_off[b - b0] + 0.. as
    // tkey = term << 16 | block_local[b - b0], tval = value
    const int64_t* kept_off;
    const uint16_t* block_local;
    int64_t b0;
    uint32_t* tkey;
    float* tval;
};

struct SumCut {
    int keep;   // pairs kept
    int vstar;  // the level the cut falls in (-1: every pair is kept)
    int r;      // that level's pairs kept (its smallest terms)
};

// The alpha cut (inverted_list_clusters.cpp:43-51) from the histogram of a
// block's maxima, by one warp: walking the pairs by value descending, the
// first count whose running sum `addup` satisfies addup / sum >= alpha. The
// running sums are integers below 2^24, so (float) of each is the reference's
// float accumulation; the division is the same correctly rounded one. No
// such count (sum 0, or alpha above 1): every pair is kept.
__device__ SumCut sum_u8_cut(const uint32_t* hist, uint32_t mass, int n_pairs, float alpha,
                             int lane) {
    uint32_t c[8];
    uint32_t cs = 0, ss = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int v = 255 - 8 * lane - i;  // lane 0 holds the top levels
        c[i] = hist[v];
        cs += c[i];
        ss += c[i] * static_cast<uint32_t>(v);
    }
    // counts and sums of the levels above this lane's
    uint32_t ci = cs, si = ss;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t cu = __shfl_up_sync(kFull, ci, o);
        const uint32_t su = __shfl_up_sync(kFull, si, o);
        if (lane >= o) {
            ci += cu;
            si += su;
        }
    }
    uint32_t cnt_above = ci - cs, sum_above = si - ss;
    const float fm = static_cast<float>(mass);
    int found = -1;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t v = static_cast<uint32_t>(255 - 8 * lane - i);
        if (found < 0 && c[i] > 0) {
            const uint32_t end = sum_above + c[i] * v;
            if (__fdiv_rn(static_cast<float>(end), fm) >= alpha) {
                found = i;
            } else {
                sum_above = end;
                cnt_above += c[i];
            }
        }
    }
    const unsigned hit = __ballot_sync(kFull, found >= 0);
    SumCut out{n_pairs, -1, 0};
    if (hit == 0u) return out;
    const int src = __ffs(hit) - 1;
    int keep = 0, vstar = 0, r = 0;
    if (lane == src) {
        uint32_t cf = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if (i == found) cf = c[i];
        const uint32_t v = static_cast<uint32_t>(255 - 8 * lane - found);
        // the smallest j in [1, cf] whose sum satisfies the test (the test
        // only turns true as j grows)
        uint32_t lo = 1, hi = cf;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__fdiv_rn(static_cast<float>(sum_above + mid * v), fm) >= alpha)
                hi = mid;
            else
                lo = mid + 1;
        }
        keep = static_cast<int>(cnt_above + lo);
        vstar = static_cast<int>(v);
        r = static_cast<int>(lo);
    }
    out.keep = __shfl_sync(kFull, keep, src);
    out.vstar = __shfl_sync(kFull, vstar, src);
    out.r = __shfl_sync(kFull, r, src);
    return out;
}

// Position of this lane's item among the warp's `pred` items appended to
// *counter (every lane of the warp calls it).
__device__ __forceinline__ int warp_append(unsigned* counter, bool pred, int lane) {
    const unsigned m = __ballot_sync(kFull, pred);
    if (m == 0u) return -1;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<unsigned>(__popc(m)));
    base = __shfl_sync(kFull, base, leader);
    return pred ? static_cast<int>(base + __popc(m & ((1u << lane) - 1u))) : -1;
}

// One row's 8 elements per lane from element e (rows start on 64-element
// boundaries and are padded to them, so the 16- and 8-byte loads are aligned
// and inside the row's padding).
__device__ __forceinline__ void row8(const nsp::FwdView& f, int64_t rb, int e, uint32_t (&t)[4],
                                     uint2& c) {
    const uint4 tv = __ldg(reinterpret_cast<const uint4*>(f.idx + rb + e));
    t[0] = tv.x;
    t[1] = tv.y;
    t[2] = tv.z;
    t[3] = tv.w;
    c = __ldg(reinterpret_cast<const uint2*>(static_cast<const uint8_t*>(f.val) + rb + e));
}

__device__ __forceinline__ uint32_t term8(const uint32_t (&t)[4], int u) {
    return (u & 1) ? (t[u >> 1] >> 16) : (t[u >> 1] & 0xffffu);
}

__device__ __forceinline__ uint32_t code8(const uint2& c, int u) {
    return ((u < 4 ? c.x : c.y) >> (8 * (u & 3))) & 0xffu;
}

// Writes the kept pairs of block b. `pair_at(i)` gives pair i of the block's
// nu pairs as (term << 8 | value); ties at the cut level are ranked by term
// in `tied` (scratch of kSumTieScratch terms) or, when more, against all pairs.
template <class PairAt>
__device__ void sum_u8_write(const SumU8Args& a, int64_t b, int nu, const SumCut& cut,
                             uint32_t ntied, PairAt pair_at, uint16_t* tied, unsigned* s_out,
                             unsigned* s_ntied, int tid, int nthreads) {
    const int lane = tid & 31;
    const int64_t out0 = a.kept_off[b - a.b0];
    const uint32_t bl = a.block_local[b - a.b0];
    const bool partial = cut.vstar >= 0 && static_cast<uint32_t>(cut.r) < ntied;
    const bool scratch = ntied <= static_cast<uint32_t>(kSumTieScratch);
    for (int base = 0; base < nu; base += nthreads) {
        const int i = base + tid;
        uint32_t p = 0;
        if (i < nu) p = pair_at(i);
        const int v = static_cast<int>(p & 0xffu);
        const uint32_t t = p >> 8;
        const bool kept = i < nu && (cut.vstar < 0 || v > cut.vstar || (v == cut.vstar && !partial));
        const int o = warp_append(s_out, kept, lane);
        if (kept) {
            a.tkey[out0 + o] = (t << 16) | bl;
            a.tval[out0 + o] = static_cast<float>(v);
        }
        const bool tie = partial && scratch && i < nu && v == cut.vstar;
        const int q = warp_append(s_ntied, tie, lane);
        if (tie) tied[q] = static_cast<uint16_t>(t);
    }
    __syncthreads();
    if (!partial) return;
    if (scratch) {
        for (int base = 0; base < static_cast<int>(ntied); base += nthreads) {
            const int i = base + tid;
            bool take = false;
            uint32_t t = 0;
            if (i < static_cast<int>(ntied)) {
                t = tied[i];
                int rank = 0;
                for (uint32_t j = 0; j < ntied; ++j) rank += tied[j] < t ? 1 : 0;
                take = rank < cut.r;
            }
            const int o = warp_append(s_out, take, lane);
            if (take) {
                a.tkey[out0 + o] = (t << 16) | bl;
                a.tval[out0 + o] = static_cast<float>(cut.vstar);
            }
        }
    } else {
        for (int base = 0; base < nu; base += nthreads) {
            const int i = base + tid;
            bool take = false;
            uint32_t t = 0;
            if (i < nu) {
                const uint32_t p = pair_at(i);
                t = p >> 8;
                if (static_cast<int>(p & 0xffu) == cut.vstar) {
                    int rank = 0;
                    for (int j = 0; j < nu; ++j) {
                        const uint32_t q = pair_at(j);
                        rank += (static_cast<int>(q & 0xffu) == cut.vstar && (q >> 8) < t) ? 1 : 0;
                    }
                    take = rank < cut.r;
                }
            }
            const int o = warp_append(s_out, take, lane);
            if (take) {
                a.tkey[out0 + o] = (t << 16) | bl;
                a.tval[out0 + o] = static_cast<float>(cut.vstar);
            }
        }
    }
}

// Blocks of at most kSumHashEntries entries: (term + 1) << 8 | max in an
// open-addressing table of kSumSlots words; warp w takes the block's docs
// w, w + 4, ..., 8 row elements per lane per step.
template <bool kWrite>
__global__ void __launch_bounds__(kSumHashThreads) sum_u8_hash_kernel(SumU8Args a) {
    __shared__ uint32_t tab[kSumSlots];
    __shared__ uint32_t hist[256];
    __shared__ uint16_t uslot[kSumHashEntries];
    __shared__ unsigned s_nu, s_out, s_ntied;
    __shared__ uint32_t s_mass;
    __shared__ SumCut s_cut;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = kSumHashThreads / 32;
    for (int i = tid; i < kSumSlots; i += kSumHashThreads) tab[i] = 0u;
    for (int i = tid; i < 256; i += kSumHashThreads) hist[i] = 0u;
    for (int64_t j = blockIdx.x; j < a.n_ids; j += gridDim.x) {
        const int64_t b = a.ids[j];
        if (tid == 0) {
            s_nu = 0u;
            s_out = 0u;
            s_ntied = 0u;
            s_mass = 0u;
        }
        __syncthreads();
        // 1. per-term maxima (inverted_list_clusters.cpp:89-115: the first
        // value of a term is max(0, v), a uint8 code is never below 0)
        const int64_t d0 = a.bdp[b], d1 = a.bdp[b + 1];
        for (int64_t d = d0 + warp; d < d1; d += kWarps) {
            const uint2 ri = __ldg(a.f.rowinfo + a.docs[d]);
            const int64_t rb = static_cast<int64_t>(ri.x) * nsp::kRowAlign;
            const int len = static_cast<int>(ri.y);
            for (int e0 = 0; e0 < len; e0 += 256) {
                const int e = e0 + 8 * lane;
                uint32_t tw[4] = {0u, 0u, 0u, 0u};
                uint2 cw = make_uint2(0u, 0u);
                if (e < len) row8(a.f, rb, e, tw, cw);
                unsigned nnew = 0u;
                uint32_t slots[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    slots[u] = 0xffffffffu;
                    if (e + u < len) {
                        const uint32_t t = term8(tw, u);
                        const uint32_t key = ((t + 1u) << 8) | code8(cw, u);
                        uint32_t h = (t * 0x9E3779B1u) >> (32 - kSumSlotsLog);
                        // at most kSumHashEntries keys in kSumSlots slots:
                        // an empty slot or the term's own is always found
                        for (int p = 0; p < kSumSlots; ++p) {
                            const uint32_t old = atomicCAS(&tab[h], 0u, key);
                            if (old == 0u) {
                                slots[u] = h;
                                ++nnew;
                                break;
                            }
                            if ((old >> 8) == t + 1u) {
                                if ((old & 0xffu) < (key & 0xffu)) atomicMax(&tab[h], key);
                                break;
                            }
                            h = (h + 1u) & (kSumSlots - 1);
                        }
                    }
                }
                // new slots appended to the block's list
                unsigned incl = nnew;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned x = __shfl_up_sync(kFull, incl, o);
                    if (lane >= o) incl += x;
                }
                unsigned base = 0u;
                const unsigned total = __shfl_sync(kFull, incl, 31);
                if (lane == 31 && total > 0u) base = atomicAdd(&s_nu, total);
                base = __shfl_sync(kFull, base, 31) + incl - nnew;
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (slots[u] != 0xffffffffu) uslot[base++] = static_cast<uint16_t>(slots[u]);
            }
        }
        __syncthreads();
        // 2. mass and histogram of the maxima
        const int nu = static_cast<int>(s_nu);
        uint32_t m = 0u;
        for (int i = tid; i < nu; i += kSumHashThreads) {
            const uint32_t v = tab[uslot[i]] & 0xffu;
            m += v;
            atomicAdd(&hist[v], 1u);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(kFull, m, o);
        if (lane == 0 && m > 0u) atomicAdd(&s_mass, m);
        __syncthreads();
        // 3. the cut
        if (warp == 0) {
            const SumCut c = sum_u8_cut(hist, s_mass, nu, a.alpha, lane);
            if (lane == 0) s_cut = c;
        }
        __syncthreads();
        const SumCut cut = s_cut;
        if constexpr (!kWrite) {
            if (tid == 0) a.keep[b] = cut.keep;
        } else {
            const uint32_t ntied = cut.vstar >= 0 ? hist[cut.vstar] : 0u;
            __syncthreads();  // the histogram becomes the tie scratch
            sum_u8_write(
                a, b, nu, cut, ntied,
                [&](int i) {
                    const uint32_t k = tab[uslot[i]];
                    return (((k >> 8) - 1u) << 8) | (k & 0xffu);
                },
                reinterpret_cast<uint16_t*>(hist), &s_out, &s_ntied, tid, kSumHashThreads);
        }
        __syncthreads();
        // 4. the table and histogram back to zero
        for (int i = tid; i < nu; i += kSumHashThreads) tab[uslot[i]] = 0u;
        for (int i = tid; i < 256; i += kSumHashThreads) hist[i] = 0u;
        __syncthreads();
    }
}

// Larger blocks: the max + 1 of every term in a table of `dim` words (0: the
// term is not in the block), the block's terms listed as first met.
// Ties at the cut level are taken in term order by a scan of the table.
template <bool kWrite>
__global__ void __launch_bounds__(kSumDenseThreads) sum_u8_dense_kernel(SumU8Args a) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int dim = a.f.dim;
    uint32_t* tab = reinterpret_cast<uint32_t*>(sm);
    uint32_t* hist = tab + dim;
    uint16_t* ulist = reinterpret_cast<uint16_t*>(hist + 256);
    __shared__ unsigned s_nu, s_out, s_ntied;
    __shared__ uint32_t s_mass;
    __shared__ SumCut s_cut;
    __shared__ unsigned wtot[kSumDenseThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = kSumDenseThreads / 32;
    for (int i = tid; i < dim; i += kSumDenseThreads) tab[i] = 0u;
    for (int i = tid; i < 256; i += kSumDenseThreads) hist[i] = 0u;
    for (int64_t j = blockIdx.x; j < a.n_ids; j += gridDim.x) {
        const int64_t b = a.ids[j];
        if (tid == 0) {
            s_nu = 0u;
            s_out = 0u;
            s_ntied = 0u;
            s_mass = 0u;
        }
        __syncthreads();
        const int64_t d0 = a.bdp[b], d1 = a.bdp[b + 1];
        for (int64_t d = d0 + warp; d < d1; d += kWarps) {
            const uint2 ri = __ldg(a.f.rowinfo + a.docs[d]);
            const int64_t rb = static_cast<int64_t>(ri.x) * nsp::kRowAlign;
            const int len = static_cast<int>(ri.y);
            for (int e0 = 0; e0 < len; e0 += 256) {
                const int e = e0 + 8 * lane;
                uint32_t tw[4] = {0u, 0u, 0u, 0u};
                uint2 cw = make_uint2(0u, 0u);
                if (e < len) row8(a.f, rb, e, tw, cw);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    bool first = false;
                    uint32_t t = 0u;
                    if (e + u < len) {
                        t = term8(tw, u);
                        first = atomicMax(&tab[t], code8(cw, u) + 1u) == 0u;
                    }
                    const int o = warp_append(&s_nu, first, lane);
                    if (first) ulist[o] = static_cast<uint16_t>(t);
                }
            }
        }
        __syncthreads();
        const int nu = static_cast<int>(s_nu);
        uint32_t m = 0u;
        for (int i = tid; i < nu; i += kSumDenseThreads) {
            const uint32_t v = tab[ulist[i]] - 1u;
            m += v;
            atomicAdd(&hist[v], 1u);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(kFull, m, o);
        if (lane == 0 && m > 0u) atomicAdd(&s_mass, m);
        __syncthreads();
        if (warp == 0) {
            const SumCut c = sum_u8_cut(hist, s_mass, nu, a.alpha, lane);
            if (lane == 0) s_cut = c;
        }
        __syncthreads();
        const SumCut cut = s_cut;
        if constexpr (!kWrite) {
            if (tid == 0) a.keep[b] = cut.keep;
        } else {
            const uint32_t ntied = cut.vstar >= 0 ? hist[cut.vstar] : 0u;
            const bool partial = cut.vstar >= 0 && static_cast<uint32_t>(cut.r) < ntied;
            const int64_t out0 = a.kept_off[b - a.b0];
            const uint32_t bl = a.block_local[b - a.b0];
            // every pair above the cut level (all of that level when it is
            // kept whole)
            for (int base = 0; base < nu; base += kSumDenseThreads) {
                const int i = base + tid;
                uint32_t t = 0u;
                int v = -1;
                if (i < nu) {
                    t = ulist[i];
                    v = static_cast<int>(tab[t]) - 1;
                }
                const bool kept =
                    i < nu && (cut.vstar < 0 || v > cut.vstar || (v == cut.vstar && !partial));
                const int o = warp_append(&s_out, kept, lane);
                if (kept) {
                    a.tkey[out0 + o] = (t << 16) | bl;
                    a.tval[out0 + o] = static_cast<float>(v);
                }
            }
            if (partial) {
                // the level's first r terms in term order: thread i scans
                // terms [i * span, (i + 1) * span)
                const int span = (dim + kSumDenseThreads - 1) / kSumDenseThreads;
                const int lo = tid * span, hi = min(dim, lo + span);
                const uint32_t want = static_cast<uint32_t>(cut.vstar) + 1u;
                unsigned mine = 0u;
                for (int t = lo; t < hi; ++t) mine += tab[t] == want ? 1u : 0u;
                unsigned incl = mine;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned x = __shfl_up_sync(kFull, incl, o);
                    if (lane >= o) incl += x;
                }
                if (lane == 31) wtot[warp] = incl;
                __syncthreads();
                unsigned before = incl - mine;
                for (int w = 0; w < warp; ++w) before += wtot[w];
                for (int t = lo; t < hi && before < static_cast<unsigned>(cut.r); ++t) {
                    if (tab[t] != want) continue;
                    const unsigned o = atomicAdd(&s_out, 1u);
                    a.tkey[out0 + o] = (static_cast<uint32_t>(t) << 16) | bl;
                    a.tval[out0 + o] = static_cast<float>(cut.vstar);
                    ++before;
                }
            }
        }
        __syncthreads();
        for (int i = tid; i < nu; i += kSumDenseThreads) tab[ulist[i]] = 0u;
        for (int i = tid; i < 256; i += kSumDenseThreads) hist[i] = 0u;
        __syncthreads();
    }
}

struct SumPool {
    DevArray<int64_t> doc_eoff, flag, pos, first_run, pair_off, kept_off, rflag, rpos, o_start,
        o_lcol;
    DevArray<uint16_t> ekey, skey, block_local, o_blk, o_term;
    DevArray<uint32_t> eidx, sidx, tkey, tkey2, mass_u;
    DevArray<float> eval, delta, mass, tval, tval2;
    DevArray<int32_t> boff, entry_block, run_start, pblock, pair_off32, keep, list_koff;
    DevArray<uint8_t> has_delta, o_val, sort_tmp, tie;
    DevArray<uint64_t> pkey, pkey2;
};

// Kept summary pairs of the lists [t0, t1) -- tkey (term << 16 | block
// within its list) and tval in P, list_koff[l] the first pair of list t0 + l
// -- become the lists' summary columns, term-major per list
// (build_transpose, inverted_list_clusters.cpp:230-293), appended to `out`.
template <int ESZ>
void emit_columns(nsp::SeismicHost& L, int32_t t0, int32_t t1,
                  const std::vector<int64_t>& list_koff, int64_t n_kept, cudaStream_t s,
                  SumPool& P, DevColumns& out) {
    const int sms = nsp::device_sm_count();
    const int64_t nk1 = std::max<int64_t>(n_kept, 1);
    const std::vector<int32_t> list_koff32 = to_i32_offsets(list_koff);
    P.list_koff.upload(list_koff32.data(), list_koff32.size(), s);
    segmented_sort_pairs(P.tkey.data(), P.tkey2.data(), P.tval.data(), P.tval2.data(), n_kept,
                         t1 - t0, P.list_koff.data(), s, /*stable=*/false, &P.sort_tmp);
    g_steps.mark("transpose sort");
    // columns assembled on the device: block ids, values, and one run per
    // (list, term) with its start
    const int32_t nl = t1 - t0;
    P.o_blk.grow(nk1);
    P.o_val.grow(nk1 * ESZ);
    P.rflag.grow(n_kept + 1);
    P.rpos.grow(n_kept + 1);
    columns_kernel<ESZ><<<sms * 8, 256, 0, s>>>(P.tkey2.data(), P.tval2.data(), n_kept,
                                                P.o_blk.data(), P.o_val.data(), P.rflag.data());
    cuda_check(cudaGetLastError(), "columns_kernel");
    list_start_kernel<<<std::max(1, (nl + 255) / 256), 256, 0, s>>>(P.list_koff.data(), nl,
                                                                    n_kept, P.rflag.data());
    cuda_check(cudaGetLastError(), "list_start_kernel");
    nsp::exclusive_scan_i64(P.rflag.data(), P.rpos.data(), n_kept + 1, s);
    int64_t n_cols = 0;
    cuda_check(cudaMemcpyAsync(&n_cols, P.rpos.data() + n_kept, 8, cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    P.o_term.grow(std::max<int64_t>(n_cols, 1));
    P.o_start.grow(std::max<int64_t>(n_cols, 1));
    P.o_lcol.grow(static_cast<size_t>(nl) + 1);
    column_compact_kernel<<<sms * 8, 256, 0, s>>>(P.tkey2.data(), P.rflag.data(), P.rpos.data(),
                                                  n_kept, P.o_term.data(), P.o_start.data());
    cuda_check(cudaGetLastError(), "column_compact_kernel");
    list_cols_kernel<<<std::max(1, (nl + 1 + 255) / 256), 256, 0, s>>>(
        P.list_koff.data(), nl, P.rpos.data(), P.o_lcol.data());
    cuda_check(cudaGetLastError(), "list_cols_kernel");
    // appended to the index's device columns; only the per-list column
    // counts come back to the host
    const size_t eb = out.n_entries, cb = out.n_cols;
    dev_append(out.sblk, eb, P.o_blk.data(), static_cast<size_t>(n_kept), s);
    dev_append(out.sval, eb * ESZ, P.o_val.data(), static_cast<size_t>(n_kept) * ESZ, s);
    dev_append(out.sterm, cb, P.o_term.data(), static_cast<size_t>(n_cols), s);
    if (out.srun.size() < cb + 1 + static_cast<size_t>(n_cols)) {
        DevArray<int64_t> bigger(
            std::max(out.srun.size() * 2, cb + 1 + static_cast<size_t>(n_cols)));
        cuda_check(cudaMemcpyAsync(bigger.data(), out.srun.data(), (cb + 1) * sizeof(int64_t),
                                   cudaMemcpyDeviceToDevice, s),
                   "D2D");
        cuda_check(cudaStreamSynchronize(s), "sync");
        out.srun = std::move(bigger);
    }
    if (n_cols > 0)
        column_bounds_kernel<<<sms * 4, 256, 0, s>>>(P.o_start.data(), n_cols,
                                                     static_cast<int64_t>(eb), n_kept,
                                                     out.srun.data() + cb + 1);
    cuda_check(cudaGetLastError(), "column_bounds_kernel");
    std::vector<int64_t> h_lcol(static_cast<size_t>(nl) + 1);
    P.o_lcol.download(h_lcol.data(), h_lcol.size(), s);
    cuda_check(cudaStreamSynchronize(s), "D2H");
    out.n_entries += static_cast<size_t>(n_kept);
    out.n_cols += static_cast<size_t>(n_cols);
    for (int32_t l = 0; l < nl; ++l) L.ltp.push_back(static_cast<int64_t>(cb) + h_lcol[l + 1]);
    g_steps.mark("columns");
}

template <int ESZ>
void summarize_batch(const nsp::FwdView& f, const DevArray<int32_t>& d_docs,
                     const DevArray<int64_t>& d_bdp, nsp::SeismicHost& L, int32_t t0, int32_t t1,
                     const std::vector<int64_t>& doc_eoff, const std::vector<int64_t>& blk_e,
                     float alpha, cudaStream_t s, SumPool& P, DevColumns& out,
                     const nsp::HostCsr* host) {
    const int sms = nsp::device_sm_count();
    const int64_t b0 = L.lbp[t0], b1 = L.lbp[t1];
    const int64_t nb = b1 - b0;
    const int64_t e0 = blk_e[b0], ne = blk_e[b1] - e0;
    // entries in block order
    const int64_t* ed = doc_eoff.data() + L.bdp[b0];
    P.doc_eoff.upload(ed, static_cast<size_t>(L.bdp[b1] - L.bdp[b0] + 1), s);
    P.ekey.grow(ne);
    P.skey.grow(ne);
    P.eidx.grow(ne);
    P.sidx.grow(ne);
    P.eval.grow(ne);
    entries_kernel<ESZ><<<sms * 8, 256, 0, s>>>(f, d_docs.data(), d_bdp.data(), b0, nb,
                                                P.doc_eoff.data(), e0, P.ekey.data(),
                                                P.eidx.data(), P.eval.data());
    cuda_check(cudaGetLastError(), "entries_kernel");
    g_steps.mark("entries");
    std::vector<int64_t> boff64(blk_e.begin() + b0, blk_e.begin() + b1 + 1);
    for (auto& v : boff64) v -= e0;
    const std::vector<int32_t> boff32 = to_i32_offsets(boff64);
    P.boff.upload(boff32.data(), boff32.size(), s);
    // stable: entries of a term stay in block order
    segmented_sort_pairs(P.ekey.data(), P.skey.data(), P.eidx.data(), P.sidx.data(), ne, nb,
                         P.boff.data(), s, /*stable=*/true, &P.sort_tmp);
    g_steps.mark("sort entries");
    P.entry_block.grow(ne);
    fill_block_kernel<<<sms * 8, 256, 0, s>>>(P.boff.data(), nb, P.entry_block.data());
    cuda_check(cudaGetLastError(), "fill_block_kernel");
    P.flag.grow(ne);
    P.pos.grow(ne);
    run_flag_kernel<<<sms * 8, 256, 0, s>>>(P.skey.data(), P.entry_block.data(), ne,
                                            P.flag.data());
    cuda_check(cudaGetLastError(), "run_flag_kernel");
    nsp::exclusive_scan_i64(P.flag.data(), P.pos.data(), ne, s);
    int64_t last_pos = 0, last_flag = 0;
    cuda_check(cudaMemcpyAsync(&last_pos, P.pos.data() + ne - 1, 8, cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaMemcpyAsync(&last_flag, P.flag.data() + ne - 1, 8, cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    const int64_t n_runs = last_pos + last_flag;
    g_steps.mark("runs scan");
    const int64_t nr1 = std::max<int64_t>(n_runs, 1);
    P.run_start.grow(nr1);
    run_compact_kernel<<<sms * 8, 256, 0, s>>>(P.flag.data(), P.pos.data(), ne,
                                               P.run_start.data());
    cuda_check(cudaGetLastError(), "run_compact_kernel");
    // pairs per block: the run index at each block's first entry
    std::vector<int64_t> pair_off(static_cast<size_t>(nb) + 1);
    {
        P.first_run.grow(nb);
        block_first_run_kernel<<<sms * 4, 256, 0, s>>>(P.pos.data(), P.boff.data(), nb, ne,
                                                       n_runs, P.first_run.data());
        cuda_check(cudaGetLastError(), "block_first_run_kernel");
        P.first_run.download(pair_off.data(), static_cast<size_t>(nb), s);
        cuda_check(cudaStreamSynchronize(s), "D2H");
        pair_off[nb] = n_runs;
        // an empty block has no runs: its offset is the next block's
        for (int64_t b = nb - 1; b >= 0; --b)
            if (boff64[b] == boff64[b + 1]) pair_off[b] = pair_off[b + 1];
    }
    if constexpr (ESZ != 1) {
        P.delta.grow(ne);
        P.has_delta.grow(ne);
    }
    P.pkey.grow(nr1);
    P.pkey2.grow(nr1);
    P.pblock.grow(nr1);
    P.mass.grow(nb);
    if constexpr (ESZ == 1) {
        P.mass_u.grow(nb);
        cuda_check(cudaMemsetAsync(P.mass_u.data(), 0, static_cast<size_t>(nb) * 4, s), "memset");
    }
    runs_kernel<ESZ><<<sms * 8, 256, 0, s>>>(P.skey.data(), P.sidx.data(), P.eval.data(),
                                             P.run_start.data(), n_runs, ne,
                                             P.entry_block.data(), P.delta.data(),
                                             P.has_delta.data(), P.pkey.data(), P.pblock.data(),
                                             ESZ == 1 ? P.mass_u.data() : nullptr);
    cuda_check(cudaGetLastError(), "runs_kernel");
    if constexpr (ESZ == 1) {
        mass_from_int_kernel<<<sms * 4, 256, 0, s>>>(P.mass_u.data(), nb, P.mass.data());
        cuda_check(cudaGetLastError(), "mass_from_int_kernel");
    } else {
        mass_kernel<<<sms * 4, 128, 0, s>>>(P.delta.data(), P.has_delta.data(), P.boff.data(), nb,
                                            P.mass.data());
        cuda_check(cudaGetLastError(), "mass_kernel");
    }
    g_steps.mark("runs, mass");
    // alpha cut over each block's maxima, value descending
    const std::vector<int32_t> pair_off32 = to_i32_offsets(pair_off);
    P.pair_off32.upload(pair_off32.data(), pair_off32.size(), s);
    segmented_sort_keys(P.pkey.data(), P.pkey2.data(), n_runs, nb, P.pair_off32.data(), s,
                        &P.sort_tmp);
    P.pair_off.upload(pair_off.data(), pair_off.size(), s);
    g_steps.mark("sort maxima");
    P.keep.grow(nb);
    cut_kernel<<<sms * 4, 128, 0, s>>>(P.pkey2.data(), P.pair_off.data(), nb, P.mass.data(),
                                       alpha, P.keep.data());
    cuda_check(cudaGetLastError(), "cut_kernel");
    std::vector<int32_t> h_keep(static_cast<size_t>(nb));
    P.keep.download(h_keep.data(), h_keep.size(), s);
    cuda_check(cudaStreamSynchronize(s), "D2H");
    if (host != nullptr) {
        // fp32: where equal maxima straddle the cut, take the reference's
        // choice -- its kept terms move to the front of the block's pairs
        // (the count is the same: equal values give equal running sums)
        P.tie.grow(nb);
        cut_tie_kernel<<<sms * 4, 128, 0, s>>>(P.pkey2.data(), P.pair_off.data(), nb,
                                               P.keep.data(), P.tie.data());
        cuda_check(cudaGetLastError(), "cut_tie_kernel");
        std::vector<uint8_t> tie(static_cast<size_t>(nb));
        P.tie.download(tie.data(), tie.size(), s);
        cuda_check(cudaStreamSynchronize(s), "D2H");
        for (int64_t b = 0; b < nb; ++b) {
            if (!tie[b]) continue;
            const int64_t gb = b0 + b;
            const std::vector<uint16_t> kept = nsp::reference_summary_kept(
                *host, L.docs.data() + L.bdp[gb], static_cast<size_t>(L.bdp[gb + 1] - L.bdp[gb]),
                alpha);
            const int64_t ps = pair_off[b], pn = pair_off[b + 1] - ps;
            std::vector<uint64_t> seg(static_cast<size_t>(pn));
            cuda_check(cudaMemcpyAsync(seg.data(), P.pkey2.data() + ps, seg.size() * 8,
                                       cudaMemcpyDeviceToHost, s), "D2H");
            cuda_check(cudaStreamSynchronize(s), "D2H");
            std::vector<uint8_t> keep_term(65536, 0);
            for (const uint16_t t : kept) keep_term[t] = 1;
            std::stable_partition(seg.begin(), seg.end(),
                                  [&](uint64_t k) { return keep_term[k & 0xffffu] != 0; });
            h_keep[b] = static_cast<int32_t>(kept.size());
            cuda_check(cudaMemcpyAsync(P.pkey2.data() + ps, seg.data(), seg.size() * 8,
                                       cudaMemcpyHostToDevice, s), "H2D");
            cuda_check(cudaMemcpyAsync(P.keep.data() + b, &h_keep[b], sizeof(int32_t),
                                       cudaMemcpyHostToDevice, s), "H2D");
            cuda_check(cudaStreamSynchronize(s), "sync");
        }
    }
    std::vector<int64_t> kept_off(static_cast<size_t>(nb) + 1, 0);
    for (int64_t b = 0; b < nb; ++b) kept_off[b + 1] = kept_off[b] + h_keep[b];
    const int64_t n_kept = kept_off[nb];
    std::vector<uint16_t> block_local(static_cast<size_t>(nb));
    std::vector<int64_t> list_koff(static_cast<size_t>(t1 - t0) + 1, 0);
    for (int32_t t = t0; t < t1; ++t) {
        for (int64_t b = L.lbp[t]; b < L.lbp[t + 1]; ++b)
            block_local[b - b0] = static_cast<uint16_t>(b - L.lbp[t]);
        list_koff[t - t0 + 1] = kept_off[L.lbp[t + 1] - b0];
    }
    P.kept_off.upload(kept_off.data(), kept_off.size(), s);
    P.block_local.upload(block_local.data(), block_local.size(), s);
    const int64_t nk1 = std::max<int64_t>(n_kept, 1);
    P.tkey.grow(nk1);
    P.tkey2.grow(nk1);
    P.tval.grow(nk1);
    P.tval2.grow(nk1);
    kept_pairs_kernel<<<sms * 8, 128, 0, s>>>(P.pkey2.data(), P.pair_off.data(), P.keep.data(),
                                              P.kept_off.data(), P.block_local.data(), nb,
                                              P.tkey.data(), P.tval.data());
    cuda_check(cudaGetLastError(), "kept_pairs_kernel");
    g_steps.mark("alpha cut");
    emit_columns<ESZ>(L, t0, t1, list_koff, n_kept, s, P, out);
}

// Entries of each block (its docs' row lengths summed), for the choice
// between the two kernels.
__global__ void block_entries_kernel(nsp::FwdView f, const int32_t* docs, const int64_t* bdp,
                                     int64_t nb, int32_t* ent) {
    for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b < nb;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t e = 0;
        for (int64_t j = bdp[b]; j < bdp[b + 1]; ++j) e += f.rowinfo[docs[j]].y;
        ent[b] = static_cast<int32_t>(e < INT32_MAX ? e : INT32_MAX);
    }
}

std::vector<int32_t> block_entries(const nsp::FwdView& f, const DevArray<int32_t>& d_docs,
                                   const DevArray<int64_t>& d_bdp, int64_t nb, cudaStream_t s) {
    if (nb == 0) return {};
    DevArray<int32_t> ent(static_cast<size_t>(nb));
    const int sms = nsp::device_sm_count();
    block_entries_kernel<<<sms * 8, 256, 0, s>>>(f, d_docs.data(), d_bdp.data(), nb, ent.data());
    cuda_check(cudaGetLastError(), "block_entries_kernel");
    return to_host(ent, static_cast<size_t>(nb), s);
}

// Dynamic shared memory of the large-block kernel: a word and a list entry
// per term, and the histogram.
size_t sum_u8_dense_smem(int dim) {
    return static_cast<size_t>(dim) * 4 + 256 * 4 + static_cast<size_t>(dim) * 2;
}

// Whether the fused uint8 summaries run on this device for this dimension.
bool sum_u8_fits(int dim) {
    int dev = 0, optin = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
               "cudaDeviceGetAttribute");
    return sum_u8_dense_smem(dim) <= static_cast<size_t>(optin);
}

// Summaries of every block of a uint8 index (section 5' above): a count
// pass over all blocks, then, per batch of lists bounded by kept pairs, a
// write pass and the term-major columns.
void summarize_u8(const nsp::FwdView& f, const DevArray<int32_t>& d_docs,
                  const DevArray<int64_t>& d_bdp, nsp::SeismicHost& L,
                  const std::vector<int32_t>& blk_n, float alpha, cudaStream_t s, SumPool& P,
                  DevColumns& out) {
    const int sms = nsp::device_sm_count();
    const int64_t n_blocks = L.lbp.back();
    const int32_t n_lists = L.n_lists();
    std::vector<int64_t> small, big;
    for (int64_t b = 0; b < n_blocks; ++b)
        (blk_n[b] <= kSumHashEntries ? small : big).push_back(b);
    DevArray<int64_t> d_small, d_big;
    if (!small.empty()) to_dev(d_small, small, s);
    if (!big.empty()) to_dev(d_big, big, s);
    const size_t dense_smem = sum_u8_dense_smem(f.dim);
    cuda_check(cudaFuncSetAttribute(sum_u8_dense_kernel<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(dense_smem)),
               "cudaFuncSetAttribute");
    cuda_check(cudaFuncSetAttribute(sum_u8_dense_kernel<true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(dense_smem)),
               "cudaFuncSetAttribute");
    auto launch = [&](SumU8Args a, int64_t s0, int64_t s1, int64_t g0, int64_t g1, bool write) {
        if (s1 > s0) {
            a.ids = d_small.data() + s0;
            a.n_ids = s1 - s0;
            const int grid = static_cast<int>(std::min<int64_t>(a.n_ids, int64_t{sms} * 8));
            if (write)
                sum_u8_hash_kernel<true><<<grid, kSumHashThreads, 0, s>>>(a);
            else
                sum_u8_hash_kernel<false><<<grid, kSumHashThreads, 0, s>>>(a);
            cuda_check(cudaGetLastError(), "sum_u8_hash_kernel");
        }
        if (g1 > g0) {
            a.ids = d_big.data() + g0;
            a.n_ids = g1 - g0;
            const int grid = static_cast<int>(std::min<int64_t>(a.n_ids, sms));
            if (write)
                sum_u8_dense_kernel<true><<<grid, kSumDenseThreads, dense_smem, s>>>(a);
            else
                sum_u8_dense_kernel<false><<<grid, kSumDenseThreads, dense_smem, s>>>(a);
            cuda_check(cudaGetLastError(), "sum_u8_dense_kernel");
        }
    };
    SumU8Args a{};
    a.f = f;
    a.docs = d_docs.data();
    a.bdp = d_bdp.data();
    a.alpha = alpha;
    DevArray<int32_t> keep(static_cast<size_t>(std::max<int64_t>(n_blocks, 1)));
    a.keep = keep.data();
    launch(a, 0, static_cast<int64_t>(small.size()), 0, static_cast<int64_t>(big.size()), false);
    const std::vector<int32_t> h_keep = to_host(keep, static_cast<size_t>(n_blocks), s);
    std::vector<int64_t> kept_off(static_cast<size_t>(n_blocks) + 1, 0);
    for (int64_t b = 0; b < n_blocks; ++b) kept_off[b + 1] = kept_off[b] + h_keep[b];
    g_steps.mark("u8 count");
    const int64_t budget = int64_t{1} << 27;  // kept pairs per batch
    int32_t t0 = 0;
    while (t0 < n_lists) {
        int32_t t1 = t0 + 1;
        while (t1 < n_lists && kept_off[L.lbp[t1 + 1]] - kept_off[L.lbp[t0]] <= budget) ++t1;
        const int64_t b0 = L.lbp[t0], b1 = L.lbp[t1];
        const int64_t nb = b1 - b0;
        const int64_t n_kept = kept_off[b1] - kept_off[b0];
        if (n_kept == 0) {
            for (int32_t t = t0; t < t1; ++t) L.ltp.push_back(L.ltp.back());
            t0 = t1;
            continue;
        }
        std::vector<int64_t> rel(static_cast<size_t>(nb) + 1);
        for (int64_t b = 0; b <= nb; ++b) rel[b] = kept_off[b0 + b] - kept_off[b0];
        std::vector<uint16_t> block_local(static_cast<size_t>(nb));
        std::vector<int64_t> list_koff(static_cast<size_t>(t1 - t0) + 1, 0);
        for (int32_t t = t0; t < t1; ++t) {
            for (int64_t b = L.lbp[t]; b < L.lbp[t + 1]; ++b)
                block_local[b - b0] = static_cast<uint16_t>(b - L.lbp[t]);
            list_koff[t - t0 + 1] = rel[L.lbp[t + 1] - b0];
        }
        P.kept_off.upload(rel.data(), rel.size(), s);
        P.block_local.upload(block_local.data(), block_local.size(), s);
        const size_t nk1 = static_cast<size_t>(std::max<int64_t>(n_kept, 1));
        P.tkey.grow(nk1);
        P.tkey2.grow(nk1);
        P.tval.grow(nk1);
        P.tval2.grow(nk1);
        SumU8Args w = a;
        w.kept_off = P.kept_off.data();
        w.block_local = P.block_local.data();
        w.b0 = b0;
        w.tkey = P.tkey.data();
        w.tval = P.tval.data();
        const int64_t s0 = std::lower_bound(small.begin(), small.end(), b0) - small.begin();
        const int64_t s1 = std::lower_bound(small.begin(), small.end(), b1) - small.begin();
        const int64_t g0 = std::lower_bound(big.begin(), big.end(), b0) - big.begin();
        const int64_t g1 = std::lower_bound(big.begin(), big.end(), b1) - big.begin();
        launch(w, s0, s1, g0, g1, true);
        g_steps.mark("u8 write");
        emit_columns<1>(L, t0, t1, list_koff, n_kept, s, P, out);
        t0 = t1;
    }
}

// fp32 lists whose kept postings hold tied values get the reference's kept
// order from the host (ref_order.cpp); every other list's device order
// (value desc, then doc asc) is already the reference's.
void reference_tie_order(const nsp::HostCsr& h, const std::vector<int64_t>& post,
                         const std::vector<int64_t>& kept_ptr, const std::vector<uint8_t>& tie,
                         int64_t cap, DevArray<int32_t>& kept, cudaStream_t s) {
    std::vector<int32_t> lists;
    for (int32_t t = 0; t < static_cast<int32_t>(tie.size()); ++t)
        if (tie[t]) lists.push_back(t);
    if (lists.empty()) return;
    std::vector<int32_t> out;
    nsp::reference_kept_order(h, post, lists, cap, out);
    for (size_t j = 0; j < lists.size(); ++j)
        cuda_check(cudaMemcpyAsync(kept.data() + kept_ptr[lists[j]], out.data() + j * cap,
                                   static_cast<size_t>(cap) * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, s),
                   "H2D kept order");
    cuda_check(cudaStreamSynchronize(s), "sync");
}

// Phase timings on stderr when NSP_VERBOSE=1 (the engine's one debug switch).
struct PhaseClock {
    cudaStream_t s;
    bool on;
    std::chrono::steady_clock::time_point t;
    explicit PhaseClock(cudaStream_t st) : s(st) {
        const char* v = std::getenv("NSP_VERBOSE");
        on = v != nullptr && v[0] == '1';
        t = std::chrono::steady_clock::now();
    }
    void mark(const char* what) {
        if (!on) return;
        cudaStreamSynchronize(s);
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[nsparse build] %-12s %8.3f s\n", what,
                     std::chrono::duration<double>(now - t).count());
        t = now;
    }
};

template <int ESZ>
void build_typed(SeismicState& st, int dim, const SeismicClusterParameters& p) {
    const nsp::HostCsr& h = st.vectors.host;
    cudaStream_t s = nsp::Workspace::get().stream();
    const int64_t n_docs = h.n();
    const int lambda = calc_lambda(p.lambda, static_cast<size_t>(n_docs));
    const int beta = calc_beta(p.beta, lambda);
    const int64_t cap = lambda <= 0 ? 0 : lambda;  // 0: keep whole lists (inverted_lists.cpp:114)
    const uint32_t base_seed =
        p.seed == -1 ? std::random_device{}() : static_cast<uint32_t>(p.seed);
    st.vectors.ensure_device();
    const nsp::FwdView f = st.vectors.dev.view();
    const int32_t n_lists = dim;
    const int sms = nsp::device_sm_count();
    PhaseClock clock(s);

    // ---- 1. postings
    DevArray<unsigned long long> cnt(static_cast<size_t>(n_lists) + 1);
    cuda_check(cudaMemsetAsync(cnt.data(), 0, cnt.size() * 8, s), "memset");
    post_count_kernel<<<sms * 8, 256, 0, s>>>(f, cnt.data());
    cuda_check(cudaGetLastError(), "post_count_kernel");
    DevArray<int64_t> post_ptr(static_cast<size_t>(n_lists) + 1);
    nsp::exclusive_scan_i64(reinterpret_cast<const int64_t*>(cnt.data()), post_ptr.data(),
                            n_lists + 1, s);
    const std::vector<int64_t> h_post = to_host(post_ptr, n_lists + 1, s);
    const int64_t nnz = h_post.back();
    DevArray<uint64_t> keys(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    DevArray<uint64_t> keys2(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    cuda_check(cudaMemsetAsync(cnt.data(), 0, cnt.size() * 8, s), "memset");
    post_scatter_kernel<ESZ><<<sms * 8, 256, 0, s>>>(f, post_ptr.data(), cnt.data(), cap, keys.data());
    cuda_check(cudaGetLastError(), "post_scatter_kernel");
    {
        DevArray<int32_t> off32;
        to_dev(off32, to_i32_offsets(h_post), s);
        segmented_sort_keys(keys.data(), keys2.data(), nnz, n_lists, off32.data(), s);
    }
    keys.reset();
    std::vector<int32_t> kept_len(n_lists);
    std::vector<int64_t> kept_ptr(n_lists + 1, 0);
    for (int32_t t = 0; t < n_lists; ++t) {
        const int64_t len = h_post[t + 1] - h_post[t];
        kept_len[t] = static_cast<int32_t>(cap > 0 && len > cap ? cap : len);
        kept_ptr[t + 1] = kept_ptr[t] + kept_len[t];
    }
    const int64_t total_kept = kept_ptr.back();
    DevArray<int64_t> d_kept_ptr;
    to_dev(d_kept_ptr, kept_ptr, s);
    DevArray<int32_t> kept(static_cast<size_t>(std::max<int64_t>(total_kept, 1)));
    kept_copy_kernel<<<sms * 8, 256, 0, s>>>(keys2.data(), post_ptr.data(), d_kept_ptr.data(),
                                             n_lists, kept.data());
    cuda_check(cudaGetLastError(), "kept_copy_kernel");
    std::vector<uint8_t> tie(static_cast<size_t>(n_lists), 0);
    if (ESZ == 4 && cap > 0) {
        DevArray<uint8_t> d_tie(static_cast<size_t>(n_lists));
        tie_flag_kernel<<<sms * 8, 256, 0, s>>>(keys2.data(), post_ptr.data(), n_lists, cap,
                                                d_tie.data());
        cuda_check(cudaGetLastError(), "tie_flag_kernel");
        d_tie.download(tie.data(), tie.size(), s);
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
    keys2.reset();
    if (ESZ == 4) reference_tie_order(h, h_post, kept_ptr, tie, cap, kept, s);

    clock.mark("postings");
    // ---- 2. centroid positions (host; depends on list lengths only)
    std::vector<int64_t> cptr(n_lists + 1, 0);
    for (int32_t t = 0; t < n_lists; ++t)
        cptr[t + 1] = cptr[t] + (kept_len[t] > 0 ? static_cast<int64_t>(clusters_for(kept_len[t], beta)) : 0);
    int32_t max_nc = 0;
    int64_t max_kept = 0;
    for (int32_t t = 0; t < n_lists; ++t) {
        max_nc = std::max<int32_t>(max_nc, static_cast<int32_t>(cptr[t + 1] - cptr[t]));
        max_kept = std::max<int64_t>(max_kept, kept_len[t]);
    }
    if (max_nc > 65536)
        throw std::invalid_argument("more than 65536 blocks in one posting list");
    std::vector<int32_t> cpos(static_cast<size_t>(std::max<int64_t>(cptr.back(), 1)));
    {
        const int nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (int w = 0; w < nth; ++w) {
            pool.emplace_back([&, w] {
                std::vector<int32_t> perm;
                for (int32_t t = w; t < n_lists; t += nth) {
                    if (kept_len[t] == 0) continue;
                    draw_positions(static_cast<size_t>(kept_len[t]),
                                   static_cast<size_t>(cptr[t + 1] - cptr[t]),
                                   base_seed + static_cast<uint32_t>(t), perm, cpos.data() + cptr[t]);
                }
            });
        }
        for (auto& th : pool) th.join();
    }
    DevArray<int64_t> d_cptr;
    DevArray<int32_t> d_cpos;
    to_dev(d_cptr, cptr, s);
    to_dev(d_cpos, cpos, s);

    clock.mark("centroids");
    // ---- 3. assignment
    DevArray<uint32_t> akey(static_cast<size_t>(std::max<int64_t>(total_kept, 1)));
    if (total_kept > 0) {
        // centroid entries per list bound: max_nc rows of the longest rows
        int64_t max_row = 0;
        for (int64_t d = 0; d < n_docs; ++d)
            max_row = std::max<int64_t>(max_row, h.indptr[d + 1] - h.indptr[d]);
        const int64_t max_ce = std::max<int64_t>(1, static_cast<int64_t>(max_nc) * max_row);
        const int wpb = 32;
        const size_t acc_bytes = sizeof(assign_acc_t<ESZ>);
        const size_t sims_smem = static_cast<size_t>(wpb) * std::max(max_nc, 1) * acc_bytes;
        const bool sims_in_smem = sims_smem <= 160u * 1024u;
        const size_t smem = sims_in_smem ? sims_smem : 0;
        if (sims_in_smem) cuda_check(nsp::allow_opt_in_smem(assign_kernel<ESZ>), "assign smem");
        // one CTA of 32 warps per SM: as many warps as four CTAs of 8 hide
        // the memory round trips with, and a quarter of the per-CTA term
        // tables (trun, tcnt, ...), which then stay in L2 (8.8M SQ docs:
        // 6.4 -> 5.5 s against four CTAs of 8 warps; two of 16: 5.7 s)
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, assign_kernel<ESZ>,
                                                                 wpb * 32, smem),
                   "assign occupancy");
        const int ctas = sms * std::max(1, std::min(per_sm, 1));
        DevArray<int32_t> tcnt(static_cast<size_t>(ctas) * dim), tstart(static_cast<size_t>(ctas) * dim),
            tcur(static_cast<size_t>(ctas) * dim), touched(static_cast<size_t>(ctas) * max_ce);
        DevArray<int2> trun(static_cast<size_t>(ctas) * dim);
        DevArray<uint16_t> ccl(static_cast<size_t>(ctas) * max_ce);
        DevArray<uint8_t> cw(static_cast<size_t>(ctas) * max_ce * ESZ);
        DevArray<uint8_t> isc(static_cast<size_t>(ctas) * std::max<int64_t>(max_kept, 1));
        DevArray<uint8_t> sims(static_cast<size_t>(ctas) * wpb * std::max(max_nc, 1) * 8);
        DevArray<int32_t> work(1);
        cuda_check(cudaMemsetAsync(tcnt.data(), 0, tcnt.size() * 4, s), "memset");
        cuda_check(cudaMemsetAsync(trun.data(), 0, trun.size() * sizeof(int2), s), "memset");
        cuda_check(cudaMemsetAsync(work.data(), 0, 4, s), "memset");
        AssignArgs a{};
        a.f = f;
        a.n_lists = n_lists;
        a.kept_ptr = d_kept_ptr.data();
        a.kept = kept.data();
        a.cptr = d_cptr.data();
        a.cpos = d_cpos.data();
        a.out_key = akey.data();
        a.work = work.data();
        a.tcnt = tcnt.data();
        a.tstart = tstart.data();
        a.tcur = tcur.data();
        a.trun = trun.data();
        a.touched = touched.data();
        a.ccl = ccl.data();
        a.cw = cw.data();
        a.is_centroid = isc.data();
        a.sims = sims.data();
        a.max_centroid_entries = max_ce;
        a.max_kept = std::max<int64_t>(max_kept, 1);
        a.max_nc = std::max(max_nc, 1);
        a.sims_in_smem = sims_in_smem ? 1 : 0;
        assign_kernel<ESZ><<<ctas, wpb * 32, smem, s>>>(a);
        cuda_check(cudaGetLastError(), "assign_kernel");
        cuda_check(cudaStreamSynchronize(s), "assign sync");
    }

    clock.mark("assignment");
    // ---- 4. blocks: centroid first, members in list order
    DevArray<int32_t> bdocs(static_cast<size_t>(std::max<int64_t>(total_kept, 1)));
    DevArray<uint32_t> akey2(static_cast<size_t>(std::max<int64_t>(total_kept, 1)));
    {
        DevArray<int32_t> off32;
        to_dev(off32, to_i32_offsets(kept_ptr), s);
        segmented_sort_pairs(akey.data(), akey2.data(), kept.data(), bdocs.data(), total_kept,
                             n_lists, off32.data(), s, /*stable=*/true);
    }
    const std::vector<uint32_t> h_akey = to_host(akey2, static_cast<size_t>(total_kept), s);
    akey.reset();
    akey2.reset();
    kept.reset();
    nsp::SeismicHost L;
    L.esz = ESZ;
    L.lbp.assign(1, 0);
    L.bdp.assign(1, 0);
    L.docs = to_host(bdocs, static_cast<size_t>(total_kept), s);
    for (int32_t t = 0; t < n_lists; ++t) {
        const int64_t nc = cptr[t + 1] - cptr[t];
        L.lbp.push_back(L.lbp.back() + nc);
        int64_t i = kept_ptr[t];
        for (int64_t c = 0; c < nc; ++c) {
            while (i < kept_ptr[t + 1] && static_cast<int64_t>(h_akey[i] >> 1) == c) ++i;
            L.bdp.push_back(i);
        }
    }
    const int64_t n_blocks = L.lbp.back();

    clock.mark("blocks");
    // ---- 5. summaries, in batches of lists bounded by entry count
    const bool fused_u8 = ESZ == 1 && sum_u8_fits(dim);
    DevArray<int64_t> d_bdp;
    to_dev(d_bdp, L.bdp, s);
    DevArray<int32_t> d_docs = std::move(bdocs);  // the block-ordered docs, still resident
    std::vector<int64_t> doc_eoff, blk_e;
    std::vector<int32_t> blk_n;  // fused uint8 path: entries per block
    if (fused_u8) {
        blk_n = block_entries(f, d_docs, d_bdp, n_blocks, s);
    } else {
        std::vector<int64_t> doc_len(static_cast<size_t>(total_kept));
        for (int64_t j = 0; j < total_kept; ++j) {
            const int32_t d = L.docs[j];
            doc_len[j] = h.indptr[d + 1] - h.indptr[d];
        }
        doc_eoff.assign(static_cast<size_t>(total_kept) + 1, 0);
        for (int64_t j = 0; j < total_kept; ++j) doc_eoff[j + 1] = doc_eoff[j] + doc_len[j];
        blk_e.assign(static_cast<size_t>(n_blocks) + 1, 0);
        for (int64_t b = 0; b <= n_blocks; ++b) blk_e[b] = doc_eoff[L.bdp[b]];
    }
    const int64_t budget = int64_t{1} << 27;  // entries per batch
    g_steps.start(s);
    SumPool pool;
    L.ltp.assign(1, 0);
    L.srun.assign(1, 0);
    L.sterm.clear();
    L.sblk.clear();
    L.sval.clear();
    DevColumns cols;
    cols.srun.resize(1);
    cuda_check(cudaMemsetAsync(cols.srun.data(), 0, sizeof(int64_t), s), "memset");
    int32_t t0 = 0;
    if (fused_u8) {
        summarize_u8(f, d_docs, d_bdp, L, blk_n, p.alpha, s, pool, cols);
        t0 = n_lists;
    }
    while (t0 < n_lists) {
        int32_t t1 = t0 + 1;
        while (t1 < n_lists && blk_e[L.lbp[t1 + 1]] - blk_e[L.lbp[t0]] <= budget) ++t1;
        const int64_t b0 = L.lbp[t0], b1 = L.lbp[t1];
        const int64_t nb = b1 - b0;
        const int64_t e0 = blk_e[b0], ne = blk_e[b1] - e0;
        if (nb == 0 || ne == 0) {
            for (int32_t t = t0; t < t1; ++t) L.ltp.push_back(L.ltp.back());
            t0 = t1;
            continue;
        }
        summarize_batch<ESZ>(f, d_docs, d_bdp, L, t0, t1, doc_eoff, blk_e, p.alpha, s, pool,
                             cols, ESZ == 4 ? &st.vectors.host : nullptr);
        t0 = t1;
    }

    clock.mark("summaries");
    g_steps.print();
    // ---- 6. publish: the device image takes the built arrays; the host copy
    // is filled on demand (host_lists)
    std::lock_guard<std::mutex> g(st.mu);
    st.lists_dev.adopt(L.lbp, L.bdp, L.ltp, ESZ, dim, std::move(d_docs), std::move(cols.sterm),
                       std::move(cols.srun), std::move(cols.sblk), std::move(cols.sval));
    st.lists = nsp::SeismicHost{};
    st.lists.esz = ESZ;
    st.list_esz.assign(static_cast<size_t>(n_lists), static_cast<uint8_t>(ESZ));
    st.host_valid = false;
    st.dev_valid = true;
}

}  // namespace

void seismic_build(SeismicState& st, int dim, const SeismicClusterParameters& params) {
    if (!st.vectors.terms_in_range(dim)) throw std::invalid_argument("term_id out of range");
    const int esz = st.vectors.host.esz;
    if (st.vectors.host.n() == 0) {
        // no documents: one empty list per term
        nsp::SeismicHost L;
        L.esz = esz;
        L.lbp.assign(static_cast<size_t>(dim) + 1, 0);
        L.ltp.assign(static_cast<size_t>(dim) + 1, 0);
        std::lock_guard<std::mutex> g(st.mu);
        st.lists = std::move(L);
        st.list_esz.assign(static_cast<size_t>(dim), static_cast<uint8_t>(esz));
        st.host_valid = true;
        st.dev_valid = false;
        return;
    }
    if (esz == 4) build_typed<4>(st, dim, params);
    else if (esz == 2) build_typed<2>(st, dim, params);
    else build_typed<1>(st, dim, params);
}

}  // namespace detail
}  // namespace nsparse
