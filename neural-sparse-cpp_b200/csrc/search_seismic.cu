// SEISMIC / SEISMIC-SQ search on sm_100a: one warp walks one query at a time,
// a persistent grid steals queries from a global counter.
//
// Per query (seismic_index.cpp:231-274, seismic_scalar_quantized_index.cpp:
// 307-357), in the warp's shared-memory slice:
//   1. the query becomes a bitmap over the vocabulary plus a popcount prefix
//      per 32-term word: a doc term is looked up with one shared load (miss)
//      or three (hit), replacing the reference's dimension-sized dense buffer;
//   2. the query cut (utils/vector_process.h:18-30) is a rank selection;
//   3. per cut list, summary scores (inverted_list_clusters.cpp:295-331) are
//      accumulated hit term by hit term, in ascending term order, lanes spread
//      over the term's (block, value) run;
//   4. blocks are visited in order -- the first list by summary score
//      descending (extracted one at a time by a warp argmax until the pruning
//      test breaks), later lists in block order -- and pruned against the heap
//      minimum times heap_factor (seismic_index.cpp:78-86);
//   5. a visited block's docs are scored four at a time, eight lanes per doc,
//      from aligned 16-byte loads of the padded forward rows. fp32 products
//      that hit the query are summed by one lane in row order, so every score
//      is bit-identical to the reference's sequential sum
//      (utils/distance.h:29-37); uint8/uint16 sums are exact integers;
//   6. scores enter a shared-memory top-k in the reference's insertion order.
//      A doc already in the heap is skipped; a doc scored before and evicted
//      or rejected scores <= the (monotone) heap minimum and is rejected
//      again, so this reproduces the reference's visited set
//      (seismic_index.cpp:104-107) without an O(n_docs) bitmap per query.
#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cstdint>

#include "nsp_device.h"
#include "search_common.cuh"
#include "tma.h"

namespace nsp {
namespace {

using detail_search::heap_emit;
using detail_search::heap_offer;
using detail_search::kFull;
using detail_search::ValT;

__device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Shared-memory slice of one warp.
template <typename V>
struct WarpSlice {
    uint32_t* qbits;   // [words]
    uint16_t* qpre;    // [words]
    uint16_t* qterm;   // [qcap]
    V* qval;           // [qcap]
    uint16_t* cuts;    // [qcap]
    float* hs;         // [k]
    int32_t* hid;      // [k]
    float* stage;      // [4][64] ordered-sum staging (fp32 only)
    int32_t* cdoc;     // [32]
    uint32_t* coff;    // [32]
    uint32_t* clen;    // [32]
    float* csc;        // [32]
    // staged variant only (nullptr otherwise)
    float* bscore_s;        // [bcap] block scores of the current list
    unsigned char* sbuf;    // [2][stage_bytes] bulk-copied doc rows
    uint64_t* mbar;         // [2]
    int32_t* sdoc;          // [2][32] docs of each staged chunk, list order
    uint32_t* slen;         // [2][32] their row lengths
    uint32_t* soff;         // [2][32] their byte offsets in the stage buffer
    int32_t* smeta;         // [2][2] doc count, direct flag per buffer
};

__host__ __device__ inline size_t slice_bytes(int vsize, int words, int qcap, int k, int bcap = 0,
                                              int stage_bytes = 0) {
    size_t b = 0;
    b += ((size_t)words * 4 + 15) & ~size_t(15);
    b += ((size_t)words * 2 + 15) & ~size_t(15);
    b += ((size_t)qcap * 2 + 15) & ~size_t(15);
    b += ((size_t)qcap * vsize + 15) & ~size_t(15);
    b += ((size_t)qcap * 2 + 15) & ~size_t(15);
    b += ((size_t)k * 4 + 15) & ~size_t(15);
    b += ((size_t)k * 4 + 15) & ~size_t(15);
    b += 4 * 64 * 4;
    b += 32 * 4 * 4;
    if (stage_bytes > 0) {
        b += ((size_t)bcap * 4 + 15) & ~size_t(15);
        b += 2 * (size_t)stage_bytes;
        b += 16;                 // two mbarriers
        b += 2 * 32 * 4 * 3;     // chunk descriptors
        b += 16;                 // chunk meta
    }
    return b;
}

template <typename V>
__device__ WarpSlice<V> carve(unsigned char* base, int words, int qcap, int k, int bcap = 0,
                              int stage_bytes = 0) {
    WarpSlice<V> w;
    size_t o = 0;
    w.bscore_s = nullptr;
    w.sbuf = nullptr;
    w.mbar = nullptr;
    if (stage_bytes > 0) {
        // stage buffers first: bulk copies need 16-byte aligned destinations
        w.sbuf = base + o;                                 o += 2 * (size_t)stage_bytes;
        w.mbar = reinterpret_cast<uint64_t*>(base + o);    o += 16;
        w.bscore_s = bcap > 0 ? reinterpret_cast<float*>(base + o) : nullptr;
        o += align16((size_t)bcap * 4);
        w.sdoc = reinterpret_cast<int32_t*>(base + o);     o += 2 * 32 * 4;
        w.slen = reinterpret_cast<uint32_t*>(base + o);    o += 2 * 32 * 4;
        w.soff = reinterpret_cast<uint32_t*>(base + o);    o += 2 * 32 * 4;
        w.smeta = reinterpret_cast<int32_t*>(base + o);    o += 16;
    }
    w.qbits = reinterpret_cast<uint32_t*>(base + o); o += align16((size_t)words * 4);
    w.qpre = reinterpret_cast<uint16_t*>(base + o);  o += align16((size_t)words * 2);
    w.qterm = reinterpret_cast<uint16_t*>(base + o); o += align16((size_t)qcap * 2);
    w.qval = reinterpret_cast<V*>(base + o);         o += align16((size_t)qcap * sizeof(V));
    w.cuts = reinterpret_cast<uint16_t*>(base + o);  o += align16((size_t)qcap * 2);
    w.hs = reinterpret_cast<float*>(base + o);       o += align16((size_t)k * 4);
    w.hid = reinterpret_cast<int32_t*>(base + o);    o += align16((size_t)k * 4);
    w.stage = reinterpret_cast<float*>(base + o);    o += 4 * 64 * 4;
    w.cdoc = reinterpret_cast<int32_t*>(base + o);   o += 32 * 4;
    w.coff = reinterpret_cast<uint32_t*>(base + o);  o += 32 * 4;
    w.clen = reinterpret_cast<uint32_t*>(base + o);  o += 32 * 4;
    w.csc = reinterpret_cast<float*>(base + o);      o += 32 * 4;
    return w;
}

// ----------------------------------------------------------- doc scoring --

__device__ __forceinline__ void unpack_terms(const uint4& v, uint32_t t[8]) {
    t[0] = v.x & 0xffffu; t[1] = v.x >> 16;
    t[2] = v.y & 0xffffu; t[3] = v.y >> 16;
    t[4] = v.z & 0xffffu; t[5] = v.z >> 16;
    t[6] = v.w & 0xffffu; t[7] = v.w >> 16;
}

template <typename V>
__device__ __forceinline__ void load_vals(const V* vp, int e, V out[8]);

template <>
__device__ __forceinline__ void load_vals<float>(const float* vp, int e, float out[8]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(vp + e));
    const float4 b = __ldg(reinterpret_cast<const float4*>(vp + e + 4));
    out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
    out[4] = b.x; out[5] = b.y; out[6] = b.z; out[7] = b.w;
}
template <>
__device__ __forceinline__ void load_vals<uint8_t>(const uint8_t* vp, int e, uint8_t out[8]) {
    const uint2 a = __ldg(reinterpret_cast<const uint2*>(vp + e));
#pragma unroll
    for (int u = 0; u < 4; ++u) out[u] = static_cast<uint8_t>(a.x >> (8 * u));
#pragma unroll
    for (int u = 0; u < 4; ++u) out[4 + u] = static_cast<uint8_t>(a.y >> (8 * u));
}
template <>
__device__ __forceinline__ void load_vals<uint16_t>(const uint16_t* vp, int e, uint16_t out[8]) {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(vp + e));
    uint32_t t[8];
    unpack_terms(a, t);
#pragma unroll
    for (int u = 0; u < 8; ++u) out[u] = static_cast<uint16_t>(t[u]);
}

// Looks up term t in the query bitmap; returns the query's rank of t or -1.
__device__ __forceinline__ int query_rank(const uint32_t* qbits, const uint16_t* qpre,
                                          uint32_t t) {
    const uint32_t w = qbits[t >> 5];
    const uint32_t bit = 1u << (t & 31);
    if (!(w & bit)) return -1;
    return static_cast<int>(qpre[t >> 5]) + __popc(w & (bit - 1));
}

// Rows are consumed 192 elements at a time: each of the 8 lanes of a sub-warp
// issues all of its loads for three 64-element chunks before using any, so a
// typical row (~130 nnz) costs one memory round trip.
constexpr int kChunks = 3;

// Scores one row with the 8 lanes of a sub-warp. fp32: the hit products are
// summed by the sub-warp's first lane in row order (exact reference order).
// Returns the score on sub-lane 0.
__device__ float score_row_f32(const uint16_t* ip, const float* vp, int len, int sub,
                               unsigned submask, const uint32_t* qbits,
                               const uint16_t* qpre, const float* qval, float* stage) {
    float acc = 0.0f;
    for (int e0 = 0; e0 < len; e0 += 64 * kChunks) {
        uint4 iv[kChunks];
        float v[kChunks][8];
#pragma unroll
        for (int j = 0; j < kChunks; ++j) {
            const int e = e0 + j * 64 + sub * 8;
            if (e < len) {
                iv[j] = __ldg(reinterpret_cast<const uint4*>(ip + e));
                load_vals<float>(vp, e, v[j]);
            } else {
                iv[j] = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                for (int u = 0; u < 8; ++u) v[j][u] = 0.0f;
            }
        }
#pragma unroll
        for (int j = 0; j < kChunks; ++j) {
            if (e0 + j * 64 >= len) break;  // uniform across the sub-warp
            const int e = e0 + j * 64 + sub * 8;
            uint32_t t[8];
            unpack_terms(iv[j], t);
            float p[8];
            unsigned hm = 0u;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                p[u] = 0.0f;
                if (e + u < len) {
                    const int r = query_rank(qbits, qpre, t[u]);
                    if (r >= 0) {
                        p[u] = __fmul_rn(v[j][u], qval[r]);
                        hm |= 1u << u;
                    }
                }
            }
            const int hits = __popc(hm);
            int incl = hits;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const int y = __shfl_up_sync(submask, incl, o, 8);
                if (sub >= o) incl += y;
            }
            const int total = __shfl_sync(submask, incl, 7, 8);
            int c = incl - hits;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (hm & (1u << u)) stage[c++] = p[u];
            __syncwarp(submask);
            if (sub == 0)
                for (int h = 0; h < total; ++h) acc = __fadd_rn(acc, stage[h]);
            __syncwarp(submask);
        }
    }
    return acc;
}

// Integer codes: sum of code products is exact in any order (int for uint8,
// utils/distance.h:39-47; int64 for uint16, distance.h:49-57), cast to float.
template <typename V>
__device__ float score_row_int(const uint16_t* ip, const V* vp, int len, int sub,
                               unsigned submask, const uint32_t* qbits,
                               const uint16_t* qpre, const V* qval) {
    long long acc = 0;
    for (int e0 = 0; e0 < len; e0 += 64 * kChunks) {
        uint4 iv[kChunks];
        V v[kChunks][8];
#pragma unroll
        for (int j = 0; j < kChunks; ++j) {
            const int e = e0 + j * 64 + sub * 8;
            if (e < len) {
                iv[j] = __ldg(reinterpret_cast<const uint4*>(ip + e));
                load_vals<V>(vp, e, v[j]);
            } else {
                iv[j] = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                for (int u = 0; u < 8; ++u) v[j][u] = 0;
            }
        }
#pragma unroll
        for (int j = 0; j < kChunks; ++j) {
            const int e = e0 + j * 64 + sub * 8;
            uint32_t t[8];
            unpack_terms(iv[j], t);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (e + u < len) {
                    const int r = query_rank(qbits, qpre, t[u]);
                    if (r >= 0)
                        acc += static_cast<long long>(v[j][u]) * static_cast<long long>(qval[r]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) acc += __shfl_xor_sync(submask, acc, o, 8);
    if (sizeof(V) == 1) return static_cast<float>(static_cast<int>(acc));
    return static_cast<float>(acc);
}

template <typename V>
__device__ __forceinline__ float score_row(const FwdView& fwd, uint32_t off16, uint32_t len,
                                           int sub, unsigned submask, const WarpSlice<V>& w,
                                           int sw) {
    const uint16_t* ip = fwd.idx + static_cast<size_t>(off16) * kRowAlign;
    const V* vp = static_cast<const V*>(fwd.val) + static_cast<size_t>(off16) * kRowAlign;
    if constexpr (sizeof(V) == 4) {
        return score_row_f32(ip, vp, static_cast<int>(len), sub, submask, w.qbits, w.qpre,
                             w.qval, w.stage + sw * 64);
    } else {
        return score_row_int<V>(ip, vp, static_cast<int>(len), sub, submask, w.qbits, w.qpre,
                                w.qval);
    }
}

// Scores `cnt` (<= 32) compacted docs of w.cdoc/coff/clen into w.csc.
template <typename V>
__device__ __forceinline__ void score_chunk(const FwdView& fwd, const WarpSlice<V>& w, int cnt,
                                            int lane) {
    const int sw = lane >> 3;
    const int sub = lane & 7;
    const unsigned submask = 0xffu << (sw * 8);
    for (int g0 = 0; g0 < cnt; g0 += 4) {
        const int gi = g0 + sw;
        const bool act = gi < cnt;
        const uint32_t off = act ? w.coff[gi] : 0u;
        const uint32_t len = act ? w.clen[gi] : 0u;
        const float s = score_row<V>(fwd, off, len, sub, submask, w, sw);
        if (act && sub == 0) w.csc[gi] = s;
    }
    __syncwarp();
}

// Visits block B: scores its (selector-admitted) docs and offers them to the
// heap in the block's doc order (seismic_index.cpp:94-116).
// `bytes` is warp-uniform; `lane_bytes` collects per-lane row bytes.
template <typename V>
__device__ void visit_block(const SeismicLaunch& a, const WarpSlice<V>& w, int64_t B, int& n,
                            int lane, unsigned long long& docs_scored,
                            unsigned long long& bytes, unsigned long long& lane_bytes) {
    const int64_t d0 = a.ix.bdp[B];
    const int64_t d1 = a.ix.bdp[B + 1];
    bytes += 16 + 4ull * static_cast<unsigned long long>(d1 - d0);
    constexpr int vsz = static_cast<int>(sizeof(V));
    for (int64_t base = d0; base < d1; base += 32) {
        const int64_t j = base + lane;
        bool valid = j < d1;
        int32_t doc = valid ? __ldg(a.ix.docs + j) : -1;
        if (valid && a.sel_bits != nullptr)
            valid = (__ldg(a.sel_bits + (doc >> 6)) >> (doc & 63)) & 1ull;
        uint2 ri = make_uint2(0u, 0u);
        if (valid) ri = __ldg(a.fwd.rowinfo + doc);
        const unsigned vm = __ballot_sync(kFull, valid);
        const int pos = __popc(vm & ((1u << lane) - 1u));
        if (valid) {
            w.cdoc[pos] = doc;
            w.coff[pos] = ri.x;
            w.clen[pos] = ri.y;
            lane_bytes += 8ull + static_cast<unsigned long long>(ri.y) * (2 + vsz);
        }
        __syncwarp();
        const int cnt = __popc(vm);
        docs_scored += static_cast<unsigned long long>(cnt);
        score_chunk<V>(a.fwd, w, cnt, lane);
        for (int i = 0; i < cnt; ++i) heap_offer(w.csc[i], w.cdoc[i], w.hs, w.hid, n, a.k, lane);
        __syncwarp();
    }
}

// ------------------------------------------------------ staged variant --
// Rows of a block arrive in shared memory by bulk copy (cp.async.bulk), in
// chunks that fill a stage buffer; two buffers alternate, so the next chunk is
// in flight while the current one is scored. A row too long for a buffer is
// scored straight from global memory, in its place in the block order.

// Scores a row staged at `row` (ids, then values at row + 2 * padded len).
template <typename V>
__device__ float score_row_staged(const unsigned char* row, int len, int sub, unsigned submask,
                                  const WarpSlice<V>& w, int sw) {
    const int plen = (len + 15) & ~15;
    const unsigned char* vrow = row + plen * 2;
    if constexpr (sizeof(V) == 4) {
        float acc = 0.0f;
        float* stage = w.stage + sw * 64;
        for (int e0 = 0; e0 < len; e0 += 64) {
            const int e = e0 + sub * 8;
            float p[8];
            unsigned hm = 0u;
#pragma unroll
            for (int u = 0; u < 8; ++u) p[u] = 0.0f;
            if (e < len) {
                uint32_t t[8];
                unpack_terms(lds128(row + e * 2), t);
                const uint4 a0 = lds128(vrow + e * 4);
                const uint4 a1 = lds128(vrow + e * 4 + 16);
                const float v[8] = {__uint_as_float(a0.x), __uint_as_float(a0.y),
                                    __uint_as_float(a0.z), __uint_as_float(a0.w),
                                    __uint_as_float(a1.x), __uint_as_float(a1.y),
                                    __uint_as_float(a1.z), __uint_as_float(a1.w)};
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (e + u < len) {
                        const int r = query_rank(w.qbits, w.qpre, t[u]);
                        if (r >= 0) {
                            p[u] = __fmul_rn(v[u], w.qval[r]);
                            hm |= 1u << u;
                        }
                    }
                }
            }
            const int hits = __popc(hm);
            int incl = hits;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const int y = __shfl_up_sync(submask, incl, o, 8);
                if (sub >= o) incl += y;
            }
            const int total = __shfl_sync(submask, incl, 7, 8);
            int c = incl - hits;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (hm & (1u << u)) stage[c++] = p[u];
            __syncwarp(submask);
            if (sub == 0)
                for (int h = 0; h < total; ++h) acc = __fadd_rn(acc, stage[h]);
            __syncwarp(submask);
        }
        return acc;
    } else {
        long long acc = 0;
        for (int e0 = 0; e0 < len; e0 += 64) {
            const int e = e0 + sub * 8;
            if (e < len) {
                uint32_t t[8];
                unpack_terms(lds128(row + e * 2), t);
                uint32_t v[8];
                if constexpr (sizeof(V) == 1) {
                    const uint2 a0 = lds64(vrow + e);
#pragma unroll
                    for (int u = 0; u < 4; ++u) v[u] = (a0.x >> (8 * u)) & 0xffu;
#pragma unroll
                    for (int u = 0; u < 4; ++u) v[4 + u] = (a0.y >> (8 * u)) & 0xffu;
                } else {
                    unpack_terms(lds128(vrow + e * 2), v);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (e + u < len) {
                        const int r = query_rank(w.qbits, w.qpre, t[u]);
                        if (r >= 0)
                            acc += static_cast<long long>(v[u]) * static_cast<long long>(w.qval[r]);
                    }
                }
            }
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) acc += __shfl_xor_sync(submask, acc, o, 8);
        if (sizeof(V) == 1) return static_cast<float>(static_cast<int>(acc));
        return static_cast<float>(acc);
    }
}

// Takes block docs [pos, d1) into stage buffer `buf`: as many as fit, in order,
// with the selector applied; issues their bulk copies. Returns the number of
// doc-list entries consumed (a row larger than a buffer becomes a one-doc
// "direct" chunk).
template <typename V>
__device__ int64_t issue_chunk(const SeismicLaunch& a, const WarpSlice<V>& w, int buf,
                               int64_t pos, int64_t d1, int lane,
                               unsigned long long& lane_bytes) {
    constexpr int vsz = static_cast<int>(sizeof(V));
    const uint32_t cap = static_cast<uint32_t>(a.stage_bytes);
    const int64_t j = pos + lane;
    const bool valid = j < d1;
    const int32_t doc = valid ? __ldg(a.ix.docs + j) : -1;
    bool member = valid;
    if (member && a.sel_bits != nullptr) member = (__ldg(a.sel_bits + (doc >> 6)) >> (doc & 63)) & 1ull;
    const uint2 ri = member ? __ldg(a.fwd.rowinfo + doc) : make_uint2(0u, 0u);
    const uint32_t plen = (ri.y + 15u) & ~15u;
    const uint32_t bytes = member ? plen * (2 + vsz) : 0u;
    const bool big = bytes > cap;
    uint32_t incl = bytes;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    const unsigned brk = __ballot_sync(kFull, valid && (big || incl > cap));
    const int64_t left = d1 - pos;
    const int avail = left < 32 ? static_cast<int>(left) : 32;
    const int c = brk ? __ffs(brk) - 1 : avail;
    int32_t* sdoc = w.sdoc + buf * 32;
    uint32_t* slen = w.slen + buf * 32;
    uint32_t* soff = w.soff + buf * 32;
    int32_t* meta = w.smeta + buf * 2;
    uint64_t* bar = w.mbar + buf;
    __syncwarp();
    if (c == 0) {
        // lane 0's row exceeds a buffer: score it from global memory
        if (lane == 0) {
            sdoc[0] = doc;
            slen[0] = ri.y;
            soff[0] = ri.x;
            meta[0] = 1;
            meta[1] = 1;
            mbar_arrive_expect_tx(bar, 0u);
            lane_bytes += 8ull + static_cast<unsigned long long>(ri.y) * (2 + vsz);
        }
        __syncwarp();
        return 1;
    }
    const bool take = member && lane < c;
    const unsigned tm = __ballot_sync(kFull, take);
    const int p = __popc(tm & ((1u << lane) - 1u));
    const uint32_t excl = incl - bytes;
    if (take) {
        sdoc[p] = doc;
        slen[p] = ri.y;
        soff[p] = excl;
    }
    const uint32_t total = __shfl_sync(kFull, incl, c - 1);
    if (lane == 0) {
        meta[0] = __popc(tm);
        meta[1] = 0;
    }
    // the buffer's previous contents were read by this warp: order those
    // reads before the copies that overwrite them
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(bar, total);
    __syncwarp();
    if (take && plen > 0) {  // an empty row needs no copy (and adds no bytes)
        unsigned char* dst = w.sbuf + static_cast<size_t>(buf) * cap + excl;
        const size_t e0 = static_cast<size_t>(ri.x) * kRowAlign;
        bulk_copy_g2s(dst, a.fwd.idx + e0, plen * 2u, bar);
        bulk_copy_g2s(dst + plen * 2u, static_cast<const unsigned char*>(a.fwd.val) + e0 * vsz,
                      plen * static_cast<uint32_t>(vsz), bar);
        lane_bytes += 8ull + static_cast<unsigned long long>(ri.y) * (2 + vsz);
    }
    __syncwarp();
    return c;
}

// Waits for buffer `buf`, scores its docs and offers them to the heap in
// order. False if the wait gave up (error recorded).
template <typename V>
__device__ bool process_chunk(const SeismicLaunch& a, const WarpSlice<V>& w, int buf,
                              uint32_t& phase_bits, int& n, int lane,
                              unsigned long long& docs_scored) {
    const uint32_t phase = (phase_bits >> buf) & 1u;
    if (!mbar_wait_bounded(w.mbar + buf, phase)) {
        if (lane == 0 && a.err != nullptr) atomicExch(a.err, 1);
        mbar_wait_bounded(w.mbar + buf, phase);  // let copies in flight land
        return false;
    }
    phase_bits ^= 1u << buf;
    const int32_t* meta = w.smeta + buf * 2;
    const int cnt = meta[0];
    const bool direct = meta[1] != 0;
    const int32_t* sdoc = w.sdoc + buf * 32;
    const uint32_t* slen = w.slen + buf * 32;
    const uint32_t* soff = w.soff + buf * 32;
    const int sw = lane >> 3;
    const int sub = lane & 7;
    const unsigned submask = 0xffu << (sw * 8);
    if (direct) {
        const float s = score_row<V>(a.fwd, soff[0], slen[0], sub, submask, w, sw);
        if (lane == 0) w.csc[0] = s;
    } else {
        const unsigned char* base = w.sbuf + static_cast<size_t>(buf) * a.stage_bytes;
        for (int g0 = 0; g0 < cnt; g0 += 4) {
            const int gi = g0 + sw;
            const bool act = gi < cnt;
            const float s = score_row_staged<V>(base + (act ? soff[gi] : 0u),
                                                act ? static_cast<int>(slen[gi]) : 0, sub,
                                                submask, w, sw);
            if (act && sub == 0) w.csc[gi] = s;
        }
    }
    __syncwarp();
    docs_scored += static_cast<unsigned long long>(cnt);
    for (int i = 0; i < cnt; ++i) heap_offer(w.csc[i], sdoc[i], w.hs, w.hid, n, a.k, lane);
    __syncwarp();
    return true;
}

template <typename V>
__device__ bool visit_block_staged(const SeismicLaunch& a, const WarpSlice<V>& w, int64_t B, int& n,
                                   int lane, uint32_t& phase_bits, unsigned long long& docs_scored,
                                   unsigned long long& bytes, unsigned long long& lane_bytes) {
    const int64_t d0 = a.ix.bdp[B];
    const int64_t d1 = a.ix.bdp[B + 1];
    bytes += 16 + 4ull * static_cast<unsigned long long>(d1 - d0);
    if (d1 <= d0) return true;
    int buf = 0;
    int64_t pos = d0 + issue_chunk<V>(a, w, buf, d0, d1, lane, lane_bytes);
    for (;;) {
        const bool more = pos < d1;
        if (more) pos += issue_chunk<V>(a, w, buf ^ 1, pos, d1, lane, lane_bytes);
        if (!process_chunk<V>(a, w, buf, phase_bits, n, lane, docs_scored)) {
            // give the other buffer's copies a bounded chance to land, then stop
            if (more) mbar_wait_bounded(w.mbar + (buf ^ 1), (phase_bits >> (buf ^ 1)) & 1u);
            return false;
        }
        if (!more) return true;
        buf ^= 1;
    }
}

// Returns false if a bounded wait gave up (the query's results are then
// padding and the warp stops).
template <typename V, bool kStaged>
__device__ bool run_query(const SeismicLaunch& a, const WarpSlice<V>& w, float* bscore_g, int q,
                          int lane, uint32_t& phase_bits) {
    // block scores of the current list: shared memory when they fit
    float* bscore = (kStaged && w.bscore_s != nullptr && a.ix.max_blocks <= a.bcap) ? w.bscore_s
                                                                                   : bscore_g;
    bool ok = true;
    const int words = a.ix.words;
    const int32_t qs = a.q.indptr[q];
    int qn = a.q.indptr[q + 1] - qs;
    // The warp's shared slice holds a.qcap query entries. A longer row (the
    // caller's max_nnz was wrong) or one past the query arrays is treated as
    // empty -- padding -- and reported.
    if (qn > a.qcap || qn < 0 || qs < 0 || (a.nnz_cap >= 0 && qs + qn > a.nnz_cap)) {
        if (lane == 0 && a.err != nullptr) atomicExch(a.err, 3);
        qn = 0;
    }
    const uint16_t* gq_idx = a.q.idx + qs;
    const V* gq_val = static_cast<const V*>(a.q.val) + qs;

    // 1. bitmap + prefix
    for (int i = lane; i < words; i += 32) w.qbits[i] = 0u;
    __syncwarp();
    for (int i = lane; i < qn; i += 32) {
        const uint32_t t = gq_idx[i];
        w.qterm[i] = static_cast<uint16_t>(t);
        w.qval[i] = gq_val[i];
        atomicOr(&w.qbits[t >> 5], 1u << (t & 31));
    }
    __syncwarp();
    {
        const int cs = (words + 31) / 32;
        const int w0 = lane * cs;
        const int w1 = min(words, w0 + cs);
        int local = 0;
        for (int i = w0; i < w1; ++i) local += __popc(w.qbits[i]);
        int incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        int run = incl - local;
        for (int i = w0; i < w1; ++i) {
            w.qpre[i] = static_cast<uint16_t>(run);
            run += __popc(w.qbits[i]);
        }
    }
    // 2. query cut (utils/vector_process.h:18-30): the query's order when
    // cut >= nnz, else the reference's TopKHolder over (value, position)
    int ncut;
    if (a.cut >= qn) {
        ncut = qn;
        for (int i = lane; i < qn; i += 32) w.cuts[i] = w.qterm[i];
    } else {
        ncut = a.cut;
        if (lane == 0)
            ranking::cut_like_reference(w.cuts, qn, ncut, detail_search::QueryWeight<V>{w.qval});
        __syncwarp();
        for (int i = lane; i < ncut; i += 32) w.cuts[i] = w.qterm[w.cuts[i]];
    }
    __syncwarp();

    int n = 0;  // heap size
    bool first = true;
    unsigned long long docs_scored = 0, blocks_visited = 0, bytes = 0, lists = 0, lane_bytes = 0;
    constexpr int vsz = static_cast<int>(sizeof(V));
    for (int c = 0; c < ncut; ++c) {
        const int t = w.cuts[c];
        if (t >= a.ix.n_lists) continue;  // seismic_index.cpp:254-256
        const int64_t lb0 = a.ix.lbp[t];
        const int nb = static_cast<int>(a.ix.lbp[t + 1] - lb0);
        if (nb > 0) {
            ++lists;
            for (int b = lane; b < nb; b += 32) bscore[b] = 0.0f;
            __syncwarp();
            // 3. summary scores, hit terms in ascending term order
            const uint2* meta = a.ix.lmeta + static_cast<size_t>(t) * words;
            const int64_t colbase = a.ix.ltp[t];
            for (int i0 = 0; i0 < qn; i0 += 32) {
                const int i = i0 + lane;
                bool hit = false;
                int64_t r0 = 0, r1 = 0;
                float qv = 0.0f;
                if (i < qn) {
                    const uint32_t term = w.qterm[i];
                    const uint2 m = __ldg(meta + (term >> 5));
                    const uint32_t bit = 1u << (term & 31);
                    if (m.x & bit) {
                        const int64_t col = colbase + m.y + __popc(m.x & (bit - 1));
                        r0 = __ldg(a.ix.srun + col);
                        r1 = __ldg(a.ix.srun + col + 1);
                        qv = ValT<V>::f(w.qval[i]);
                        hit = true;
                    }
                }
                bytes += 8ull * static_cast<unsigned long long>(min(32, qn - i0));
                unsigned hm = __ballot_sync(kFull, hit);
                bytes += 16ull * __popc(hm);
                while (hm) {
                    const int src = __ffs(hm) - 1;
                    hm &= hm - 1;
                    const int64_t R0 = __shfl_sync(kFull, r0, src);
                    const int64_t R1 = __shfl_sync(kFull, r1, src);
                    const float QV = __shfl_sync(kFull, qv, src);
                    bytes += static_cast<unsigned long long>(R1 - R0) * (2 + vsz);
                    const V* sv = static_cast<const V*>(a.ix.sval);
                    for (int64_t e = R0 + lane; e < R1; e += 32) {
                        const int blk = __ldg(a.ix.sblk + e);
                        const float p = __fmul_rn(QV, ValT<V>::f(__ldg(sv + e)));
                        bscore[blk] = __fadd_rn(bscore[blk], p);
                    }
                    __syncwarp();
                }
            }
            // 4. block traversal
            if (first) {
                // the reference's visiting order (seismic_common.h:105-115)
                ranking::Blk* items = reinterpret_cast<ranking::Blk*>(
                    bscore_g + ((a.ix.max_blocks + 1) & ~1));
                for (int b = lane; b < nb; b += 32) items[b] = ranking::Blk{bscore[b], b};
                __syncwarp();
                ranking::warp_sort_blocks_like_reference(items, nb, lane);
                for (int o = 0; o < nb; ++o) {
                    const ranking::Blk it = items[o];
                    if (n == a.k && __fmul_rn(it.s, a.heap_factor) < w.hs[0]) break;
                    ++blocks_visited;
                    if constexpr (kStaged) {
                        ok = visit_block_staged<V>(a, w, lb0 + it.b, n, lane, phase_bits,
                                                   docs_scored, bytes, lane_bytes);
                        if (!ok) break;
                    } else {
                        visit_block<V>(a, w, lb0 + it.b, n, lane, docs_scored, bytes, lane_bytes);
                    }
                }
            } else {
                for (int b0 = 0; b0 < nb; b0 += 32) {
                    const int b = b0 + lane;
                    const float s = b < nb ? bscore[b] : 0.0f;
                    const bool cand =
                        b < nb && !(n == a.k && __fmul_rn(s, a.heap_factor) < w.hs[0]);
                    unsigned cm = __ballot_sync(kFull, cand);
                    while (cm) {
                        const int src = __ffs(cm) - 1;
                        cm &= cm - 1;
                        const float S = __shfl_sync(kFull, s, src);
                        if (n == a.k && __fmul_rn(S, a.heap_factor) < w.hs[0]) continue;
                        ++blocks_visited;
                        if constexpr (kStaged) {
                            ok = visit_block_staged<V>(a, w, lb0 + b0 + src, n, lane, phase_bits,
                                                       docs_scored, bytes, lane_bytes);
                            if (!ok) break;
                        } else {
                            visit_block<V>(a, w, lb0 + b0 + src, n, lane, docs_scored, bytes,
                                           lane_bytes);
                        }
                    }
                    if (!ok) break;
                }
            }
        }
        if (!ok) break;
        first = false;  // seismic_index.cpp:261
    }
    if (!ok) n = 0;  // a gave-up wait leaves this query's results as padding

    // 6. results, padded with (-1.0, -1); SQ scores decoded
    //    (seismic_scalar_quantized_index.cpp:345-355).
    heap_emit(w.hs, w.hid, n, a.k, a.decode_scale, a.out_d + static_cast<size_t>(q) * a.k,
              a.out_l + static_cast<size_t>(q) * a.k, lane);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lane_bytes += __shfl_xor_sync(kFull, lane_bytes, o);
    bytes += lane_bytes;
    if (a.stats != nullptr && lane == 0) {
        atomicAdd(a.stats + kStatDocsScored, docs_scored);
        atomicAdd(a.stats + kStatBlocksVisited, blocks_visited);
        atomicAdd(a.stats + kStatBytes, bytes);
        atomicAdd(a.stats + kStatListsProbed, lists);
        atomicAdd(a.stats + kStatRowBytes, lane_bytes);
    }
    __syncwarp();
    return ok;
}

template <typename V, bool kStaged>
__global__ void __launch_bounds__(256) seismic_search_kernel(SeismicLaunch a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int bcap = kStaged ? a.bcap : 0;
    const int sb = kStaged ? a.stage_bytes : 0;
    const size_t per = slice_bytes(static_cast<int>(sizeof(V)), a.ix.words, a.qcap, a.k, bcap, sb);
    WarpSlice<V> w = carve<V>(smem + per * warp, a.ix.words, a.qcap, a.k, bcap, sb);
    const int wpb = blockDim.x >> 5;
    const int gw = blockIdx.x * wpb + warp;
    float* bscore = a.bscore + static_cast<size_t>(gw) * one_warp_slot(a.ix.max_blocks);
    uint32_t phase_bits = 0;
    if constexpr (kStaged) {
        if (lane == 0) {
            mbar_init(w.mbar, 1);
            mbar_init(w.mbar + 1, 1);
            fence_mbar_init();
        }
        __syncwarp();
    }
    if (a.work_counter != nullptr) {
        for (;;) {
            int q = 0;
            if (lane == 0) q = atomicAdd(a.work_counter, 1);
            q = __shfl_sync(kFull, q, 0);
            if (q >= a.q.n) break;
            if (!run_query<V, kStaged>(a, w, bscore, q, lane, phase_bits)) break;
        }
    } else {
        const int total = gridDim.x * wpb;
        for (int q = a.first_query + gw; q < a.q.n; q += total)
            if (!run_query<V, kStaged>(a, w, bscore, q, lane, phase_bits)) break;
    }
}

// ---------------------------------------------- exact list (ExactMatcher) --

template <typename V>
__global__ void __launch_bounds__(32) exact_list_kernel(FwdView fwd, QueryView qv, const int32_t* ids,
                                                        int n_ids, int k, float decode_scale,
                                                        int words, int qcap, float* out_d,
                                                        int32_t* out_l) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    WarpSlice<V> w = carve<V>(smem, words, qcap, k);
    const int q = blockIdx.x;
    const int32_t qs = qv.indptr[q];
    const int qn = qv.indptr[q + 1] - qs;
    for (int i = lane; i < words; i += 32) w.qbits[i] = 0u;
    __syncwarp();
    for (int i = lane; i < qn; i += 32) {
        const uint32_t t = qv.idx[qs + i];
        w.qval[i] = static_cast<const V*>(qv.val)[qs + i];
        atomicOr(&w.qbits[t >> 5], 1u << (t & 31));
    }
    __syncwarp();
    {
        const int cs = (words + 31) / 32;
        const int w0 = lane * cs;
        const int w1 = min(words, w0 + cs);
        int local = 0;
        for (int i = w0; i < w1; ++i) local += __popc(w.qbits[i]);
        int incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        int run = incl - local;
        for (int i = w0; i < w1; ++i) {
            w.qpre[i] = static_cast<uint16_t>(run);
            run += __popc(w.qbits[i]);
        }
    }
    __syncwarp();
    int n = 0;
    for (int base = 0; base < n_ids; base += 32) {
        const int j = base + lane;
        const bool valid = j < n_ids && ids[j] >= 0 && ids[j] < fwd.n_docs;
        const int32_t doc = valid ? ids[j] : -1;
        uint2 ri = make_uint2(0u, 0u);
        if (valid) ri = fwd.rowinfo[doc];
        const unsigned vm = __ballot_sync(kFull, valid);
        const int pos = __popc(vm & ((1u << lane) - 1u));
        if (valid) {
            w.cdoc[pos] = doc;
            w.coff[pos] = ri.x;
            w.clen[pos] = ri.y;
        }
        __syncwarp();
        const int cnt = __popc(vm);
        score_chunk<V>(fwd, w, cnt, lane);
        for (int i = 0; i < cnt; ++i) heap_offer(w.csc[i], w.cdoc[i], w.hs, w.hid, n, k, lane);
        __syncwarp();
    }
    heap_emit(w.hs, w.hid, n, k, decode_scale, out_d + static_cast<size_t>(q) * k,
              out_l + static_cast<size_t>(q) * k, lane);
}

// ------------------------------------------------------- quantize (SQ) --
// encode_8bit / encode_16bit (utils/scalar_quantizer.h:97-118): the scale
// kMax / (vmax - vmin) is formed on the host in float, exactly as the
// reference forms it, and passed in.
__global__ void sq_encode_kernel(const float* vals, void* codes, int64_t n, int qbits, float vmin,
                                 float scale) {
    const float kmax = qbits == 16 ? 65535.0f : 255.0f;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float scaled = __fmul_rn(__fsub_rn(vals[i], vmin), scale);
        const float lo = (scaled < kmax) ? scaled : kmax;  // std::min(kMax, x)
        const float c = (0.0f < lo) ? lo : 0.0f;           // std::max(0, x)
        const long r = lroundf(c);
        if (qbits == 16)
            static_cast<uint16_t*>(codes)[i] = static_cast<uint16_t>(r);
        else
            static_cast<uint8_t*>(codes)[i] = static_cast<uint8_t>(r);
    }
}

}  // namespace

size_t seismic_smem_per_warp(int val_kind, int dim_words, int qcap, int k, int bcap,
                             int stage_bytes) {
    return slice_bytes(val_kind, dim_words, qcap, k, bcap, stage_bytes);
}

template <typename V, bool kStaged>
static int max_blocks_typed(int wpb, size_t smem) {
    // the occupancy calculator only admits dynamic shared memory the kernel
    // has been allowed to use
    if (allow_opt_in_smem(seismic_search_kernel<V, kStaged>) != cudaSuccess)
        return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, seismic_search_kernel<V, kStaged>,
                                                      wpb * 32, smem) != cudaSuccess)
        return 0;
    return blocks;
}

int seismic_max_blocks_per_sm(int val_kind, int variant, int wpb, size_t smem) {
    if (val_kind == kF32)
        return variant ? max_blocks_typed<float, true>(wpb, smem) : max_blocks_typed<float, false>(wpb, smem);
    if (val_kind == kU8)
        return variant ? max_blocks_typed<uint8_t, true>(wpb, smem)
                       : max_blocks_typed<uint8_t, false>(wpb, smem);
    return variant ? max_blocks_typed<uint16_t, true>(wpb, smem)
                   : max_blocks_typed<uint16_t, false>(wpb, smem);
}

int seismic_max_blocks_per_sm(int val_kind, int wpb, size_t smem) {
    return seismic_max_blocks_per_sm(val_kind, 0, wpb, smem);
}

template <typename V, bool kStaged>
static cudaError_t launch_typed(const SeismicLaunch& a, int wpb, int blocks, cudaStream_t s) {
    const size_t smem = slice_bytes(static_cast<int>(sizeof(V)), a.ix.words, a.qcap, a.k,
                                    kStaged ? a.bcap : 0, kStaged ? a.stage_bytes : 0) *
                        wpb;
    cudaError_t e = allow_opt_in_smem(seismic_search_kernel<V, kStaged>);
    if (e != cudaSuccess) return e;
    seismic_search_kernel<V, kStaged><<<blocks, wpb * 32, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_seismic(int val_kind, const SeismicLaunch& a, int wpb, int blocks,
                           cudaStream_t s) {
    const bool staged = a.variant == 1 && a.stage_bytes > 0;
    if (val_kind == kF32)
        return staged ? launch_typed<float, true>(a, wpb, blocks, s)
                      : launch_typed<float, false>(a, wpb, blocks, s);
    if (val_kind == kU8)
        return staged ? launch_typed<uint8_t, true>(a, wpb, blocks, s)
                      : launch_typed<uint8_t, false>(a, wpb, blocks, s);
    return staged ? launch_typed<uint16_t, true>(a, wpb, blocks, s)
                  : launch_typed<uint16_t, false>(a, wpb, blocks, s);
}

template <typename V>
static cudaError_t launch_exact_list_t(const FwdView& fwd, const QueryView& q, const int32_t* ids,
                                       int n_ids, int k, float decode_scale, int32_t qcap,
                                       float* out_d, int32_t* out_l, cudaStream_t s) {
    const int words = (fwd.dim + 31) / 32;
    const size_t smem = slice_bytes(static_cast<int>(sizeof(V)), words, qcap, k);
    cudaError_t e = allow_opt_in_smem(exact_list_kernel<V>);
    if (e != cudaSuccess) return e;
    if (q.n == 0) return cudaSuccess;
    exact_list_kernel<V><<<q.n, 32, smem, s>>>(fwd, q, ids, n_ids, k, decode_scale, words, qcap,
                                               out_d, out_l);
    return cudaGetLastError();
}

cudaError_t launch_exact_list(int val_kind, const FwdView& fwd, const QueryView& q,
                              const int32_t* ids, int n_ids, int k, float decode_scale,
                              int32_t qcap, float* out_d, int32_t* out_l, cudaStream_t s) {
    if (val_kind == kF32)
        return launch_exact_list_t<float>(fwd, q, ids, n_ids, k, decode_scale, qcap, out_d, out_l, s);
    if (val_kind == kU8)
        return launch_exact_list_t<uint8_t>(fwd, q, ids, n_ids, k, decode_scale, qcap, out_d, out_l,
                                            s);
    return launch_exact_list_t<uint16_t>(fwd, q, ids, n_ids, k, decode_scale, qcap, out_d, out_l, s);
}

cudaError_t launch_sq_encode(const float* vals, void* codes, int64_t n, int qbits, float vmin,
                             float scale, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    const int64_t want = (n + threads - 1) / threads;
    const int blocks = static_cast<int>(want < 148 * 32 ? want : 148 * 32);
    sq_encode_kernel<<<blocks, threads, 0, s>>>(vals, codes, n, qbits, vmin, scale);
    return cudaGetLastError();
}

}  // namespace nsp
