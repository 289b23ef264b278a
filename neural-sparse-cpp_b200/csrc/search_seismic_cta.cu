// SEISMIC / SEISMIC-SQ search on sm_100a, one CTA per query (kernel
// variants 2-5). A persistent grid steals queries from a global counter; the
// CTA's warps walk the query's blocks together.
//
// Per query (seismic_index.cpp:231-274, seismic_scalar_quantized_index.cpp:
// 307-357):
//   1. the query is scattered into a dense per-term table in shared memory --
//      the reference's dimension-sized dense buffer (seismic_index.cpp:243-
//      246), one byte per term: fp32 queries store the term's rank (0 = not
//      in the query; the rank indexes a table of the query's values, entry 0
//      holding 0.0f), SQ queries store the code itself;
//   2. the query cut (utils/vector_process.h:18-30) is a rank selection;
//   3. block summary scores (inverted_list_clusters.cpp:295-331) of up to
//      one list per warp are accumulated at once, each warp hit term by hit
//      term in ascending term order;
//   4. the first list's blocks are sorted (score desc, block asc) by a
//      bitonic sort (seismic_common.h:105-115); later lists keep block order;
//   5. blocks are taken in that order into batches of up to `batch_docs`
//      docs. A block that fails the pruning test (seismic_index.cpp:78-86)
//      against the current heap minimum is skipped (or ends the first list);
//      the heap minimum only grows, so a block that fails now fails at its
//      turn too. Blocks that pass are gathered, their docs scored in
//      parallel, and then -- in block order -- each block is tested again
//      against the heap as it stands when its turn comes, exactly as the
//      reference tests it, and its docs are offered in order. Docs of a block
//      that fails the second test are dropped: the result is the reference's,
//      only some scoring work is speculative;
//   6. a group of kG lanes (1, 2, 4 or 8) scores one doc at a time, 16 row
//      elements per lane per step from 256-bit loads of the padded forward
//      rows, and takes the next doc of the batch as soon as its row ends, so
//      groups stay busy across rows of different lengths. fp32 scores are the
//      reference's sequential sum result += w * dense[t] over the whole row
//      (utils/distance.h:29-37), with the same round-to-nearest products and
//      sums in the same order: bit-identical. The zero padding after a row
//      adds +-0.0, which leaves every sum unchanged unless the query holds a
//      non-finite value, in which case padding elements are masked out. SQ
//      sums are exact integers (distance.h:39-57);
//   7. scores enter a shared-memory top-k in the reference's insertion order;
//      a doc already in the heap is skipped and one scored before and
//      evicted or rejected scores <= the (monotone) heap minimum and is
//      rejected again: the reference's visited set (seismic_index.cpp:104-
//      107) without an O(n_docs) bitmap per query.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cstdint>
#include <type_traits>

#include "nsp_device.h"
#include "search_common.cuh"

namespace nsp {
namespace {

namespace cg = cooperative_groups;
using detail_search::heap_emit;
using detail_search::QueryWeight;
using detail_search::heap_offer;
using detail_search::kFull;
using detail_search::ValT;

constexpr int kSegCap = 128;    // block segments per batch, one CTA per query
constexpr int kSegCapMax = 1024;  // the most any launch asks for (a cluster per query)

// A run of consecutive docs of one block inside a batch.
struct Seg {
    int64_t d0;     // position of the first doc in ix.docs
    int32_t cnt;    // docs in the segment
    int32_t cand0;  // first candidate slot of the batch
    int32_t blk;    // block index within its list
    float bs;       // the block's summary score
    int32_t head;   // 1 when the block starts here (its pruning test applies)
    int32_t surv;   // 1 when a doc of it may still enter the heap (set after scoring)
};

struct Ctl {
    int32_t q;
    int32_t nseg;
    int32_t total;
    int32_t next;   // claim counter of the scoring phase
    int32_t nheap;  // heap size when the batch was gathered (warp 0's)
    int32_t pad[3];
};

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

struct CtaLayout {
    size_t tbl, qv, qterm, qraw, cuts, hs, hid, cdoc, coff, clen, csc, segs, cseg, wsum, cur, uq,
        total;
};

// Shared-memory layout of one CTA. The four candidate arrays are contiguous
// (16 * batch bytes) and double as the sort-key buffer of the first list.
__host__ __device__ inline CtaLayout cta_layout(int vsize, int tsize, int dim, int qcap, int k,
                                                int batch, int seg_cap) {
    CtaLayout L;
    size_t o = a16(sizeof(Ctl));
    L.tbl = o;   o += a16(static_cast<size_t>(dim + 1) * tsize);
    L.qv = o;    o += a16(static_cast<size_t>(qcap + 1) * 4);
    L.qterm = o; o += a16(static_cast<size_t>(qcap) * 2);
    L.qraw = o;  o += a16(static_cast<size_t>(qcap) * vsize);
    L.cuts = o;  o += a16(static_cast<size_t>(qcap) * 2);
    L.hs = o;    o += a16(static_cast<size_t>(k) * 4);
    L.hid = o;   o += a16(static_cast<size_t>(k) * 4);
    L.cdoc = o;  o += static_cast<size_t>(batch) * 4;
    L.coff = o;  o += static_cast<size_t>(batch) * 4;
    L.clen = o;  o += static_cast<size_t>(batch) * 4;
    L.csc = o;   o += static_cast<size_t>(batch) * 4;
    L.segs = o;  o += static_cast<size_t>(seg_cap) * sizeof(Seg);
    L.cseg = o;  o += a16(static_cast<size_t>(batch) * 2);
    L.wsum = o;  o += 32 * 4;
    L.cur = o;   o += 64;  // warp 0's Cursor
    L.uq = o;    o += 2 * 32 * 4;  // counting pass: warp 0's per-lane unique docs, row bytes
    L.total = o;
    return L;
}

// ------------------------------------------------------------ row loads --
// 256-bit loads (sm_100): a lane reads 16 term ids (32 bytes) per step and
// their values (64 bytes fp32, 32 bytes uint16, 16 bytes uint8).
__device__ __forceinline__ void ldg256(const void* p, uint32_t (&r)[8]) {
    asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "l"(p));
}

__device__ __forceinline__ uint32_t term_of(const uint32_t (&t)[8], int u) {
    return (u & 1) ? (t[u >> 1] >> 16) : (t[u >> 1] & 0xffffu);
}

// One bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned) into L2
// (the TMA unit fetches it; no registers, no L1 traffic).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// A candidate row's ids and values from element `from` to the row's end on
// its 64-element boundary. Rows start on 64-element boundaries, so both
// ranges are 16-byte aligned multiples of 16 bytes.
template <typename V>
__device__ __forceinline__ void prefetch_row(const uint16_t* idx_base, const V* val_base,
                                             uint32_t off, uint32_t len, uint32_t from) {
    const uint32_t padded = (len + kRowAlign - 1) & ~static_cast<uint32_t>(kRowAlign - 1);
    if (padded <= from) return;
    const size_t e0 = static_cast<size_t>(off) * kRowAlign + from;
    prefetch_l2(idx_base + e0, (padded - from) * 2u);
    prefetch_l2(val_base + e0, (padded - from) * static_cast<uint32_t>(sizeof(V)));
}

template <typename V>
struct Acc;
template <>
struct Acc<float> {
    using T = float;
};
template <>
struct Acc<uint8_t> {
    using T = int;
};
template <>
struct Acc<uint16_t> {
    using T = long long;
};

// Products of one lane's 16 row elements at ip/vp, `rem` of them real (the
// rest are the row's zero padding, or nothing when rem <= 0).
// fp32: p[u] = w[u] * qv[tbl[t[u]]], the reference's product; with kMask the
// padding gives +0.0.
template <typename TE, bool kMask>
__device__ __forceinline__ void products(const uint16_t* ip, const float* vp, int rem,
                                         const TE* tbl, const float* qv, float (&p)[16]) {
    if (rem <= 0) {
#pragma unroll
        for (int u = 0; u < 16; ++u) p[u] = 0.0f;
        return;
    }
    uint32_t t[8], v0[8], v1[8];
    ldg256(ip, t);
    ldg256(vp, v0);
    ldg256(vp + 8, v1);
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const float q = qv[tbl[term_of(t, u)]];
        const float x = __uint_as_float(u < 8 ? v0[u] : v1[u - 8]);
        p[u] = __fmul_rn(x, q);
        if (kMask && u >= rem) p[u] = 0.0f;
    }
}

// uint8 codes: the sum of code products as int (distance.h:39-47); padding
// codes are 0. (Packing four looked-up codes for __dp4a measured slower: the
// packing waits for all four lookups.)
template <typename TE>
__device__ __forceinline__ int partial(const uint16_t* ip, const uint8_t* vp, int rem,
                                       const TE* tbl) {
    if (rem <= 0) return 0;
    uint32_t t[8];
    ldg256(ip, t);
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(vp));
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    int acc = 0;
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int q = static_cast<int>(tbl[term_of(t, u)]);
        const int x = static_cast<int>((w[u >> 2] >> (8 * (u & 3))) & 0xffu);
        acc += x * q;
    }
    return acc;
}

// kSteps consecutive steps of uint8 codes (elements at ip + s * stride,
// `rem - s * stride` of them real for step s): every step's loads are issued
// before any is used, so a row of up to kSteps steps costs one memory round
// trip.
template <typename TE, int kSteps>
__device__ __forceinline__ int partial_steps(const uint16_t* ip, const uint8_t* vp, int rem,
                                             int stride, const TE* tbl) {
    if (rem <= 0) return 0;
    uint32_t t[kSteps][8];
    uint4 v[kSteps];
#pragma unroll
    for (int s = 0; s < kSteps; ++s) {
        v[s] = make_uint4(0u, 0u, 0u, 0u);
        if (s == 0 || rem > s * stride) {
            ldg256(ip + s * stride, t[s]);
            v[s] = __ldg(reinterpret_cast<const uint4*>(vp + s * stride));
        }
    }
    // four independent sums (integer: exact in any order), so the products
    // do not wait on one another
    int acc[4] = {0, 0, 0, 0};
#pragma unroll
    for (int s = 0; s < kSteps; ++s) {
        if (s == 0 || rem > s * stride) {
            const uint32_t w[4] = {v[s].x, v[s].y, v[s].z, v[s].w};
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int q = static_cast<int>(tbl[term_of(t[s], u)]);
                // code byte u & 3 of its word, zero-extended (one byte permute)
                const uint32_t x = __byte_perm(w[u >> 2], 0u, 0x4440u | (u & 3));
                acc[u & 3] += static_cast<int>(x) * q;
            }
        }
    }
    return (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

// uint16 codes: int64 sum (distance.h:49-57).
template <typename TE>
__device__ __forceinline__ long long partial(const uint16_t* ip, const uint16_t* vp, int rem,
                                             const TE* tbl) {
    if (rem <= 0) return 0;
    uint32_t t[8], v[8];
    ldg256(ip, t);
    ldg256(vp, v);
    long long acc = 0;
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const unsigned long long q = static_cast<unsigned long long>(tbl[term_of(t, u)]);
        const unsigned long long x = static_cast<unsigned long long>(term_of(v, u));
        acc += static_cast<long long>(x * q);
    }
    return acc;
}

// fp32: folds the group's products into acc in row order -- lane 0's 16,
// then lane 1's, ... -- one FADD per product, the reference's sequence of
// roundings. Every lane of the warp takes part (the shuffles are warp-wide);
// `acc` is the same on every lane of a group and comes back the same.
template <int kG>
__device__ __forceinline__ float fold(float acc, const float (&p)[16], int gbase) {
    if constexpr (kG == 1) {
#pragma unroll
        for (int u = 0; u < 16; ++u) acc = __fadd_rn(acc, p[u]);
        return acc;
    } else {
        float a = acc;
#pragma unroll
        for (int l = 0; l < kG; ++l) {
            float r = a;
#pragma unroll
            for (int u = 0; u < 16; ++u) r = __fadd_rn(r, p[u]);
            a = __shfl_sync(kFull, r, gbase + l);
        }
        return a;
    }
}

// Integer partial sums of a group, exact in any order.
template <int kG, typename A>
__device__ __forceinline__ A group_sum(A x) {
#pragma unroll
    for (int o = kG / 2; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    return x;
}

__device__ __forceinline__ float finish(float a) { return a; }
__device__ __forceinline__ float finish(int a) { return static_cast<float>(a); }
__device__ __forceinline__ float finish(long long a) { return static_cast<float>(a); }

// Scoring phase. Lanes work in groups of kG (aligned within the warp); a
// group claims one candidate of the batch at a time and walks its row kG*16
// elements per step, lane l of the group taking elements 16l..16l+15 of the
// step, so a step's loads are kG*32 contiguous bytes of ids and the matching
// contiguous values (uint8 rows: two steps per iteration). A group whose row
// ends takes the next candidate at the following iteration.
template <typename V, typename TE, bool kMask, int kG>
__device__ void score_batch(const FwdView& fwd, Ctl* ctl, const TE* tbl, const float* qv,
                            const uint32_t* coff, const uint32_t* clen, float* csc, int total,
                            int lane) {
    using A = typename Acc<V>::T;
    constexpr bool kF32 = std::is_same<V, float>::value;
    // uint8 rows advance kU8Steps steps per iteration (partial_steps)
    constexpr bool kU8 = std::is_same<V, uint8_t>::value;
    constexpr int kU8Steps = 2;
    constexpr int kStep = (kU8 ? 16 * kU8Steps : 16) * kG;
    // rows handed to L2 ahead of their scoring, in claims (3M-doc SQ
    // launch: 16 -> -1.4%, 32 -> -2.0%, 64 -> +0.6%, 128 -> +3.7% in time)
    constexpr int kPrefetchAhead = 32;
    const uint16_t* idx_base = fwd.idx;
    const V* val_base = static_cast<const V*>(fwd.val);
    const int gl = lane & (kG - 1);
    const int gbase = lane - gl;
    int i = -1;  // the group's candidate (the same on every lane of the group)
    const uint16_t* ip = nullptr;
    const V* vp = nullptr;
    int rem = 0;  // row elements from this step on
    A acc = 0;
    bool fin = false;
    for (;;) {
        const bool want = !fin && i < 0;
        const unsigned wm = __ballot_sync(kFull, want && gl == 0);
        if (wm) {
            const int leader = __ffs(wm) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&ctl->next, __popc(wm));
            base = __shfl_sync(kFull, base, leader);
            if (want) {
                const int j = base + __popc(wm & ((1u << gbase) - 1u));
                if (j < total) {
                    i = j;
                    if (kPrefetchAhead > 0 && gl == 0) {
                        // the row a group will claim about one round of
                        // claims from now goes to L2; the first round's own
                        // rows past their first iteration too
                        const int jn = j + kPrefetchAhead;
                        if (jn < total) prefetch_row<V>(idx_base, val_base, coff[jn], clen[jn], 0);
                        if (j < kPrefetchAhead)
                            prefetch_row<V>(idx_base, val_base, coff[j], clen[j], kStep);
                    }
                    const size_t e0 = static_cast<size_t>(coff[j]) * kRowAlign + 16 * gl;
                    ip = idx_base + e0;
                    vp = val_base + e0;
                    rem = static_cast<int>(clen[j]);
                    acc = 0;
                } else {
                    fin = true;
                }
            }
        }
        const bool act = i >= 0;
        if (!__any_sync(kFull, act)) break;
        const int mine = act ? rem - 16 * gl : 0;  // this lane's real elements
        if constexpr (kF32) {
            float p[16];
            products<TE, kMask>(ip, vp, mine, tbl, qv, p);
            acc = fold<kG>(acc, p, gbase);
        } else if constexpr (kU8) {
            acc += group_sum<kG>(partial_steps<TE, kU8Steps>(ip, vp, mine, 16 * kG, tbl));
        } else {
            acc += group_sum<kG>(partial<TE>(ip, vp, mine, tbl));
        }
        if (act) {
            ip += kStep;
            vp += kStep;
            rem -= kStep;
            if (rem <= 0) {
                if (gl == 0) csc[i] = finish(acc);
                i = -1;
            }
        }
    }
}

// Summary scores of list t into bscore[0..nb): hit terms in ascending term
// order, lanes spread over the term's (block, value) run.
template <typename V>
__device__ void list_summaries(const SeismicLaunch& a, int t, int nb, const uint16_t* qterm,
                               const V* qraw, int qn, float* bscore, int lane,
                               uint32_t& bytes) {
    constexpr int vsz = static_cast<int>(sizeof(V));
    // uint8 codes: a block's score is a sum of at most qn products of two
    // codes (<= 255 * 255 each), an integer below 2^24 -- exact in fp32 --
    // while qn * 65025 < 2^24 (the reference sums these integer-valued floats
    // in float as well, inverted_list_clusters.cpp:295-331)
    const bool exact_any_order =
        std::is_same<V, uint8_t>::value && static_cast<long long>(qn) * 65025ll < (1ll << 24);
    for (int b = lane; b < nb; b += 32) bscore[b] = 0.0f;
    __syncwarp();
    const uint2* meta = a.ix.lmeta + static_cast<size_t>(t) * a.ix.words;
    const int64_t colbase = a.ix.ltp[t];
    for (int i0 = 0; i0 < qn; i0 += 32) {
        const int i = i0 + lane;
        bool hit = false;
        int64_t r0 = 0, r1 = 0;
        float qv = 0.0f;
        if (i < qn && qterm[i] < static_cast<uint32_t>(a.fwd.dim)) {
            const uint32_t term = qterm[i];
            const uint2 m = __ldg(meta + (term >> 5));
            const uint32_t bit = 1u << (term & 31);
            if (m.x & bit) {
                const int64_t col = colbase + m.y + __popc(m.x & (bit - 1));
                r0 = __ldg(a.ix.srun + col);
                r1 = __ldg(a.ix.srun + col + 1);
                qv = ValT<V>::f(qraw[i]);
                hit = true;
            }
        }
        bytes += 8u * static_cast<uint32_t>(min(32, qn - i0));
        unsigned hm = __ballot_sync(kFull, hit);
        bytes += 16u * __popc(hm);
        while (hm) {
            const int src = __ffs(hm) - 1;
            hm &= hm - 1;
            const int64_t R0 = __shfl_sync(kFull, r0, src);
            const int64_t R1 = __shfl_sync(kFull, r1, src);
            const float QV = __shfl_sync(kFull, qv, src);
            bytes += static_cast<uint32_t>(R1 - R0) * (2 + vsz);
            const V* sv = static_cast<const V*>(a.ix.sval);
            if (exact_any_order) {
                // integer products and sums below 2^24: every order of the
                // float additions gives the same sum, so the updates need not
                // wait for one another
                for (int64_t e = R0 + lane; e < R1; e += 32) {
                    const int blk = __ldg(a.ix.sblk + e);
                    atomicAdd(bscore + blk, __fmul_rn(QV, ValT<V>::f(__ldg(sv + e))));
                }
            } else {
                for (int64_t e = R0 + lane; e < R1; e += 32) {
                    const int blk = __ldg(a.ix.sblk + e);
                    const float p = __fmul_rn(QV, ValT<V>::f(__ldg(sv + e)));
                    bscore[blk] = __fadd_rn(bscore[blk], p);
                }
                __syncwarp();
            }
        }
    }
}

// The first list's visiting order: the reference's std::ranges::sort of the
// block indices by summary score descending (seismic_common.h:105-115),
// restated in ref_ranking.cuh -- equal scores keep the order the reference's
// unstable sort leaves. Warp 0 sorts (score, block) pairs in `items`; the
// other warps wait at the barrier.
__device__ void sort_blocks(const float* bscore, int nb, ranking::Blk* items, uint16_t* order,
                            int tid, int warp, int lane) {
    if (warp == 0) {
        for (int i = lane; i < nb; i += 32) items[i] = ranking::Blk{__ldcg(bscore + i), i};
        __syncwarp();
        ranking::warp_sort_blocks_like_reference(items, nb, lane);
        for (int i = lane; i < nb; i += 32) order[i] = static_cast<uint16_t>(items[i].b);
    }
    __syncthreads();
}

// Cursor of warp 0 over one list's visiting order. It lives in shared memory:
// only warp 0 uses it (its lanes write the same values), and held in every
// thread's registers it would cost the scoring loop registers.
struct Cursor {
    int o;            // next position in the visiting order
    bool dead;        // the first list's walk has ended
    bool split;       // a block is part-way through
    int64_t split_d;  // its next doc position
    int split_left;
    int split_blk;
    float split_bs;
};

// Warp 0: fills the next batch with segments of blocks that pass the pruning
// test against the current heap, taking blocks in the list's visiting order
// `order[0..nb)` (the first list: sorted; later lists: the blocks that passed
// when the list began, in block order). Returns the number of segments;
// `total` receives the number of docs.
__device__ int gather(const SeismicLaunch& a, Cursor& c, bool first, int64_t lb0, int nb,
                      const float* bscore, const uint16_t* order, int n, const float* hs,
                      Seg* segs, int batch, int seg_cap, int& total, int lane) {
    int room = batch;
    int nseg = 0;
    total = 0;
    if (c.split) {
        const int take = min(room, c.split_left);
        if (lane == 0) {
            Seg g;
            g.d0 = c.split_d;
            g.cnt = take;
            g.cand0 = 0;
            g.blk = c.split_blk;
            g.bs = c.split_bs;
            g.head = 0;
            g.surv = 0;
            segs[0] = g;
        }
        nseg = 1;
        total = take;
        room -= take;
        c.split_d += take;
        c.split_left -= take;
        if (c.split_left == 0) c.split = false;
    }
    const bool full = n == a.k;
    const float hmin = full ? hs[0] : 0.0f;
    while (!c.split && !c.dead && room > 0 && nseg < seg_cap && c.o < nb) {
        const int p = c.o + lane;
        const bool in = p < nb;
        int blk = 0;
        float bs = 0.0f;
        int64_t d0 = 0, d1 = 0;
        if (in) {
            blk = static_cast<int>(order[p]);
            // the block's doc range is loaded with its score, before the test
            bs = __ldcg(bscore + blk);
            d0 = __ldg(a.ix.bdp + lb0 + blk);
            d1 = __ldg(a.ix.bdp + lb0 + blk + 1);
        }
        const bool pass = in && !(full && __fmul_rn(bs, a.heap_factor) < hmin);
        const unsigned inm = __ballot_sync(kFull, in);
        const unsigned pm = __ballot_sync(kFull, pass);
        int lim = __popc(inm);
        bool brk = false;
        if (first) {
            const unsigned fm = inm & ~pm;
            if (fm) {
                lim = __ffs(fm) - 1;
                brk = true;
            }
        }
        const bool cand = pass && lane < lim;
        const int sz = cand ? static_cast<int>(d1 - d0) : 0;
        int incl = sz;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - sz;
        const unsigned cm = __ballot_sync(kFull, cand);
        const int r = __popc(cm & ((1u << lane) - 1u));
        const bool take = cand && excl < room && nseg + r < seg_cap;
        const unsigned tm = __ballot_sync(kFull, take);
        if (take) {
            Seg g;
            g.d0 = d0;
            g.cnt = min(sz, room - excl);
            g.cand0 = total + excl;
            g.blk = blk;
            g.bs = bs;
            g.head = 1;
            g.surv = 0;
            segs[nseg + r] = g;
        }
        int taken_docs = 0;
        if (tm) {
            const int last = 31 - __clz(tm);
            const int lsz = __shfl_sync(kFull, sz, last);
            const int lexcl = __shfl_sync(kFull, excl, last);
            const int lcnt = min(lsz, room - lexcl);
            const int64_t ld0 = __shfl_sync(kFull, d0, last);
            const int lblk = __shfl_sync(kFull, blk, last);
            const float lbs = __shfl_sync(kFull, bs, last);
            taken_docs = lexcl + lcnt;
            if (lcnt < lsz) {
                c.split = true;
                c.split_d = ld0 + lcnt;
                c.split_left = lsz - lcnt;
                c.split_blk = lblk;
                c.split_bs = lbs;
            }
        }
        const unsigned nt = cm & ~tm;  // candidates left for the next batch
        if (nt) {
            c.o += __ffs(nt) - 1;
        } else {
            c.o += lim;
            // the failing block ends the first list once the blocks before it
            // (including a block cut short) are done
            if (brk && !c.split) c.dead = true;
        }
        nseg += __popc(tm);
        total += taken_docs;
        room -= taken_docs;
    }
    __syncwarp();
    return nseg;
}

// All threads: the blocks of a later list that pass the pruning test against
// the heap as it stands when the list begins, in block order, into
// order[0..return). The heap minimum only grows, so a block failing now fails
// at its turn too; the walk then visits only these (the reference tests and
// skips every block, seismic_index.cpp:78-86).
__device__ int passing_blocks(const float* bscore, int nb, bool full, float hmin, float hf,
                              uint16_t* order, int* wsum, int tid, int lane, int warp,
                              int nwarps) {
    int base = 0;
    for (int i0 = 0; i0 < nb; i0 += nwarps * 32) {
        const int i = i0 + tid;
        const bool pass = i < nb && !(full && __fmul_rn(__ldcg(bscore + i), hf) < hmin);
        const unsigned m = __ballot_sync(kFull, pass);
        if (lane == 0) wsum[warp] = __popc(m);
        __syncthreads();
        int off = 0, all = 0;
        for (int w = 0; w < nwarps; ++w) {
            const int c = wsum[w];
            off += w < warp ? c : 0;
            all += c;
        }
        if (pass) order[base + off + __popc(m & ((1u << lane) - 1u))] = static_cast<uint16_t>(i);
        base += all;
        __syncthreads();
    }
    return base;
}

// A cluster's CTAs meet here (barrier.cluster arrive + wait: release and
// acquire of shared memory across the cluster).
__device__ __forceinline__ void cluster_sync() { cg::this_cluster().sync(); }

// The leader writes a control word into every other CTA of its cluster.
__device__ __forceinline__ void push_to_cluster(int32_t* field, int32_t v) {
    cg::cluster_group cl = cg::this_cluster();
    for (unsigned r = 1; r < cl.num_blocks(); ++r) *cl.map_shared_rank(field, r) = v;
}

template <typename V, typename TE, int kG, bool kCl>
__global__ void __launch_bounds__(1024, 1) seismic_cta_kernel(SeismicLaunch a) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr bool kRank = std::is_same<V, float>::value;
    constexpr int vsz = static_cast<int>(sizeof(V));
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nwarps = blockDim.x >> 5;
    const int dim = a.fwd.dim;
    const int batch = a.batch_docs;
    const CtaLayout L =
        cta_layout(vsz, static_cast<int>(sizeof(TE)), dim, a.qcap, a.k, batch, a.seg_cap);
    Ctl* ctl = reinterpret_cast<Ctl*>(smem);
    TE* tbl = reinterpret_cast<TE*>(smem + L.tbl);
    float* qv = reinterpret_cast<float*>(smem + L.qv);
    uint16_t* qterm = reinterpret_cast<uint16_t*>(smem + L.qterm);
    V* qraw = reinterpret_cast<V*>(smem + L.qraw);
    uint16_t* cuts = reinterpret_cast<uint16_t*>(smem + L.cuts);
    float* hs = reinterpret_cast<float*>(smem + L.hs);
    int32_t* hid = reinterpret_cast<int32_t*>(smem + L.hid);
    int32_t* cdoc = reinterpret_cast<int32_t*>(smem + L.cdoc);
    uint32_t* coff = reinterpret_cast<uint32_t*>(smem + L.coff);
    uint32_t* clen = reinterpret_cast<uint32_t*>(smem + L.clen);
    float* csc = reinterpret_cast<float*>(smem + L.csc);
    Seg* segs = reinterpret_cast<Seg*>(smem + L.segs);
    uint16_t* cseg = reinterpret_cast<uint16_t*>(smem + L.cseg);  // each candidate's segment
    int* wsum = reinterpret_cast<int*>(smem + L.wsum);

    const int maxb = a.ix.max_blocks;
    float* bscore_cta = a.bscore + static_cast<size_t>(blockIdx.x) * nwarps * maxb;
    uint16_t* order = a.order + static_cast<size_t>(blockIdx.x) * a.order_stride;
    unsigned long long* keys_g =
        a.sortkeys != nullptr ? a.sortkeys + static_cast<size_t>(blockIdx.x) * a.sort_stride
                              : nullptr;

    for (int i = tid; i <= dim; i += blockDim.x) tbl[i] = 0;
    if (tid == 0) qv[0] = 0.0f;

    // With a cluster per query, the scoring phase of every CTA claims the
    // leader's (rank 0) candidates and writes the scores back there; the
    // pointers below are the leader's arrays as the cluster addresses them.
    Ctl* sctl = ctl;
    const uint32_t* scoff = coff;
    const uint32_t* sclen = clen;
    float* scsc = csc;
    unsigned cid = blockIdx.x, ncl = gridDim.x;  // this CTA's query slot, and the slots
    if constexpr (kCl) {
        cg::cluster_group cl = cg::this_cluster();
        sctl = cl.map_shared_rank(ctl, 0);
        scoff = cl.map_shared_rank(coff, 0);
        sclen = cl.map_shared_rank(clen, 0);
        scsc = cl.map_shared_rank(csc, 0);
        asm("mov.u32 %0, %%clusterid.x;" : "=r"(cid));
        asm("mov.u32 %0, %%nclusterid.x;" : "=r"(ncl));
        // every CTA of the cluster runs before any touches another's memory
        __syncthreads();
        cluster_sync();
        if (cl.block_rank() != 0) {
            // A scoring CTA: per query, the leader publishes the query index
            // (q >= n: none left), then each batch's candidate count (-1:
            // the query is done); barriers pair one to one with the leader's.
            for (;;) {
                __syncthreads();
                cluster_sync();
                const int q = ctl->q;
                if (q >= a.q.n) break;
                const int32_t qs = a.q.indptr[q];
                int qn = a.q.indptr[q + 1] - qs;
                // the leader reports it
                if (qn > a.qcap || qn < 0 || qs < 0 || (a.nnz_cap >= 0 && qs + qn > a.nnz_cap))
                    qn = 0;
                bool bad = false;
                for (int i = tid; i < qn; i += blockDim.x) {
                    const uint32_t t = a.q.idx[qs + i];
                    const V v = static_cast<const V*>(a.q.val)[qs + i];
                    qterm[i] = static_cast<uint16_t>(t);
                    if (t < static_cast<uint32_t>(dim)) {
                        if constexpr (kRank) {
                            tbl[t] = static_cast<TE>(i + 1);
                        } else {
                            tbl[t] = static_cast<TE>(v);
                        }
                    }
                    if constexpr (kRank) {
                        qv[i + 1] = ValT<V>::f(v);
                        bad |= !isfinite(ValT<V>::f(v));
                    }
                }
                const bool nonfinite = __syncthreads_or(bad) != 0;
                for (;;) {
                    cluster_sync();
                    const int total = ctl->total;
                    if (total < 0) break;
                    if (kRank && nonfinite)
                        score_batch<V, TE, true, kG>(a.fwd, sctl, tbl, qv, scoff, sclen, scsc,
                                                     total, lane);
                    else
                        score_batch<V, TE, false, kG>(a.fwd, sctl, tbl, qv, scoff, sclen, scsc,
                                                      total, lane);
                    cluster_sync();
                }
                __syncthreads();
                for (int i = tid; i < qn; i += blockDim.x) {
                    const uint32_t t = qterm[i];
                    if (t < static_cast<uint32_t>(dim)) tbl[t] = 0;
                }
            }
            return;
        }
    }

    int iter = 0;
    for (;;) {
        if (tid == 0) {
            int q;
            if (a.work_counter != nullptr) {
                q = atomicAdd(a.work_counter, 1);
                if (a.qorder != nullptr && q < a.q.n) q = a.qorder[q];
            } else
                q = a.first_query + static_cast<int>(cid) + iter * static_cast<int>(ncl);
            ctl->q = q;
            ctl->nheap = 0;  // the query's heap starts empty
            if constexpr (kCl) push_to_cluster(&ctl->q, q);
        }
        ++iter;
        __syncthreads();
        if constexpr (kCl) cluster_sync();
        const int q = ctl->q;
        if (q >= a.q.n) break;

        const uint64_t* sel = a.sel_q != nullptr ? a.sel_q[q] : a.sel_bits;
        // 1. scatter the query
        const int32_t qs = a.q.indptr[q];
        int qn = a.q.indptr[q + 1] - qs;
        // the caller's max_nnz was wrong, or the row lies past the query
        // arrays: padding, and the error is reported
        if (qn > a.qcap || qn < 0 || qs < 0 || (a.nnz_cap >= 0 && qs + qn > a.nnz_cap)) {
            if (tid == 0 && a.err != nullptr) atomicExch(a.err, 3);
            qn = 0;
        }
        bool bad = false;
        for (int i = tid; i < qn; i += blockDim.x) {
            const uint32_t t = a.q.idx[qs + i];
            const V v = static_cast<const V*>(a.q.val)[qs + i];
            qterm[i] = static_cast<uint16_t>(t);
            qraw[i] = v;
            if (t < static_cast<uint32_t>(dim)) {
                if constexpr (kRank) {
                    tbl[t] = static_cast<TE>(i + 1);
                } else {
                    tbl[t] = static_cast<TE>(v);
                }
            }
            if constexpr (kRank) {
                qv[i + 1] = ValT<V>::f(v);
                bad |= !isfinite(ValT<V>::f(v));
            }
        }
        const bool nonfinite = __syncthreads_or(bad) != 0;

        // 2. query cut (utils/vector_process.h:18-30): the query's order when
        // cut >= nnz, else the reference's TopKHolder over (value, position)
        int ncut;
        if (a.cut >= qn) {
            ncut = qn;
            for (int i = tid; i < qn; i += blockDim.x) cuts[i] = qterm[i];
        } else {
            ncut = a.cut;
            if (tid == 0) ranking::cut_like_reference(cuts, qn, ncut, QueryWeight<V>{qraw});
            __syncthreads();
            for (int i = tid; i < ncut; i += blockDim.x) cuts[i] = qterm[cuts[i]];
        }
        __syncthreads();

        // counting pass: this CTA's stamps, and warp 0's per-lane counts
        uint32_t* uq = reinterpret_cast<uint32_t*>(smem + L.uq);
        if (a.visit != nullptr && warp == 0) {
            uq[lane] = 0;
            uq[32 + lane] = 0;
        }
        int n = 0;  // heap size (warp 0)
        bool first = true;
        // Counters of this query (32 bits: a query reads far less than 4 GB).
        // docs_scored / row_bytes: every thread adds the member docs of each
        // batch it checks after scoring; warp 0 takes back those of segments
        // the second test drops, so a thread's value may be negative.
        uint32_t blocks_visited = 0, bytes = 0, lists = 0;
        int32_t docs_scored = 0, row_bytes = 0;
        for (int c = 0; c < ncut; ++c) {
            // 3. summary scores of the next nwarps lists, one warp per list
            if (c % nwarps == 0) {
                const int cw = c + warp;
                if (cw < ncut) {
                    const int tw = cuts[cw];
                    if (tw < a.ix.n_lists) {
                        const int nbw = static_cast<int>(a.ix.lbp[tw + 1] - a.ix.lbp[tw]);
                        if (nbw > 0)
                            list_summaries<V>(a, tw, nbw, qterm, qraw, qn,
                                              bscore_cta + static_cast<size_t>(warp) * maxb,
                                              lane, bytes);
                    }
                }
                __syncthreads();
            }
            const int t = cuts[c];
            if (t >= a.ix.n_lists) continue;  // seismic_index.cpp:254-256
            const int64_t lb0 = a.ix.lbp[t];
            const int nb = static_cast<int>(a.ix.lbp[t + 1] - lb0);
            if (nb > 0) {
                ++lists;
                const float* bscore = bscore_cta + static_cast<size_t>(c % nwarps) * maxb;
                // 4. visiting order: the first list's blocks sorted; a later
                // list's blocks that can still pass, in block order
                int nbv = nb;
                if (first) {
                    int p2 = 1;
                    while (p2 < nb) p2 <<= 1;
                    ranking::Blk* items = reinterpret_cast<ranking::Blk*>(
                        p2 <= 2 * batch ? reinterpret_cast<unsigned long long*>(cdoc) : keys_g);
                    if (items == nullptr) {  // the host sizes sortkeys; never taken
                        if (tid == 0) atomicExch(a.err, 2);
                        break;
                    }
                    sort_blocks(bscore, nb, items, order, tid, warp, lane);
                } else {
                    const int nh = ctl->nheap;
                    nbv = passing_blocks(bscore, nb, nh == a.k, nh == a.k ? hs[0] : 0.0f,
                                         a.heap_factor, order, wsum, tid, lane, warp, nwarps);
                }
                // 5. batches
                Cursor& cur = *reinterpret_cast<Cursor*>(smem + L.cur);
                if (warp == 0) {
                    cur.o = 0;
                    cur.dead = false;
                    cur.split = false;
                    cur.split_d = 0;
                    cur.split_left = 0;
                    cur.split_blk = 0;
                    cur.split_bs = 0.0f;
                }
                for (;;) {
                    if (warp == 0) {
                        int total = 0;
                        const int nseg = gather(a, cur, first, lb0, nbv, bscore, order, n, hs,
                                                segs, batch, a.seg_cap, total, lane);
                        if (lane == 0) {
                            ctl->nseg = nseg;
                            ctl->total = total;
                            ctl->next = 0;
                            ctl->nheap = n;
                        }
                    }
                    __syncthreads();
                    const int nseg = ctl->nseg;
                    const int total = ctl->total;
                    if (nseg == 0) break;
                    if (total > 0) {
                        // candidates: doc ids and row info of every segment's docs
                        for (int i = tid; i < total; i += blockDim.x) {
                            int lo = 0, hi = nseg - 1;
                            while (lo < hi) {
                                const int mid = (lo + hi + 1) >> 1;
                                if (segs[mid].cand0 <= i)
                                    lo = mid;
                                else
                                    hi = mid - 1;
                            }
                            const Seg& g = segs[lo];
                            const int64_t pj = g.d0 + (i - g.cand0);
                            const int32_t d = __ldg(a.ix.docs + pj);
                            // row info stored with the posting, else looked up
                            uint2 ri = a.ix.drow != nullptr ? __ldg(a.ix.drow + pj)
                                                            : __ldg(a.fwd.rowinfo + d);
                            bool member = true;
                            if (sel != nullptr)
                                member = (__ldg(sel + (d >> 6)) >> (d & 63)) & 1ull;
                            if (!member) ri = make_uint2(0u, 0u);
                            cdoc[i] = member ? d : -1;
                            coff[i] = ri.x;
                            clen[i] = ri.y;
                            cseg[i] = static_cast<uint16_t>(lo);
                        }
                        __syncthreads();
                        // 6. scores (with the cluster's other CTAs)
                        if constexpr (kCl) {
                            if (tid == 0) push_to_cluster(&ctl->total, total);
                            cluster_sync();
                        }
                        if (kRank && nonfinite)
                            score_batch<V, TE, true, kG>(a.fwd, sctl, tbl, qv, scoff, sclen, scsc,
                                                         total, lane);
                        else
                            score_batch<V, TE, false, kG>(a.fwd, sctl, tbl, qv, scoff, sclen,
                                                          scsc, total, lane);
                        if constexpr (kCl) cluster_sync();
                        __syncthreads();
                    }
                    // 7. second pruning test and heap offers, in block order.
                    // (a) All threads: a doc can still enter the heap only if
                    // it is a member scoring above the heap minimum as it
                    // stood when the batch was gathered (the minimum only
                    // grows); segments holding such docs are flagged.
                    {
                        const int nh = ctl->nheap;
                        const float hmin0 = nh == a.k ? hs[0] : 0.0f;
                        for (int i = tid; i < total; i += blockDim.x) {
                            if (cdoc[i] >= 0) {
                                ++docs_scored;
                                row_bytes += 8 + static_cast<int32_t>(clen[i]) * (2 + vsz);
                                // a flag: every writer stores the same 1
                                if (nh < a.k || !(csc[i] <= hmin0)) segs[cseg[i]].surv = 1;
                            }
                        }
                        __syncthreads();
                    }
                    // (b) Warp 0 walks the segments in block order as the
                    // reference walks its blocks (seismic_index.cpp:78-117):
                    // each block head is tested against the heap as it stands
                    // at its turn, then its docs are offered in order. A run
                    // of segments without survivors leaves the heap as it is,
                    // so all its tests see one minimum and one ballot settles
                    // up to 32 of them; a segment with survivors offers those.
                    if (warp == 0) {
                        // the work counters give back a dropped segment's docs
                        auto give_back = [&](int t) {
                            const Seg g = segs[t];
                            for (int j = lane; j < g.cnt; j += 32) {
                                const int i = g.cand0 + j;
                                if (cdoc[i] >= 0) {
                                    --docs_scored;
                                    row_bytes -= 8 + static_cast<int32_t>(clen[i]) * (2 + vsz);
                                }
                            }
                        };
                        // counting pass: the member docs of a visited block,
                        // each counted the first time the query meets it
                        auto count_visits = [&](int t) {
                            if (a.visit == nullptr) return;
                            uint32_t* stamp = a.visit + static_cast<size_t>(blockIdx.x) *
                                                            static_cast<size_t>(a.fwd.n_docs);
                            const Seg g = segs[t];
                            for (int j = lane; j < g.cnt; j += 32) {
                                const int i = g.cand0 + j;
                                const int32_t d = cdoc[i];
                                if (d >= 0 && atomicExch(stamp + d, static_cast<uint32_t>(iter)) !=
                                                  static_cast<uint32_t>(iter)) {
                                    uq[lane] += 1;
                                    uq[32 + lane] += 8u + clen[i] * (2 + vsz);
                                }
                            }
                        };
                        auto end_first_list = [&](int from) {
                            for (int t = from; t < nseg; ++t) give_back(t);
                            cur.dead = true;
                            cur.split = false;
                        };
                        int s = 0;
                        bool ended = false;
                        while (s < nseg && !ended) {
                            const int sl = s + lane;
                            const bool valid = sl < nseg;
                            int head = 0, cnt = 0, surv = 0;
                            float bs = 0.0f;
                            if (valid) {
                                const Seg g = segs[sl];
                                head = g.head;
                                cnt = g.cnt;
                                surv = g.surv;
                                bs = g.bs;
                            }
                            const int w = __popc(__ballot_sync(kFull, valid));
                            const unsigned sm = __ballot_sync(kFull, valid && surv > 0);
                            const int S = sm ? __ffs(sm) - 1 : w;  // first that may change the heap
                            const bool full = n == a.k;
                            const float hmin = full ? hs[0] : 0.0f;
                            const bool fail =
                                lane < S && head && full && __fmul_rn(bs, a.heap_factor) < hmin;
                            const unsigned fm = __ballot_sync(kFull, fail);
                            // the first list ends at its first failing block
                            const int upto = (first && fm) ? __ffs(fm) - 1 : S;
                            const bool taken = lane < upto && !fail;
                            blocks_visited += __popc(__ballot_sync(kFull, taken && head));
                            bytes += 16u * __popc(__ballot_sync(kFull, taken && head)) +
                                     4u * __reduce_add_sync(kFull, taken ? cnt : 0);
                            if (a.visit != nullptr) {
                                unsigned tm = __ballot_sync(kFull, taken);
                                while (tm) {
                                    const int t = __ffs(tm) - 1;
                                    tm &= tm - 1;
                                    count_visits(s + t);
                                }
                            }
                            unsigned dm = __ballot_sync(kFull, lane < upto && fail);
                            while (dm) {  // later lists skip a failing block
                                const int t = __ffs(dm) - 1;
                                dm &= dm - 1;
                                give_back(s + t);
                                if (s + t == nseg - 1) cur.split = false;
                            }
                            if (first && fm) {
                                end_first_list(s + upto);
                                ended = true;
                                break;
                            }
                            s += upto;
                            if (upto == w) continue;
                            // segment s holds survivors: its test, then its offers
                            const Seg g = segs[s];
                            if (g.head && n == a.k &&
                                __fmul_rn(g.bs, a.heap_factor) < hs[0]) {
                                if (first) {
                                    end_first_list(s);
                                    ended = true;
                                    break;
                                }
                                give_back(s);
                                if (s == nseg - 1) cur.split = false;
                            } else {
                                if (g.head) {
                                    ++blocks_visited;
                                    bytes += 16;
                                }
                                bytes += 4u * static_cast<uint32_t>(g.cnt);
                                count_visits(s);
                                for (int b = 0; b < g.cnt; b += 32) {
                                    const int j = b + lane;
                                    float sc = 0.0f;
                                    int32_t d = -1;
                                    if (j < g.cnt) {
                                        d = cdoc[g.cand0 + j];
                                        sc = csc[g.cand0 + j];
                                    }
                                    unsigned m = __ballot_sync(
                                        kFull, d >= 0 && (n < a.k || !(sc <= hs[0])));
                                    while (m) {
                                        const int src = __ffs(m) - 1;
                                        m &= m - 1;
                                        const float S2 = __shfl_sync(kFull, sc, src);
                                        const int32_t D2 = __shfl_sync(kFull, d, src);
                                        heap_offer(S2, D2, hs, hid, n, a.k, lane);
                                    }
                                }
                            }
                            ++s;
                        }
                    }
                }
            }
            first = false;  // seismic_index.cpp:261
        }

        if constexpr (kCl) {  // the query is done: the scoring CTAs move on
            __syncthreads();
            if (tid == 0) push_to_cluster(&ctl->total, -1);
            cluster_sync();
        }
        // results, padded with (-1.0, -1); SQ scores decoded
        // (seismic_scalar_quantized_index.cpp:345-355)
        if (warp == 0) {
            heap_emit(hs, hid, n, a.k, a.decode_scale, a.out_d + static_cast<size_t>(q) * a.k,
                      a.out_l + static_cast<size_t>(q) * a.k, lane);
            if (a.done != nullptr) {
                // every lane's results reach memory (mapped host memory
                // included) before the flag does
                __threadfence_system();
                __syncwarp();
                if (lane == 0) *reinterpret_cast<volatile int32_t*>(a.done + q) = 1;
            }
        }
        if (a.stats != nullptr) {
            // per warp: its threads' doc counts and row bytes, plus its
            // summary bytes (the same on every lane) and, for warp 0, the
            // block counts
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                row_bytes += __shfl_xor_sync(kFull, row_bytes, o);
                docs_scored += __shfl_xor_sync(kFull, docs_scored, o);
            }
            if (lane == 0) {
                if (warp == 0) {
                    atomicAdd(a.stats + kStatBlocksVisited,
                              static_cast<unsigned long long>(blocks_visited));
                    atomicAdd(a.stats + kStatListsProbed, static_cast<unsigned long long>(lists));
                }
                // a warp's net counts can be negative: widened with their sign,
                // they add up modulo 2^64 to the exact total
                atomicAdd(a.stats + kStatDocsScored,
                          static_cast<unsigned long long>(static_cast<long long>(docs_scored)));
                atomicAdd(a.stats + kStatBytes,
                          static_cast<unsigned long long>(bytes) +
                              static_cast<unsigned long long>(static_cast<long long>(row_bytes)));
                atomicAdd(a.stats + kStatRowBytes,
                          static_cast<unsigned long long>(static_cast<long long>(row_bytes)));
            }
            if (a.visit != nullptr && warp == 0) {
                uint32_t ud = uq[lane], ub = uq[32 + lane];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ud += __shfl_xor_sync(kFull, ud, o);
                    ub += __shfl_xor_sync(kFull, ub, o);
                }
                if (lane == 0) {
                    atomicAdd(a.stats + kStatUniqueDocs, static_cast<unsigned long long>(ud));
                    atomicAdd(a.stats + kStatUniqueRowBytes, static_cast<unsigned long long>(ub));
                }
            }
        }
        // restore the all-zero table for the next query
        __syncthreads();
        for (int i = tid; i < qn; i += blockDim.x) {
            const uint32_t t = qterm[i];
            if (t < static_cast<uint32_t>(dim)) tbl[t] = 0;
        }
    }
}

template <typename V, typename TE>
size_t smem_typed(int dim, int qcap, int k, int batch, int seg_cap) {
    return cta_layout(static_cast<int>(sizeof(V)), static_cast<int>(sizeof(TE)), dim, qcap, k,
                      batch, seg_cap)
        .total;
}

template <typename V, typename TE, int kG>
int max_blocks_cta_g(int threads, size_t smem) {
    if (allow_opt_in_smem(seismic_cta_kernel<V, TE, kG, false>) != cudaSuccess)
        return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, seismic_cta_kernel<V, TE, kG, false>,
                                                      threads, smem) != cudaSuccess)
        return 0;
    return blocks;
}

template <typename V, typename TE>
int max_blocks_cta_typed(int group, int threads, size_t smem) {
    if (group == 8) return max_blocks_cta_g<V, TE, 8>(threads, smem);
    if (group == 4) return max_blocks_cta_g<V, TE, 4>(threads, smem);
    if (group == 2) return max_blocks_cta_g<V, TE, 2>(threads, smem);
    return max_blocks_cta_g<V, TE, 1>(threads, smem);
}

template <typename V, typename TE, int kG>
cudaError_t launch_cta_g(const SeismicLaunch& a, int warps, int blocks, size_t smem,
                         cudaStream_t s) {
    if (a.cluster > 1) {
        // one cluster of a.cluster CTAs per query; the grid is whole clusters
        auto* f = seismic_cta_kernel<V, TE, kG, true>;
        cudaError_t e = allow_opt_in_smem(f);
        if (e != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(static_cast<unsigned>(blocks));
        cfg.blockDim = dim3(static_cast<unsigned>(warps * 32));
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = static_cast<unsigned>(a.cluster);
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int fits = 0;
        if (cudaOccupancyMaxActiveClusters(&fits, f, &cfg) == cudaSuccess && fits > 0)
            return cudaLaunchKernelEx(&cfg, f, a);
        // A device that cannot place such a cluster runs the query on one CTA
        // (same results): the same grid walks the same queries, the extra
        // CTAs of a one-query launch find none left.
        (void)cudaGetLastError();
        SeismicLaunch one = a;
        one.cluster = 1;
        e = allow_opt_in_smem(seismic_cta_kernel<V, TE, kG, false>);
        if (e != cudaSuccess) return e;
        seismic_cta_kernel<V, TE, kG, false><<<blocks, warps * 32, smem, s>>>(one);
        return cudaGetLastError();
    }
    cudaError_t e = allow_opt_in_smem(seismic_cta_kernel<V, TE, kG, false>);
    if (e != cudaSuccess) return e;
    seismic_cta_kernel<V, TE, kG, false><<<blocks, warps * 32, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename V, typename TE>
cudaError_t launch_cta_typed(const SeismicLaunch& a, int warps, int blocks, cudaStream_t s) {
    const size_t smem = smem_typed<V, TE>(a.fwd.dim, a.qcap, a.k, a.batch_docs, a.seg_cap);
    if (a.group_lanes == 8) return launch_cta_g<V, TE, 8>(a, warps, blocks, smem, s);
    if (a.group_lanes == 4) return launch_cta_g<V, TE, 4>(a, warps, blocks, smem, s);
    if (a.group_lanes == 2) return launch_cta_g<V, TE, 2>(a, warps, blocks, smem, s);
    return launch_cta_g<V, TE, 1>(a, warps, blocks, smem, s);
}

}  // namespace

// Table entries: fp32 queries hold ranks, one byte while the query has at
// most 255 terms; SQ queries hold their codes.
// Claim order of a batched launch: queries by row length, longest first (a
// counting sort over lengths clamped to 255, one CTA).
__global__ void __launch_bounds__(1024) order_by_length_kernel(const int32_t* indptr, int32_t n,
                                                               int32_t* order) {
    __shared__ int32_t bin[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) bin[i] = 0;
    __syncthreads();
    auto key = [&](int32_t i) {
        const int32_t len = indptr[i + 1] - indptr[i];
        return 255 - (len < 0 ? 0 : (len > 255 ? 255 : len));
    };
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&bin[key(i)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t run = 0;
        for (int b = 0; b < 256; ++b) {
            const int32_t c = bin[b];
            bin[b] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) order[atomicAdd(&bin[key(i)], 1)] = i;
}

static bool wide_table(int val_kind, int qcap) {
    return val_kind == kU16 || (val_kind == kF32 && qcap > 255);
}

size_t seismic_cta_smem(int val_kind, int dim, int qcap, int k, int batch, int seg_cap) {
    if (val_kind == kF32)
        return wide_table(val_kind, qcap)
                   ? smem_typed<float, uint16_t>(dim, qcap, k, batch, seg_cap)
                   : smem_typed<float, uint8_t>(dim, qcap, k, batch, seg_cap);
    if (val_kind == kU8) return smem_typed<uint8_t, uint8_t>(dim, qcap, k, batch, seg_cap);
    return smem_typed<uint16_t, uint16_t>(dim, qcap, k, batch, seg_cap);
}

int seismic_cta_seg_cap(int cluster) { return cluster > 1 ? kSegCapMax : kSegCap; }

int seismic_cta_max_blocks_per_sm(int val_kind, int qcap, int group, int warps, size_t smem) {
    const int th = warps * 32;
    if (val_kind == kF32)
        return wide_table(val_kind, qcap)
                   ? max_blocks_cta_typed<float, uint16_t>(group, th, smem)
                   : max_blocks_cta_typed<float, uint8_t>(group, th, smem);
    if (val_kind == kU8) return max_blocks_cta_typed<uint8_t, uint8_t>(group, th, smem);
    return max_blocks_cta_typed<uint16_t, uint16_t>(group, th, smem);
}

cudaError_t launch_seismic_cta(int val_kind, const SeismicLaunch& a, int warps, int blocks,
                               cudaStream_t s) {
    if (val_kind == kF32)
        return wide_table(val_kind, a.qcap) ? launch_cta_typed<float, uint16_t>(a, warps, blocks, s)
                                            : launch_cta_typed<float, uint8_t>(a, warps, blocks, s);
    if (val_kind == kU8) return launch_cta_typed<uint8_t, uint8_t>(a, warps, blocks, s);
    return launch_cta_typed<uint16_t, uint16_t>(a, warps, blocks, s);
}

cudaError_t launch_order_by_length(const int32_t* indptr, int32_t n, int32_t* order,
                                   cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    order_by_length_kernel<<<1, 1024, 0, s>>>(indptr, n, order);
    return cudaGetLastError();
}

}  // namespace nsp
