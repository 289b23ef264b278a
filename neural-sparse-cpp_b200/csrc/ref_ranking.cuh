// The reference's ranking order, restated for the device (and the host, for
// the tests that pin it):
//
//  * its first list's visiting order, std::ranges::sort of the block indices
//    by summary score descending (seismic_common.h:105-115) -- an unstable
//    sort, so the order of equal scores is whatever the C++ standard
//    library's introsort leaves. The steps below are that introsort's
//    (median of three moved to the front, unguarded partition, recursion on
//    the right part, a heap sort once the depth budget 2*floor(log2 n) is
//    spent, ranges of at most 16 left to a final insertion sort), so equal
//    scores end up where the reference's sort puts them;
//  * its top-k holder, a std::priority_queue ordered by std::greater on the
//    score (utils/ranker.h:34-138): the smallest score on top, a full holder
//    rejects score <= top, otherwise pops the top and pushes; results come
//    out by popping into the array from its end. Equal scores are ordered by
//    the binary heap's sift steps, restated here.
//
// Both only permute; the comparisons are the reference's (strict `>` on
// float scores; +0.0 and -0.0 compare equal).
#ifndef NSP_REF_RANKING_CUH
#define NSP_REF_RANKING_CUH

#include <cstdint>

#if defined(__CUDACC__)
#define NSP_RR __host__ __device__ __forceinline__
// kept out of line on the device: its stack stays out of the search
// kernels' register allocation
#define NSP_RR_CALL static __host__ __device__ __noinline__
#else
#define NSP_RR inline
#define NSP_RR_CALL inline
#endif

namespace nsp {
namespace ranking {

// A block of the first list: summary score and block index.
struct Blk {
    float s;
    int32_t b;
};

// The reference's comparator: x before y when x scores higher.
NSP_RR bool before(const Blk& x, const Blk& y) { return x.s > y.s; }

NSP_RR void swap_blk(Blk* a, int i, int j) {
    const Blk t = a[i];
    a[i] = a[j];
    a[j] = t;
}

NSP_RR int floor_log2(int n) {
    int r = 0;
    while (n > 1) {
        n >>= 1;
        ++r;
    }
    return r;
}

// Moves the median of a[x], a[y], a[z] (under `before`) into a[r].
NSP_RR void median_to(Blk* a, int r, int x, int y, int z) {
    int m;
    if (before(a[x], a[y])) {
        if (before(a[y], a[z])) m = y;
        else if (before(a[x], a[z])) m = z;
        else m = x;
    } else if (before(a[x], a[z])) {
        m = x;
    } else if (before(a[y], a[z])) {
        m = z;
    } else {
        m = y;
    }
    swap_blk(a, r, m);
}

// One partition step of [f, l) (l - f > 16): the median of a[f+1], the
// middle element and a[l-1] becomes the pivot at a[f]; returns the cut.
NSP_RR int partition_step(Blk* a, int f, int l) {
    median_to(a, f, f + 1, f + (l - f) / 2, l - 1);
    const Blk p = a[f];  // never moved by the scan below
    int lo = f + 1, hi = l;
    for (;;) {
        while (before(a[lo], p)) ++lo;
        --hi;
        while (before(p, a[hi])) --hi;
        if (!(lo < hi)) return lo;
        swap_blk(a, lo, hi);
        ++lo;
    }
}

// Heap primitives over a[0, len) under `Less(x, y)` (x below y in the heap
// order): the sift-up from a hole, and the sift-down that walks the hole to
// a leaf along the larger child and then sifts the value up.
template <typename T, typename Less>
NSP_RR void heap_sift_up(T* a, int hole, int top, T v, Less less) {
    int parent = (hole - 1) / 2;
    while (hole > top && less(a[parent], v)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

template <typename T, typename Less>
NSP_RR void heap_sift_down(T* a, int hole, int len, T v, Less less) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (less(a[child], a[child - 1])) --child;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    heap_sift_up(a, hole, top, v, less);
}

struct BlkLess {
    NSP_RR bool operator()(const Blk& x, const Blk& y) const { return before(x, y); }
};

// The depth-budget fallback: make a heap of a[f, l), then pop it empty.
NSP_RR void heap_sort_range(Blk* a, int f, int l) {
    Blk* h = a + f;
    const int len = l - f;
    if (len < 2) return;
    for (int parent = (len - 2) / 2;; --parent) {
        heap_sift_down(h, parent, len, h[parent], BlkLess{});
        if (parent == 0) break;
    }
    for (int n = len; n > 1;) {
        --n;
        const Blk v = h[n];
        h[n] = h[0];
        heap_sift_down(h, 0, n, v, BlkLess{});
    }
}

// Insertion sort of a[f, l) that moves an element left only past elements it
// is strictly `before`: equal scores keep their order. Over a range whose
// partition steps are done it is the reference's final insertion pass
// (an element never moves past a cut: everything left of a cut scores at
// least as high as everything right of it).
NSP_RR void insertion_range(Blk* a, int f, int l) {
    for (int i = f + 1; i < l; ++i) {
        const Blk v = a[i];
        int j = i;
        while (j > f && before(v, a[j - 1])) {
            a[j] = a[j - 1];
            --j;
        }
        a[j] = v;
    }
}

constexpr int kSortThreshold = 16;
// Pending ranges: their depth budgets strictly decrease from the bottom of
// the stack to its top, so at most 2 * floor(log2 n) + 1 <= 63 wait at once.
constexpr int kSortStack = 64;

// The introsort loop over a[f, l) with depth budget d (the order in which
// independent ranges are finished does not change the result), then the
// insertion pass over the range.
NSP_RR_CALL void sort_range(Blk* a, int f, int l, int d) {
    int sf[kSortStack], sl[kSortStack];
    uint8_t sd[kSortStack];
    int top = 0;
    sf[0] = f;
    sl[0] = l;
    sd[0] = static_cast<uint8_t>(d);
    top = 1;
    while (top > 0) {
        --top;
        int cf = sf[top], cl = sl[top], cd = sd[top];
        while (cl - cf > kSortThreshold) {
            if (cd == 0) {
                heap_sort_range(a, cf, cl);
                break;
            }
            --cd;
            const int cut = partition_step(a, cf, cl);
            // the right part waits on the stack (its size is bounded by the
            // depth budget, at most 2 * 31 entries)
            sf[top] = cut;
            sl[top] = cl;
            sd[top] = static_cast<uint8_t>(cd);
            ++top;
            cl = cut;
        }
    }
    insertion_range(a, f, l);
}

// The reference's sort of a[0, n) on one thread.
NSP_RR void sort_blocks_like_reference(Blk* a, int n) {
    if (n <= 0) return;
    sort_range(a, 0, n, 2 * floor_log2(n));
}

// Splits of the sort handed out to more lanes: lane j of round r takes the
// left (j even) or right (j odd) part of lane j/2's range; a range that is
// not partitioned (at most 16 entries, or its depth budget spent) stays whole
// with the even lane. After kSortSplitRounds rounds each lane finishes its
// range with sort_range. Ranges are disjoint, so the result is the
// one-thread sort's.
constexpr int kSortSplitRounds = 5;

struct SortRange {
    int f, l, d;  // [f, l), depth budget d
};

// One lane's range after a split round, from its parent's range and cut
// (cut < 0: not partitioned).
NSP_RR SortRange split_child(SortRange parent, int cut, bool odd) {
    SortRange r;
    if (cut < 0) {
        r.f = odd ? 0 : parent.f;
        r.l = odd ? 0 : parent.l;
        r.d = parent.d;
    } else {
        r.f = odd ? cut : parent.f;
        r.l = odd ? parent.l : cut;
        r.d = parent.d - 1;
    }
    return r;
}

NSP_RR int split_cut(Blk* a, SortRange r) {
    return (r.l - r.f > kSortThreshold && r.d > 0) ? partition_step(a, r.f, r.l) : -1;
}

#if defined(__CUDACC__)
// The reference's sort of a[0, n) by one warp (all lanes call).
__device__ __forceinline__ void warp_sort_blocks_like_reference(Blk* a, int n, int lane) {
    SortRange r{0, lane == 0 ? n : 0, n > 0 ? 2 * floor_log2(n) : 0};
    for (int round = 0; round < kSortSplitRounds; ++round) {
        const int active = 1 << round;
        const int cut = lane < active ? split_cut(a, r) : -1;
        __syncwarp();
        const int src = lane >> 1;
        SortRange p;
        p.f = __shfl_sync(0xffffffffu, r.f, src);
        p.l = __shfl_sync(0xffffffffu, r.l, src);
        p.d = __shfl_sync(0xffffffffu, r.d, src);
        const int pc = __shfl_sync(0xffffffffu, cut, src);
        if (lane < 2 * active) r = split_child(p, pc, (lane & 1) != 0);
    }
    if (r.l > r.f) sort_range(a, r.f, r.l, r.d);
    __syncwarp();
}
#endif

// ---- the top-k holder ------------------------------------------------

// Heap order of the reference's priority_queue<..., CompareItem> with
// CompareItem = std::greater on the score: x below y when x.score > y.score,
// so the top holds the smallest score.
struct ScoreLess {
    NSP_RR bool operator()(float x, float y) const { return x > y; }
};

// Heap entries live as two arrays (scores, ids); these helpers move both.
struct TopK {
    float* s;
    int32_t* id;
};

NSP_RR void topk_sift_up(TopK h, int hole, float vs, int32_t vi) {
    int parent = (hole - 1) / 2;
    while (hole > 0 && h.s[parent] > vs) {
        h.s[hole] = h.s[parent];
        h.id[hole] = h.id[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    h.s[hole] = vs;
    h.id[hole] = vi;
}

NSP_RR void topk_sift_down(TopK h, int len, float vs, int32_t vi) {
    int hole = 0, child = 0;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (h.s[child] > h.s[child - 1]) --child;
        h.s[hole] = h.s[child];
        h.id[hole] = h.id[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        h.s[hole] = h.s[child - 1];
        h.id[hole] = h.id[child - 1];
        hole = child - 1;
    }
    topk_sift_up(h, hole, vs, vi);
}

// push: append, sift up.
NSP_RR void topk_push(TopK h, int& n, float s, int32_t id) {
    topk_sift_up(h, n, s, id);
    ++n;
}

// pop: the last entry fills the top's place by the sift-down.
NSP_RR void topk_pop(TopK h, int& n) {
    if (n > 1) {
        const float vs = h.s[n - 1];
        const int32_t vi = h.id[n - 1];
        h.s[n - 1] = h.s[0];
        h.id[n - 1] = h.id[0];
        topk_sift_down(h, n - 1, vs, vi);
    }
    --n;
}

// TopKHolder::add (ranker.h:58-72): a full holder rejects score <= its top;
// otherwise a full holder pops, then pushes.
NSP_RR void topk_add(TopK h, int& n, int k, float s, int32_t id) {
    if (n >= k && s <= h.s[0]) return;
    if (n >= k) topk_pop(h, n);
    topk_push(h, n, s, id);
}

// TopKHolder::top_k_items_descending (ranker.h:113-127): pops into the
// arrays from the end; empties the holder.
NSP_RR void topk_drain_descending(TopK h, int n, float* out_s, int32_t* out_id) {
    for (int i = n - 1; i >= 0; --i) {
        out_s[i] = h.s[0];
        out_id[i] = h.id[0];
        topk_pop(h, n);
    }
}

// ---- the query cut ----------------------------------------------------

// top_k_tokens (utils/vector_process.h:18-30) when cut < n: a TopKHolder of
// size `cut` offered (value, position) for positions 0..n-1 in order, then
// top_k_descending (ranker.h:95-106). The holder is an array of positions
// `heap` (cut entries); `value(i)` is position i's weight as a float. Popping
// the holder empty in place leaves it in top_k_descending order (each pop
// moves the top to the end of the shrinking heap). One thread.
template <typename Value>
struct WeightGreater {
    Value v;
    NSP_RR bool operator()(uint16_t x, uint16_t y) const { return v(x) > v(y); }
};

template <typename Value>
NSP_RR void cut_like_reference(uint16_t* heap, int n, int cut, Value value) {
    const WeightGreater<Value> less{value};
    int m = 0;
    for (int i = 0; i < n; ++i) {
        const float s = value(static_cast<uint16_t>(i));
        if (m >= cut && s <= value(heap[0])) continue;
        if (m >= cut) {
            if (m > 1) {
                const uint16_t v = heap[m - 1];
                heap[m - 1] = heap[0];
                heap_sift_down(heap, 0, m - 1, v, less);
            }
            --m;
        }
        heap_sift_up(heap, m, 0, static_cast<uint16_t>(i), less);
        ++m;
    }
    while (m > 1) {
        const uint16_t v = heap[m - 1];
        heap[m - 1] = heap[0];
        heap_sift_down(heap, 0, m - 1, v, less);
        --m;
    }
}

}  // namespace ranking
}  // namespace nsp

#endif  // NSP_REF_RANKING_CUH
