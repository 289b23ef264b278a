// Exact top-k over every document: BrutalIndex (brutal_index.cpp:75-96) and
// InvertedIndex (inverted_index.cpp:295-365) semantics on sm_100a.
//
// A CTA owns 32 queries (one per lane) and a contiguous tile of documents.
// The 32 query bitmaps (+ popcount prefixes) sit in shared memory with an odd
// word stride, so the 32 lanes probing the same term hit 32 distinct banks.
// Each warp streams its share of the tile's rows: a row is staged once in
// shared memory (the next row's loads are in flight meanwhile) and every lane
// walks it sequentially against its own query -- the reference's exact fp32
// summation order (utils/distance.h:29-37) falls out for free, and each row is
// read from HBM/L2 once per 32 queries.
//
// Top-k: every lane keeps a k-entry list for its query in global scratch with
// its threshold in a register (inserts are rare once it fills); a warp visits
// its docs in ascending id order, so "reject score <= min" resolves ties to
// the lower id (utils/ranker.h:147-200). The CTA merges its warps' lists per
// query, and a second kernel merges the tiles.
//
// The term-at-a-time kernel below is the default for indexes whose rows hold
// strictly ascending terms and for k <= kTaatMaxK; the tile kernel serves the
// rest.
#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cstdint>

#include "nsp_device.h"

namespace nsp {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 8;
constexpr int kQG = 32;        // queries per CTA
constexpr int kStageElems = 256;

__host__ __device__ inline int odd_stride(int words) { return words | 1; }

// qcap_smem = 0 keeps the query values in global scratch (long queries).
__host__ __device__ inline size_t exact_smem_bytes(int words, int qcap_smem) {
    const size_t S = static_cast<size_t>(odd_stride(words));
    size_t b = 0;
    b += kQG * S * 4;                                   // bitmaps
    b += ((kQG * S * 2) + 15) & ~size_t(15);            // prefixes (uint16)
    b += ((static_cast<size_t>(kQG) * qcap_smem * 4) + 15) & ~size_t(15);  // values
    b += static_cast<size_t>(kWarps) * kStageElems * 6;  // row stage (u16 + f32)
    return b;
}

__device__ __forceinline__ bool better(float s1, int32_t i1, float s2, int32_t i2) {
    return s1 > s2 || (s1 == s2 && i1 < i2);
}

// Inserts into a sorted (score desc, id asc) list of size n <= k. Caller has
// already checked the threshold.
__device__ __forceinline__ void list_insert(float* ls, int32_t* li, int& n, int k, float s,
                                            int32_t d) {
    int pos = n < k ? n : k - 1;
    if (n < k) ++n;
    while (pos > 0 && better(s, d, ls[pos - 1], li[pos - 1])) {
        ls[pos] = ls[pos - 1];
        li[pos] = li[pos - 1];
        --pos;
    }
    ls[pos] = s;
    li[pos] = d;
}

__global__ void __launch_bounds__(kWarps * 32) exact_tile_kernel(ExactLaunch a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int words = (a.fwd.dim + 31) / 32;
    const int S = odd_stride(words);
    uint32_t* qbits = reinterpret_cast<uint32_t*>(smem);
    uint16_t* qpre = reinterpret_cast<uint16_t*>(smem + static_cast<size_t>(kQG) * S * 4);
    float* qval_smem = reinterpret_cast<float*>(
        smem + static_cast<size_t>(kQG) * S * 4 + ((static_cast<size_t>(kQG) * S * 2 + 15) & ~size_t(15)));
    const int qcap_smem = a.qval_global != nullptr ? 0 : a.qcap;
    unsigned char* stage_base = reinterpret_cast<unsigned char*>(qval_smem) +
                                ((static_cast<size_t>(kQG) * qcap_smem * 4 + 15) & ~size_t(15));
    float* qval = a.qval_global != nullptr
                      ? a.qval_global + static_cast<size_t>(blockIdx.y * gridDim.x + blockIdx.x) *
                                            kQG * a.qcap
                      : qval_smem;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int tile = blockIdx.x;
    const int group = blockIdx.y;
    const int tiles = gridDim.x;
    const int q0 = group * kQG;
    const int nq_here = min(kQG, a.q.n - q0);

    // Build the group's bitmaps: warp w builds queries w, w+8, ...
    for (int g = warp; g < kQG; g += kWarps) {
        uint32_t* bits = qbits + static_cast<size_t>(g) * S;
        for (int i = lane; i < words; i += 32) bits[i] = 0u;
        __syncwarp();
        if (g < nq_here) {
            const int32_t qs = a.q.indptr[q0 + g];
            const int qn = a.q.indptr[q0 + g + 1] - qs;
            const float* qv = static_cast<const float*>(a.q.val);
            for (int i = lane; i < qn; i += 32) {
                const uint32_t t = a.q.idx[qs + i];
                qval[static_cast<size_t>(g) * a.qcap + i] = qv[qs + i];
                atomicOr(&bits[t >> 5], 1u << (t & 31));
            }
        }
        __syncwarp();
        const int cs = (words + 31) / 32;
        const int w0 = lane * cs;
        const int w1 = min(words, w0 + cs);
        int local = 0;
        for (int i = w0; i < w1; ++i) local += __popc(bits[i]);
        int incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        int run = incl - local;
        uint16_t* pre = qpre + static_cast<size_t>(g) * S;
        for (int i = w0; i < w1; ++i) {
            pre[i] = static_cast<uint16_t>(run);
            run += __popc(bits[i]);
        }
    }
    __syncthreads();

    // This lane's query and its top-k list in scratch.
    const int g = lane;
    const bool live = g < nq_here;
    const uint32_t* mybits = qbits + static_cast<size_t>(g) * S;
    const uint16_t* mypre = qpre + static_cast<size_t>(g) * S;
    const float* myval = qval + static_cast<size_t>(g) * a.qcap;
    const size_t slot = ((static_cast<size_t>(group) * tiles + tile) * kWarps + warp) * kQG + lane;
    float* ls = a.heap_d + slot * a.k;
    int32_t* li = a.heap_l + slot * a.k;
    int n = 0;
    float thr = -FLT_MAX;  // meaningful once n == k

    uint16_t* sidx = reinterpret_cast<uint16_t*>(stage_base + static_cast<size_t>(warp) * kStageElems * 6);
    float* sval = reinterpret_cast<float*>(stage_base + static_cast<size_t>(warp) * kStageElems * 6 +
                                           kStageElems * 2);

    const int32_t tile_lo = tile * a.docs_per_tile;
    const int32_t tile_hi = min(a.fwd.n_docs, tile_lo + a.docs_per_tile);
    const int32_t per_warp = (tile_hi - tile_lo + kWarps - 1) / kWarps;
    const int32_t d_lo = tile_lo + warp * per_warp;
    const int32_t d_hi = min(tile_hi, d_lo + per_warp);
    const float* fval = static_cast<const float*>(a.fwd.val);
    unsigned long long bytes = 0;

    for (int32_t d = d_lo; d < d_hi; ++d) {
        const uint2 ri = __ldg(a.fwd.rowinfo + d);
        const int len = static_cast<int>(ri.y);
        const uint16_t* ip = a.fwd.idx + static_cast<size_t>(ri.x) * kRowAlign;
        const float* vp = fval + static_cast<size_t>(ri.x) * kRowAlign;
        bytes += 8ull + 6ull * static_cast<unsigned long long>(len);
        bool member = true;
        if (a.mode == 1 && a.sel_bits != nullptr)
            member = (__ldg(a.sel_bits + (d >> 6)) >> (d & 63)) & 1ull;
        float acc = 0.0f;
        for (int e0 = 0; e0 < len; e0 += kStageElems) {
            const int chunk = min(kStageElems, len - e0);
            // stage: each lane loads 8 elements (16 B of ids, 32 B of values)
            const int e = e0 + lane * 8;
            if (e < len) {
                const uint4 iv = __ldg(reinterpret_cast<const uint4*>(ip + e));
                const float4 va = __ldg(reinterpret_cast<const float4*>(vp + e));
                const float4 vb = __ldg(reinterpret_cast<const float4*>(vp + e + 4));
                *reinterpret_cast<uint4*>(sidx + lane * 8) = iv;
                *reinterpret_cast<float4*>(sval + lane * 8) = va;
                *reinterpret_cast<float4*>(sval + lane * 8 + 4) = vb;
            }
            __syncwarp();
            if (live && member) {
                for (int x = 0; x < chunk; ++x) {
                    const uint32_t t = sidx[x];
                    const uint32_t wbits = mybits[t >> 5];
                    const uint32_t bit = 1u << (t & 31);
                    if (wbits & bit) {
                        const int r = static_cast<int>(mypre[t >> 5]) + __popc(wbits & (bit - 1));
                        acc = __fadd_rn(acc, __fmul_rn(sval[x], myval[r]));
                    }
                }
            }
            __syncwarp();
        }
        if (!live || !member) continue;
        if (a.mode == 1 && !(acc > 0.0f)) continue;
        if (n == a.k && !(acc > thr)) continue;
        list_insert(ls, li, n, a.k, acc, d);
        if (n == a.k) thr = ls[a.k - 1];
    }
    // pad the unused tail so merges can treat every list as k long
    for (int i = n; i < a.k; ++i) {
        ls[i] = -FLT_MAX;
        li[i] = INT_MAX;
    }
    if (a.stats != nullptr) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(kFull, bytes, o);
        if (lane == 0) atomicAdd(a.stats + kStatBytes, bytes / 32);  // row bytes counted per lane
    }
    __syncthreads();

    // Merge the warps' lists for each query: thread g of warp 0.
    if (warp == 0 && live) {
        int head[kWarps];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) head[w] = 0;
        const size_t base_slot = ((static_cast<size_t>(group) * tiles + tile) * kWarps) * kQG;
        float* cd = a.cand_d + (static_cast<size_t>(q0 + g) * tiles + tile) * a.k;
        int32_t* cl = a.cand_l + (static_cast<size_t>(q0 + g) * tiles + tile) * a.k;
        for (int r = 0; r < a.k; ++r) {
            int bw = -1;
            float bs = -FLT_MAX;
            int32_t bi = INT_MAX;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                if (head[w] >= a.k) continue;
                const size_t sl = (base_slot + static_cast<size_t>(w) * kQG + g) * a.k + head[w];
                const float s = a.heap_d[sl];
                const int32_t i = a.heap_l[sl];
                if (i == INT_MAX) continue;
                if (bw < 0 || better(s, i, bs, bi)) {
                    bw = w;
                    bs = s;
                    bi = i;
                }
            }
            if (bw < 0) {
                cd[r] = -FLT_MAX;
                cl[r] = INT_MAX;
            } else {
                cd[r] = bs;
                cl[r] = bi;
                ++head[bw];
            }
        }
    }
}

// Merges each query's per-tile candidates (each sorted) into the final top-k,
// padded with (-1.0, -1) (brutal_index.cpp:93-95).
__global__ void __launch_bounds__(32) exact_merge_kernel(const float* cand_d, const int32_t* cand_l,
                                                         int tiles, int k, float* out_d,
                                                         int32_t* out_l) {
    extern __shared__ __align__(16) unsigned char smem[];
    int* head = reinterpret_cast<int*>(smem);
    const int q = blockIdx.x;
    const int lane = threadIdx.x;
    for (int t = lane; t < tiles; t += 32) head[t] = 0;
    __syncwarp();
    const float* cd = cand_d + static_cast<size_t>(q) * tiles * k;
    const int32_t* cl = cand_l + static_cast<size_t>(q) * tiles * k;
    for (int r = 0; r < k; ++r) {
        float bs = -FLT_MAX;
        int32_t bi = INT_MAX;
        int bt = -1;
        for (int t = lane; t < tiles; t += 32) {
            const int h = head[t];
            if (h >= k) continue;
            const float s = cd[static_cast<size_t>(t) * k + h];
            const int32_t i = cl[static_cast<size_t>(t) * k + h];
            if (i == INT_MAX) continue;
            if (bt < 0 || better(s, i, bs, bi)) {
                bs = s;
                bi = i;
                bt = t;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float s2 = __shfl_xor_sync(kFull, bs, o);
            const int32_t i2 = __shfl_xor_sync(kFull, bi, o);
            const int t2 = __shfl_xor_sync(kFull, bt, o);
            if (t2 >= 0 && (bt < 0 || better(s2, i2, bs, bi))) {
                bs = s2;
                bi = i2;
                bt = t2;
            }
        }
        if (lane == 0) {
            const size_t o = static_cast<size_t>(q) * k + r;
            if (bt < 0) {
                out_d[o] = -1.0f;
                out_l[o] = -1;
            } else {
                out_d[o] = bs;
                out_l[o] = bi;
                head[bt] += 1;
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------- term at a time --
// One CTA per (query, doc chunk): the chunk's scores live in shared memory,
// and the query's terms are applied one after another in ascending term order
// -- term t adds w * q_t to every doc of the chunk in t's postings, a barrier
// between terms. A doc's score thus receives its nonzero products in
// ascending term order, which for a row stored with strictly ascending terms
// is its row order: the reference's sequential sum (utils/distance.h:29-37)
// with the zero products of non-query terms left out, and adding +-0 to a sum
// that starts at +0 changes nothing. The host takes this path only for such
// rows. Work per query is the postings of its terms (~8% of the index on
// the reference corpus shape) instead of every row.
constexpr int kTWarps = 8;
constexpr int kTermWin = 256;  // query terms whose runs are located at once

__host__ __device__ inline size_t taat_smem_bytes(int chunk_docs, int k) {
    return static_cast<size_t>(chunk_docs) * 4 + static_cast<size_t>(kTermWin) * 12 +
           static_cast<size_t>(kTWarps) * k * 8;
}

__global__ void __launch_bounds__(kTWarps * 32) exact_taat_kernel(ExactLaunch a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const PostingsView& P = a.post;
    const int nq = a.q.n;
    const int c = static_cast<int>(blockIdx.x / static_cast<unsigned>(nq));  // chunk-major
    const int qi = static_cast<int>(blockIdx.x - static_cast<unsigned>(c) * nq);
    float* sc = reinterpret_cast<float*>(smem);
    int32_t* tlo = reinterpret_cast<int32_t*>(sc + P.chunk_docs);
    int32_t* thi = tlo + kTermWin;
    float* tqv = reinterpret_cast<float*>(thi + kTermWin);
    float* lsd = tqv + kTermWin;
    int32_t* lsi = reinterpret_cast<int32_t*>(lsd + kTWarps * a.k);

    const int32_t d0 = c * P.chunk_docs;
    const int nd = min(P.chunk_docs, a.fwd.n_docs - d0);
    for (int i = threadIdx.x; i < nd; i += blockDim.x) sc[i] = 0.0f;
    const int32_t qs = a.q.indptr[qi];
    const int qn = a.q.indptr[qi + 1] - qs;
    const uint16_t* qt = a.q.idx + qs;
    const float* qv = static_cast<const float*>(a.q.val) + qs;
    const int stride = P.n_chunks + 1;
    const int B = blockDim.x;
    unsigned long long postings = 0;
    for (int w0 = 0; w0 < qn; w0 += kTermWin) {
        const int wn = min(kTermWin, qn - w0);
        __syncthreads();  // zeroing, or the previous window's runs, done
        for (int i = threadIdx.x; i < wn; i += B) {
            const size_t row = static_cast<size_t>(qt[w0 + i]) * stride + c;
            tlo[i] = __ldg(P.chunk_at + row);
            thi[i] = __ldg(P.chunk_at + row + 1);
            tqv[i] = qv[w0 + i];
        }
        __syncthreads();
        for (int i = 0; i < wn; ++i) {
            const int32_t lo = tlo[i];
            const int32_t hi = thi[i];
            const float q = tqv[i];
            postings += static_cast<unsigned long long>(hi - lo);
            int32_t p = lo + static_cast<int32_t>(threadIdx.x);
            // four postings' loads in flight before their updates; a term's
            // docs are distinct, so the updates of one term never collide
            for (; p + 3 * B < hi; p += 4 * B) {
                int32_t d[4];
                float w[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    d[u] = __ldg(P.doc + p + u * B);
                    w[u] = __ldg(P.val + p + u * B);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    float* s = sc + (d[u] - d0);
                    *s = __fadd_rn(*s, __fmul_rn(w[u], q));
                }
            }
            for (; p < hi; p += B) {
                float* s = sc + (__ldg(P.doc + p) - d0);
                *s = __fadd_rn(*s, __fmul_rn(__ldg(P.val + p), q));
            }
            __syncthreads();
        }
    }
    __syncthreads();

    // Top-k of the chunk: warp w keeps a sorted list of its contiguous docs,
    // visited in ascending id order, so "reject score <= min" once full
    // resolves ties to the lower id (utils/ranker.h:147-200).
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int per = (nd + kTWarps - 1) / kTWarps;
    const int lo = warp * per;
    const int hi = min(nd, lo + per);
    float* ls = lsd + warp * a.k;
    int32_t* li = lsi + warp * a.k;
    int n = 0;
    float thr = -FLT_MAX;
    for (int b = lo; b < hi; b += 32) {
        const int i = b + lane;
        bool ok = i < hi;
        const float s = ok ? sc[i] : 0.0f;
        const int32_t d = d0 + i;
        if (ok && a.mode == 1) {
            if (!(s > 0.0f)) ok = false;
            if (a.sel_bits != nullptr && !((__ldg(a.sel_bits + (d >> 6)) >> (d & 63)) & 1ull))
                ok = false;
        }
        unsigned m = __ballot_sync(kFull, ok && (n < a.k || s > thr));
        while (m != 0u) {
            const int L = __ffs(m) - 1;
            m &= m - 1u;
            const float sL = __shfl_sync(kFull, s, L);
            if (n == a.k && !(sL > thr)) continue;  // the list moved on
            if (lane == 0) {
                int nn = n;
                list_insert(ls, li, nn, a.k, sL, d0 + b + L);
            }
            if (n < a.k) ++n;
            __syncwarp();
            if (n == a.k) thr = ls[a.k - 1];
        }
    }
    for (int i = n + lane; i < a.k; i += 32) {
        ls[i] = -FLT_MAX;
        li[i] = INT_MAX;
    }
    if (a.stats != nullptr && threadIdx.x == 0)
        atomicAdd(a.stats + kStatBytes, postings * 8ull + static_cast<unsigned long long>(qn) * 8ull);
    __syncthreads();

    // Merge the warps' lists into the chunk's candidates: lane w < kTWarps
    // holds list w's head; lane 0's choice is the warp's.
    if (warp == 0) {
        int head = 0;
        float* cd = a.cand_d + (static_cast<size_t>(qi) * P.n_chunks + c) * a.k;
        int32_t* cl = a.cand_l + (static_cast<size_t>(qi) * P.n_chunks + c) * a.k;
        for (int r = 0; r < a.k; ++r) {
            float bs = -FLT_MAX;
            int32_t bi = INT_MAX;
            int bl = -1;
            if (lane < kTWarps && head < a.k) {
                const int32_t id = lsi[lane * a.k + head];
                if (id != INT_MAX) {
                    bs = lsd[lane * a.k + head];
                    bi = id;
                    bl = lane;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float s2 = __shfl_xor_sync(kFull, bs, o);
                const int32_t i2 = __shfl_xor_sync(kFull, bi, o);
                const int l2 = __shfl_xor_sync(kFull, bl, o);
                if (l2 >= 0 && (bl < 0 || better(s2, i2, bs, bi))) {
                    bs = s2;
                    bi = i2;
                    bl = l2;
                }
            }
            bl = __shfl_sync(kFull, bl, 0);
            bs = __shfl_sync(kFull, bs, 0);
            bi = __shfl_sync(kFull, bi, 0);
            if (lane == 0) {
                cd[r] = bl < 0 ? -FLT_MAX : bs;
                cl[r] = bl < 0 ? INT_MAX : bi;
            }
            if (lane == bl) ++head;
        }
    }
}

}  // namespace

size_t exact_smem(int dim_words, int qcap_smem) { return exact_smem_bytes(dim_words, qcap_smem); }

int exact_taat_chunk_docs() {
    int dev = 0;
    int per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
            cudaSuccess)
        per_sm = 228 * 1024;
    // four CTAs per SM (1 KB of each CTA's share is reserved by the device)
    const long long room = per_sm / 4 - 1024 - static_cast<long long>(taat_smem_bytes(0, kTaatMaxK));
    const long long docs = (room / 4) & ~255ll;
    return static_cast<int>(docs < 1024 ? 1024 : docs);
}

cudaError_t launch_exact_taat(const ExactLaunch& a, cudaStream_t s) {
    if (a.q.n == 0) return cudaSuccess;
    if (a.k > kTaatMaxK) return cudaErrorInvalidValue;
    const size_t smem = taat_smem_bytes(a.post.chunk_docs, a.k);
    cudaError_t e = allow_opt_in_smem(exact_taat_kernel);
    if (e != cudaSuccess) return e;
    const long long grid = static_cast<long long>(a.post.n_chunks) * a.q.n;
    if (grid > 0x7fffffffll) return cudaErrorInvalidValue;
    exact_taat_kernel<<<static_cast<unsigned>(grid), kTWarps * 32, smem, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    exact_merge_kernel<<<a.q.n, 32, static_cast<size_t>(a.post.n_chunks) * sizeof(int), s>>>(
        a.cand_d, a.cand_l, a.post.n_chunks, a.k, a.out_d, a.out_l);
    return cudaGetLastError();
}

cudaError_t launch_exact(const ExactLaunch& a, int tiles, cudaStream_t s) {
    if (a.q.n == 0) return cudaSuccess;
    const int words = (a.fwd.dim + 31) / 32;
    const size_t smem = exact_smem_bytes(words, a.qval_global != nullptr ? 0 : a.qcap);
    cudaError_t e = allow_opt_in_smem(exact_tile_kernel);
    if (e != cudaSuccess) return e;
    const int groups = (a.q.n + kQG - 1) / kQG;
    exact_tile_kernel<<<dim3(tiles, groups), kWarps * 32, smem, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    exact_merge_kernel<<<a.q.n, 32, static_cast<size_t>(tiles) * sizeof(int), s>>>(
        a.cand_d, a.cand_l, tiles, a.k, a.out_d, a.out_l);
    return cudaGetLastError();
}

}  // namespace nsp
