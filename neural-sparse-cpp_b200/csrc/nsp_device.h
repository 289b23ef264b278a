// Device-side data layouts and kernel launchers of the B200 sparse-retrieval
// engine. Everything here is internal to libnsparse_b200.so; the public
// surface is include/nsparse_c.h (C ABI) and include/nsparse/*.h (C++ API).
//
// HBM layouts
// -----------
// Forward index (the reference's SparseVectors CSR, sparse_vectors.h:36-111)
//   rowinfo[d] = {start / 64, length}: row d's elements begin at element
//   64*rowinfo[d].x of `idx` (uint16 term ids) and `val` (float32, uint8 or
//   uint16 codes). Every row starts on a 64-element boundary and is padded to
//   a multiple of 64 elements, so a row is read with aligned vector loads of
//   16 elements (ids 32 bytes, values 16-64 bytes) and a lane never reads
//   past its row's padding. 64 elements put every row's ids on a 128-byte
//   and its uint8 codes on a 64-byte boundary: a random row then costs DRAM
//   no partly used 64-byte access at its start (measured on the SEISMIC-SQ
//   search at 3M docs: DRAM reads 1.20x -> 1.10x the bytes the kernel uses).
//
// SEISMIC index (the reference's InvertedListClusters per term,
// cluster/inverted_list_clusters.h:75-84), flattened over the lists:
//   list t owns blocks [lbp[t], lbp[t+1]); block b owns docs[bdp[b]..bdp[b+1]).
//   Summaries are term-major (CSC) per list: summary column c of list t is the
//   term whose bit is set in the list's term bitmap `lmeta`; its (block, value)
//   run is sblk/sval[srun[ltp[t]+c] .. srun[ltp[t]+c+1]).
//   lmeta[t*W + w] = {bits of terms 32w..32w+31 present in list t's summaries,
//   number of present terms below 32w}. A query term is located in a list with
//   one 8-byte load and a popcount, instead of the reference's binary search
//   over term_ids (inverted_list_clusters.cpp:302-304).
#ifndef NSP_DEVICE_H
#define NSP_DEVICE_H

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace nsp {

constexpr int kRowAlign = 64;  // elements

enum ValKind : int { kF32 = 4, kU8 = 1, kU16 = 2 };

struct FwdView {
    int32_t n_docs;
    int32_t dim;
    const uint2* rowinfo;
    const uint16_t* idx;
    const void* val;
};

struct SeismicView {
    int32_t n_lists;
    int32_t words;          // ceil(dim / 32)
    int32_t max_blocks;     // max blocks in one list
    const int64_t* lbp;     // [n_lists + 1]
    const int64_t* bdp;     // [n_blocks + 1]
    const int32_t* docs;    // [n_list_docs]
    const uint2* drow;      // [n_list_docs] forward rowinfo of each posting, or nullptr
    const uint2* lmeta;     // [n_lists * words]
    const int64_t* ltp;     // [n_lists + 1], column base per list
    const int64_t* srun;    // [n_columns + 1]
    const uint16_t* sblk;   // [n_entries]
    const void* sval;       // [n_entries], float32 / uint8 / uint16
};

// A query batch in canonical form: each row's terms ascending and unique.
struct QueryView {
    int32_t n;
    const int32_t* indptr;
    const uint16_t* idx;
    const void* val;        // same element type as the index values
};

// Counters the search kernels accumulate (unsigned long long each).
// kStatBytes counts every byte a kernel reads, rows included as often as they
// are scored; kStatRowBytes is the rows' share of it. A doc met again in a
// later list is scored again (the reference skips it with its visited set,
// seismic_index.cpp:104-107), so the reference's algorithmic bytes are
// kStatBytes - kStatRowBytes + kStatUniqueRowBytes, the last counted only by
// a launch with `visit` stamps (SeismicLaunch).
enum StatSlot : int {
    kStatDocsScored = 0,
    kStatBlocksVisited = 1,
    kStatBytes = 2,
    kStatListsProbed = 3,
    kStatRowBytes = 4,
    kStatUniqueDocs = 5,
    kStatUniqueRowBytes = 6,
    kStatCount = 7,
};

// One-warp kernels (variants 0-1): floats per warp of `bscore` -- the
// current list's block scores, then the first list's (score, block) pairs
// sorted into the reference's visiting order (8 bytes each).
__host__ __device__ inline size_t one_warp_slot(int max_blocks) {
    return 3 * static_cast<size_t>((max_blocks + 1) & ~1);
}

struct SeismicLaunch {
    FwdView fwd;
    SeismicView ix;
    QueryView q;
    int k;
    int cut;
    float heap_factor;
    float decode_scale;         // SQ: quantized score -> float (0 = none)
    const uint64_t* sel_bits;   // doc bitmap or nullptr
    float* out_d;
    int32_t* out_l;
    int32_t qcap;               // max query nnz in the batch
    int32_t* work_counter;      // work stealing over queries, or nullptr
    float* bscore;              // scratch: per warp slot (one_warp_slot floats for
                                // variants 0-1; wpb * max_blocks per CTA otherwise)
    unsigned long long* stats;  // kStatCount counters, or nullptr
    int32_t first_query;        // static mode: queries first_query.. strided
    // Variant 1 (staged): doc rows arrive in shared memory by bulk copy,
    // double-buffered, stage_bytes per buffer; block scores of lists with at
    // most bcap blocks stay in shared memory. Variant 0 loads rows directly.
    int32_t variant;
    int32_t stage_bytes;
    int32_t bcap;
    int32_t* err;               // nonzero: a kernel-side error (see check_kernel_error)
    // variants 2-5, batched, or nullptr: the order queries are claimed in
    // (longest rows first, so the launch does not end on a long query
    // claimed last); results do not depend on it
    const int32_t* qorder;
    // variants 2-5, or nullptr: done[q] is set to 1 once query q's results are
    // written (system scope: the host may read both from mapped memory)
    int32_t* done;
    // Variants 2-5 (one CTA per query): candidate docs per batch, lanes per
    // scored doc (1, 2, 4, 8), and per-CTA scratch -- `bscore` holds warps *
    // max_blocks floats per CTA, `order` the first list's visiting order,
    // `sortkeys` the sort buffer of lists too long to sort in shared memory
    // (nullptr when none is).
    int32_t batch_docs;
    int32_t group_lanes;
    const uint64_t* const* sel_q;  // per-query doc bitmaps (null entry: none), or nullptr
    uint16_t* order;
    int32_t order_stride;
    unsigned long long* sortkeys;
    int32_t sort_stride;
    // Block segments a batch may hold, and CTAs per query: with cluster > 1
    // each query runs on a thread-block cluster of that many CTAs, rank 0
    // walking the query and every CTA scoring its batches.
    int32_t seg_cap;
    int32_t cluster;
    // Entries the query arrays hold (negative: not checked). A row that ends
    // past it is treated as empty and reported through `err`, like a row
    // longer than qcap.
    int32_t nnz_cap;
    // Counting pass only (variants 2-5), else nullptr: per CTA, one stamp per
    // doc (n_docs of them); the walk stamps each doc of a visited block with
    // the CTA's query number and counts a member doc's row the first time
    // (kStatUniqueDocs / kStatUniqueRowBytes). Zero on entry.
    uint32_t* visit;
};

// Doc-ascending postings of an fp32 forward index (the exact search's
// term-at-a-time path): term t's postings are doc/val[chunk_at[t * (n_chunks
// + 1)] .. chunk_at[t * (n_chunks + 1) + n_chunks]), docs ascending, and
// chunk_at[t * (n_chunks + 1) + c] is the first of them with doc >= c *
// chunk_docs, so a CTA scoring doc chunk c finds each query term's run with
// two loads.
struct PostingsView {
    int32_t n_chunks;
    int32_t chunk_docs;
    const int32_t* doc;
    const float* val;
    const int32_t* chunk_at;    // [dim][n_chunks + 1]
};

struct ExactLaunch {
    FwdView fwd;
    PostingsView post;          // term-at-a-time path (launch_exact_taat)
    QueryView q;
    int k;
    int mode;                   // 0 brutal (all docs), 1 inverted (score > 0)
    const uint64_t* sel_bits;   // honoured in mode 1
    int32_t qcap;
    float* qval_global;         // query values in global scratch, or nullptr
    int32_t docs_per_tile;
    float* cand_d;              // scratch [n_q][tiles][k]
    int32_t* cand_l;
    float* heap_d;              // scratch per (tile, group, warp, lane) k
    int32_t* heap_l;
    float* out_d;
    int32_t* out_l;
    unsigned long long* stats;
};

// Lets kernel `f` use the device's whole opt-in shared memory (less its own
// static shared memory, which counts against the same limit). Every call sets
// the same value, so launches from several host threads cannot undo one
// another's setting, as a per-launch size could between a set and a launch.
template <class F>
inline cudaError_t allow_opt_in_smem(F f) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int v = 0;
    e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa{};
    e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return e;
    const int dyn = v - static_cast<int>(fa.sharedSizeBytes);
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn > 0 ? dyn : 0);
}

// Launchers (return cudaError_t of the launch). `sm_count` sizes persistent
// grids; `plan_*` report the dynamic shared memory a launch needs.
size_t seismic_smem_per_warp(int val_kind, int dim_words, int qcap, int k, int bcap = 0,
                             int stage_bytes = 0);
cudaError_t launch_seismic(int val_kind, const SeismicLaunch& a, int warps_per_block,
                           int blocks, cudaStream_t s);
int seismic_max_blocks_per_sm(int val_kind, int variant, int warps_per_block, size_t smem);
int seismic_max_blocks_per_sm(int val_kind, int warps_per_block, size_t smem);  // variant 0

// Variants 2-5: one CTA of `warps` warps per query (search_seismic_cta.cu).
size_t seismic_cta_smem(int val_kind, int dim, int qcap, int k, int batch_docs, int seg_cap);
// Block segments per batch the kernel is laid out for (more with a cluster).
int seismic_cta_seg_cap(int cluster);
int seismic_cta_max_blocks_per_sm(int val_kind, int qcap, int group_lanes, int warps,
                                  size_t smem);
cudaError_t launch_seismic_cta(int val_kind, const SeismicLaunch& a, int warps, int blocks,
                               cudaStream_t s);

size_t exact_smem(int dim_words, int qcap_smem);  // qcap_smem 0: values in global
cudaError_t launch_exact(const ExactLaunch& a, int tiles, cudaStream_t s);

// Term-at-a-time exact search (search_exact_taat.cu): one CTA per (query, doc
// chunk of a.post), k <= kTaatMaxK; candidates per chunk in a.cand_d/l
// [n_q][n_chunks][k], then the tile path's merge.
constexpr int kTaatMaxK = 128;
int exact_taat_chunk_docs();  // docs per chunk that keep 4 CTAs per SM
cudaError_t launch_exact_taat(const ExactLaunch& a, cudaStream_t s);

// Exact scoring of an explicit doc list per query (the reference's
// ExactMatcher, exact_matcher.h:23-58): ids ascending, at most k of them.
cudaError_t launch_exact_list(int val_kind, const FwdView& fwd, const QueryView& q,
                              const int32_t* ids, int n_ids, int k, float decode_scale,
                              int32_t qcap, float* out_d, int32_t* out_l,
                              cudaStream_t s);

// The claim order of a batched launch's queries: row lengths descending
// (one CTA; any order among equal lengths).
cudaError_t launch_order_by_length(const int32_t* indptr, int32_t n, int32_t* order,
                                   cudaStream_t s);

// ScalarQuantizer::encode (utils/scalar_quantizer.h:97-118) on the device.
cudaError_t launch_sq_encode(const float* vals, void* codes, int64_t n, int qbits,
                             float vmin, float inv_range_scaled, cudaStream_t s);

}  // namespace nsp

#endif  // NSP_DEVICE_H
