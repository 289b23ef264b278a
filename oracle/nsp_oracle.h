/*
 * TEST INFRASTRUCTURE -- the checker, never the product.
 *
 * Plain-C restatement of the reference's search hot path
 * (opensearch-project/neural-sparse-cpp). Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it. Each function names the reference
 * file:line it restates. Where the reference's order of equal values comes
 * from its std::priority_queue (TopKHolder, utils/ranker.h) and its unstable
 * std::ranges::sort, SEISMIC search follows the C++ library's own steps for
 * them, as the device kernels do:
 *   - the query cut: a TopKHolder of size cut over (value, term) in query
 *     order, popped into top_k_descending order; the query's own order when
 *     cut >= nnz (utils/vector_process.h:18-30);
 *   - the first list's blocks: std::ranges::sort by summary score descending
 *     (seismic_common.h:105-115), the library's introsort;
 *   - the results: a TopKHolder (rejects score <= its top; pops, then pushes)
 *     drained by top_k_items_descending (seismic_index.cpp:263-273).
 * Exact search (BrutalIndex, InvertedIndex) fixes one total order instead:
 * score descending, then doc id ascending; a full top-k rejects a score <= its
 * minimum and evicts its worst entry (lowest score, then highest id).
 * Pinned by tests/test_oracle.py against the reference library compiled from
 * its sources (oracle/_ref) and against fixtures under tests/golden/.
 */
#ifndef NSP_ORACLE_H
#define NSP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Exact top-k over all docs. mode 0 = BrutalIndex (every doc eligible, zero
 * scores included: brutal_index.cpp:75-96); mode 1 = InvertedIndex (positive
 * scores only, selector honoured: inverted_index.cpp:152-212). `sel_bits` is a
 * doc bitmap (bit d set = member) or NULL. Scores are sequential fp32 sums in
 * the doc's stored term order (utils/distance.h:29-37). */
int nspo_exact_search(int dim, int32_t n_docs, const int32_t* d_indptr,
                      const uint16_t* d_indices, const float* d_values,
                      int32_t n_q, const int32_t* q_indptr,
                      const uint16_t* q_indices, const float* q_values, int k,
                      int mode, const uint64_t* sel_bits, float* out_d,
                      int32_t* out_l);

/* SEISMIC search (seismic_index.cpp:53-274; SQ variant
 * seismic_scalar_quantized_index.cpp:67-357) over a flattened index:
 *   list l owns blocks [list_block_ptr[l], list_block_ptr[l+1]);
 *   block b owns docs[block_doc_ptr[b] .. block_doc_ptr[b+1]);
 *   list l's summary terms are sum_terms[list_term_ptr[l] .. list_term_ptr[l+1])
 *   (ascending); term j's (block, value) run is
 *   sum_block/sum_val[sum_run_ptr[j] .. sum_run_ptr[j+1]) with block ids local
 *   to the list.
 * esz = 4: fp32 values/summaries/query; esz = 1: uint8 codes throughout (the
 * query codes are passed in q_codes), scores are int sums cast to float and the
 * caller decodes; esz = 2: uint16 codes, int64 doc sums cast to float
 * (utils/distance.h:49-57), summary products and sums in float as for every
 * code width (inverted_list_clusters.cpp:295-315). `sel_bits` as above. */
int nspo_seismic_search(int dim, int esz, int32_t n_docs, const int32_t* d_indptr,
                        const uint16_t* d_indices, const void* d_values,
                        int32_t n_lists, const int64_t* list_block_ptr,
                        const int64_t* block_doc_ptr, const int32_t* docs,
                        const int64_t* list_term_ptr, const uint16_t* sum_terms,
                        const int64_t* sum_run_ptr, const uint16_t* sum_block,
                        const void* sum_val, int32_t n_q, const int32_t* q_indptr,
                        const uint16_t* q_indices, const void* q_values, int k,
                        int cut, float heap_factor, const uint64_t* sel_bits,
                        float* out_d, int32_t* out_l, int64_t* stats);

/* ScalarQuantizer::encode_8bit/16bit (utils/scalar_quantizer.h:97-118). */
void nspo_sq_encode_u8(float vmin, float vmax, const float* vals, uint8_t* codes,
                       int64_t n);
void nspo_sq_encode_u16(float vmin, float vmax, const float* vals, uint16_t* codes,
                        int64_t n);
/* ScalarQuantizer::decode_dot_product scale (utils/scalar_quantizer.h:85-93). */
float nspo_sq_scale(int qbits, float vmin, float vmax, float qvmin, float qvmax);

/* Query cut (utils/vector_process.h:18-30) with the tie order above. esz 4, 2 or 1. */
int nspo_cut(const uint16_t* idx, const void* vals, int esz, int len, int cut,
             uint16_t* out);

#ifdef __cplusplus
}
#endif
#endif
