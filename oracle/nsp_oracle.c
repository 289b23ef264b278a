/*
 * TEST INFRASTRUCTURE -- the checker, never the product. See nsp_oracle.h for
 * the contract and the tie order it fixes. Built by oracle/Makefile with
 * -ffp-contract=off so every float product and sum rounds separately, as the
 * reference's generic build does.
 */
#include "nsp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- bounded top-k: utils/ranker.h:34-138 (TopKHolder::add) ------------- */

typedef struct {
    float s;
    int32_t id;
} item_t;

typedef struct {
    item_t* a; /* sorted: score desc, id asc */
    int n, k;
} topk_t;

static inline int better(float s1, int32_t i1, float s2, int32_t i2) {
    return s1 > s2 || (s1 == s2 && i1 < i2);
}

/* Full heap rejects score <= min (ranker.h:58-60); otherwise the worst entry
 * (lowest score, highest id) is replaced (ranker.h:67-71). */
static void topk_add(topk_t* h, float s, int32_t id) {
    if (h->n == h->k && s <= h->a[h->n - 1].s) return;
    int pos = h->n == h->k ? h->k - 1 : h->n;
    if (h->n < h->k) h->n++;
    while (pos > 0 && better(s, id, h->a[pos - 1].s, h->a[pos - 1].id)) {
        h->a[pos] = h->a[pos - 1];
        --pos;
    }
    h->a[pos].s = s;
    h->a[pos].id = id;
}

static int topk_contains(const topk_t* h, int32_t id) {
    for (int i = 0; i < h->n; ++i)
        if (h->a[i].id == id) return 1;
    return 0;
}

/* Pads with (-1.0, -1): brutal_index.cpp:93-95, seismic_index.cpp:270-273. */
static void topk_emit(const topk_t* h, float* d, int32_t* l) {
    for (int i = 0; i < h->k; ++i) {
        if (i < h->n) {
            d[i] = h->a[i].s;
            l[i] = h->a[i].id;
        } else {
            d[i] = -1.0f;
            l[i] = -1;
        }
    }
}

/* ---- the reference's TopKHolder for SEISMIC: utils/ranker.h:34-138 -------
 * A std::priority_queue with std::greater on the score: a binary heap with the
 * smallest score at a[0]. The sift steps are the C++ library's push_heap /
 * pop_heap (bits/stl_heap.h: __push_heap, __adjust_heap), which decide which
 * of several equal scores is dropped and in which order equal scores leave. */

typedef struct {
    item_t* a; /* binary heap, smallest score on top */
    int n, k;
} rheap_t;

static void rh_sift_up(item_t* a, int hole, item_t v) {
    int parent = (hole - 1) / 2;
    while (hole > 0 && a[parent].s > v.s) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

static void rh_sift_down(item_t* a, int len, item_t v) {
    int hole = 0, child = 0;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (a[child].s > a[child - 1].s) --child;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    rh_sift_up(a, hole, v);
}

static void rh_pop(rheap_t* h) {
    if (h->n > 1) {
        item_t v = h->a[h->n - 1];
        h->a[h->n - 1] = h->a[0];
        rh_sift_down(h->a, h->n - 1, v);
    }
    h->n--;
}

/* TopKHolder::add (ranker.h:58-72) */
static void rh_add(rheap_t* h, float s, int32_t id) {
    item_t v;
    if (h->n >= h->k && s <= h->a[0].s) return;
    if (h->n >= h->k) rh_pop(h);
    v.s = s;
    v.id = id;
    rh_sift_up(h->a, h->n, v);
    h->n++;
}

/* top_k_items_descending (ranker.h:113-127), padded with (-1.0, -1)
 * (seismic_index.cpp:270-273); empties the heap. */
static void rh_emit(rheap_t* h, float* d, int32_t* l) {
    const int n = h->n;
    for (int i = n - 1; i >= 0; --i) {
        d[i] = h->a[0].s;
        l[i] = h->a[0].id;
        rh_pop(h);
    }
    for (int i = n; i < h->k; ++i) {
        d[i] = -1.0f;
        l[i] = -1;
    }
}

static inline int sel_member(const uint64_t* bits, int32_t d) {
    return bits == NULL || ((bits[d >> 6] >> (d & 63)) & 1u);
}

/* ---- exact search ------------------------------------------------------- */

int nspo_exact_search(int dim, int32_t n_docs, const int32_t* d_indptr,
                      const uint16_t* d_indices, const float* d_values,
                      int32_t n_q, const int32_t* q_indptr,
                      const uint16_t* q_indices, const float* q_values, int k,
                      int mode, const uint64_t* sel_bits, float* out_d,
                      int32_t* out_l) {
    if (k <= 0 || dim <= 0) return -1;
    int err = 0;
#pragma omp parallel
    {
        float* dense = (float*)calloc((size_t)dim, sizeof(float));
        item_t* buf = (item_t*)malloc(sizeof(item_t) * (size_t)k);
        if (!dense || !buf) err = 1;
#pragma omp for schedule(dynamic, 4)
        for (int32_t q = 0; q < n_q; ++q) {
            if (!dense || !buf) continue;
            /* get_dense_vector_float: later duplicates overwrite earlier
             * (sparse_vectors.cpp:157-177). */
            for (int32_t j = q_indptr[q]; j < q_indptr[q + 1]; ++j)
                dense[q_indices[j]] = q_values[j];
            topk_t h = {buf, 0, k};
            for (int32_t d = 0; d < n_docs; ++d) {
                float s = 0.0f;
                for (int32_t j = d_indptr[d]; j < d_indptr[d + 1]; ++j) {
                    float p = d_values[j] * dense[d_indices[j]];
                    s = s + p;
                }
                if (mode == 0) {
                    topk_add(&h, s, d);
                } else {
                    if (!(s > 0.0f)) continue;
                    if (!sel_member(sel_bits, d)) continue;
                    topk_add(&h, s, d);
                }
            }
            topk_emit(&h, out_d + (int64_t)q * k, out_l + (int64_t)q * k);
            for (int32_t j = q_indptr[q]; j < q_indptr[q + 1]; ++j)
                dense[q_indices[j]] = 0.0f;
        }
        free(dense);
        free(buf);
    }
    return err ? -1 : 0;
}

/* ---- scalar quantizer: utils/scalar_quantizer.h:85-118 ------------------- */

void nspo_sq_encode_u8(float vmin, float vmax, const float* vals, uint8_t* codes,
                       int64_t n) {
    const float kmax = 255.0f;
    const float range = vmax - vmin;
    const float inv = kmax / range;
    for (int64_t i = 0; i < n; ++i) {
        float scaled = (vals[i] - vmin) * inv;
        /* std::min(kMax, scaled) then std::max(0, .): NaN maps to kMax. */
        float lo = (scaled < kmax) ? scaled : kmax;
        float c = (0.0f < lo) ? lo : 0.0f;
        codes[i] = (uint8_t)lroundf(c);
    }
}

/* encode_16bit: the same clamp and lround against 65535 (scalar_quantizer.h:108-113). */
void nspo_sq_encode_u16(float vmin, float vmax, const float* vals, uint16_t* codes,
                        int64_t n) {
    const float kmax = 65535.0f;
    const float range = vmax - vmin;
    const float inv = kmax / range;
    for (int64_t i = 0; i < n; ++i) {
        float scaled = (vals[i] - vmin) * inv;
        float lo = (scaled < kmax) ? scaled : kmax;
        float c = (0.0f < lo) ? lo : 0.0f;
        codes[i] = (uint16_t)lroundf(c);
    }
}

float nspo_sq_scale(int qbits, float vmin, float vmax, float qvmin, float qvmax) {
    const float in_range = vmax - vmin;
    const float q_range = qvmax - qvmin;
    const float m = qbits == 16 ? 65535.0f : 255.0f;
    return (in_range * q_range) / (m * m);
}

/* ---- query cut: utils/vector_process.h:18-30 ---------------------------- */

static inline float val_at(const void* v, int esz, int64_t i) {
    if (esz == 4) return ((const float*)v)[i];
    if (esz == 2) return (float)((const uint16_t*)v)[i];
    return (float)((const uint8_t*)v)[i];
}

int nspo_cut(const uint16_t* idx, const void* vals, int esz, int len, int cut,
             uint16_t* out) {
    if (cut >= len) {
        for (int i = 0; i < len; ++i) out[i] = idx[i];
        return len;
    }
    /* a TopKHolder of size cut offered (value, term) in query order, then
     * top_k_descending: the heap's pops fill the result from its end */
    {
        item_t* hp = (item_t*)malloc(sizeof(item_t) * (size_t)cut);
        rheap_t h;
        if (!hp) return -1;
        h.a = hp;
        h.n = 0;
        h.k = cut;
        for (int i = 0; i < len; ++i) rh_add(&h, val_at(vals, esz, i), (int32_t)idx[i]);
        for (int i = h.n - 1; i >= 0; --i) {
            out[i] = (uint16_t)h.a[0].id;
            rh_pop(&h);
        }
        free(hp);
    }
    return cut;
}

/* ---- SEISMIC search ----------------------------------------------------- */

static int find_term(const uint16_t* terms, int64_t n, uint16_t t) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (terms[mid] < t) lo = mid + 1; else hi = mid;
    }
    return (lo < n && terms[lo] == t) ? (int)lo : -1;
}

typedef struct {
    float s;
    int32_t b;
} blk_t;

/* reorder_clusters (seismic_common.h:105-115): std::ranges::sort of the block
 * indices by score descending -- the C++ library's introsort
 * (bits/stl_algo.h: __introsort_loop, __unguarded_partition_pivot,
 * __final_insertion_sort; heap sort past the depth budget), whose steps
 * decide where equal scores land. */
static int blk_before(blk_t x, blk_t y) { return x.s > y.s; }

static void blk_swap(blk_t* a, int64_t i, int64_t j) {
    blk_t t = a[i];
    a[i] = a[j];
    a[j] = t;
}

static void blk_heap_up(blk_t* a, int64_t hole, int64_t top, blk_t v) {
    int64_t parent = (hole - 1) / 2;
    while (hole > top && blk_before(a[parent], v)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

static void blk_heap_adjust(blk_t* a, int64_t hole, int64_t len, blk_t v) {
    const int64_t top = hole;
    int64_t child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (blk_before(a[child], a[child - 1])) child--;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    blk_heap_up(a, hole, top, v);
}

static void blk_heap_sort(blk_t* a, int64_t len) {
    if (len < 2) return;
    for (int64_t parent = (len - 2) / 2;; parent--) {
        blk_heap_adjust(a, parent, len, a[parent]);
        if (parent == 0) break;
    }
    while (len > 1) {
        blk_t v;
        len--;
        v = a[len];
        a[len] = a[0];
        blk_heap_adjust(a, 0, len, v);
    }
}

static void blk_introsort(blk_t* a, int64_t f, int64_t l, int depth) {
    while (l - f > 16) {
        int64_t mid, lo, hi;
        blk_t piv;
        if (depth == 0) {
            blk_heap_sort(a + f, l - f);
            return;
        }
        depth--;
        /* median of a[f+1], a[mid], a[l-1] to the front */
        mid = f + (l - f) / 2;
        if (blk_before(a[f + 1], a[mid])) {
            if (blk_before(a[mid], a[l - 1])) blk_swap(a, f, mid);
            else if (blk_before(a[f + 1], a[l - 1])) blk_swap(a, f, l - 1);
            else blk_swap(a, f, f + 1);
        } else if (blk_before(a[f + 1], a[l - 1])) {
            blk_swap(a, f, f + 1);
        } else if (blk_before(a[mid], a[l - 1])) {
            blk_swap(a, f, l - 1);
        } else {
            blk_swap(a, f, mid);
        }
        piv = a[f];
        lo = f + 1;
        hi = l;
        for (;;) {
            while (blk_before(a[lo], piv)) lo++;
            hi--;
            while (blk_before(piv, a[hi])) hi--;
            if (!(lo < hi)) break;
            blk_swap(a, lo, hi);
            lo++;
        }
        blk_introsort(a, lo, l, depth);
        l = lo;
    }
}

static void blk_linear_insert(blk_t* a, int64_t i) {
    blk_t v = a[i];
    while (blk_before(v, a[i - 1])) {
        a[i] = a[i - 1];
        i--;
    }
    a[i] = v;
}

static void blk_insertion(blk_t* a, int64_t f, int64_t l) {
    for (int64_t i = f + 1; i < l; ++i) {
        if (blk_before(a[i], a[f])) {
            blk_t v = a[i];
            memmove(a + f + 1, a + f, (size_t)(i - f) * sizeof(blk_t));
            a[f] = v;
        } else {
            blk_linear_insert(a, i);
        }
    }
}

static void blk_sort_like_reference(blk_t* a, int64_t n) {
    int lg = 0;
    if (n <= 0) return;
    while ((n >> (lg + 1)) > 0) lg++;
    blk_introsort(a, 0, n, 2 * lg);
    if (n > 16) {
        blk_insertion(a, 0, 16);
        for (int64_t i = 16; i < n; ++i) blk_linear_insert(a, i);
    } else {
        blk_insertion(a, 0, n);
    }
}

int nspo_seismic_search(int dim, int esz, int32_t n_docs, const int32_t* d_indptr,
                        const uint16_t* d_indices, const void* d_values,
                        int32_t n_lists, const int64_t* list_block_ptr,
                        const int64_t* block_doc_ptr, const int32_t* docs,
                        const int64_t* list_term_ptr, const uint16_t* sum_terms,
                        const int64_t* sum_run_ptr, const uint16_t* sum_block,
                        const void* sum_val, int32_t n_q, const int32_t* q_indptr,
                        const uint16_t* q_indices, const void* q_values, int k,
                        int cut, float heap_factor, const uint64_t* sel_bits,
                        float* out_d, int32_t* out_l, int64_t* stats) {
    if (k <= 0 || cut <= 0 || dim <= 0 || (esz != 4 && esz != 2 && esz != 1)) return -1;
    int64_t max_blocks = 0;
    for (int32_t l = 0; l < n_lists; ++l) {
        int64_t nb = list_block_ptr[l + 1] - list_block_ptr[l];
        if (nb > max_blocks) max_blocks = nb;
    }
    int err = 0;
#pragma omp parallel
    {
        float* dense = (float*)calloc((size_t)dim, sizeof(float));
        uint8_t* dense8 = (uint8_t*)calloc((size_t)dim, 1);
        uint16_t* dense16 = (uint16_t*)calloc((size_t)dim, 2);
        uint64_t* visited = (uint64_t*)calloc(((size_t)n_docs + 64) / 64, 8);
        blk_t* blocks = (blk_t*)malloc(sizeof(blk_t) * (size_t)(max_blocks + 1));
        item_t* buf = (item_t*)malloc(sizeof(item_t) * (size_t)k);
        uint16_t* cuts = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)(dim + 1));
        if (!dense || !dense8 || !dense16 || !visited || !blocks || !buf || !cuts) err = 1;
#pragma omp for schedule(dynamic, 4)
        for (int32_t q = 0; q < n_q; ++q) {
            if (err) continue;
            const int32_t qs = q_indptr[q];
            const int qlen = q_indptr[q + 1] - qs;
            const uint16_t* qi = q_indices + qs;
            const float* qf = esz == 4 ? (const float*)q_values + qs : NULL;
            const uint8_t* q8 = esz == 1 ? (const uint8_t*)q_values + qs : NULL;
            const uint16_t* q16 = esz == 2 ? (const uint16_t*)q_values + qs : NULL;
            const void* qany = esz == 4 ? (const void*)qf
                                        : (esz == 2 ? (const void*)q16 : (const void*)q8);
            /* seismic_index.cpp:244-246: scatter all query terms */
            for (int i = 0; i < qlen; ++i) {
                if (esz == 4) dense[qi[i]] = qf[i];
                else if (esz == 2) dense16[qi[i]] = q16[i];
                else dense8[qi[i]] = q8[i];
            }
            int ncut = nspo_cut(qi, qany, esz, qlen, cut, cuts);
            rheap_t h = {buf, 0, k};
            int64_t n_scored = 0, n_blk_visit = 0, n_blk_seen = 0, n_revisit = 0;
            int first = 1;
            for (int c = 0; c < ncut; ++c) {
                const int t = cuts[c];
                if (t >= n_lists) continue; /* seismic_index.cpp:254-256 */
                const int64_t b0 = list_block_ptr[t];
                const int64_t nb = list_block_ptr[t + 1] - b0;
                if (nb > 0) {
                    /* score_summaries_typed: inverted_list_clusters.cpp:295-315 */
                    for (int64_t b = 0; b < nb; ++b) {
                        blocks[b].s = 0.0f;
                        blocks[b].b = (int32_t)b;
                    }
                    const int64_t tp0 = list_term_ptr[t];
                    const int64_t ntm = list_term_ptr[t + 1] - tp0;
                    if (ntm > 0) {
                        for (int i = 0; i < qlen; ++i) {
                            int col = find_term(sum_terms + tp0, ntm, qi[i]);
                            if (col < 0) continue;
                            const float qv = val_at(qany, esz, i);
                            for (int64_t j = sum_run_ptr[tp0 + col];
                                 j < sum_run_ptr[tp0 + col + 1]; ++j) {
                                const float sv = val_at(sum_val, esz, j);
                                const float p = qv * sv;
                                blocks[sum_block[j]].s = blocks[sum_block[j]].s + p;
                            }
                        }
                    }
                    /* reorder_clusters: seismic_common.h:105-115 */
                    if (first) blk_sort_like_reference(blocks, nb);
                    /* query_single_inverted_list: seismic_index.cpp:78-117 */
                    for (int64_t o = 0; o < nb; ++o) {
                        const float bs = blocks[o].s;
                        const int64_t b = b0 + blocks[o].b;
                        ++n_blk_seen;
                        if (h.n == h.k && bs * heap_factor < h.a[0].s) {
                            if (first) break;
                            continue;
                        }
                        ++n_blk_visit;
                        for (int64_t j = block_doc_ptr[b]; j < block_doc_ptr[b + 1];
                             ++j) {
                            const int32_t d = docs[j];
                            if ((visited[d >> 6] >> (d & 63)) & 1u) {
                                ++n_revisit;
                                continue;
                            }
                            visited[d >> 6] |= (uint64_t)1 << (d & 63);
                            if (!sel_member(sel_bits, d)) continue;
                            float s;
                            if (esz == 4) {
                                const float* dv = (const float*)d_values;
                                s = 0.0f;
                                for (int32_t e = d_indptr[d]; e < d_indptr[d + 1]; ++e) {
                                    float p = dv[e] * dense[d_indices[e]];
                                    s = s + p;
                                }
                            } else if (esz == 2) {
                                /* dot_product_uint16_dense: int64 sum (distance.h:49-57) */
                                const uint16_t* dv = (const uint16_t*)d_values;
                                int64_t acc = 0;
                                for (int32_t e = d_indptr[d]; e < d_indptr[d + 1]; ++e)
                                    acc += (int64_t)dv[e] * (int64_t)dense16[d_indices[e]];
                                s = (float)acc;
                            } else {
                                const uint8_t* dv = (const uint8_t*)d_values;
                                int acc = 0;
                                for (int32_t e = d_indptr[d]; e < d_indptr[d + 1]; ++e)
                                    acc += (int)dv[e] * (int)dense8[d_indices[e]];
                                s = (float)acc;
                            }
                            ++n_scored;
                            rh_add(&h, s, d);
                        }
                    }
                }
                first = 0; /* seismic_index.cpp:261: set after every list */
            }
            rh_emit(&h, out_d + (int64_t)q * k, out_l + (int64_t)q * k);
            if (stats) {
                stats[(int64_t)q * 4 + 0] = n_scored;
                stats[(int64_t)q * 4 + 1] = n_blk_visit;
                stats[(int64_t)q * 4 + 2] = n_blk_seen;
                stats[(int64_t)q * 4 + 3] = n_revisit;
            }
            /* clear scratch */
            for (int i = 0; i < qlen; ++i) {
                dense[qi[i]] = 0.0f;
                dense8[qi[i]] = 0;
                dense16[qi[i]] = 0;
            }
            for (int c = 0; c < ncut; ++c) {
                const int t = cuts[c];
                if (t >= n_lists) continue;
                const int64_t b0 = list_block_ptr[t];
                for (int64_t b = b0; b < list_block_ptr[t + 1]; ++b)
                    for (int64_t j = block_doc_ptr[b]; j < block_doc_ptr[b + 1]; ++j)
                        visited[docs[j] >> 6] = 0;
            }
        }
        free(dense);
        free(dense8);
        free(dense16);
        free(visited);
        free(blocks);
        free(buf);
        free(cuts);
    }
    (void)topk_contains;
    return err ? -1 : 0;
}
