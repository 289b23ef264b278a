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
    /* rank by (value desc, position asc): O(len*cut) selection, taken mask */
    unsigned char* taken = (unsigned char*)calloc((size_t)len, 1);
    if (!taken) return -1;
    for (int r = 0; r < cut; ++r) {
        int best = -1;
        float bv = 0.0f;
        for (int i = 0; i < len; ++i) {
            if (taken[i]) continue;
            float vi = val_at(vals, esz, i);
            if (best < 0 || vi > bv) {
                best = i;
                bv = vi;
            }
        }
        taken[best] = 1;
        out[r] = idx[best];
    }
    free(taken);
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

static int blk_cmp(const void* x, const void* y) {
    const blk_t* a = (const blk_t*)x;
    const blk_t* b = (const blk_t*)y;
    if (a->s > b->s) return -1;
    if (a->s < b->s) return 1;
    return a->b - b->b;
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
            topk_t h = {buf, 0, k};
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
                    if (first) qsort(blocks, (size_t)nb, sizeof(blk_t), blk_cmp);
                    /* query_single_inverted_list: seismic_index.cpp:78-117 */
                    for (int64_t o = 0; o < nb; ++o) {
                        const float bs = blocks[o].s;
                        const int64_t b = b0 + blocks[o].b;
                        ++n_blk_seen;
                        if (h.n == h.k && bs * heap_factor < h.a[h.n - 1].s) {
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
                            topk_add(&h, s, d);
                        }
                    }
                }
                first = 0; /* seismic_index.cpp:261: set after every list */
            }
            topk_emit(&h, out_d + (int64_t)q * k, out_l + (int64_t)q * k);
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
