/*
 * Seeded synthetic sparse corpora with the shape of a SPLADE-style index
 * (MS MARCO: ~8.8M docs over the 30,522-term BERT vocabulary, ~120-130 nnz per
 * doc), which stand in for the real dataset in benchmarks and tests.
 *
 * Row r of stream `stream` draws from its own counter-based generator seeded
 * by (seed, stream, r), so the output does not depend on thread count.
 *   nnz   lognormal(ln median, sigma) rounded and clipped to [lo, hi], or
 *         uniform on [lo, hi]
 *   terms Zipf(s) over ranks 1..dim (term id = rank - 1), drawn without
 *         replacement per row, stored ascending
 *   vals  lognormal(mu, sigma) as float32 (> 0)
 *
 * Plain C, OpenMP over rows. Exported with C linkage for ctypes.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t s;
} rng_t;

static inline uint64_t splitmix64(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static inline rng_t row_rng(uint64_t seed, uint64_t stream, int64_t row) {
    uint64_t x = seed * 0xD1B54A32D192ED03ULL ^ (stream + 1) * 0xABC98388FB8FAC03ULL;
    (void)splitmix64(&x);
    x ^= (uint64_t)row * 0x8CB92BA72F3D8DD7ULL;
    (void)splitmix64(&x);
    rng_t r = {x};
    return r;
}

static inline double uniform01(rng_t* r) {
    return (double)(splitmix64(&r->s) >> 11) * (1.0 / 9007199254740992.0);
}

static inline double normal01(rng_t* r) {
    double u1 = uniform01(r);
    double u2 = uniform01(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static int row_nnz(rng_t* r, int kind, double p0, double p1, int lo, int hi) {
    int n;
    if (kind == 0) {
        n = (int)lround(exp(log(p0) + p1 * normal01(r)));
    } else {
        n = lo + (int)(uniform01(r) * (double)(hi - lo + 1));
    }
    if (n < lo) n = lo;
    if (n > hi) n = hi;
    return n;
}

/* Row lengths: writes indptr[0..n] (int32, exclusive prefix) and returns the
 * total nnz, or -1 if it does not fit int32 offsets. */
int64_t nsp_synth_indptr(uint64_t seed, uint64_t stream, int64_t n, int kind,
                         double p0, double p1, int lo, int hi, int dim,
                         int32_t* indptr) {
    if (hi > dim) hi = dim;
    if (lo > hi) lo = hi;
    int32_t* lens = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    if (!lens) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        rng_t r = row_rng(seed, stream * 2 + 0, i);
        lens[i] = row_nnz(&r, kind, p0, p1, lo, hi);
    }
    int64_t acc = 0;
    indptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        acc += lens[i];
        if (acc > 2147483647LL) {
            free(lens);
            return -1;
        }
        indptr[i + 1] = (int32_t)acc;
    }
    free(lens);
    return acc;
}

static int cmp_u16(const void* a, const void* b) {
    return (int)*(const uint16_t*)a - (int)*(const uint16_t*)b;
}

/* Fills indices/values for rows [0, n) given indptr from nsp_synth_indptr. */
int nsp_synth_fill(uint64_t seed, uint64_t stream, int64_t n, int dim,
                   double zipf_s, double val_mu, double val_sigma,
                   const int32_t* indptr, uint16_t* indices, float* values) {
    if (dim <= 0 || dim > 65536) return -1;
    double* cdf = (double*)malloc(sizeof(double) * (size_t)dim);
    if (!cdf) return -1;
    double acc = 0.0;
    for (int i = 0; i < dim; ++i) {
        acc += pow((double)(i + 1), -zipf_s);
        cdf[i] = acc;
    }
    for (int i = 0; i < dim; ++i) cdf[i] /= acc;
    cdf[dim - 1] = 1.0;
    int err = 0;
#pragma omp parallel
    {
        uint32_t* seen = (uint32_t*)calloc((size_t)dim, sizeof(uint32_t));
        if (!seen) {
#pragma omp atomic write
            err = 1;
        }
        uint32_t epoch = 0;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; ++i) {
            if (!seen) continue;
            rng_t r = row_rng(seed, stream * 2 + 1, i);
            const int32_t start = indptr[i];
            const int32_t len = indptr[i + 1] - start;
            if (++epoch == 0) {
                memset(seen, 0, sizeof(uint32_t) * (size_t)dim);
                epoch = 1;
            }
            int32_t got = 0;
            while (got < len) {
                double u = uniform01(&r);
                int lo = 0, hi = dim - 1;
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if (cdf[mid] < u) lo = mid + 1; else hi = mid;
                }
                if (seen[lo] == epoch) continue;
                seen[lo] = epoch;
                indices[start + got] = (uint16_t)lo;
                ++got;
            }
            qsort(indices + start, (size_t)len, sizeof(uint16_t), cmp_u16);
            for (int32_t j = 0; j < len; ++j) {
                values[start + j] = (float)exp(val_mu + val_sigma * normal01(&r));
            }
        }
        free(seen);
    }
    free(cdf);
    return err ? -1 : 0;
}
