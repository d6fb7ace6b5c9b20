/*
 * sift_oracle.c - CPU restatement of the reference's 2-NN and LSH algorithms.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA product
 * is compared against; only tests/, the smoke check and bench.py's CPU-baseline
 * leg may load it. The product library never links or calls it.
 *
 * What it restates (paths are within the reference project):
 *   oracle_2nn_u8 / metric 0 : host_brute + host_lenght, src/knn_brute.cu:801-835, :873-885.
 *       Full squared Euclidean distance, candidates visited in increasing index
 *       order with strict '<' updates, i.e. lexicographic (distance, index)
 *       top-2 where the lower index wins a tie. Integer arithmetic here is exact
 *       (128 * 255^2 < 2^31), so the result is what the reference's FP32 loop
 *       produces on integer-valued descriptors.
 *   oracle_2nn_u8 / metric 1 : cublas_2nn_brute_f, src/knn_brute.cu:579-606.
 *       The reference ranks by -2 q.r only (its GEMM uses alpha = -2 and never
 *       adds norms). Same lexicographic top-2 rule.
 *   oracle_2nn_f64           : the same two metrics in FP64 for float inputs.
 *   oracle_ratio_match       : the Lowe ratio test of find_matches,
 *       src/knn_brute.cu:430-442, stated on true squared distances:
 *       sqrtf(d1) / sqrtf(d2) < threshold in IEEE single precision.
 *       For unit-norm inputs the reference's d + 2 equals the squared distance.
 *   oracle_lsh_codes         : set_bit_h, src/lsh_h.cu:265-317: bit j of a
 *       point's code is set when its dot product with hyperplane j is < 0.
 *   oracle_bucket_sort       : lsh_thread_sort_reduce, src/lsh_h.cu:565-629:
 *       points ordered by code (ties by point id) and run-length grouped.
 *   oracle_lsh_scan          : the candidate scan of brute_2nn_h,
 *       src/lsh_h.cu:441-562, over the true bucket members of every table
 *       (the reference indexes sorted positions by point id; see its
 *       bucket-offset defect at src/lsh_h.cu:599,617 vs :469,482).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define D 128
#define NONE_I (-1)

typedef struct {
    int64_t d1, d2, i1, i2;
} top2_t;

static inline void top2_push(top2_t *t, int64_t d, int64_t i) {
    /* candidates arrive in increasing index order: strict '<' keeps the
       lexicographic (d, i) order of host_brute (src/knn_brute.cu:816-831) */
    if (d < t->d1) {
        t->d2 = t->d1; t->i2 = t->i1;
        t->d1 = d; t->i1 = i;
    } else if (d < t->d2) {
        t->d2 = d; t->i2 = i;
    }
}

/* lexicographic merge of an arbitrary (d, i) candidate into a top-2 */
static inline int lex_less(int64_t da, int64_t ia, int64_t db, int64_t ib) {
    return da < db || (da == db && ia < ib);
}
static inline void top2_push_lex(top2_t *t, int64_t d, int64_t i) {
    if (i == t->i1 || i == t->i2) return;
    if (lex_less(d, i, t->d1, t->i1)) {
        t->d2 = t->d1; t->i2 = t->i1;
        t->d1 = d; t->i1 = i;
    } else if (lex_less(d, i, t->d2, t->i2)) {
        t->d2 = d; t->i2 = i;
    }
}

static inline int32_t l2_u8(const uint8_t *a, const uint8_t *b) {
    int32_t s = 0;
    for (int k = 0; k < D; ++k) {
        int32_t c = (int32_t)a[k] - (int32_t)b[k];
        s += c * c;
    }
    return s;
}

static inline int32_t dot_u8(const uint8_t *a, const uint8_t *b) {
    int32_t s = 0;
    for (int k = 0; k < D; ++k) s += (int32_t)a[k] * (int32_t)b[k];
    return s;
}

typedef struct {
    const uint8_t *q, *r;
    const float *qf, *rf;
    int64_t q_begin, q_end, r_n;
    int metric;
    int64_t *out_i;
    int64_t *out_d;
    double *out_df;
} job_t;

static void *run_u8(void *arg) {
    job_t *j = (job_t *)arg;
    for (int64_t qi = j->q_begin; qi < j->q_end; ++qi) {
        top2_t t = {INT64_MAX, INT64_MAX, NONE_I, NONE_I};
        const uint8_t *qv = j->q + qi * D;
        if (j->metric == 0) {
            for (int64_t ri = 0; ri < j->r_n; ++ri) top2_push(&t, l2_u8(qv, j->r + ri * D), ri);
        } else {
            for (int64_t ri = 0; ri < j->r_n; ++ri) top2_push(&t, -2 * (int64_t)dot_u8(qv, j->r + ri * D), ri);
        }
        j->out_d[2 * qi] = t.d1; j->out_d[2 * qi + 1] = t.d2;
        j->out_i[2 * qi] = t.i1; j->out_i[2 * qi + 1] = t.i2;
    }
    return NULL;
}

static void *run_f64(void *arg) {
    job_t *j = (job_t *)arg;
    for (int64_t qi = j->q_begin; qi < j->q_end; ++qi) {
        double d1 = INFINITY, d2 = INFINITY;
        int64_t i1 = NONE_I, i2 = NONE_I;
        const float *qv = j->qf + qi * D;
        for (int64_t ri = 0; ri < j->r_n; ++ri) {
            const float *rv = j->rf + ri * D;
            double s = 0.0;
            if (j->metric == 0) {
                for (int k = 0; k < D; ++k) { double c = (double)qv[k] - (double)rv[k]; s += c * c; }
            } else {
                for (int k = 0; k < D; ++k) s += (double)qv[k] * (double)rv[k];
                s = -2.0 * s;
            }
            if (s < d1) { d2 = d1; i2 = i1; d1 = s; i1 = ri; }
            else if (s < d2) { d2 = s; i2 = ri; }
        }
        j->out_df[2 * qi] = d1; j->out_df[2 * qi + 1] = d2;
        j->out_i[2 * qi] = i1; j->out_i[2 * qi + 1] = i2;
    }
    return NULL;
}

static int run_threads(void *(*fn)(void *), job_t base, int64_t q_n, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (nthreads > q_n) nthreads = (int)(q_n > 0 ? q_n : 1);
    pthread_t th[256];
    job_t jobs[256];
    int64_t per = (q_n + nthreads - 1) / nthreads;
    int started = 0;
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = base;
        jobs[t].q_begin = t * per;
        jobs[t].q_end = (t + 1) * per < q_n ? (t + 1) * per : q_n;
        if (jobs[t].q_begin >= jobs[t].q_end) break;
        if (nthreads == 1) { fn(&jobs[t]); started = 0; break; }
        if (pthread_create(&th[t], NULL, fn, &jobs[t]) != 0) return -1;
        started = t + 1;
    }
    for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
    return 0;
}

/* Exact 2-NN of u8 descriptors. out_d[2q] / out_d[2q+1]: best and second
   distance (INT64_MAX when absent); out_i likewise (-1 when absent). */
int oracle_2nn_u8(const uint8_t *q, const uint8_t *r, int64_t q_n, int64_t r_n, int metric, int nthreads,
                  int64_t *out_d, int64_t *out_i) {
    if (q_n < 0 || r_n < 0 || (metric != 0 && metric != 1)) return -1;
    job_t j = {q, r, NULL, NULL, 0, 0, r_n, metric, out_i, out_d, NULL};
    return run_threads(run_u8, j, q_n, nthreads);
}

/* FP64 2-NN of float descriptors (same metrics); distances as double. */
int oracle_2nn_f64(const float *q, const float *r, int64_t q_n, int64_t r_n, int metric, int nthreads,
                   double *out_d, int64_t *out_i) {
    if (q_n < 0 || r_n < 0 || (metric != 0 && metric != 1)) return -1;
    job_t j = {NULL, NULL, q, r, 0, 0, r_n, metric, out_i, NULL, out_d};
    return run_threads(run_f64, j, q_n, nthreads);
}

/* Lowe ratio test on squared distances: match when sqrtf(d1)/sqrtf(d2) < thr.
   A missing second neighbour counts as an infinite distance (ratio 0), a
   missing first neighbour never matches. */
void oracle_ratio_match(const int64_t *nn_d, const int64_t *nn_i, int64_t q_n, float thr, uint32_t *matches) {
    for (int64_t k = 0; k < q_n; ++k) {
        int64_t d1 = nn_d[2 * k], d2 = nn_d[2 * k + 1];
        if (nn_i[2 * k] < 0) { matches[k] = UINT32_MAX; continue; }
        float f1 = sqrtf((float)d1);
        float f2 = nn_i[2 * k + 1] < 0 ? INFINITY : sqrtf((float)d2);
        matches[k] = (f1 / f2 < thr) ? (uint32_t)nn_i[2 * k] : UINT32_MAX;
    }
}

/* ---------------------------------------------------------------- LSH --- */

/* Sign-bit codes: code[i] bit j = (x_i . h_j < 0), dots in FP64 over u8 points
   and float hyperplanes (nbits rows of 128). Also returns the dots (FP64) so a
   test can tell sign flips caused by rounding (|dot| tiny) from real errors. */
void oracle_lsh_codes(const uint8_t *x, int64_t n, const float *planes, int nbits, uint32_t *code, double *dots) {
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c = 0;
        for (int j = 0; j < nbits; ++j) {
            double s = 0.0;
            for (int k = 0; k < D; ++k) s += (double)x[i * D + k] * (double)planes[j * D + k];
            if (dots) dots[i * nbits + j] = s;
            if (s < 0.0) c |= 1u << j;
        }
        code[i] = c;
    }
}

static const uint32_t *g_sort_code;
static int cmp_by_code(const void *a, const void *b) {
    int64_t ia = *(const int64_t *)a, ib = *(const int64_t *)b;
    uint32_t ca = g_sort_code[ia], cb = g_sort_code[ib];
    if (ca != cb) return ca < cb ? -1 : 1;
    return ia < ib ? -1 : (ia > ib);
}

/* Order point ids by (code, id) and run-length group them. Outputs:
   order[n] (ids), bucket_code[nb], bucket_start[nb] (position in order),
   bucket_count[nb]; returns nb. */
int64_t oracle_bucket_sort(const uint32_t *code, int64_t n, int64_t *order, uint32_t *bucket_code,
                           int64_t *bucket_start, int64_t *bucket_count) {
    for (int64_t i = 0; i < n; ++i) order[i] = i;
    g_sort_code = code;
    qsort(order, (size_t)n, sizeof(int64_t), cmp_by_code);
    int64_t nb = 0;
    for (int64_t p = 0; p < n; ++p) {
        uint32_t c = code[order[p]];
        if (nb == 0 || bucket_code[nb - 1] != c) {
            bucket_code[nb] = c; bucket_start[nb] = p; bucket_count[nb] = 0; ++nb;
        }
        bucket_count[nb - 1]++;
    }
    return nb;
}

/* Exact lexicographic 2-NN of each query over the union of the base points
   that share its code in any of the L tables. q_code / r_code: [L][n] codes.
   Distances are full squared L2; absent neighbours are (INT64_MAX, -1). */
int oracle_lsh_scan(const uint8_t *q, int64_t q_n, const uint8_t *r, int64_t r_n, const uint32_t *q_code,
                    const uint32_t *r_code, int L, int64_t *out_d, int64_t *out_i) {
    int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)(r_n > 0 ? r_n : 1) * (size_t)L);
    uint32_t *bcode = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(r_n > 0 ? r_n : 1) * (size_t)L);
    int64_t *bstart = (int64_t *)malloc(sizeof(int64_t) * (size_t)(r_n > 0 ? r_n : 1) * (size_t)L);
    int64_t *bcount = (int64_t *)malloc(sizeof(int64_t) * (size_t)(r_n > 0 ? r_n : 1) * (size_t)L);
    int64_t *nbk = (int64_t *)malloc(sizeof(int64_t) * (size_t)L);
    if (!order || !bcode || !bstart || !bcount || !nbk) return -1;
    for (int t = 0; t < L; ++t)
        nbk[t] = oracle_bucket_sort(r_code + (size_t)t * r_n, r_n, order + (size_t)t * r_n, bcode + (size_t)t * r_n,
                                    bstart + (size_t)t * r_n, bcount + (size_t)t * r_n);
    for (int64_t qi = 0; qi < q_n; ++qi) {
        top2_t best = {INT64_MAX, INT64_MAX, NONE_I, NONE_I};
        for (int t = 0; t < L; ++t) {
            uint32_t c = q_code[(size_t)t * q_n + qi];
            /* binary search the bucket with code c */
            int64_t lo = 0, hi = nbk[t];
            const uint32_t *bc = bcode + (size_t)t * r_n;
            while (lo < hi) {
                int64_t mid = (lo + hi) / 2;
                if (bc[mid] < c) lo = mid + 1; else hi = mid;
            }
            if (lo >= nbk[t] || bc[lo] != c) continue;
            int64_t s = bstart[(size_t)t * r_n + lo], cnt = bcount[(size_t)t * r_n + lo];
            for (int64_t p = s; p < s + cnt; ++p) {
                int64_t ri = order[(size_t)t * r_n + p];
                top2_push_lex(&best, l2_u8(q + qi * D, r + ri * D), ri);
            }
        }
        out_d[2 * qi] = best.d1; out_d[2 * qi + 1] = best.d2;
        out_i[2 * qi] = best.i1; out_i[2 * qi + 1] = best.i2;
    }
    free(order); free(bcode); free(bstart); free(bcount); free(nbk);
    return 0;
}
