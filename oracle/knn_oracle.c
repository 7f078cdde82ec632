/*
 * knn_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU oracle for the exact brute-force k-NN path.  Only the test suite, the
 * smoke check and bench.py's CPU-baseline leg load this library; the product
 * library (libknnb200.so) never links or calls it.
 *
 * It restates, in plain C, the reference's single-threaded ground truth
 * `knn_c` (code/test.cpp:129-175) together with its two helpers
 * `compute_distance` (code/test.cpp:54-67) and `modified_insertion_sort`
 * (code/test.cpp:85-114), using the same FP32 arithmetic in the same order
 * (no FMA contraction: built with -ffp-contract=off), so that its output is
 * bit-identical to the reference's own knn_c on the same inputs.  That
 * identity is pinned by the test suite against the reference compiled from
 * its sources (oracle/_ref) and against committed golden fixtures.
 *
 * It adds an FP64 brute force (`oracle_knn_f64`) ordered by (distance,
 * index), the stricter criterion used for near-tie analysis, and a
 * pthread driver that splits the query set into contiguous slices.
 *
 * Data layout (code/test.cpp:63, README.md "Data storage"): a point set of n
 * points of dimension dim is a dim x n row-major array, x[d*n + i].  Outputs
 * are k x query_nb row-major: knn_dist[j*query_nb + i] (code/test.cpp:164-165).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* code/test.cpp:54-67: FP32 sum of squared differences over d, then sqrtf. */
static float oracle_compute_distance(const float *ref, int ref_nb,
                                     const float *query, int query_nb,
                                     int dim, int ref_index, int query_index) {
    float sum = 0.f;
    for (int d = 0; d < dim; ++d) {
        const float diff = ref[(size_t)d * ref_nb + ref_index] -
                           query[(size_t)d * query_nb + query_index];
        sum += diff * diff;
    }
    return sqrtf(sum);
}

/* code/test.cpp:85-114: partial insertion sort keeping the k smallest at the
 * front.  A value equal to the current k-th is skipped (:98) and the shift
 * is on strict '>' (:104), so equal distances keep the lower index first. */
static void oracle_insertion_sort(float *dist, int *index, int length, int k) {
    index[0] = 0;
    for (int i = 1; i < length; ++i) {
        float curr_dist = dist[i];
        int curr_index = i;
        if (i >= k && curr_dist >= dist[k - 1]) continue;
        int j = i < k - 1 ? i : k - 1;
        while (j > 0 && dist[j - 1] > curr_dist) {
            dist[j] = dist[j - 1];
            index[j] = index[j - 1];
            --j;
        }
        dist[j] = curr_dist;
        index[j] = curr_index;
    }
}

/* code/test.cpp:129-175 restricted to the query range [q0, q1). */
static int oracle_knn_c_range(const float *ref, int ref_nb, const float *query,
                              int query_nb, int dim, int k, float *knn_dist,
                              int *knn_index, int q0, int q1) {
    float *dist = (float *)malloc((size_t)ref_nb * sizeof(float));
    int *index = (int *)malloc((size_t)ref_nb * sizeof(int));
    if (!dist || !index) {
        free(dist);
        free(index);
        return 0;
    }
    for (int i = q0; i < q1; ++i) {
        for (int j = 0; j < ref_nb; ++j) {
            dist[j] = oracle_compute_distance(ref, ref_nb, query, query_nb, dim, j, i);
            index[j] = j;
        }
        oracle_insertion_sort(dist, index, ref_nb, k);
        for (int j = 0; j < k; ++j) {
            knn_dist[(size_t)j * query_nb + i] = dist[j];
            knn_index[(size_t)j * query_nb + i] = index[j];
        }
    }
    free(dist);
    free(index);
    return 1;
}

/* FP64 brute force: squared differences accumulated in double, sqrt in
 * double, partial insertion sort ordered by (distance, index).  Outputs are
 * double so that FP32 results can be measured against it. */
static int oracle_knn_f64_range(const float *ref, int ref_nb, const float *query,
                                int query_nb, int dim, int k, double *knn_dist,
                                int *knn_index, int q0, int q1) {
    double *dist = (double *)malloc((size_t)ref_nb * sizeof(double));
    int *index = (int *)malloc((size_t)ref_nb * sizeof(int));
    double *qv = (double *)malloc((size_t)dim * sizeof(double));
    if (!dist || !index || !qv) {
        free(dist);
        free(index);
        free(qv);
        return 0;
    }
    for (int i = q0; i < q1; ++i) {
        for (int d = 0; d < dim; ++d) qv[d] = query[(size_t)d * query_nb + i];
        for (int j = 0; j < ref_nb; ++j) dist[j] = 0.0;
        /* d-outer loop keeps the reads of ref rows contiguous */
        for (int d = 0; d < dim; ++d) {
            const float *row = ref + (size_t)d * ref_nb;
            const double q = qv[d];
            for (int j = 0; j < ref_nb; ++j) {
                const double diff = (double)row[j] - q;
                dist[j] += diff * diff;
            }
        }
        /* same partial insertion sort as above, in double */
        int kept = 0;
        for (int j = 0; j < ref_nb; ++j) {
            double cd = dist[j];
            if (kept == k && cd >= dist[k - 1]) continue;
            int p = kept < k ? kept : k - 1;
            while (p > 0 && dist[p - 1] > cd) {
                dist[p] = dist[p - 1];
                index[p] = index[p - 1];
                --p;
            }
            dist[p] = cd;
            index[p] = j;
            if (kept < k) ++kept;
        }
        for (int j = 0; j < k; ++j) {
            knn_dist[(size_t)j * query_nb + i] = sqrt(dist[j]);
            knn_index[(size_t)j * query_nb + i] = index[j];
        }
    }
    free(dist);
    free(index);
    free(qv);
    return 1;
}

typedef struct {
    const float *ref, *query;
    int ref_nb, query_nb, dim, k, q0, q1, f64, ok;
    void *knn_dist;
    int *knn_index;
} oracle_job;

static void *oracle_worker(void *arg) {
    oracle_job *j = (oracle_job *)arg;
    if (j->f64)
        j->ok = oracle_knn_f64_range(j->ref, j->ref_nb, j->query, j->query_nb, j->dim, j->k,
                                     (double *)j->knn_dist, j->knn_index, j->q0, j->q1);
    else
        j->ok = oracle_knn_c_range(j->ref, j->ref_nb, j->query, j->query_nb, j->dim, j->k,
                                   (float *)j->knn_dist, j->knn_index, j->q0, j->q1);
    return NULL;
}

static int oracle_run(const float *ref, int ref_nb, const float *query, int query_nb,
                      int dim, int k, void *knn_dist, int *knn_index, int threads,
                      int f64) {
    if (!ref || !query || !knn_dist || !knn_index || ref_nb < 1 || query_nb < 1 ||
        dim < 1 || k < 1 || k > ref_nb)
        return 0;
    if (threads < 1) threads = 1;
    if (threads > query_nb) threads = query_nb;
    oracle_job *jobs = (oracle_job *)calloc((size_t)threads, sizeof(oracle_job));
    pthread_t *tids = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!jobs || !tids) {
        free(jobs);
        free(tids);
        return 0;
    }
    for (int t = 0; t < threads; ++t) {
        oracle_job *j = &jobs[t];
        j->ref = ref; j->query = query; j->ref_nb = ref_nb; j->query_nb = query_nb;
        j->dim = dim; j->k = k; j->f64 = f64; j->knn_dist = knn_dist; j->knn_index = knn_index;
        j->q0 = (int)((long long)query_nb * t / threads);
        j->q1 = (int)((long long)query_nb * (t + 1) / threads);
    }
    for (int t = 1; t < threads; ++t)
        if (pthread_create(&tids[t], NULL, oracle_worker, &jobs[t]) != 0)
            jobs[t].ok = -1;              /* could not start: run inline below */
    oracle_worker(&jobs[0]);
    int ok = jobs[0].ok;
    for (int t = 1; t < threads; ++t) {
        if (jobs[t].ok == -1)
            oracle_worker(&jobs[t]);
        else
            pthread_join(tids[t], NULL);
        ok = ok && jobs[t].ok == 1;
    }
    free(jobs);
    free(tids);
    return ok;
}

/* Exported: restatement of knn_c (FP32, sqrt'ed, (dist,index) order). */
int oracle_knn_c(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                 int k, float *knn_dist, int *knn_index, int threads) {
    return oracle_run(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index, threads, 0);
}

/* Exported: FP64 brute force; knn_dist is double[k*query_nb]. */
int oracle_knn_f64(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                   int k, double *knn_dist, int *knn_index, int threads) {
    return oracle_run(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index, threads, 1);
}
