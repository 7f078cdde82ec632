// ref_glue.cpp -- TEST INFRASTRUCTURE ONLY (linked into oracle/_ref/).
//
// Glue that lets the reference's own CPU ground truth, `knn_c`
// (code/test.cpp:129-175), be called from the test suite and from bench.py's
// CPU-baseline / reference arm.  The reference's test.cpp is compiled
// unmodified from its source tree with `-Dmain=ref_test_main`; its driver
// calls the three GPU entry points, which this CPU-only library does not
// carry, so this file defines them as stubs that always fail.  Nothing here
// calls them.
//
// `ref_knn_c_mt` runs the reference knn_c on contiguous query slices in
// parallel.  knn_c reads queries as query[d*query_nb + i]
// (code/test.cpp:63), so each slice is first transposed into its own
// dim x slice array; per-query work is independent (code/test.cpp:151-167),
// so the result equals a single call on the whole query set.
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <vector>

bool knn_c(const float *ref, int ref_nb, const float *query, int query_nb, int dim, int k,
           float *knn_dist, int *knn_index);

bool knn_cuda_global(const float *, int, const float *, int, int, int, float *, int *) {
    std::printf("ERROR: reference GPU path is not part of this CPU library\n");
    return false;
}
bool knn_cuda_texture(const float *, int, const float *, int, int, int, float *, int *) {
    std::printf("ERROR: reference GPU path is not part of this CPU library\n");
    return false;
}
bool knn_cublas(const float *, int, const float *, int, int, int, float *, int *) {
    std::printf("ERROR: reference GPU path is not part of this CPU library\n");
    return false;
}

extern "C" int ref_knn_c(const float *ref, int ref_nb, const float *query, int query_nb,
                         int dim, int k, float *knn_dist, int *knn_index) {
    return knn_c(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) ? 1 : 0;
}

extern "C" int ref_knn_c_mt(const float *ref, int ref_nb, const float *query, int query_nb,
                            int dim, int k, float *knn_dist, int *knn_index, int threads) {
    if (threads <= 1 || query_nb < 2)
        return ref_knn_c(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index);
    if (threads > query_nb) threads = query_nb;
    std::vector<int> ok(threads, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        pool.emplace_back([&, t]() {
            const int q0 = (int)((long long)query_nb * t / threads);
            const int q1 = (int)((long long)query_nb * (t + 1) / threads);
            const int qn = q1 - q0;
            std::vector<float> qs((size_t)dim * qn), dd((size_t)k * qn);
            std::vector<int> ii((size_t)k * qn);
            for (int d = 0; d < dim; ++d)
                for (int i = 0; i < qn; ++i)
                    qs[(size_t)d * qn + i] = query[(size_t)d * query_nb + q0 + i];
            ok[t] = knn_c(ref, ref_nb, qs.data(), qn, dim, k, dd.data(), ii.data()) ? 1 : 0;
            for (int j = 0; j < k; ++j)
                for (int i = 0; i < qn; ++i) {
                    knn_dist[(size_t)j * query_nb + q0 + i] = dd[(size_t)j * qn + i];
                    knn_index[(size_t)j * query_nb + q0 + i] = ii[(size_t)j * qn + i];
                }
        });
    }
    int all = 1;
    for (int t = 0; t < threads; ++t) {
        pool[t].join();
        all = all && ok[t];
    }
    return all;
}
