/*
 * knncuda.h -- drop-in replacement header for the reference's code/knncuda.h.
 *
 * Same three functions, same signatures, same C++ linkage, so a program
 * written against the reference (e.g. its code/test.cpp) compiles and links
 * unchanged against libknnb200.so.  Exported (mangled) symbols:
 *   _Z15knn_cuda_globalPKfiS0_iiiPfPi
 *   _Z16knn_cuda_texturePKfiS0_iiiPfPi
 *   _Z10knn_cublasPKfiS0_iiiPfPi
 * C callers use the extern "C" aliases in knn_b200.h.
 *
 * Contract shared by all three (reference semantics):
 *   ref        dim x ref_nb   row-major host array, ref[d*ref_nb + i]
 *   query      dim x query_nb row-major host array
 *   knn_dist   k x query_nb   host output, ascending Euclidean distances,
 *              knn_dist[j*query_nb + i] = distance of query i to its j-th NN
 *   knn_index  k x query_nb   host output, 0-based reference indices;
 *              equal distances are ordered by ascending index
 *   returns    true on success; on failure prints "ERROR: ..." to stdout and
 *              returns false (outputs undefined).
 * Calls are synchronous and run on the calling thread's current CUDA device
 * (device 0 in a fresh process).  Unlike the reference, k is validated
 * (1 <= k <= ref_nb) and the ref_nb x query_nb distance matrix is never
 * allocated.
 */
#ifndef KNNB200_KNNCUDA_H
#define KNNB200_KNNCUDA_H

#ifndef KNNB200_API
#define KNNB200_API __attribute__((visibility("default")))
#endif

/* Replaces knn_cuda_global, code/knncuda.h:14-21 (body code/knncuda.cu:271-415).
 * Exact FP32 direct-form distances, fused distance + top-k + sqrt kernel. */
KNNB200_API bool knn_cuda_global(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                     int k, float *knn_dist, int *knn_index);

/* Replaces knn_cuda_texture, code/knncuda.h:37-44 (body code/knncuda.cu:418-609).
 * Same arithmetic as knn_cuda_global; reference points are staged by TMA
 * instead of a texture, so the reference's texture-size limits do not apply. */
KNNB200_API bool knn_cuda_texture(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                      int k, float *knn_dist, int *knn_index);

/* Replaces knn_cublas, code/knncuda.h:61-68 (body code/knncuda.cu:612-832).
 * The ||r||^2 - 2 r.q + ||q||^2 expansion method; returns exact results. */
KNNB200_API bool knn_cublas(const float *ref, int ref_nb, const float *query, int query_nb, int dim, int k,
                float *knn_dist, int *knn_index);

#endif /* KNNB200_KNNCUDA_H */
