/*
 * knn_b200.h -- C ABI of libknnb200.so (extern "C", plain pointers and sizes).
 *
 * Layout conventions (the reference's, README.md "Data storage"):
 *   a point set of n points in dim dimensions is a dim x n row-major FP32
 *   array, x[d*ld + i] with ld >= n (ld = n for the host entry points);
 *   results are k x query_nb row-major, dist[j*out_ld + i], index likewise,
 *   ascending distance with ties ordered by ascending index.
 *
 * Return codes of the int-returning functions: KNNB200_OK (0) or one of the
 * KNNB200_E* codes below; knnb200_status_string() names them.
 */
#ifndef KNNB200_KNN_B200_H
#define KNNB200_KNN_B200_H

#include <stddef.h>

#ifndef KNNB200_API
#define KNNB200_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define KNNB200_OK 0
#define KNNB200_EINVAL 1        /* invalid argument (sizes, k, pointers, alignment) */
#define KNNB200_ENODEV 2        /* no CUDA device */
#define KNNB200_ENOMEM 3        /* device allocation failed */
#define KNNB200_ELAUNCH 4       /* kernel launch failed */
#define KNNB200_ETIMEOUT 5      /* a kernel wait hit its time limit and returned early */
#define KNNB200_ECUDA 6         /* other CUDA runtime error */
#define KNNB200_EUNSUPPORTED 7  /* shape not supported by the requested method */
#define KNNB200_ESCRATCH 8      /* caller-provided scratch too small */
#define KNNB200_ETENSORMAP 9    /* TMA descriptor could not be encoded */

/* Methods for the device entry points. */
#define KNNB200_METHOD_GLOBAL 0   /* fused exact FP32 direct form (knn_cuda_global) */
#define KNNB200_METHOD_TEXTURE 1  /* same kernel as GLOBAL (knn_cuda_texture) */
#define KNNB200_METHOD_CUBLAS 2   /* expansion method (knn_cublas) */
#define KNNB200_METHOD_FP8 3      /* expansion method with an FP8 (e4m3) candidate scan; same
                                     exact results; as CUBLAS where the FP8 scan does not apply
                                     (d > 1024) or where its sample pass predicts that most
                                     candidate lists would overflow */

/* C-linkage aliases of the three drop-in entry points of knncuda.h.
 * Replace knn_cuda_global / knn_cuda_texture / knn_cublas,
 * code/knncuda.h:14-21, :37-44, :61-68; identical arguments and semantics
 * (bool result as int: 1 success, 0 failure with "ERROR: ..." on stdout). */
KNNB200_API int knnb200_cuda_global(const float *ref, int ref_nb, const float *query, int query_nb,
                        int dim, int k, float *knn_dist, int *knn_index);
KNNB200_API int knnb200_cuda_texture(const float *ref, int ref_nb, const float *query, int query_nb,
                         int dim, int k, float *knn_dist, int *knn_index);
KNNB200_API int knnb200_cublas(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                   int k, float *knn_dist, int *knn_index);

/* Device-resident variant of the same computation: every pointer is device
 * memory on the current device, work is queued on `stream` (a cudaStream_t,
 * NULL = legacy default stream) and the call returns without synchronising.
 * It replaces the compute part of the reference host bodies
 * (code/knncuda.cu:352-394 and :709-805) for callers whose data already
 * lives in HBM.  ref_ld / query_ld are row pitches in elements (multiples of
 * 4, base pointers 16-byte aligned); out_ld >= query_nb.  Scratch comes from
 * a per-device library workspace (grown with cudaMalloc when needed, so the
 * first call of a new size may synchronise the device); consecutive calls on
 * one device are ordered by the library so they never share scratch.
 * Device-side status (a timed-out wait) is reported by knnb200_sync_status. */
KNNB200_API int knnb200_knn_device(const float *ref, int ref_nb, long long ref_ld, const float *query,
                       int query_nb, long long query_ld, int dim, int k, int method,
                       float *knn_dist, int *knn_index, long long out_ld, void *stream);

/* The exact k-NN of knnb200_knn_device (method GLOBAL) for callers that
 * cannot allocate device memory: their memory is handed out by their own
 * pool, or cudaMalloc / cudaFree (which can stall the device) are not
 * allowed where they call from.  It has no counterpart in the reference
 * (whose functions allocate and free every buffer per call).  Inputs and
 * outputs are caller-owned device memory as for knnb200_knn_device; the
 * scratch is a static 64 MiB device array inside this library, held on
 * every GPU that loads it until exit.  A call needs the exact path's whole
 * scratch there: the duplicated query copy (dim * round_up(query_nb, 32) * 8
 * bytes), 256 bytes, and the per-split lists (splits * query_nb *
 * min(k, 256) * 8 bytes when the reference set is split; query_nb * 8 more
 * for k > 256).
 * knnb200_scratch_bytes(..., KNNB200_METHOD_GLOBAL) gives the exact figure;
 * shapes needing more than 64 MiB are rejected with KNNB200_ESCRATCH.  The
 * first call on a device looks up the array's device address (make that
 * first call before any stream capture).  All calls share the array and its
 * status word: calls that overlap on the GPU race and must be serialised by
 * the caller.  The call synchronises `stream` (it reads the status word back
 * into host memory) and returns after the results are written (KNNB200_OK,
 * or KNNB200_ETIMEOUT if a kernel wait gave up). */
KNNB200_API int knnb200_knn_device_noalloc(const float *ref, int ref_nb, long long ref_ld,
                                           const float *query, int query_nb,
                                           long long query_ld, int dim, int k, float *knn_dist,
                                           int *knn_index, long long out_ld, void *stream);

/* ---- Resident reference sets (no counterpart in the reference, which
 * re-uploads the reference set on every call, code/knncuda.cu:341, :695). */
typedef struct knnb200_refset knnb200_refset;

/* Copy a dim x ref_nb reference set (row pitch ref_ld elements; host memory,
 * or device memory when on_device != 0) into a resident set on the current
 * device, with the tensor-core view prepared when the shape qualifies. */
KNNB200_API int knnb200_refset_create(const float *ref, int ref_nb, long long ref_ld, int dim,
                                      int on_device, knnb200_refset **out);
KNNB200_API void knnb200_refset_destroy(knnb200_refset *rs);
/* Device bytes held by the resident set. */
KNNB200_API size_t knnb200_refset_device_bytes(const knnb200_refset *rs);
/* k-NN of device-resident queries (dim x query_nb, pitch query_ld, a multiple
 * of 4) against the resident set; results k x query_nb (pitch out_ld) in
 * device memory.  Synchronises `stream` before returning.  Same methods and
 * results as knnb200_knn_device. */
KNNB200_API int knnb200_refset_knn(knnb200_refset *rs, const float *query, int query_nb,
                                   long long query_ld, int k, int method, float *knn_dist,
                                   int *knn_index, long long out_ld, void *stream);

/* ---- Continuous-batching server over a resident set.  `slots` worker
 * threads, each with its own stream and scratch, form batches of up to
 * max_batch_queries queries from the head of the request queue; a batch is
 * admitted only while the working memory of all batches in flight stays
 * within memory_budget_bytes (one batch is always admitted).  Requests of
 * different k share a batch (top-k_max, each takes its first k rows), and a
 * request's result does not depend on its batch.  Each slot's device buffers
 * are allocated at creation for a full batch at k = 128 (KNNB200_ENOMEM if
 * they do not fit), so no allocation happens on the request path unless a
 * batch needs k > 128. */
typedef struct knnb200_server knnb200_server;
KNNB200_API int knnb200_server_create(knnb200_refset *rs, int slots, size_t memory_budget_bytes,
                                      int max_batch_queries, int method, knnb200_server **out);
/* Queue a request: host queries dim x query_nb (contiguous), host outputs
 * k x query_nb filled on completion.  Buffers must stay valid until
 * knnb200_server_wait returns.  Returns a ticket > 0, or -KNNB200_E*. */
KNNB200_API long long knnb200_server_submit(knnb200_server *s, const float *query, int query_nb,
                                            int k, float *knn_dist, int *knn_index);
/* Block until the request is done; returns its status and (optionally) its
 * latency from submit to completion. */
KNNB200_API int knnb200_server_wait(knnb200_server *s, long long ticket, double *latency_ms);
/* Latency percentiles of completed requests, totals, and wall time from the
 * first submit to the last completion. */
KNNB200_API int knnb200_server_stats(knnb200_server *s, double *p50_ms, double *p99_ms,
                                     long long *queries_done, long long *batches_done,
                                     double *wall_seconds);
/* Drain the queue, stop the workers and free the server (not the refset). */
KNNB200_API void knnb200_server_destroy(knnb200_server *s);

/* ---- Many independent problems in one persistent launch (no counterpart
 * in the reference, which solves one problem per call,
 * code/knncuda.cu:271-278).  All pointers are device memory; the reference
 * set of each problem must have a row pitch that is a multiple of 4 and a
 * 16-byte-aligned base.  k <= 256 for every problem. */
typedef struct knnb200_problem {
    const float *ref;       /* dim x ref_nb, pitch ref_ld */
    int ref_nb;
    long long ref_ld;
    const float *query;     /* dim x query_nb, pitch query_ld */
    int query_nb;
    long long query_ld;
    int dim;
    int k;
    float *knn_dist;        /* k x query_nb, pitch out_ld */
    int *knn_index;
    long long out_ld;
} knnb200_problem;
typedef struct knnb200_batched_plan knnb200_batched_plan;
/* Build a plan: problem table, TMA descriptors and scratch on the current
 * device (this call allocates and synchronises).  item_stages sets the work-
 * item granularity in pipeline stages (<= 0: 256); see the autotuner. */
KNNB200_API int knnb200_batched_plan_create(const knnb200_problem *problems, int count,
                                            int item_stages, knnb200_batched_plan **out);
/* Queue the plan's work on `stream`: one persistent exact kernel over a
 * device work queue plus a batched split merge.  Allocates nothing and does
 * not synchronise. */
KNNB200_API int knnb200_batched_run(knnb200_batched_plan *plan, void *stream);
/* Synchronise `stream` and report the device status of the last run. */
KNNB200_API int knnb200_batched_status(knnb200_batched_plan *plan, void *stream);
/* Number of work items of the plan. */
KNNB200_API long long knnb200_batched_items(const knnb200_batched_plan *plan);
KNNB200_API void knnb200_batched_plan_destroy(knnb200_batched_plan *plan);
/* Capture knnb200_batched_run(plan) into an instantiated CUDA graph
 * (cudaGraphExec_t returned as void*); launch with knnb200_graph_launch. */
KNNB200_API int knnb200_batched_graph_create(knnb200_batched_plan *plan, void **graph_exec);
KNNB200_API int knnb200_graph_launch(void *graph_exec, void *stream);
KNNB200_API void knnb200_graph_destroy(void *graph_exec);
/* Time plans of several work-item granularities on `stream` and return the
 * fastest (and its time per run in ms). */
KNNB200_API int knnb200_batched_autotune(const knnb200_problem *problems, int count,
                                         void *stream, int *best_item_stages, float *best_ms);

/* Plan configuration: the work-item size in pipeline stages (<= 0: 256),
 * the queries per consumer warp of the persistent kernel (its query tile is
 * 16 x that: 4 -> 64-query tiles, 2 -> 32-query tiles for small query
 * counts; 0: 4, or 2 when some k > 128), and whether problems with dim <= 4
 * and k <= 16 run the low-dimension kernel in launches of their own
 * (queued by knnb200_batched_run) instead of the persistent launch. */
typedef struct knnb200_batched_config {
    int item_stages;
    int queries_per_warp;
    int lowdim_kernel;
} knnb200_batched_config;
KNNB200_API int knnb200_batched_plan_create_config(const knnb200_problem *problems, int count,
                                                   const knnb200_batched_config *config,
                                                   knnb200_batched_plan **out);
/* The configuration a plan was built with and the number of problems it
 * routes to the low-dimension kernel. */
KNNB200_API int knnb200_batched_plan_config(const knnb200_batched_plan *plan,
                                            knnb200_batched_config *config,
                                            int *lowdim_problems);
/* Autotuner over the whole configuration: the work-item size with the
 * default tile, then both tile shapes with and without low-d routing at
 * that size; returns the fastest configuration and its ms per run. */
KNNB200_API int knnb200_batched_autotune_config(const knnb200_problem *problems, int count,
                                                void *stream, knnb200_batched_config *best,
                                                float *best_ms);

/* Synchronise `stream` and return the status of the last device-resident
 * call on the current device (KNNB200_OK or KNNB200_ETIMEOUT / ECUDA). */
KNNB200_API int knnb200_sync_status(void *stream);

/* Bytes of scratch the device entry point needs for this shape and method. */
KNNB200_API size_t knnb200_scratch_bytes(int ref_nb, int query_nb, int dim, int k, int method);

/* Number of reference splits the exact kernel uses for this shape. */
KNNB200_API int knnb200_plan_splits(int ref_nb, int query_nb, int dim, int k);

/* Memory admission of the host and device entry points (the reference's
 * legacy code split the queries by free memory,
 * legacy/KNN.CUDA.with.indexes/knn_cuda_with_indexes.cu:348-349, :406-444):
 * a call whose buffers for all query_nb queries do not fit in the device's
 * free memory (plus what the library's workspace already holds) runs its
 * queries in chunks that do, with the same results.  knnb200_set_memory_cap
 * lowers the memory the library assumes it may use to `bytes` (0 = no cap;
 * a host-side setting, used to test the chunked path); knnb200_last_query_chunks
 * returns the number of chunks of the last host or device call. */
KNNB200_API void knnb200_set_memory_cap(size_t bytes);
KNNB200_API int knnb200_last_query_chunks(void);
/* Device bytes the library estimates for one call of this shape run as one
 * chunk: host != 0 for the host entry points (reference and query copies,
 * outputs, scratch), 0 for knnb200_knn_device (scratch only). */
KNNB200_API size_t knnb200_call_bytes(int ref_nb, int query_nb, int dim, int k, int method,
                                      int host);

/* Free the current device's workspace (the next call re-allocates). */
KNNB200_API void knnb200_release_workspace(void);

/* Human-readable name of a KNNB200_* code. */
KNNB200_API const char *knnb200_status_string(int code);

/* Calibration: FP32 CUDA-core multiply-add throughput of the current device
 * in FLOP/s (2 flops per multiply-add), measured by a packed-FMA kernel of
 * `iters` inner iterations on `stream`; synchronises; -1 on error.  Used as
 * the roofline denominator of the FP32 direct-form path. */
KNNB200_API double knnb200_measure_fp32_peak(int iters, void *stream);

/* Self-test of the bounded waits (no counterpart in the reference, whose
 * kernels have no waits): one warp waits on an mbarrier that nothing
 * completes, gives up after limit_ns (0 < limit_ns <= 1e9) like every
 * pipelined kernel of this library does after its own limit, and the call
 * returns KNNB200_ETIMEOUT with the device context still usable.
 * KNNB200_OK would mean the wait completed, which cannot happen. */
KNNB200_API int knnb200_selftest_wait_timeout(long long limit_ns, void *stream);

/* For the last knn_cublas-method call on the current device: the total
 * number of candidates the first tensor-core scan emitted (*candidates), the
 * number of queries that failed the first certification and were scanned a
 * second time (*second_scan), and of those the number recomputed by the
 * exact kernel (*exact).  All 0 when the call ran the exact kernel only.
 * Any pointer may be NULL. */
KNNB200_API void knnb200_last_tc_stats(long long *candidates, int *second_scan, int *exact);

/* Test-only check of the tensor path's error bound (no counterpart in the
 * reference, whose knn_cublas has no bound).  While enabled, every
 * knn_cublas-method call on the current device that runs the tensor path
 * records, over all candidates its exact re-rank sees, the largest
 * |a + ||q||^2 - D| / E_q: a the candidate's BF16-expansion value, D its
 * exact FP32 squared distance, E_q the bound the certification assumes
 * for the query.  A ratio below 1 is what the certification needs; the
 * test asserts a margin.  The check runs a separate instantiation of the
 * re-rank kernel; off by default (enable = 0 turns it off). */
KNNB200_API int knnb200_set_bound_check(int enable);
/* Waits for the current device (cudaDeviceSynchronize) and returns the ratio and the
 * number of candidates checked by the last such call (KNNB200_EINVAL if
 * the check was never enabled). */
KNNB200_API int knnb200_last_bound_check(double *max_ratio, long long *checked);

/* Scan kinds of the last knn_cublas- or FP8-method call on the current
 * device: *first = the kind of its candidate scan over the whole set,
 * *second = the kind of the second scan of uncertified queries; 0 BF16,
 * 1 split BF16 (hi + lo parts), 2 FP8 e4m3, -1 none (exact kernel only, or
 * no second scan).  Either pointer may be NULL. */
KNNB200_API void knnb200_last_tc_kinds(int *first, int *second);

/* Test and measurement override of the pass-2 kind of the device-entry
 * tensor path (no counterpart in the reference): 0 BF16, 1 split BF16,
 * 2 FP8 (FP8-method calls only), -1 none (the default: the kind the
 * threshold pass predicts to fit).  Results stay exact whatever the kind:
 * a forced kind whose lists overflow only costs time (second scan, exact
 * kernel).  Process-wide. */
KNNB200_API void knnb200_set_tc_kind_override(int kind);

/* Per-phase device timing of the calls on the current device (CUDA events on
 * the launching stream between the kernels of a call).  Off by default. */
KNNB200_API void knnb200_set_phase_timing(int enable);

/* Durations in ms of the phases of the last timed call on the current device,
 * indexed by phase: 0 tensor-path reference prep, 1 query prep, 2 pass-1 scan,
 * 3 thresholds, 4 pass-2 scan, 5 exact re-rank, 6 uncertified-query fallback,
 * 7 fused exact kernel, 8 split merge, 9 second-chance scan of uncertified
 * queries (with the host round trip before it), 10 their re-rank; -1 for
 * phases the call did not run.  Waits for the call's last event.  Returns
 * the number of phases (11), or 0 when nothing was timed. */
KNNB200_API int knnb200_last_phase_times(float *ms, int n);

/* Library version string. */
KNNB200_API const char *knnb200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* KNNB200_KNN_B200_H */
