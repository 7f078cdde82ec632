// knn_kernels.h -- internal interface between the host runtime (knn_api.cu)
// and the kernels.  Not installed; the public C-ABI is include/knn_b200.h.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace knnb200 {

// Internal result codes (mirrored by the public KNNB200_* codes).
enum Result : int {
    kOk = 0,
    kErrInvalid = 1,
    kErrNoDevice = 2,
    kErrNoMemory = 3,
    kErrLaunch = 4,
    kErrDeviceTimeout = 5,
    kErrCuda = 6,
    kErrUnsupported = 7,
    kErrScratch = 8,
    kErrTensorMap = 9,
};

// Optional per-phase device timing: CUDA events recorded on the launching
// stream between the kernels of one call.
enum Phase : int {
    kPhaseTcPrepRef = 0,
    kPhaseTcPrepQuery = 1,
    kPhaseTcPass1 = 2,
    kPhaseTcThreshold = 3,
    kPhaseTcPass2 = 4,
    kPhaseTcRerank = 5,
    kPhaseTcFallback = 6,
    kPhaseExactMain = 7,
    kPhaseExactMerge = 8,
    kPhaseTcRetryScan = 9,     // second-chance scan of uncertified queries
    kPhaseTcRetryRerank = 10,
    kNumPhases = 11,
};

struct PhaseTimer {
    static constexpr int kMaxMarks = 16;
    bool on = false;
    int marks = 0;                    // events recorded so far in this call
    int phase[kMaxMarks];             // phase ended by event i (i >= 1)
    cudaEvent_t ev[kMaxMarks];
    void begin(cudaStream_t st) {
        marks = 0;
        if (on) cudaEventRecord(ev[marks++], st);
    }
    void mark(cudaStream_t st, int ph) {
        if (on && marks > 0 && marks < kMaxMarks) {
            phase[marks] = ph;
            cudaEventRecord(ev[marks++], st);
        }
    }
};

// Kernel-side arguments of the fused exact kernel.
struct ExactArgs {
    int N, Q, d, k;
    int n_rtiles, n_splits, n_dchunks;
    float *out_dist;
    int *out_idx;
    long long ld_out;
    unsigned long long *part;   // [n_splits][Q][k] keys when n_splits > 1
    int *status;                // device status word (DeviceStatus)
    // k > 256 runs in passes of up to 256 ranks: pass p selects keys >= lb[q]
    // (LB kernels only), writes output rows row0 .. row0 + k - 1 and, when
    // lb_out is set, lb_out[q] = (its k-th key) + 1 for the next pass
    const unsigned long long *lb;
    unsigned long long *lb_out;
    int row0;
};

// One exact k-NN problem on device-resident, dim x n row-major inputs.
struct ExactProblem {
    const float *ref;   // [d][ldr]
    int N;
    long long ldr;
    const float *qry;   // [d][ldq]
    int Q;
    long long ldq;
    int d, k;
    float *out_dist;    // [k][ld_out]
    int *out_idx;
    long long ld_out;
    void *scratch;
    size_t scratch_bytes;
    int *status;
    int num_sms;
    int force_splits;   // 0 = automatic
    PhaseTimer *timer = nullptr;
};

// Encode a 2-D tensor map (cols = contiguous axis, row pitch ld_elems) with
// zero out-of-bounds fill.
bool encode_2d(CUtensorMap *map, CUtensorMapDataType dtype, int elem_bytes, const void *base,
               uint64_t cols, uint64_t rows, uint64_t ld_elems, uint32_t box_cols,
               uint32_t box_rows, CUtensorMapSwizzle swizzle);
inline bool encode_f32_2d(CUtensorMap *map, const void *base, uint64_t cols, uint64_t rows,
                          uint64_t ld_elems, uint32_t box_cols, uint32_t box_rows) {
    return encode_2d(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, cols, rows, ld_elems,
                     box_cols, box_rows, CU_TENSOR_MAP_SWIZZLE_NONE);
}

bool exact_supported_k(int k);
// Low-dimension path (d <= 4, k <= 16): chosen by launch_exact itself.
bool lowdim_applies(int N, int Q, int d, int k);
size_t lowdim_scratch_bytes(int N, int Q, int d, int k, int num_sms);
int lowdim_plan_splits(int N, int Q, int d, int k, int num_sms);
int launch_lowdim(const ExactProblem &p, cudaStream_t st);
// Merge per-split sorted key lists [S][Q][k] into rows row0 .. row0 + k - 1
// of the output; with lb_out, lb_out[q] = (k-th merged key) + 1.
int launch_split_merge(const unsigned long long *part, int S, int Q, int k, float *out_dist,
                       int *out_idx, long long ld_out, cudaStream_t st, int row0 = 0,
                       unsigned long long *lb_out = nullptr);
size_t exact_scratch_bytes(int N, int Q, int d, int k, int num_sms);
int exact_plan_splits(int N, int Q, int d, int k, int num_sms);
int launch_exact(const ExactProblem &p, cudaStream_t st);

// Host-side state of a prepared reference set: which of the optional
// copies exist, and the FP8 scales (known once the set's largest |r - c|
// and ||r - c||^2 have been read back).
struct TcRefState {
    bool lo_ready = false;   // refBlo holds the split-BF16 lo parts
    bool f8_scaled = false;  // s_r, kappa set (from the set's maxima)
    bool f8_ready = false;   // ref8 / refN8 hold the FP8 copy
    float s_r = 0.f, kappa = 0.f, resid8 = 0.f;   // FP8 scale, norm-step unit, norm residual
    float absmax_r = 0.f, r2max = 0.f;            // read back with the FP8 prep
};

// Prepared reference set of the tensor-core path (see knn_tc.cu).
struct TcRefView {
    __nv_bfloat16 *refB;    // [N][d_pad] BF16 of r - c, K-major
    float *refT;            // [N][d_pad] FP32 point-major (re-rank gathers)
    __nv_bfloat16 *refN;    // [N][16] squared norm as three BF16 parts, then zeros
    unsigned *rmax_bits;    // largest squared norm of ref - center (float bits)
    unsigned *absmax_bits;  // largest |r - c| of any coordinate (float bits)
    unsigned *resid8_bits;  // FP8 norm-split residual (float bits)
    float *center;          // [d_pad] translation of both sets before the expansion
    __nv_bfloat16 *refBlo;  // [N][d_pad] split-BF16 lo parts (prepared when first needed)
    unsigned char *ref8;    // [N][d_pad8] FP8 e4m3 of s_r (r - c) (prepared when first needed)
    unsigned char *refN8;   // [N][32] FP8 norm-step parts
    // every TC_SAMPLE_EVERY-th point's BF16 row and norm-step row
    // ([ceil(N / TC_SAMPLE_EVERY)][d_pad] and [..][16]), written by the
    // preparation: the threshold sample of a set prepared as a whole
    __nv_bfloat16 *sampB;
    __nv_bfloat16 *sampN;
    TcRefState *state;      // host-side flags and scales
};

// First-scan kind requested of the tensor path.
enum TcRequest : int {
    kTcReqBf16 = 0,   // BF16 scan; split BF16 when BF16 is predicted to overflow
    kTcReqFp8 = 1,    // FP8 e4m3 scan
};

struct TcProblem {
    const float *ref;       // original dim x N FP32 set (exact fallback)
    int N;
    long long ldr;
    const float *qry;       // dim x Q FP32 queries
    int Q;
    long long ldq;
    int d, k;
    float *out_dist;
    int *out_idx;
    long long ld_out;
    void *scratch;
    size_t scratch_bytes;
    int *status;
    int num_sms;
    PhaseTimer *timer = nullptr;
    // test-only bound check of the re-rank (nullptr = off): [0] max over
    // re-ranked candidates of |a + ||q||^2 - D| / E_q (float bits), [2..3]
    // candidates checked (64-bit)
    unsigned *bound_stat = nullptr;
    int request = kTcReqBf16;
    int *host_tmp = nullptr;   // pinned, >= 2 ints: read-backs inside the run
    // the first scan's kind may switch to split BF16 after the threshold
    // pass (not with a reference set still streaming in)
    bool adaptive = true;
    // pass-2 kind forced regardless of the overflow prediction (-1: none;
    // a kind that does not fit the shape is ignored); tests and benchmarks
    int force_kind = -1;
    // the threshold sample is every (16 m)-th point of the prepared set
    // (TcRefView::sampB, whole set prepared before pass 1) rather than runs
    // of tiles (a set still streaming in): a sample spread over every part
    // of the set, whatever its order
    bool point_sample = false;
};

// A sample of the 256-point tiles: `run` consecutive tiles out of every
// `period` (unit u is tile (u / run) * period + u % run), `units` of them.
// Runs rather than single tiles keep the host-to-device copy of a sample in
// long contiguous segments.
struct TileRuns {
    int run, period, units;
    __host__ __device__ int tile(int u) const { return (u / run) * period + u % run; }
    // tile(u), tile(u + 1), ... without a division per step
    struct Iter {
        int t, r, run, skip;
        __host__ __device__ int operator*() const { return t; }
        __host__ __device__ void next() {
            if (++r == run) {
                r = 0;
                t += skip;
            } else {
                ++t;
            }
        }
    };
    __host__ __device__ Iter from(int u) const { return Iter{tile(u), u % run, run, period - run + 1}; }
    // units of the pattern among the tiles [0, t)
    __host__ __device__ int count_below(int t) const {
        return (t / period) * run + (t % period < run ? t % period : run);
    }
};

bool tc_supported(int N, int Q, int d, int k);
bool tc_fp8_supported(int d);
size_t tc_ref_bytes(int N, int d);
size_t tc_scratch_bytes(int N, int Q, int d, int k, int num_sms);
// Carves the view out of `mem` (tc_ref_bytes); a non-null `state` is reset.
TcRefView tc_carve_ref(void *mem, int N, int d, TcRefState *state);
int tc_prepare_ref(const TcRefView &v, const float *ref, int N, long long ldr, int d,
                   cudaStream_t st);
// Staged form of launch_tc, for callers that stream the reference set in:
// tc_run_begin (scratch carve, query prep), tc_run_pass1 (threshold sample:
// the tiles of tc_sample_runs must be prepared), tc_run_pass2 over 256-point
// tile ranges as they become ready (each range prepared), tc_run_finish
// (re-rank, certification, second chance; every tile prepared and the
// maximum norm final).  launch_tc = all four over the whole set.
struct TcRun {
    TcProblem P;
    TcRefView R;
    TileRuns sample;
    int p1_rows, p1_every;  // point sample: rows scanned by pass 1, in units of 16 points
    int d_pad, d_pad8, qtiles, n_tiles2, splits1, cmax;
    int kind;               // kind of the first scan's pass 2 (TcKind in knn_tc.cu)
    bool want_fp8;          // FP8 requested: pass 2 in FP8 if predicted to fit
    float s_q, scale;       // FP8: query scale, accumulator units per a unit (s_q s_r)
    long long ldf;
    __nv_bfloat16 *qB, *qBlo;
    unsigned char *q8;
    float *qn, *thr, *thr_raw, *retry, *retry_f, *retry_s, *p1, *qsub, *sd;
    int *count, *fail, *fail2, *nfail, *si, *nwide, *nsel;
    unsigned long long *cand_total, *cand;
    unsigned char *xs;
    size_t xcap;
    // incremental re-rank (tc_run_rerank_piece): running k smallest exact
    // keys per query and list entries consumed, in the exact-fallback
    // scratch (idle until certification)
    bool pieces;
    unsigned long long *run_keys;
    int *done;
};
int tc_tile_points();   // points per tile of the staged API (256)
TileRuns tc_sample_runs(int N, int Q, int d, int k, int num_sms);
// The translation (center) from the tiles of units 0, step, 2 step, ... of
// `tiles`; must run before any tile is prepared.
int tc_center_from_tiles(const TcRefView &v, const float *ref, int N, long long ldr, int d,
                         const TileRuns &tiles, int step, cudaStream_t st);
// Prepare the tiles tile0 + tiles.tile(u), u < tiles.units (the maximum
// norm accumulates; tc_prepare_ref zeroes it, computes the center and
// prepares all).
int tc_prepare_ref_tiles(const TcRefView &v, const float *ref, int N, long long ldr, int d,
                         int tile0, const TileRuns &tiles, cudaStream_t st);
// Every tile of [tile0, tile0 + n) as a pattern.
inline TileRuns contiguous_tiles(int n) { return TileRuns{1, 1, n}; }
int tc_run_begin(const TcProblem &P, const TcRefView &R, cudaStream_t st, TcRun &run);
int tc_run_pass1(TcRun &run, cudaStream_t st);
int tc_run_pass2(TcRun &run, int tile_begin, int tile_end, cudaStream_t st);
// Exact re-rank of the candidates found since the last call, merged into
// running per-query lists; when it has run after the last tc_run_pass2,
// tc_run_finish only certifies (and handles the second chance).  Optional:
// without it tc_run_finish re-ranks all candidates at once.
int tc_run_rerank_piece(TcRun &run, cudaStream_t st);
int tc_run_finish(TcRun &run, cudaStream_t st, int *host_stats);

// Prepares the optional copies of a prepared set (split-BF16 lo parts, the
// FP8 copy) now rather than on first use; synchronises `st`.  host_tmp:
// pinned, >= 2 ints.  For sets shared by several streams.
int tc_prepare_extras(const TcRefView &v, int N, int d, cudaStream_t st, int *host_tmp);

// Queues the tensor-core k-NN.  Synchronises once to learn how many queries
// failed certification; those get a second scan with thresholds that
// certify, and queries whose candidate list overflowed are recomputed by the
// exact kernel.  host_stats (pinned, 8 ints, 8-byte aligned): [0] queries
// given the second scan, [1] queries recomputed by the exact kernel, [2..3]
// scratch, [4..5] total first-scan candidates (64-bit), [6] kind of the
// first scan's pass 2, [7] kind of the second scan (-1: none); kinds are
// 0 BF16, 1 split BF16, 2 FP8 (an FP8 request whose BF16 sample pass
// predicts overflowing FP8 lists runs BF16 and reports that).
int launch_tc(const TcProblem &P, const TcRefView &R, cudaStream_t st, int *host_stats);

}  // namespace knnb200
