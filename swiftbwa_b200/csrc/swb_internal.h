// swb_internal.h -- declarations shared by the CUDA translation units of
// libswb_cuda.so.  Not part of the public C ABI (include/swb_cuda.h).
#pragma once

#include <initializer_list>

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/swb_cuda.h"

namespace swb {

// -------------------------------------------------------------- limits
// Queries up to this length run in the shared-memory extension kernels;
// longer ones (and scores that do not fit int16) use the global-scratch
// int32 kernel.
constexpr int kExtSmemMaxQ = 256;
// Hard cap on any query or target length (the reference's extension target
// window is capped at 10000 bases, ExtensionAligner.swift:214,277).
constexpr int kMaxLen = 65535;

// Device-side copy of swb_scoring plus derived constants.
struct DevScoring {
    int a, b, o_ins, e_ins, o_del, e_del, zdrop, pen_clip5, pen_clip3, band_width, min_seed_len;
    int max_mat;        // max over the 5x5 matrix, starting from 0 (BandedSWScalar.swift:54-58)
};

inline DevScoring make_dev_scoring(const swb_scoring &s) {
    DevScoring d{s.a, s.b, s.o_ins, s.e_ins, s.o_del, s.e_del, s.zdrop, s.pen_clip5, s.pen_clip3,
                 s.band_width, s.min_seed_len, 0};
    int m = 0;
    // scoringMatrix(): a on the diagonal, -b off it, -1 for N (ScoringParameters.swift:65-73)
    int vals[3] = {(int)(int8_t)s.a, (int)(int8_t)(-s.b), -1};
    for (int v : vals) m = v > m ? v : m;
    d.max_mat = m;
    return d;
}

// True when every H/E of an extension task fits int16: H <= h0 + qlen*maxMat
// (each row adds at most the best match score) and E, F <= H.
__device__ __host__ __forceinline__ bool fits16(int qlen, int h0, int max_mat) {
    long long hi = (long long)h0 + (long long)qlen * (max_mat > 0 ? max_mat : 0);
    return h0 >= 0 && hi <= 32000;
}

// The band half-width an extension runs with: the task's w clamped by the
// longest insertion and deletion that can still score
// (BandedSWScalar.swift:52-62).
__device__ __host__ __forceinline__ int ext_band_w(int qlen, int w, int end_bonus, const DevScoring &sc) {
    const int maxIns = (int)((double)(qlen * sc.max_mat + end_bonus - sc.o_ins) / (double)sc.e_ins + 1.0);
    w = w < (maxIns > 1 ? maxIns : 1) ? w : (maxIns > 1 ? maxIns : 1);
    const int maxDel = (int)((double)(qlen * sc.max_mat + end_bonus - sc.o_del) / (double)sc.e_del + 1.0);
    return w < (maxDel > 1 ? maxDel : 1) ? w : (maxDel > 1 ? maxDel : 1);
}

// Columns a two-row extension keeps in shared memory, less one: the whole
// query (qlen + 1 words), or, when the band is narrower than the query, a
// ring of 2w + 3 words -- every column a row pair reads or writes lies within
// [i - w, i + w + 2] of its first row i.
__device__ __host__ __forceinline__ int ext_row_len(int qlen, int w_band) {
    return (w_band >= 0 && 2LL * w_band + 2 < (long long)qlen) ? 2 * w_band + 2 : qlen;
}

// Cell counters: one per kernel family (indices below) in ctx->d_counters.
enum CounterIdx {
    kCntExtBin0 = 0,      // extension bins 0..30 -> 0..30
    kCntGlobal = 32,
    kCntLocalStriped = 33,
    kCntLocalScalar = 34,
    kCntSeed = 35,        // backward extensions of the SMEM search
    kNumCounters = 40
};

// Extension length classes: query-length upper bounds of the shared-memory
// bins, ascending; each class has an int8-row and an int16-row bin, and one
// more bin takes everything else (int32 rows).  The bin index sits in 5 bits
// of the sort key, so 2 * 15 + 1 = 31 bins at most.
constexpr int kMaxLenClasses = 15;
constexpr int kMaxExtBins = 2 * kMaxLenClasses + 1;
struct ExtBins {
    int n = 10;
    int q[kMaxLenClasses] = {32, 48, 64, 80, 96, 112, 128, 160, 192, 256};
};

constexpr int kSideStreams = 32;   // concurrent bin launches per context
// Host-entry batches up to this many tasks run the one-launch form
// (launch_ext_plain): measured on B200, 10k config-0 tasks take 0.26 ms
// that way against 0.36 ms binned; from ~20k mixed-length tasks on, the
// binned pass is faster.
constexpr size_t kExtPlainMaxTasks = 16384;
constexpr int kMaxChunks = 16;     // pipelined chunks of one synchronous batch call

// ------------------------------------------------------------ a device arena
// Grow-only device buffer owned by a context, counted against its budget.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
};

}  // namespace swb

// ------------------------------------------------------------------ context
struct swb_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    // fork/join of the per-bin kernels
    cudaStream_t side[swb::kSideStreams] = {};
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t join_ev[swb::kSideStreams] = {};
    // host<->device copy streams and per-chunk events of the pipelined batch calls
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t chunk_in[swb::kMaxChunks] = {}, chunk_done[swb::kMaxChunks] = {};
    size_t budget = 0;       // cap on bytes the context allocates on the device
    size_t allocated = 0;    // bytes currently allocated
    std::mutex mu;
    // resident 2-bit reference (.pac layout)
    uint8_t *d_pac = nullptr;
    bool pac_owned = true;        // false for a server lane sharing its parent's reference
    uint64_t ref_bases = 0;
    size_t pac_bytes = 0;
    // named scratch buffers (grow-only)
    swb::DevBuf d_bases, d_tasks, d_out, d_keys, d_keys2, d_idx, d_idx2, d_sort_tmp, d_misc,
        d_scratch, d_cigar, d_aux, d_chain;
    swb::HostBuf h_in, h_out;
    // resident FM index (swb_upload_bwt): checkpoints, counts, length, sentinel
    swb::DevBuf d_bwt, d_seed;
    int64_t bwt_count[5] = {0, 0, 0, 0, 0};
    int64_t bwt_length = 0, bwt_sentinel = -1;
    uint64_t bwt_ncp = 0;
    unsigned long long launches = 0;
    double last_ms = 0.0;
    unsigned long long last_cells = 0;
    // per-kernel profiling
    unsigned long long *d_counters = nullptr;   // swb::kNumCounters cells counters
    swb::ExtBins ext_bins;   // extension length classes (swb_set_ext_bins / swb_tune_ext_bins)
    bool prof_on = false;
    struct ProfRec {
        const char *name;
        int counter;          // counter index or -1
        cudaEvent_t a, b;
    };
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
};

namespace swb {

// Error plumbing (thread-local message, set by every failing call).
int set_error(int code, const std::string &msg);
// Scoring ranges every entry point accepts (SWB_ERR_INVALID_ARG otherwise).
int validate_scoring(const swb_scoring *sc);
int check_cuda(cudaError_t e, const char *what);
#define SWB_CUDA(call)                                               \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return ::swb::check_cuda(_e, #call);  \
    } while (0)

// Brackets one kernel launch with events when profiling is on.
struct ProfScope {
    swb_ctx *ctx;
    cudaStream_t s;
    int idx = -1;
    ProfScope(swb_ctx *c, cudaStream_t st, const char *name, int counter);
    ~ProfScope();
};

// Downloads of a call's results into (pageable) caller arrays through the
// context's pinned staging buffer: one async copy each into pinned memory,
// then host threads unpack.  Synchronises `st` (recording after_copies, when
// given, once the copies are queued).  Pageable downloads are much slower.
struct DevSpan {
    const void *dev;
    void *dst;
    size_t bytes;
};
void par_copy(void *dst, const void *src, size_t bytes);
// True when p lies in page-locked host memory (cudaHostAlloc or registered).
bool is_pinned(const void *p);
int d2h_staged(swb_ctx *ctx, cudaStream_t st, std::initializer_list<DevSpan> parts, cudaEvent_t after_copies = nullptr);

// Grow-only allocation against the context budget.
int ensure_dev(swb_ctx *ctx, DevBuf &b, size_t bytes);
int ensure_host(swb_ctx *ctx, HostBuf &b, size_t bytes);

// -------------------------------------------------------- kernel launchers
// All enqueue on `stream` and return SWB_OK or an error status.  `cells`
// is a device counter (unsigned long long) the kernels add DP cells to.

// Extension (kernel 1).  d_tasks/d_out are device arrays of n tasks/results.
// warp_cells > 0: tasks with more DP cells (qlen * tlen) run one warp per
// extension (latency), otherwise their length bin's thread-per-task kernel.
// Pipelined passes: two scratch sets let pass k+1 sort and start its bins
// while pass k's bins finish.  The caller sizes the scratch with
// ext_reserve(cap) first and makes `stream` wait for pass k-2 to finish
// before pass k reuses its set; the bins join into `join` instead of `stream`.
struct ExtPipe {
    int slot;            // scratch set 0 or 1
    size_t cap;          // tasks per scratch set (every pass has n <= cap)
    cudaStream_t join;   // stream that waits for the bins
};
int ext_reserve(swb_ctx *ctx, size_t cap);
int launch_ext(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases,
               const swb_ext_task *d_tasks, size_t n, swb_ext_result *d_out,
               unsigned long long *d_cells, cudaStream_t stream, int max_q_hint,
               uint32_t warp_cells = 0, const ExtPipe *pipe = nullptr);

// The plain one-launch-per-batch comparator of the extension pass (the same
// two-row kernel over the batch in input order; no sort, bins or claiming).
// Reads the batch's shape back from the device: synchronises `stream` once.
int launch_ext_plain(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases, const swb_ext_task *d_tasks,
                     size_t n, swb_ext_result *d_out, unsigned long long *d_cells, cudaStream_t stream);

// Banded global + traceback (kernel 2).  Tasks with qlen <= kGlobalSmemMaxQ
// run in the shared-memory kernel, longer ones in the global-scratch kernel;
// the shape gives each group's count and largest query / target.
constexpr int kGlobalSmemMaxQ = 256;
// The int16-row NW kernel is exact for a task when (qlen + tlen + 2) times
// (a + the largest single-step cost) stays below 16000 (swb_global.cu).
__host__ __device__ inline int nw_i16_cost(int a, int b, int o_del, int e_del, int o_ins, int e_ins) {
    int p = o_del + e_del;
    p = p > o_ins + e_ins ? p : o_ins + e_ins;
    p = p > b ? p : b;
    return a + (p > 1 ? p : 1);
}
__host__ __device__ inline bool nw_fits_i16(int qlen, int tlen, int cost) {
    return (long long)(qlen + tlen + 2) * cost < 16000;
}
struct GlobalShape {
    size_t n_small = 0, n_small16 = 0, n_big = 0;
    int small_q = 0, small_t = 0, big_q = 0, big_t = 0;
    void add(int qlen, int tlen, int cost16) {
        if (qlen <= kGlobalSmemMaxQ) {
            ++n_small;
            if (nw_fits_i16(qlen, tlen, cost16)) ++n_small16;
            small_q = std::max(small_q, qlen);
            small_t = std::max(small_t, tlen);
        } else {
            ++n_big;
            big_q = std::max(big_q, qlen);
            big_t = std::max(big_t, tlen);
        }
    }
};
int launch_global(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases,
                  const swb_global_task *d_tasks, size_t n, swb_global_result *d_res,
                  uint32_t *d_cigar, unsigned long long *d_cells, cudaStream_t stream,
                  const GlobalShape &shape);

// Local SW for mate rescue (kernel 3).
int launch_local(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases,
                 const swb_local_task *d_tasks, size_t n, swb_local_result *d_out,
                 unsigned long long *d_cells, cudaStream_t stream, int max_q, int max_t);

}  // namespace swb
