// swb_ext.cu -- kernel 1: banded seed extension, bit-exact with
// BandedSWScalar.align (Sources/Alignment/BandedSWScalar.swift:21-191).
//
// Layout and schedule
//   * Tasks are binned on the device by row width and row-length class:
//     int8 rows when the score bound h0 + qlen*maxScore is at most 255,
//     int16 rows when it is at most 32000, each in the context's length
//     classes (ExtBins: up to 15 bounds, defaults 32..256, chosen by
//     swb_tune_ext_bins) of the columns the task keeps: min(qlen, 2w + 2)
//     (ext_row_len: a band narrower than the query is kept as a ring) in
//     passes of kRingAllTasks tasks and up, else its query length unless
//     the query is longer than the last bound;
//     everything else (rows above the last bound, larger scores, gap costs
//     beyond a 16-bit lane) goes to the int32 bin.
//     The bounds are static, so no row ever saturates and nothing is re-run.
//     A CUB radix sort orders the tasks by (bin, longest query, longest
//     target).
//   * Every shared-memory bin is one launch of a persistent grid of one-warp
//     blocks; lane 0 claims the next 32 sorted tasks of the bin from a device
//     counter, so long tasks start first and no block holds a bin up.  The
//     bins run on their own streams and overlap.
//   * One thread owns one extension and computes two target rows per pass in
//     the 16-bit lanes of DPX s16x2 operations (swb_ext_pair.cuh), keeping the
//     reference's row storage semantics (stale cells outside the band,
//     h[end], the last-j row-max tie, z-drop, band narrowing).  The row lives
//     in shared memory, [column][thread]: a 16-bit (int8 scores) or 32-bit
//     (int16) H|E word and a query byte per column.  A class bound sizes only
//     these rows; bounds that are multiples of 16 get a kernel instance with
//     the bound as a constant.  A warp whose tasks all keep their whole query
//     runs the plain row code, else the ring form.
//   * The int32 bin runs one warp per extension for queries up to 4096
//     (swb_ext_warp.cuh) and one thread per extension over int32 rows in
//     global scratch above that (swb_ext_dp.cuh).

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "swb_device.cuh"
#include "swb_ext_dp.cuh"
#include "swb_ext_pair.cuh"
#include "swb_ext_warp.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

// Bins for n length classes (ExtBins, from the context): 0..n-1 int8 rows
// (score bound <= 255), n..2n-1 int16 rows, by query-length class; bin 2n:
// int32 rows (one warp per extension, or global scratch above kWarpMaxQ).
constexpr int kFastT = 32;                // threads per block in the shared-memory kernels
// Per pass: bin bounds (up to 32 words), the int32 bin's longest query at
// byte 256, the bins' claim counters from byte 320.
constexpr size_t kMiscBytes = 512;
constexpr int kBigT = 64;

// True when every H/E of the task fits one byte: H <= h0 + qlen*maxMat.
__device__ __forceinline__ bool fits8(int qlen, int h0, int max_mat) {
    return h0 >= 0 && (long long)h0 + (long long)qlen * (max_mat > 0 ? max_mat : 0) <= 255;
}

// Columns the two-row code keeps for a task (less one): the query length,
// or for queries longer than `ring_above` the band's ring, ext_row_len.
// A pass of fewer than kRingAllTasks tasks sets ring_above to the last
// length class, so only queries beyond the classes take rings: binning by
// ring length mixes tasks of very different row counts in a bin, and a
// small pass ends with its slowest bin -- a serving wave of 131k
// config-2-like tasks ran a third slower that way (100M -> 67M ext/s).  A
// larger pass (0: every task whose band is narrower than its query) is
// bound by throughput and gains from the occupancy (20M config-2 tasks:
// 146.4 -> 141.3 ms).  Tasks beyond the classes take the int32 bin either
// way, since a ring is never longer than the query.
constexpr size_t kRingAllTasks = size_t(1) << 22;
__device__ __host__ __forceinline__ int task_row_len(const swb_ext_task &t, const DevScoring &sc, int ring_above) {
    return t.qlen > ring_above ? ext_row_len(t.qlen, ext_band_w(t.qlen, t.w, t.end_bonus, sc)) : t.qlen;
}

// pair_ok: the gap costs fit a 16-bit lane (the two-row kernels of both row
// widths); otherwise every task takes the int32 bin.  Columns run in 16-bit
// lanes, so queries above kMaxLen take it too (and are refused there).
__device__ __forceinline__ int ext_bin(const swb_ext_task &t, const DevScoring &sc, bool pair_ok, uint32_t warp_cells,
                                       const ExtBins &bins, int ring_above) {
    if (t.qlen <= 0 || t.tlen <= 0) return 0;
    const int big = 2 * bins.n;
    const int len = task_row_len(t, sc, ring_above);
    if (!pair_ok || len > bins.q[bins.n - 1] || t.qlen > kMaxLen || !fits16(t.qlen, t.h0, sc.max_mat)) return big;
    if (warp_cells && (unsigned long long)t.qlen * (unsigned long long)t.tlen > warp_cells) return big;
    int b = 0;
    while (len > bins.q[b]) ++b;
    return fits8(t.qlen, t.h0, sc.max_mat) ? b : bins.n + b;
}

// Sort key: bin in bits 27-31, then target length (the rows a task runs) and
// row length, longest first: within a bin the tasks with the most rows start
// first, so a band narrower than its query (a short ring row over many
// target rows) does not start last and hold the bin up.
__global__ void ext_keys_kernel(const swb_ext_task *__restrict__ tasks, size_t n, DevScoring sc, int pair_ok,
                                uint32_t warp_cells, ExtBins bins, int ring_above, uint32_t *__restrict__ keys,
                                uint32_t *__restrict__ idx, int *__restrict__ big_max_q) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const swb_ext_task t = tasks[i];
    const int b = ext_bin(t, sc, pair_ok != 0, warp_cells, bins, ring_above);
    const uint32_t q = (uint32_t)min(max(b < 2 * bins.n ? task_row_len(t, sc, ring_above) : t.qlen, 0), 4095);
    const uint32_t tl = (uint32_t)min(max(t.tlen, 0), 32767);
    // Within a bin the longest tasks come first: they are claimed first, so
    // they overlap the rest instead of finishing the bin alone.
    keys[i] = ((uint32_t)b << 27) | ((32767u - tl) << 12) | (4095u - q);
    idx[i] = (uint32_t)i;
    if (b == 2 * bins.n) atomicMax(big_max_q, t.qlen);
}

// bin_start[b] = first sorted position whose bin >= b; bin_start[nbins] = n.
__global__ void bin_bounds_kernel(const uint32_t *__restrict__ sorted_keys, size_t n,
                                  uint32_t *__restrict__ bin_start, int nbins) {
    const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (n == 0) {
        if (p <= (size_t)nbins) bin_start[p] = 0;
        return;
    }
    if (p >= n) return;
    const int b = (int)(sorted_keys[p] >> 27);
    const int bprev = p == 0 ? -1 : (int)(sorted_keys[p - 1] >> 27);
    for (int bb = bprev + 1; bb <= b; ++bb) bin_start[bb] = (uint32_t)p;
    if (p == n - 1)
        for (int bb = b + 1; bb <= nbins; ++bb) bin_start[bb] = (uint32_t)n;
}

// QMAX > 0: the class bound as a constant (the multiples of 16 from 32 to
// 256); QMAX = 0: any other bound, passed in qcap.
template <int QMAX, int T, bool U8>
__global__ void __launch_bounds__(T) ext_fast_kernel(ExtArgs a, int bin, int qcap_arg) {
    extern __shared__ uint32_t sm[];
    // Rows: (qcap + 1) words of 2 (int8 scores) or 4 bytes (int16), then
    // qcap + 1 query bytes; qcap is the bin's class bound (the rows' only use
    // of it).
    const int qcap = QMAX > 0 ? QMAX : qcap_arg;
    uint16_t *he16 = reinterpret_cast<uint16_t *>(sm) + threadIdx.x;
    uint32_t *he32 = sm + threadIdx.x;
    uint8_t *qc = reinterpret_cast<uint8_t *>(sm) + (size_t)(qcap + 1) * T * (U8 ? 2 : 4) + threadIdx.x;
    static_assert(T == 32, "one warp per block: the warp claims its tasks together");
    const uint32_t lo = a.bin_start[bin], hi = a.bin_start[bin + 1];
    unsigned long long cells = 0;
    const uint32_t span = hi - lo;
    // Resident blocks claim the next 32 sorted tasks of the bin from a
    // counter, so blocks that draw long tasks do not hold up the bin.
    for (;;) {
        uint32_t base = 0;
        if (threadIdx.x == 0) base = atomicAdd(a.claim + bin, (uint32_t)T);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= span) break;
        const uint32_t pos = lo + base + threadIdx.x;
        uint32_t ti = 0;
        swb_ext_task tk{};
        if (pos < hi) {
            ti = a.order[pos];
            tk = a.tasks[ti];
        }
        // The ring form only for warps that hold a task whose band is
        // narrower than its query.
        const bool ring = __any_sync(0xFFFFFFFFu, pos < hi && task_row_len(tk, a.sc, a.ring_above) < tk.qlen);
        if (pos < hi) {
            swb_ext_result r;
            const bool sym = a.sc.o_del + a.sc.e_del == a.sc.o_ins + a.sc.e_ins;
            if (ring) {
                if constexpr (U8) {
                    if (sym) ext_pair_one<T, true, false, true>(a, tk, he16, qc, r, cells);
                    else ext_pair_one<T, false, false, true>(a, tk, he16, qc, r, cells);
                } else {
                    if (sym) ext_pair_one<T, true, true, true>(a, tk, he32, qc, r, cells);
                    else ext_pair_one<T, false, true, true>(a, tk, he32, qc, r, cells);
                }
            } else {
                if constexpr (U8) {
                    if (sym) ext_pair_one<T, true, false, false>(a, tk, he16, qc, r, cells);
                    else ext_pair_one<T, false, false, false>(a, tk, he16, qc, r, cells);
                } else {
                    if (sym) ext_pair_one<T, true, true, false>(a, tk, he32, qc, r, cells);
                    else ext_pair_one<T, false, true, false>(a, tk, he32, qc, r, cells);
                }
            }
            a.out[ti] = r;
        }
    }
    add_cells(a.cells + kCntExtBin0 + bin, cells);
}

// Queries above 256 bases or scores beyond int16, up to kWarpMaxQ bases: one
// warp per extension (swb_ext_warp.cuh), rows in shared memory, warps claim
// tasks of the bin one at a time.
__global__ void __launch_bounds__(256) ext_warp_kernel(ExtArgs a, int bin, int qcap) {
    extern __shared__ __align__(16) uint8_t wsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t stride = ((size_t)(qcap + 1) * 8 + (size_t)qcap + 15) & ~(size_t)15;
    int *h = reinterpret_cast<int *>(wsm + warp * stride);
    int *e = h + (qcap + 1);
    uint8_t *qc = reinterpret_cast<uint8_t *>(e + (qcap + 1));
    const uint32_t lo = a.bin_start[bin], hi = a.bin_start[bin + 1];
    const uint32_t span = hi - lo;
    unsigned long long cells = 0;
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(a.claim + bin, 1u);
        k = __shfl_sync(0xFFFFFFFFu, k, 0);
        if (k >= span) break;
        const uint32_t ti = a.order[lo + k];
        const swb_ext_task tk = a.tasks[ti];
        if (tk.qlen > qcap) continue;                 // the global-scratch kernel's
        swb_ext_result r;
        ext_warp_one(a, tk, h, e, qc, r, cells);
        if (lane == 0) a.out[ti] = r;
        __syncwarp();
    }
    add_cells(a.cells + kCntExtBin0 + bin, cells);
}

// Queries above kWarpMaxQ: one thread per extension over int32 rows in
// global scratch (tasks with qlen <= skip_le belong to the warp kernel).
__global__ void __launch_bounds__(kBigT) ext_global_kernel(ExtArgs a, int bin, int *h, int *e, uint8_t *q,
                                                           size_t nslots, int skip_le) {
    const uint32_t lo = a.bin_start[bin], hi = a.bin_start[bin + 1];
    const size_t slot = blockIdx.x * (size_t)kBigT + threadIdx.x;
    Global32 st{h, e, q, nslots, slot};
    unsigned long long cells = 0;
    const uint32_t span = hi - lo;
    const uint32_t iters = (uint32_t)((span + nslots - 1) / nslots);
    for (uint32_t it = 0; it < iters; ++it) {
        const size_t pos = lo + (size_t)it * nslots + slot;
        if (pos < hi) {
            const uint32_t ti = a.order[pos];
            const swb_ext_task tk = a.tasks[ti];
            if (tk.qlen <= skip_le) continue;
            swb_ext_result r;
            ext_one(a, tk, st, r, cells);
            a.out[ti] = r;
        }
    }
    add_cells(a.cells + kCntExtBin0 + bin, cells);
}

// ------------------------------------------------------ plain comparator
// The batch as the reference's GPU dispatcher shapes it
// (BandedSWDispatcher.dispatchBatch16, Sources/MetalSW/BandedSWDispatcher.swift:107-160):
// one launch, one task per thread in input order -- no sort, no length bins,
// no claiming -- running the same two-row code (ext_pair_one) with rows sized
// for the batch's longest query: int8 rows when every task's score bound fits
// a byte, else int16 rows.  It differs from the binned pass only in the
// batching, which makes it the baseline the batching is measured against.
// Tasks the two-row code cannot take (queries above kExtSmemMaxQ, scores
// beyond int16, gap costs beyond a 16-bit lane) are collected, unordered,
// into one list that the int32 kernels of the binned pass run.

// True when the two-row code takes the task in the plain launch.
__device__ __forceinline__ bool plain_pair_task(const swb_ext_task &t, int max_mat, bool pair_ok) {
    return t.qlen <= 0 || t.tlen <= 0 || (pair_ok && t.qlen <= kExtSmemMaxQ && fits16(t.qlen, t.h0, max_mat));
}

// Shape of a plain batch (device words in the pass's misc block).
struct PlainShape {
    int pair_max_q;   // longest query the plain launch takes (at least 1 when it takes any task; 0: none)
    int need16;       // 1 when one of them needs int16 rows
    int big_max_q;    // longest query of the int32 list
};
constexpr size_t kPlainShapeOff = 64;

// Classifies every task: the plain launch's row shape, and the int32 list
// (order[0 .. bin_start[1]) with bin_start[0] = 0).
__global__ void ext_plain_scan_kernel(const swb_ext_task *__restrict__ tasks, size_t n, int max_mat, int pair_ok,
                                      uint32_t *__restrict__ bin_start, uint32_t *__restrict__ order,
                                      PlainShape *__restrict__ shape) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int pq = 0, n16 = 0, bq = 0;
    if (i < n) {
        const swb_ext_task t = tasks[i];
        if (plain_pair_task(t, max_mat, pair_ok != 0)) {
            pq = t.qlen > 0 && t.tlen > 0 ? t.qlen : 1;   // an empty task still needs its zero result
            n16 = t.qlen > 0 && t.tlen > 0 && !fits8(t.qlen, t.h0, max_mat);
        } else {
            bq = t.qlen;
            order[atomicAdd(&bin_start[1], 1u)] = (uint32_t)i;
        }
    }
    pq = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)pq);
    n16 = (int)__reduce_or_sync(0xFFFFFFFFu, (unsigned)n16);
    bq = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)bq);
    if ((threadIdx.x & 31) == 0) {
        if (pq) atomicMax(&shape->pair_max_q, pq);
        if (n16) atomicOr(&shape->need16, 1);
        if (bq) atomicMax(&shape->big_max_q, bq);
    }
}

template <int T, bool U8>
__global__ void __launch_bounds__(T) ext_plain_kernel(ExtArgs a, size_t n, int qcap, int pair_ok) {
    extern __shared__ uint32_t sm[];
    uint16_t *he16 = reinterpret_cast<uint16_t *>(sm) + threadIdx.x;
    uint32_t *he32 = sm + threadIdx.x;
    uint8_t *qc = reinterpret_cast<uint8_t *>(sm) + (size_t)(qcap + 1) * T * (U8 ? 2 : 4) + threadIdx.x;
    unsigned long long cells = 0;
    const size_t pos = blockIdx.x * (size_t)T + threadIdx.x;
    if (pos < n) {
        const swb_ext_task tk = a.tasks[pos];
        if (plain_pair_task(tk, a.sc.max_mat, pair_ok != 0)) {
            swb_ext_result r;
            const bool sym = a.sc.o_del + a.sc.e_del == a.sc.o_ins + a.sc.e_ins;
            if constexpr (U8) {
                if (sym) ext_pair_one<T, true, false, false>(a, tk, he16, qc, r, cells);
                else ext_pair_one<T, false, false, false>(a, tk, he16, qc, r, cells);
            } else {
                if (sym) ext_pair_one<T, true, true, false>(a, tk, he32, qc, r, cells);
                else ext_pair_one<T, false, true, false>(a, tk, he32, qc, r, cells);
            }
            a.out[pos] = r;
        }
    }
    add_cells(a.cells + kCntExtBin0, cells);
}

// A 16-bit (int8 scores) or 32-bit (int16) word and a query byte per column.
size_t fast_smem_bytes(int qcap, bool u8) {
    return ((size_t)(qcap + 1) * kFastT * (u8 ? sizeof(uint16_t) : sizeof(uint32_t)) + (size_t)(qcap + 1) * kFastT +
            15) &
           ~(size_t)15;
}

// Profile names of the bins, kept for the life of the process.
const char *bin_name(bool u8, int qcap) {
    static std::mutex mu;
    static std::set<std::string> names;
    std::lock_guard<std::mutex> lk(mu);
    return names.insert(std::string(u8 ? "ext_u8_q" : "ext_i16_q") + std::to_string(qcap)).first->c_str();
}

using FastKernel = void (*)(ExtArgs, int, int);

template <bool U8, int... Q>
FastKernel fast_kernel_for(int qcap, std::integer_sequence<int, Q...>) {
    FastKernel k = ext_fast_kernel<0, kFastT, U8>;
    ((qcap == 32 + 16 * Q ? (void)(k = ext_fast_kernel<32 + 16 * Q, kFastT, U8>) : (void)0), ...);
    return k;
}

// The kernel instance for a class bound: the constant-bound one for the
// multiples of 16 from 32 to 256, else the runtime-bound one.
FastKernel fast_kernel(bool u8, int qcap) {
    return u8 ? fast_kernel_for<true>(qcap, std::make_integer_sequence<int, 15>{})
              : fast_kernel_for<false>(qcap, std::make_integer_sequence<int, 15>{});
}

// Resident one-warp blocks per SM of the shared-memory kernel for a class bound.
int fast_occupancy(bool u8, int qcap) {
    static int cache[2][kExtSmemMaxQ + 1];
    static std::once_flag once;
    std::call_once(once, [] {
        for (auto &row : cache)
            for (int &v : row) v = -1;
    });
    int &occ = cache[u8 ? 1 : 0][qcap];
    if (occ < 0) {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fast_kernel(u8, qcap), kFastT, fast_smem_bytes(qcap, u8)) !=
            cudaSuccess)
            return -1;
        occ = o < 1 ? 1 : o;
    }
    return occ;
}

int launch_fast(swb_ctx *ctx, const ExtArgs &a, int bin, bool u8, int qcap, size_t n, cudaStream_t s) {
    const int occ = fast_occupancy(u8, qcap);
    if (occ < 0) return check_cuda(cudaGetLastError(), "occupancy query");
    const size_t grid = std::min<size_t>((n + kFastT - 1) / kFastT, (size_t)ctx->sm_count * occ);
    if (grid == 0) return SWB_OK;
    const size_t smem = fast_smem_bytes(qcap, u8);
    ProfScope ps(ctx, s, ctx->prof_on ? bin_name(u8, qcap) : nullptr, kCntExtBin0 + bin);
    fast_kernel(u8, qcap)<<<(unsigned)grid, kFastT, smem, s>>>(a, bin, qcap);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    return SWB_OK;
}

}  // namespace

int ext_reserve(swb_ctx *ctx, size_t cap) {
    if (cap > 0x7FFFFFF0ull) return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 tasks in one batch");
    int rc;
    size_t tmp_bytes = 0;
    SWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                             (uint32_t *)nullptr, (uint32_t *)nullptr, (int)cap, 0, 32, ctx->stream));
    if ((rc = ensure_dev(ctx, ctx->d_keys, cap * 4)) || (rc = ensure_dev(ctx, ctx->d_keys2, cap * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_idx, cap * 4)) || (rc = ensure_dev(ctx, ctx->d_idx2, 2 * cap * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_misc, 2 * kMiscBytes)) || (rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp_bytes)))
        return rc;
    return SWB_OK;
}

int launch_ext(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases,
               const swb_ext_task *d_tasks, size_t n, swb_ext_result *d_out,
               unsigned long long *d_cells, cudaStream_t s, int max_q_hint, uint32_t warp_cells,
               const ExtPipe *pipe) {
    if (n == 0) return SWB_OK;
    if (n > 0x7FFFFFF0ull) return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 tasks in one batch");
    if (pipe && n > pipe->cap) return set_error(SWB_ERR_INVALID_ARG, "pass larger than its scratch set");
    int rc;
    // keys, keys2, idx and the sort's temporary storage are used by the
    // launching stream only; the sorted order (idx2) and the bin bounds and
    // claim counters (misc) are read by the bins, one set per pipelined slot.
    const size_t set = pipe ? pipe->cap : n;
    const int slot = pipe ? pipe->slot : 0;
    if ((rc = ensure_dev(ctx, ctx->d_keys, n * 4)) || (rc = ensure_dev(ctx, ctx->d_keys2, n * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_idx, n * 4)) || (rc = ensure_dev(ctx, ctx->d_idx2, (slot + 1) * set * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_misc, (slot + 1) * kMiscBytes)))
        return rc;
    // The context's length classes at the time of the call: the keys and the
    // launches below use the same copy.
    const ExtBins bins = ctx->ext_bins;
    const int ring_above = n >= kRingAllTasks ? 0 : bins.q[bins.n - 1];
    const int nbins = 2 * bins.n + 1, big = 2 * bins.n;
    uint32_t *keys = (uint32_t *)ctx->d_keys.p, *keys2 = (uint32_t *)ctx->d_keys2.p;
    uint32_t *idx = (uint32_t *)ctx->d_idx.p, *idx2 = (uint32_t *)ctx->d_idx2.p + (size_t)slot * set;
    char *misc = (char *)ctx->d_misc.p + slot * kMiscBytes;
    uint32_t *bin_start = (uint32_t *)misc;                   // nbins + 1 words
    int *big_max_q = (int *)(misc + 256);
    uint32_t *claim = (uint32_t *)(misc + 320);               // nbins claim counters
    SWB_CUDA(cudaMemsetAsync(misc + 256, 0, kMiscBytes - 256, s));   // big_max_q and the counters
    const unsigned tb = 256;
    {
        ProfScope ps(ctx, s, "ext_keys", -1);
        // Two target rows per pass on 16-bit lanes: the gap costs must fit a lane.
        const int pair_ok = sc.o_del + sc.e_del <= 32767 && sc.o_ins + sc.e_ins <= 32767;
        ext_keys_kernel<<<(unsigned)((n + tb - 1) / tb), tb, 0, s>>>(d_tasks, n, sc, pair_ok, warp_cells, bins,
                                                                       ring_above, keys, idx, big_max_q);
    }
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0;
    SWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, idx, idx2, (int)n, 0, 32, s));
    if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp_bytes))) return rc;
    {
        ProfScope ps(ctx, s, "cub_radix_sort", -1);
        SWB_CUDA(cub::DeviceRadixSort::SortPairs(ctx->d_sort_tmp.p, tmp_bytes, keys, keys2, idx, idx2,
                                                 (int)n, 0, 32, s));
    }
    {
        ProfScope ps(ctx, s, "bin_bounds", -1);
        bin_bounds_kernel<<<(unsigned)((n + tb - 1) / tb), tb, 0, s>>>(keys2, n, bin_start, nbins);
    }
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());

    // Global-scratch bin: size its scratch from the longest query in it.
    int max_q = max_q_hint;
    if (max_q < 0) {
        SWB_CUDA(cudaMemcpyAsync(&max_q, big_max_q, sizeof(int), cudaMemcpyDeviceToHost, s));
        SWB_CUDA(cudaStreamSynchronize(s));
    }
    if (max_q > kMaxLen) return set_error(SWB_ERR_TOO_LARGE, "query longer than 65535 bases");
    const size_t nslots = (size_t)ctx->sm_count * 4 * kBigT;
    const size_t cols = (size_t)max_q + 1;
    if (max_q > kWarpMaxQ) {
        const size_t bytes = cols * nslots * (2 * sizeof(int) + 1) + 256;
        if ((rc = ensure_dev(ctx, ctx->d_scratch, bytes))) return rc;
    }
    // Warp kernel shape for the big bin: warps per block from the rows' size.
    const int wq = imin(max_q, kWarpMaxQ);
    const size_t wstride = ((size_t)(wq + 1) * 8 + (size_t)wq + 15) & ~(size_t)15;
    int wwarps = 0, wblocks = 0;
    if (max_q > 0) {
        wwarps = (int)std::max<size_t>(1, std::min<size_t>(8, (size_t)(200 * 1024) / wstride));
        SWB_CUDA(cudaFuncSetAttribute(ext_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(wwarps * wstride)));
        SWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wblocks, ext_warp_kernel, wwarps * 32,
                                                               wwarps * wstride));
        wblocks = imax(wblocks, 1) * ctx->sm_count;
    }

    // Fork: every bin runs on its own stream after the sort, then joins back
    // (into the pipeline's join stream for pipelined passes).
    ExtArgs a{sc, d_bases, ctx->d_pac, d_tasks, d_out, idx2, bin_start, d_cells, claim, ring_above};
    const cudaStream_t js = pipe ? pipe->join : s;
    ProfScope pass(ctx, s, pipe ? nullptr : "ext_pass", -1);   // fork to join, on the launching stream
    SWB_CUDA(cudaEventRecord(ctx->fork_ev, s));
    for (int b = 0; b < nbins; ++b) {
        cudaStream_t sb = ctx->side[b];
        SWB_CUDA(cudaStreamWaitEvent(sb, ctx->fork_ev, 0));
        if (b < big) {
            if ((rc = launch_fast(ctx, a, b, b < bins.n, bins.q[b % bins.n], n, sb))) return rc;
        } else if (max_q > 0) {
            ProfScope ps(ctx, sb, "ext_big_i32", kCntExtBin0 + big);
            ext_warp_kernel<<<(unsigned)wblocks, wwarps * 32, wwarps * wstride, sb>>>(a, big, wq);
            ctx->launches++;
            SWB_CUDA(cudaGetLastError());
            if (max_q > kWarpMaxQ) {
                int *hbuf = (int *)ctx->d_scratch.p;
                int *ebuf = hbuf + cols * nslots;
                uint8_t *qbuf = (uint8_t *)(ebuf + cols * nslots);
                ext_global_kernel<<<(unsigned)(nslots / kBigT), kBigT, 0, sb>>>(a, big, hbuf, ebuf, qbuf, nslots, wq);
                ctx->launches++;
                SWB_CUDA(cudaGetLastError());
            }
        }
        SWB_CUDA(cudaEventRecord(ctx->join_ev[b], sb));
        SWB_CUDA(cudaStreamWaitEvent(js, ctx->join_ev[b], 0));
    }
    return SWB_OK;
}

// Host-side twin of the device bin test: the longest query among
// tasks[lo, hi) that the int32 bin takes under the context's length classes
// (sizes its kernels' rows).
int ext_big_max_q_range(const swb_ctx *ctx, const swb_ext_task *tasks, size_t lo, size_t hi, const DevScoring &sc) {
    const bool pair_ok = sc.o_del + sc.e_del <= 32767 && sc.o_ins + sc.e_ins <= 32767;
    const int top = ctx->ext_bins.q[ctx->ext_bins.n - 1];
    int m = 0;
    for (size_t i = lo; i < hi; ++i) {
        const swb_ext_task &t = tasks[i];
        if (t.qlen <= 0 || t.tlen <= 0) continue;
        if (!pair_ok || task_row_len(t, sc, top) > top || t.qlen > kMaxLen || !fits16(t.qlen, t.h0, sc.max_mat))
            m = t.qlen > m ? t.qlen : m;
    }
    return m;
}

// The plain comparator (see ext_plain_kernel): one launch of the two-row code
// over the batch in input order, then the int32 kernels over the tasks it
// cannot take.  The batch's shape (row length and width) is read back from
// the device, which synchronises `s` once.
int launch_ext_plain(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases, const swb_ext_task *d_tasks,
                     size_t n, swb_ext_result *d_out, unsigned long long *d_cells, cudaStream_t s) {
    if (n == 0) return SWB_OK;
    if (n > 0x7FFFFFF0ull) return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 tasks in one batch");
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_idx2, n * 4)) || (rc = ensure_dev(ctx, ctx->d_misc, kMiscBytes))) return rc;
    char *misc = (char *)ctx->d_misc.p;
    uint32_t *bin_start = (uint32_t *)misc;                 // {0, int32-list length}
    PlainShape *shape = (PlainShape *)(misc + kPlainShapeOff);
    uint32_t *claim = (uint32_t *)(misc + 320);
    uint32_t *order = (uint32_t *)ctx->d_idx2.p;
    SWB_CUDA(cudaMemsetAsync(misc, 0, kMiscBytes, s));
    const int pair_ok = sc.o_del + sc.e_del <= 32767 && sc.o_ins + sc.e_ins <= 32767;
    const unsigned tb = 256;
    {
        ProfScope ps(ctx, s, "ext_plain_scan", -1);
        ext_plain_scan_kernel<<<(unsigned)((n + tb - 1) / tb), tb, 0, s>>>(d_tasks, n, sc.max_mat, pair_ok, bin_start,
                                                                            order, shape);
    }
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    PlainShape sh{};
    SWB_CUDA(cudaMemcpyAsync(&sh, shape, sizeof(sh), cudaMemcpyDeviceToHost, s));
    SWB_CUDA(cudaStreamSynchronize(s));
    if (sh.big_max_q > kMaxLen) return set_error(SWB_ERR_TOO_LARGE, "query longer than 65535 bases");
    ExtArgs a{sc, d_bases, ctx->d_pac, d_tasks, d_out, order, bin_start, d_cells, claim};
    if (sh.pair_max_q > 0) {
        // Rows for the longest query, in the kernel's word width; one
        // 32-thread block per 32 consecutive tasks.
        const int qcap = imin(sh.pair_max_q, kExtSmemMaxQ);
        const bool u8 = sh.need16 == 0;
        const size_t smem = fast_smem_bytes(qcap, u8);
        ProfScope ps(ctx, s, "ext_plain", kCntExtBin0);
        const unsigned grid = (unsigned)((n + kFastT - 1) / kFastT);
        if (u8) ext_plain_kernel<kFastT, true><<<grid, kFastT, smem, s>>>(a, n, qcap, pair_ok);
        else ext_plain_kernel<kFastT, false><<<grid, kFastT, smem, s>>>(a, n, qcap, pair_ok);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    if (sh.big_max_q > 0) {
        const int wq = imin(sh.big_max_q, kWarpMaxQ);
        const size_t wstride = ((size_t)(wq + 1) * 8 + (size_t)wq + 15) & ~(size_t)15;
        const int wwarps = (int)std::max<size_t>(1, std::min<size_t>(8, (size_t)(200 * 1024) / wstride));
        int wblocks = 0;
        SWB_CUDA(cudaFuncSetAttribute(ext_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(wwarps * wstride)));
        SWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wblocks, ext_warp_kernel, wwarps * 32,
                                                               wwarps * wstride));
        wblocks = imax(wblocks, 1) * ctx->sm_count;
        {
            ProfScope ps(ctx, s, "ext_plain_i32", kCntExtBin0 + 1);
            ext_warp_kernel<<<(unsigned)wblocks, wwarps * 32, wwarps * wstride, s>>>(a, 0, wq);
        }
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
        if (sh.big_max_q > kWarpMaxQ) {
            const size_t nslots = (size_t)ctx->sm_count * 4 * kBigT;
            const size_t cols = (size_t)sh.big_max_q + 1;
            if ((rc = ensure_dev(ctx, ctx->d_scratch, cols * nslots * (2 * sizeof(int) + 1) + 256))) return rc;
            int *hbuf = (int *)ctx->d_scratch.p;
            int *ebuf = hbuf + cols * nslots;
            uint8_t *qbuf = (uint8_t *)(ebuf + cols * nslots);
            ext_global_kernel<<<(unsigned)(nslots / kBigT), kBigT, 0, s>>>(a, 0, hbuf, ebuf, qbuf, nslots, wq);
            ctx->launches++;
            SWB_CUDA(cudaGetLastError());
        }
    }
    return SWB_OK;
}

}  // namespace swb
