// swb_ext.cu -- kernel 1: banded seed extension, bit-exact with
// BandedSWScalar.align (Sources/Alignment/BandedSWScalar.swift:21-191).
//
// Layout and schedule
//   * One thread owns one extension.  Its DP row (H and E per query column)
//     lives in shared memory as one 32-bit word per column, int16 H in the
//     low half and int16 E in the high half, interleaved across the block's
//     threads ([column][thread]) so every access is bank-conflict free.  The
//     query is staged beside it, 4 codes per word.  This keeps the
//     reference's storage semantics exactly: cells outside the current band
//     keep their stale values, h[end] receives the last H of the row, and
//     narrowing scans the same words the Swift loop scans.
//   * Tasks are binned on the device by query length (<=32, 64, 128, 256)
//     and radix-sorted by (bin, qlen, tlen) so a warp's threads walk rows of
//     similar shape; each bin runs a kernel instantiated for its row size
//     with a grid-stride loop over its slice of the sorted order.
//   * Tasks whose scores could leave int16 (h0 + qlen*maxScore > 32000) or
//     whose query exceeds 256 run in an int32 kernel with the row in global
//     scratch, same code path.
#include <cub/device/device_radix_sort.cuh>

#include "swb_device.cuh"
#include "swb_ext_dp.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

constexpr int kNumBins = 5;           // 4 shared-memory bins + 1 global-scratch bin
constexpr int kBigBin = 4;
constexpr int kSmemT = 64;            // threads per block in the shared-memory kernels
constexpr int kBigT = 64;

__device__ __forceinline__ int ext_bin(const swb_ext_task &t, int max_mat) {
    if (t.qlen <= 0 || t.tlen <= 0) return 0;
    if (t.qlen > kExtSmemMaxQ || !fits16(t.qlen, t.h0, max_mat)) return kBigBin;
    return t.qlen <= 32 ? 0 : t.qlen <= 64 ? 1 : t.qlen <= 128 ? 2 : 3;
}

// Sort key: bin in bits 28-31, query length in 16-27, target length in 0-15.
__global__ void ext_keys_kernel(const swb_ext_task *__restrict__ tasks, size_t n, int max_mat,
                                uint32_t *__restrict__ keys, uint32_t *__restrict__ idx,
                                int *__restrict__ big_max_q) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const swb_ext_task t = tasks[i];
    const int b = ext_bin(t, max_mat);
    const uint32_t q = (uint32_t)min(max(t.qlen, 0), 4095);
    const uint32_t tl = (uint32_t)min(max(t.tlen, 0), 65535);
    keys[i] = ((uint32_t)b << 28) | (q << 16) | tl;
    idx[i] = (uint32_t)i;
    if (b == kBigBin) atomicMax(big_max_q, t.qlen);
}

// bin_start[b] = first sorted position whose bin >= b; bin_start[kNumBins] = n.
__global__ void bin_bounds_kernel(const uint32_t *__restrict__ sorted_keys, size_t n,
                                  uint32_t *__restrict__ bin_start, int nbins) {
    const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (n == 0) {
        if (p <= (size_t)nbins) bin_start[p] = 0;
        return;
    }
    if (p >= n) return;
    const int b = (int)(sorted_keys[p] >> 28);
    const int bprev = p == 0 ? -1 : (int)(sorted_keys[p - 1] >> 28);
    for (int bb = bprev + 1; bb <= b; ++bb) bin_start[bb] = (uint32_t)p;
    if (p == n - 1)
        for (int bb = b + 1; bb <= nbins; ++bb) bin_start[bb] = (uint32_t)n;
}

template <int QMAX, int T>
__global__ void __launch_bounds__(T) ext_smem_kernel(ExtArgs a, int bin) {
    extern __shared__ uint32_t sm[];
    Smem16<T> st{sm, sm + (QMAX + 1) * T, (int)threadIdx.x};
    const uint32_t lo = a.bin_start[bin], hi = a.bin_start[bin + 1];
    unsigned long long cells = 0;
    // Every thread of the block runs the same number of iterations, so the
    // warp-level reduction below sees all 32 lanes.
    const uint32_t span = hi - lo;
    const uint32_t per_iter = gridDim.x * (uint32_t)T;
    const uint32_t iters = (span + per_iter - 1) / per_iter;
    for (uint32_t it = 0; it < iters; ++it) {
        const uint32_t pos = lo + it * per_iter + blockIdx.x * T + threadIdx.x;
        if (pos < hi) {
            const uint32_t ti = a.order[pos];
            const swb_ext_task tk = a.tasks[ti];
            swb_ext_result r;
            ext_one(a, tk, st, r, cells);
            a.out[ti] = r;
        }
    }
    add_cells(a.cells + kCntExtBin0 + bin, cells);
}

__global__ void __launch_bounds__(kBigT) ext_global_kernel(ExtArgs a, int *h, int *e, uint8_t *q,
                                                           size_t nslots) {
    const uint32_t lo = a.bin_start[kBigBin], hi = a.bin_start[kBigBin + 1];
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
            swb_ext_result r;
            ext_one(a, tk, st, r, cells);
            a.out[ti] = r;
        }
    }
    add_cells(a.cells + kCntExtBin0 + kBigBin, cells);
}

template <int QMAX>
size_t smem_bytes() { return (size_t)((QMAX + 1) + QMAX / 4) * kSmemT * sizeof(uint32_t); }

template <int QMAX>
int launch_bin(swb_ctx *ctx, const ExtArgs &a, int bin, size_t n, cudaStream_t s) {
    static int occ = -1;
    const size_t smem = smem_bytes<QMAX>();
    if (occ < 0) {
        SWB_CUDA(cudaFuncSetAttribute(ext_smem_kernel<QMAX, kSmemT>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        SWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ext_smem_kernel<QMAX, kSmemT>,
                                                               kSmemT, smem));
        if (occ < 1) occ = 1;
    }
    const size_t need = (n + kSmemT - 1) / kSmemT;
    const size_t grid = std::min<size_t>(need, (size_t)ctx->sm_count * occ);
    if (grid == 0) return SWB_OK;
    static const char *names[4] = {"ext_smem_q32", "ext_smem_q64", "ext_smem_q128", "ext_smem_q256"};
    ProfScope ps(ctx, s, names[bin], kCntExtBin0 + bin);
    ext_smem_kernel<QMAX, kSmemT><<<(unsigned)grid, kSmemT, smem, s>>>(a, bin);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    return SWB_OK;
}

}  // namespace

int launch_ext(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases,
               const swb_ext_task *d_tasks, size_t n, swb_ext_result *d_out,
               unsigned long long *d_cells, cudaStream_t s, int max_q_hint) {
    if (n == 0) return SWB_OK;
    if (n > 0x7FFFFFF0ull) return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 tasks in one batch");
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_keys, n * 4)) || (rc = ensure_dev(ctx, ctx->d_keys2, n * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_idx, n * 4)) || (rc = ensure_dev(ctx, ctx->d_idx2, n * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_misc, 256)))
        return rc;
    uint32_t *keys = (uint32_t *)ctx->d_keys.p, *keys2 = (uint32_t *)ctx->d_keys2.p;
    uint32_t *idx = (uint32_t *)ctx->d_idx.p, *idx2 = (uint32_t *)ctx->d_idx2.p;
    uint32_t *bin_start = (uint32_t *)ctx->d_misc.p;          // kNumBins+1 words
    int *big_max_q = (int *)((char *)ctx->d_misc.p + 64);
    SWB_CUDA(cudaMemsetAsync(big_max_q, 0, sizeof(int), s));
    const unsigned tb = 256;
    {
        ProfScope ps(ctx, s, "ext_keys", -1);
        ext_keys_kernel<<<(unsigned)((n + tb - 1) / tb), tb, 0, s>>>(d_tasks, n, sc.max_mat, keys, idx, big_max_q);
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
        bin_bounds_kernel<<<(unsigned)((n + tb - 1) / tb), tb, 0, s>>>(keys2, n, bin_start, kNumBins);
    }
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());

    ExtArgs a{sc, d_bases, ctx->d_pac, d_tasks, d_out, idx2, bin_start, d_cells};
    if ((rc = launch_bin<32>(ctx, a, 0, n, s))) return rc;
    if ((rc = launch_bin<64>(ctx, a, 1, n, s))) return rc;
    if ((rc = launch_bin<128>(ctx, a, 2, n, s))) return rc;
    if ((rc = launch_bin<256>(ctx, a, 3, n, s))) return rc;

    // Global-scratch bin: size its scratch from the longest query in it.
    int max_q = max_q_hint;
    if (max_q < 0) {
        SWB_CUDA(cudaMemcpyAsync(&max_q, big_max_q, sizeof(int), cudaMemcpyDeviceToHost, s));
        SWB_CUDA(cudaStreamSynchronize(s));
    }
    if (max_q > 0) {
        if (max_q > kMaxLen) return set_error(SWB_ERR_TOO_LARGE, "query longer than 65535 bases");
        const size_t nslots = (size_t)ctx->sm_count * 4 * kBigT;
        const size_t cols = (size_t)max_q + 1;
        const size_t bytes = cols * nslots * (2 * sizeof(int) + 1) + 256;
        if ((rc = ensure_dev(ctx, ctx->d_scratch, bytes))) return rc;
        int *hbuf = (int *)ctx->d_scratch.p;
        int *ebuf = hbuf + cols * nslots;
        uint8_t *qbuf = (uint8_t *)(ebuf + cols * nslots);
        ProfScope ps(ctx, s, "ext_global_i32", kCntExtBin0 + kBigBin);
        ext_global_kernel<<<(unsigned)(nslots / kBigT), kBigT, 0, s>>>(a, hbuf, ebuf, qbuf, nslots);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    return SWB_OK;
}

// Host-side twin of the device bin test, used to size the scratch bin.
int ext_big_max_q(const swb_ext_task *tasks, size_t n, int max_mat) {
    int m = 0;
    for (size_t i = 0; i < n; ++i) {
        const swb_ext_task &t = tasks[i];
        if (t.qlen <= 0 || t.tlen <= 0) continue;
        if (t.qlen > kExtSmemMaxQ || !fits16(t.qlen, t.h0, max_mat)) m = t.qlen > m ? t.qlen : m;
    }
    return m;
}

}  // namespace swb
