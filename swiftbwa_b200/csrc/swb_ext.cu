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
#include "swb_internal.h"

namespace swb {
namespace {

constexpr int kNumBins = 5;           // 4 shared-memory bins + 1 global-scratch bin
constexpr int kBigBin = 4;
constexpr int kSmemT = 64;            // threads per block in the shared-memory kernels
constexpr int kBigT = 64;

struct ExtArgs {
    DevScoring sc;
    const uint8_t *bases;
    const uint8_t *pac;
    const swb_ext_task *tasks;
    swb_ext_result *out;
    const uint32_t *order;      // sorted task indices
    const uint32_t *bin_start;  // kNumBins + 1 entries
    unsigned long long *cells;
};

// True when every H/E of the task fits int16: H <= h0 + qlen*maxMat
// (each row adds at most the best match score) and E, F <= H.
__device__ __host__ __forceinline__ bool fits16(int qlen, int h0, int max_mat) {
    long long hi = (long long)h0 + (long long)qlen * (max_mat > 0 ? max_mat : 0);
    return h0 >= 0 && hi <= 32000;
}

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

// ---------------------------------------------------------------- row stores
// 16-bit store: one word per column, H low half, E high half, in shared memory.
template <int T>
struct Smem16 {
    uint32_t *he;        // [(qmax+1) * T]
    uint32_t *qw;        // [(qmax/4) * T]
    int tid;
    static constexpr bool kPackedKey = true;
    __device__ __forceinline__ void load(int j, int &h, int &e) const {
        const uint32_t w = he[j * T + tid];
        h = (int)(int16_t)(w & 0xFFFFu);
        e = (int)(int16_t)(w >> 16);
    }
    __device__ __forceinline__ void store(int j, int h, int e) const {
        he[j * T + tid] = ((uint32_t)h & 0xFFFFu) | ((uint32_t)e << 16);
    }
    __device__ __forceinline__ bool zero(int j) const { return he[j * T + tid] == 0u; }
    __device__ __forceinline__ uint32_t qcode(int j) const {
        return (qw[(j >> 2) * T + tid] >> ((j & 3) << 3)) & 0xFFu;
    }
    __device__ __forceinline__ void put_query(int k, uint32_t word, int) const { qw[(k >> 2) * T + tid] = word; }
};

// 32-bit store in global scratch, [column][slot] so a warp's slots coalesce.
struct Global32 {
    int *h, *e;
    uint8_t *q;
    size_t stride;   // number of slots
    size_t slot;
    static constexpr bool kPackedKey = false;
    __device__ __forceinline__ void load(int j, int &hv, int &ev) const {
        hv = h[(size_t)j * stride + slot];
        ev = e[(size_t)j * stride + slot];
    }
    __device__ __forceinline__ void store(int j, int hv, int ev) const {
        h[(size_t)j * stride + slot] = hv;
        e[(size_t)j * stride + slot] = ev;
    }
    __device__ __forceinline__ bool zero(int j) const {
        return h[(size_t)j * stride + slot] == 0 && e[(size_t)j * stride + slot] == 0;
    }
    __device__ __forceinline__ uint32_t qcode(int j) const { return q[(size_t)j * stride + slot]; }
    __device__ __forceinline__ void put_query(int k, uint32_t word, int nvalid) const {
        for (int b = 0; b < nvalid; ++b) q[(size_t)(k + b) * stride + slot] = (uint8_t)(word >> (8 * b));
    }
};

// One extension, restating BandedSWScalar.swift:21-191 over a row store.
template <class Store>
__device__ void ext_one(const ExtArgs &a, const swb_ext_task &tk, const Store &st,
                        swb_ext_result &res, unsigned long long &cells) {
    res = swb_ext_result{0, 0, 0, 0, 0, 0};
    const int qlen = tk.qlen, tlen = tk.tlen;
    if (!(qlen > 0 && tlen > 0)) return;                                  // :33-35
    const DevScoring &sc = a.sc;
    const int oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const int zDrop = sc.zdrop;
    const int h0 = tk.h0;

    // Stage the query (4 codes per word; padding bytes are never read).
    for (int k = 0; k < qlen; k += 4) {
        uint32_t word = 0;
        for (int b = 0; b < 4 && k + b < qlen; ++b)
            word |= span_base(a.bases, a.pac, tk.q_off, k + b, qlen, tk.flags, false) << (8 * b);
        st.put_query(k, word, imin(4, qlen - k));
    }
    // w cap in double arithmetic (:52-62)
    int w = tk.w;
    {
        const int maxIns = (int)((double)(qlen * sc.max_mat + tk.end_bonus - oIns) / (double)eIns + 1.0);
        w = imin(w, imax(1, maxIns));
        const int maxDel = (int)((double)(qlen * sc.max_mat + tk.end_bonus - oDel) / (double)eDel + 1.0);
        w = imin(w, imax(1, maxDel));
    }
    // First row from h0 (:65-77)
    {
        int hv = h0;
        st.store(0, hv, 0);
        int j = 1;
        if (h0 > oIns + eIns) {
            hv = h0 - oIns - eIns;
            st.store(1, hv, 0);
            j = 2;
            while (j <= qlen && hv > eIns) {
                hv -= eIns;
                st.store(j, hv, 0);
                ++j;
            }
        }
        for (; j <= qlen; ++j) st.store(j, 0, 0);
    }
    int maxScore = h0, maxI = -1, maxJ = -1, gScore = -1, gTle = -1, maxOff = 0;
    int beg = 0, end = qlen;
    const int oeDel = oDel + eDel, oeIns = oIns + eIns;

    for (int i = 0; i < tlen; ++i) {                                      // :90
        const uint32_t tb = span_base(a.bases, a.pac, tk.t_off, i, tlen, tk.flags, true);
        const RowTable rt = row_table(sc, tb);
        if (beg < i - w) beg = i - w;                                     // :95-97
        if (end > i + w + 1) end = i + w + 1;
        if (end > qlen) end = qlen;
        int f = 0;
        int h1 = beg == 0 ? imax(h0 - (oDel + eDel * (i + 1)), 0) : 0;   // :99-107
        int rowMax = 0, rowMaxJ = -1;
        uint32_t key = 0;
        if (end > beg) cells += (unsigned long long)(end - beg);
        for (int j = beg; j < end; ++j) {                                 // :112-143
            int M, e;
            st.load(j, M, e);
            const int diag = M != 0 ? M + row_score(rt, st.qcode(j)) : 0;
            const int H = imax(imax(diag, e), f);
            const int newE = imax(e - eDel, imax(diag - oeDel, 0));
            st.store(j, h1, newE);
            h1 = H;
            if (Store::kPackedKey) {
                key = max(key, ((uint32_t)H << 16) | (uint32_t)j);
            } else {
                rowMaxJ = rowMax > H ? rowMaxJ : j;
                rowMax = rowMax > H ? rowMax : H;
            }
            f = imax(f - eIns, imax(diag - oeIns, 0));
        }
        st.store(end, h1, 0);                                             // :145-146
        if (Store::kPackedKey && end > beg) {
            rowMax = (int)(key >> 16);
            rowMaxJ = (int)(key & 0xFFFFu);
        }
        if (end == qlen) {                                                // :149-152
            gTle = gScore > h1 ? gTle : i;
            gScore = gScore > h1 ? gScore : h1;
        }
        if (rowMax == 0) break;                                           // :155
        if (rowMax > maxScore) {                                          // :158-172
            maxScore = rowMax;
            maxI = i;
            maxJ = rowMaxJ;
            const int off = abs(rowMaxJ - i);
            if (off > maxOff) maxOff = off;
        } else if (zDrop > 0) {
            const int dI = i - maxI, dJ = rowMaxJ - maxJ;
            if (dI > dJ) {
                if (maxScore - rowMax - (dI - dJ) * eDel > zDrop) break;
            } else {
                if (maxScore - rowMax - (dJ - dI) * eIns > zDrop) break;
            }
        }
        int nb = beg;                                                     // :175-180
        while (nb < end && st.zero(nb)) ++nb;
        beg = nb;
        int ne = end;
        while (ne >= beg && st.zero(ne)) --ne;
        end = imin(ne + 2, qlen);
    }
    res = swb_ext_result{maxScore, maxJ + 1, maxI + 1, gTle + 1, gScore, maxOff};   // :183-190
}

__device__ __forceinline__ void add_cells(unsigned long long *dst, unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
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
