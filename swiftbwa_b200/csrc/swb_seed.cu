// swb_seed.cu -- SMEM seeding on the resident FM index, bit-exact with
// SMEMFinder.findAllSMEMs (Sources/FMIndex/SMEMFinder.swift:28-268) over
// BWT.occ (Sources/FMIndex/BWT.swift:68-84) and BackwardSearch.backwardExt
// (Sources/FMIndex/BackwardSearch.swift:21-77).
//
// One thread owns one read and walks its start positions in the reference's
// order (each start's forward phase decides the next start), so the SMEMs,
// their order and their SA intervals are the reference's.  The work is a
// chain of rank queries into the checkpoint array (64 bytes per 64 BWT
// positions, at most 2 checkpoints per backward extension): random reads
// over the resident index, so the kernel is bound by memory latency and
// keeps as many reads in flight as the SMs hold threads.  The walk is a
// state machine (Walker) whose every step is one backward extension, so the
// lanes of a warp run their rank queries together; each lane claims its next
// read from a counter when its current one is done.  Each thread's list of
// candidate intervals (at most one per query base) keeps its first kShE
// entries in shared memory -- the entries every backward step reads and
// rewrites, off the chain of dependent loads -- and the rest in the
// thread's own row of global scratch, one 32-byte sector per entry.  A
// read's SMEMs go to its own window in the order found and are then sorted
// there (query begin, longer first), as the reference sorts its array; a
// scan of the counts and a gather pack the windows in read order, and only
// those entries are copied back to the host.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "swb_internal.h"

namespace swb {
namespace {

constexpr int kSeedT = 128;   // threads per block
// Candidate entries per thread in shared memory (32 bytes each; 28 KB per
// block of 128 threads).
constexpr int kShE = 7;

struct SeedArgs {
    const swb_bwt_checkpoint *cp;
    int64_t count[5];
    int64_t sentinel;
    const uint8_t *bases;
    const uint64_t *read_off;
    const int32_t *read_len;
    uint32_t n_reads;
    int32_t min_seed_len;
    int64_t min_intv;
    int32_t split_len, split_width;   // internal re-seeding (split_len <= 0: off)
    uint32_t cap;
    swb_smem *out;
    uint32_t *n_out;
    uint32_t *claim;            // next unclaimed position of `order`
    const uint32_t *order;      // reads, least complex (most work) first
    uint32_t *first_over;       // lowest read index with more SMEMs than cap (~0 = none)
    unsigned long long *exts;   // backward extensions (work counter)
    // candidate intervals past the first kShE: [slot][entry - kShE], 32 bytes
    // each ({k, l}, {s, m | n << 32})
    longlong2 *cand;
    size_t entries;
};

struct Intv {
    int64_t k, l, s;
};

// Ranks of the four bases before BWT position pos (BWT.occ for c = 0..3):
// the checkpoint's counts plus the set bits of the block before pos.
__device__ __forceinline__ void occ4(const swb_bwt_checkpoint *__restrict__ cp, int64_t pos, int64_t o[4]) {
    const longlong2 *p = reinterpret_cast<const longlong2 *>(cp + (pos >> 6));
    const longlong2 c01 = __ldg(p), c23 = __ldg(p + 1), b01 = __ldg(p + 2), b23 = __ldg(p + 3);
    const int y = (int)(pos & 63);
    const unsigned long long mask = y == 0 ? 0ull : ~(~0ull >> y);   // oneHotMaskArray[y]: the top y bits
    o[0] = c01.x + __popcll((unsigned long long)b01.x & mask);
    o[1] = c01.y + __popcll((unsigned long long)b01.y & mask);
    o[2] = c23.x + __popcll((unsigned long long)b23.x & mask);
    o[3] = c23.y + __popcll((unsigned long long)b23.y & mask);
}

// BackwardSearch.backwardExt: the interval of base a prepended (a < 4).
// Branch-free, so the lanes of a warp stay together: both checkpoints are
// read even when sp and ep share a block (the second read then hits the
// same cache line), and the base selects with conditional moves.
__device__ __forceinline__ Intv backward_ext(const SeedArgs &g, int64_t k, int64_t l, int64_t s, int a) {
    const int64_t sp = k, ep = k + s;
    int64_t osp[4], oep[4];
    occ4(g.cp, sp, osp);
    occ4(g.cp, ep, oep);
    const int64_t s0 = oep[0] - osp[0], s1 = oep[1] - osp[1], s2 = oep[2] - osp[2], s3 = oep[3] - osp[3];
    const int64_t sentinelOffset = (sp <= g.sentinel && ep > g.sentinel) ? 1 : 0;
    const int64_t l3 = l + sentinelOffset, l2 = l3 + s3, l1 = l2 + s2, l0 = l1 + s1;
    const int64_t c = a == 0 ? g.count[0] : a == 1 ? g.count[1] : a == 2 ? g.count[2] : g.count[3];
    const int64_t o = a == 0 ? osp[0] : a == 1 ? osp[1] : a == 2 ? osp[2] : osp[3];
    return {c + o, a == 0 ? l0 : a == 1 ? l1 : a == 2 ? l2 : l3, a == 0 ? s0 : a == 1 ? s1 : a == 2 ? s2 : s3};
}

struct Cand {   // SMEMFinder.BidiInterval
    int64_t k, l, s;
    int32_t m, n;
};

// A thread's candidate list: entries 0..kShE-1 in shared memory (this
// thread's column of two [entry][thread] arrays of 16-byte pairs), the rest
// in the thread's row of global scratch, one 32-byte sector per entry; both
// hold {k, l} and {s, m | n << 32}.  An entry is read and written through a
// generic pointer chosen by a select, so lanes whose entries live in
// different memories do not split the warp.
struct Prev {
    longlong2 *shkl, *shsm;   // shared, already offset by the thread
    longlong2 *row;           // global: entry kShE + i at row[2i], row[2i + 1]
    __device__ __forceinline__ longlong2 *kl(int e) const { return e < kShE ? shkl + e * kSeedT : row + 2 * (e - kShE); }
    __device__ __forceinline__ longlong2 *sm(int e) const {
        return e < kShE ? shsm + e * kSeedT : row + 2 * (e - kShE) + 1;
    }
    __device__ __forceinline__ Cand get(int e) const {
        const longlong2 a = *kl(e), b = *sm(e);
        return {a.x, a.y, b.x, (int)(uint32_t)b.y, (int)((unsigned long long)b.y >> 32)};
    }
    __device__ __forceinline__ void put(int e, const Cand &c) const {
        *kl(e) = make_longlong2(c.k, c.l);
        *sm(e) = make_longlong2(c.s, (long long)((unsigned long long)(uint32_t)c.m | ((unsigned long long)(uint32_t)c.n << 32)));
    }
};

struct Emit {
    swb_smem *w;      // the read's window
    uint32_t cap, n = 0;
    __device__ __forceinline__ void add(const Cand &c) {
        if (n < cap) w[n] = swb_smem{c.k, c.k + c.s - 1, c.m, c.n + 1};
        ++n;
    }
};

// Sort by query begin, longer first (SMEMFinder.swift:53-58); equal keys
// are equal SMEMs, so their order cannot differ from the reference's.
__device__ void sort_smems(swb_smem *w, uint32_t n) {
    for (uint32_t i = 1; i < n; ++i) {
        const swb_smem x = w[i];
        uint32_t j = i;
        while (j > 0 && (w[j - 1].qb > x.qb || (w[j - 1].qb == x.qb && w[j - 1].qe - w[j - 1].qb < x.qe - x.qb))) {
            w[j] = w[j - 1];
            --j;
        }
        w[j] = x;
    }
}

// SMEMFinder.findAllSMEMs for one read (SMEMFinder.swift:28-59; its
// findSMEMsAtPosition calls :89-268) followed by the internal re-seeding of
// BWAMemAligner (BWAMemAligner.swift:283-304), written as a state machine in
// which every step waits for one backward extension.  next() makes the
// transitions that need none and returns the extension the read waits for
// (false once the read is done); apply() consumes its result.  The lanes of
// a warp walk different reads, so a warp runs next(), one backward extension
// on every lane that has one, then apply(): the rank queries, which are the
// work, run with the lanes converged instead of one code path at a time.
struct Walker {
    enum State : int { kStart, kFwd, kBwd, kDone };
    const SeedArgs *g;
    const uint8_t *q;
    int len;
    State st;
    bool reseed;          // in the re-seeding pass (the first pass is sorted)
    bool phase2;          // backward row: past the first kept or emitted interval
    int pos;              // first pass: the next start position
    uint32_t ri, n0;      // re-seeding: the next original SMEM, the originals' count
    int64_t minIntv;      // of the current findSMEMsAtPosition call
    int startPos, nextPos, j, bj, p, numPrev, numCurr, bbase;
    int64_t currS;
    Cand smem, iv;
    Emit emit;

    __device__ __forceinline__ void start(const SeedArgs &args, uint32_t r) {
        g = &args;
        q = args.bases + args.read_off[r];
        len = args.read_len[r];
        st = kStart;
        reseed = false;
        pos = 0;
        emit = Emit{args.out + (size_t)r * args.cap, args.cap, 0};
    }
    __device__ __forceinline__ void end_call() {
        if (!reseed) pos = nextPos;                                          // :41-51
        st = kStart;
    }
    // One findSMEMsAtPosition call (:89-123).
    __device__ __forceinline__ void call(int sp, int64_t mi) {
        startPos = sp;
        minIntv = mi;
        nextPos = sp + 1;
        const int a = q[sp];
        if (a >= 4) {                                                        // :104-107
            end_call();
            return;
        }
        smem = Cand{g->count[a], g->count[3 - a], g->count[a + 1] - g->count[a], sp, sp};
        numPrev = 0;
        j = sp + 1;
        st = kFwd;
    }
    __device__ __forceinline__ void bwd_done(const Prev &prev) {             // :253-265
        if (numPrev != 0) {
            const Cand c = prev.get(0);
            if ((c.n - c.m + 1) >= g->min_seed_len) emit.add(c);
        }
        end_call();
    }
    // The backward phase at query position bj (:169-176).
    __device__ __forceinline__ void bwd_row(const Prev &prev) {
        if (bj < 0 || q[bj] >= 4) {
            bwd_done(prev);
            return;
        }
        bbase = q[bj];
        numCurr = 0;
        currS = -1;
        p = 0;
        phase2 = false;
        st = kBwd;
    }
    __device__ __forceinline__ void fwd_done(const Prev &prev) {             // :160-166 (longest first)
        if (smem.s >= minIntv) prev.put(numPrev++, smem);
        for (int x = 0, y = numPrev - 1; x < y; ++x, --y) {
            const Cand cx = prev.get(x), cy = prev.get(y);
            prev.put(x, cy);
            prev.put(y, cx);
        }
        bj = startPos - 1;
        bwd_row(prev);
    }
    // Transitions up to the next backward extension (its interval and base
    // in k, l, s, a); false when the read is done.
    __device__ bool next(const Prev &prev, int64_t &k, int64_t &l, int64_t &s, int &a) {
        for (;;) {
            if (st == kFwd) {                                                // :124-157
                if (j >= len) {
                    fwd_done(prev);
                    continue;
                }
                const int base = q[j];
                nextPos = j + 1;
                if (base >= 4) {
                    fwd_done(prev);
                    continue;
                }
                // Forward extension: backward extension with k/l swapped and the complement base.
                k = smem.l;
                l = smem.k;
                s = smem.s;
                a = 3 - base;
                return true;
            }
            if (st == kBwd) {
                if (p >= numPrev) {                                          // :248-249
                    numPrev = numCurr;
                    if (numCurr == 0) {
                        bwd_done(prev);
                        continue;
                    }
                    --bj;
                    bwd_row(prev);
                    continue;
                }
                iv = prev.get(p);
                k = iv.k;
                l = iv.l;
                s = iv.s;
                a = bbase;
                return true;
            }
            if (st == kDone) return false;
            // kStart
            if (!reseed) {
                if (pos < len) {                                             // :41-51
                    call(pos, g->min_intv);
                    continue;
                }
                // First pass done: sort it (:53-58); then re-seeding, unless
                // the window overflowed.
                if (emit.n > g->cap) {
                    st = kDone;
                    continue;
                }
                sort_smems(emit.w, emit.n);
                if (g->split_len <= 0) {
                    st = kDone;
                    continue;
                }
                n0 = emit.n;
                ri = 0;
                reseed = true;
                continue;
            }
            // Re-seeding: the first-pass SMEMs (w[0 .. n0), never overwritten:
            // new ones are appended behind them) that are long and rare enough.
            bool found = false;
            while (ri < n0) {
                const swb_smem sm = emit.w[ri++];
                const int64_t cnt = sm.l - sm.k + 1;
                if (sm.qe - sm.qb < g->split_len || cnt > (int64_t)g->split_width) continue;
                call((sm.qb + sm.qe) / 2, cnt + 1);
                found = true;
                break;
            }
            if (found) continue;
            if (emit.n > n0 && emit.n <= g->cap) sort_smems(emit.w, emit.n);
            st = kDone;
        }
    }
    // The result of the extension next() asked for.
    __device__ __forceinline__ void apply(const Prev &prev, const Intv &ext) {
        if (st == kFwd) {
            if (ext.s != smem.s) prev.put(numPrev++, smem);
            if (ext.s < minIntv) {
                nextPos = j;
                fwd_done(prev);
                return;
            }
            smem = Cand{ext.l, ext.k, ext.s, smem.m, j};
            ++j;
            return;
        }
        // Backward row (:177-246): until the first interval that is emitted
        // (condition 1) or kept (condition 2), then every further one kept
        // whose size differs from the last kept.
        if (!phase2) {
            if (ext.s < minIntv && (iv.n - iv.m + 1) >= g->min_seed_len) {
                emit.add(iv);
                phase2 = true;
            } else if (ext.s >= minIntv && ext.s != currS) {
                currS = ext.s;
                prev.put(numCurr++, Cand{ext.k, ext.l, ext.s, bj, iv.n});
                phase2 = true;
            }
        } else if (ext.s >= minIntv && ext.s != currS) {
            currS = ext.s;
            prev.put(numCurr++, Cand{ext.k, ext.l, ext.s, bj, iv.n});
        }
        ++p;
    }
};

__global__ void __launch_bounds__(kSeedT, 5) smem_kernel(SeedArgs g) {
    __shared__ longlong2 sh_kl[kShE * kSeedT], sh_sm[kShE * kSeedT];
    const size_t slot = blockIdx.x * (size_t)kSeedT + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const Prev prev{sh_kl + threadIdx.x, sh_sm + threadIdx.x, g.cand + 2 * slot * g.entries};
    unsigned long long exts = 0;
    // Each lane claims its next read as soon as its current one is done, so
    // the lanes of a warp keep walking while any read remains.
    Walker w;
    uint32_t c = atomicAdd(g.claim, 1u), r = 0;
    bool have = c < g.n_reads;
    if (have) r = g.order[c];
    if (have) w.start(g, r);
    for (;;) {
        int64_t k = 0, l = 0, s = 0;
        int a = 0;
        bool need = false;
        while (have) {
            need = w.next(prev, k, l, s, a);
            if (need) break;
            g.n_out[r] = w.emit.n;
            if (w.emit.n > g.cap) atomicMin(g.first_over, r);
            c = atomicAdd(g.claim, 1u);
            have = c < g.n_reads;
            if (have) r = g.order[c];
            if (have) w.start(g, r);
        }
        if (!__any_sync(0xFFFFFFFFu, need)) break;
        if (need) {
            w.apply(prev, backward_ext(g, k, l, s, a));
            ++exts;
        }
    }
    for (int o = 16; o > 0; o >>= 1) exts += __shfl_down_sync(0xFFFFFFFFu, exts, o);
    if (lane == 0 && exts) atomicAdd(g.exts, exts);
}

// Claim order of the reads: the number of distinct 4-mers of each read as
// the sort key, so the least complex reads -- tandem repeats, whose SA
// intervals stay large and whose walks take many more extensions -- are
// claimed first and the cheap ones fill the end of the launch.
__global__ void seed_order_keys_kernel(const uint8_t *__restrict__ bases, const uint64_t *__restrict__ read_off,
                                       const int32_t *__restrict__ read_len, uint32_t n_reads,
                                       uint32_t *__restrict__ keys, uint32_t *__restrict__ idx) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    const uint8_t *q = bases + read_off[r];
    const int len = read_len[r];
    uint32_t seen[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t kmer = 0;
    int run = 0;   // bases since the last N
    for (int j = 0; j < len; ++j) {
        const uint32_t b = q[j];
        if (b >= 4) {
            run = 0;
            continue;
        }
        kmer = ((kmer << 2) | b) & 0xFFu;
        if (++run >= 4) {
#pragma unroll
            for (int w = 0; w < 8; ++w)
                if ((int)(kmer >> 5) == w) seen[w] |= 1u << (kmer & 31);
        }
    }
    uint32_t d = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) d += __popc(seen[w]);
    keys[r] = d;
    idx[r] = r;
}

// Packs every read's window into the output in read order: read r's first
// min(n[r], cap) SMEMs go to off[r] (off = exclusive sum of n).
__global__ void smem_pack_kernel(const swb_smem *__restrict__ win, const uint32_t *__restrict__ n,
                                 const unsigned long long *__restrict__ off, uint32_t n_reads, uint32_t cap,
                                 swb_smem *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    const uint32_t k = min(n[r], cap);
    const swb_smem *src = win + (size_t)r * cap;
    swb_smem *dst = out + off[r];
    for (uint32_t i = 0; i < k; ++i) dst[i] = src[i];
}

__global__ void u32_to_u64_kernel(const uint32_t *__restrict__ a, unsigned long long *__restrict__ b, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" {

int swb_upload_bwt(swb_ctx *ctx, const swb_bwt_checkpoint *cp, uint64_t n_cp, const int64_t count[5], int64_t length,
                   int64_t sentinel) {
    if (!ctx || !count || (!cp && n_cp)) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    if (length < 1 || n_cp < (uint64_t)(length >> 6) + 1 || sentinel < 0 || sentinel >= length || count[4] != length)
        return set_error(SWB_ERR_INVALID_ARG, "BWT: need length >= 1, (length >> 6) + 1 checkpoints, "
                                              "0 <= sentinel < length and count[4] == length");
    for (int c = 0; c < 4; ++c)
        if (count[c] < 0 || count[c] > count[c + 1]) return set_error(SWB_ERR_INVALID_ARG, "BWT: counts must ascend");
    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_bwt, n_cp * sizeof(swb_bwt_checkpoint)))) return rc;
    SWB_CUDA(cudaMemcpy(ctx->d_bwt.p, cp, n_cp * sizeof(swb_bwt_checkpoint), cudaMemcpyHostToDevice));
    for (int c = 0; c < 5; ++c) ctx->bwt_count[c] = count[c];
    ctx->bwt_length = length;
    ctx->bwt_sentinel = sentinel;
    ctx->bwt_ncp = n_cp;
    return SWB_OK;
}

int swb_smem_batch(swb_ctx *ctx, const uint8_t *bases, size_t n_bases, const uint64_t *read_off,
                   const int32_t *read_len, size_t n_reads, int32_t min_seed_len, int64_t min_intv,
                   int32_t split_len, int32_t split_width, uint32_t cap_per_read, swb_smem *out, size_t out_cap,
                   uint32_t *n_out, uint64_t *out_off) {
    if (!ctx || (n_reads && (!read_off || !read_len || !n_out || !out_off)) || (!out && out_cap) ||
        (!bases && n_bases))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    // The claim order's sort and the offsets' scan take int counts.
    if (n_reads > 0x7FFFFFF0ull) return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 reads in one batch");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->last_ms = 0;
    ctx->last_cells = 0;
    if (n_reads == 0) return SWB_OK;
    if (ctx->bwt_ncp == 0) return set_error(SWB_ERR_NO_REFERENCE, "no FM index uploaded (swb_upload_bwt)");
    int max_len = 0;
    for (size_t r = 0; r < n_reads; ++r) {
        if (read_len[r] < 0 || read_len[r] > kMaxLen)
            return set_error(SWB_ERR_TOO_LARGE, "read " + std::to_string(r) + ": length outside 0..65535");
        if (read_off[r] + (uint64_t)read_len[r] > n_bases)
            return set_error(SWB_ERR_INVALID_ARG, "read " + std::to_string(r) + ": span outside the bases buffer");
        max_len = std::max(max_len, read_len[r]);
    }
    SWB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t b_bytes = al(n_bases), o_bytes = al(n_reads * 8), l_bytes = al(n_reads * 4);
    const size_t out_bytes = al(n_reads * (size_t)cap_per_read * sizeof(swb_smem)), n_bytes = al(n_reads * 4);
    const size_t off_bytes = al(n_reads * 8);
    size_t scan_bytes = 0;
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (unsigned long long *)nullptr,
                                           (unsigned long long *)nullptr, (int)n_reads, ctx->stream));
    size_t sort_bytes = 0;
    SWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                             (uint32_t *)nullptr, (uint32_t *)nullptr, (int)n_reads, 0, 9, ctx->stream));
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_keys, n_reads * 4)) || (rc = ensure_dev(ctx, ctx->d_keys2, n_reads * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_idx, n_reads * 4)) || (rc = ensure_dev(ctx, ctx->d_idx2, n_reads * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_sort_tmp, sort_bytes)))
        return rc;
    if ((rc = ensure_dev(ctx, ctx->d_bases, b_bytes + o_bytes + l_bytes + 256)) ||
        (rc = ensure_dev(ctx, ctx->d_out, out_bytes + n_bytes + 2 * off_bytes + al(scan_bytes) + 256)))
        return rc;
    char *in = (char *)ctx->d_bases.p;
    uint8_t *d_b = (uint8_t *)in;
    uint64_t *d_off = (uint64_t *)(in + b_bytes);
    int32_t *d_len = (int32_t *)(in + b_bytes + o_bytes);
    uint32_t *d_misc = (uint32_t *)(in + b_bytes + o_bytes + l_bytes);   // claim, first_over
    swb_smem *d_out = (swb_smem *)ctx->d_out.p;
    uint32_t *d_n = (uint32_t *)((char *)ctx->d_out.p + out_bytes);
    unsigned long long *d_n64 = (unsigned long long *)((char *)ctx->d_out.p + out_bytes + n_bytes);
    unsigned long long *d_off64 = d_n64 + off_bytes / 8;
    void *d_scan_tmp = (char *)ctx->d_out.p + out_bytes + n_bytes + 2 * off_bytes;
    // Persistent grid: resident blocks on every SM, each thread with a
    // candidate column of max_len entries (32 bytes each) past the kShE it
    // keeps in shared memory.
    int per_sm = 0;
    SWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, smem_kernel, kSeedT, 0));
    per_sm = std::max(per_sm, 1);
    size_t blocks = std::min<size_t>((size_t)ctx->sm_count * per_sm, (n_reads + kSeedT - 1) / kSeedT);
    const size_t entries = (size_t)std::max(max_len - kShE, 1);
    const size_t per_slot = entries * 32;
    const size_t avail = ctx->budget > ctx->allocated ? (ctx->budget - ctx->allocated) / 2 : 0;
    while (blocks > 1 && blocks * kSeedT * per_slot > avail) blocks /= 2;
    const size_t nslots = blocks * kSeedT;
    if ((rc = ensure_dev(ctx, ctx->d_seed, nslots * per_slot + 256))) return rc;
    char *sp = (char *)ctx->d_seed.p;
    SeedArgs g{};
    g.cp = (const swb_bwt_checkpoint *)ctx->d_bwt.p;
    for (int c = 0; c < 5; ++c) g.count[c] = ctx->bwt_count[c];
    g.sentinel = ctx->bwt_sentinel;
    g.bases = d_b;
    g.read_off = d_off;
    g.read_len = d_len;
    g.n_reads = (uint32_t)n_reads;
    g.min_seed_len = min_seed_len;
    g.min_intv = min_intv;
    g.split_len = split_len;
    g.split_width = split_width;
    g.cap = cap_per_read;
    g.out = d_out;
    g.n_out = d_n;
    g.claim = d_misc;
    g.first_over = d_misc + 1;
    g.cand = (longlong2 *)sp;
    g.entries = entries;
    // Inputs: straight from the caller's buffers when all three are pinned,
    // else through the context's pinned staging buffer in the device layout
    // (host threads copy, then one transfer).
    if (is_pinned(bases) && is_pinned(read_off) && is_pinned(read_len)) {
        SWB_CUDA(cudaMemcpyAsync(in, bases, n_bases, cudaMemcpyHostToDevice, st));
        SWB_CUDA(cudaMemcpyAsync(in + b_bytes, read_off, n_reads * 8, cudaMemcpyHostToDevice, st));
        SWB_CUDA(cudaMemcpyAsync(in + b_bytes + o_bytes, read_len, n_reads * 4, cudaMemcpyHostToDevice, st));
    } else {
        if ((rc = ensure_host(ctx, ctx->h_in, b_bytes + o_bytes + l_bytes))) return rc;
        char *stage = (char *)ctx->h_in.p;
        par_copy(stage, bases, n_bases);
        par_copy(stage + b_bytes, read_off, n_reads * 8);
        par_copy(stage + b_bytes + o_bytes, read_len, n_reads * 4);
        SWB_CUDA(cudaMemcpyAsync(in, stage, b_bytes + o_bytes + l_bytes, cudaMemcpyHostToDevice, st));
    }
    SWB_CUDA(cudaMemsetAsync(d_misc, 0, 4, st));
    SWB_CUDA(cudaMemsetAsync(d_misc + 1, 0xFF, 4, st));
    SWB_CUDA(cudaMemsetAsync(ctx->d_counters, 0, sizeof(unsigned long long) * kNumCounters, st));
    g.exts = ctx->d_counters + kCntSeed;
    SWB_CUDA(cudaEventRecord(ctx->ev_start, st));
    {
        ProfScope ps(ctx, st, "seed_order", -1);
        uint32_t *keys = (uint32_t *)ctx->d_keys.p, *keys2 = (uint32_t *)ctx->d_keys2.p;
        uint32_t *idx = (uint32_t *)ctx->d_idx.p, *order = (uint32_t *)ctx->d_idx2.p;
        const unsigned ob = 256;
        seed_order_keys_kernel<<<(unsigned)((n_reads + ob - 1) / ob), ob, 0, st>>>(d_b, d_off, d_len, (uint32_t)n_reads,
                                                                                   keys, idx);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
        SWB_CUDA(cub::DeviceRadixSort::SortPairs(ctx->d_sort_tmp.p, sort_bytes, keys, keys2, idx, order, (int)n_reads, 0,
                                                 9, st));
        g.order = order;
    }
    {
        ProfScope ps(ctx, st, "smem_search", kCntSeed);
        smem_kernel<<<(unsigned)blocks, kSeedT, 0, st>>>(g);
    }
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    SWB_CUDA(cudaEventRecord(ctx->ev_stop, st));
    // Offsets: the running sum of every read's full count.
    const unsigned cb = 256, cg = (unsigned)((n_reads + cb - 1) / cb);
    u32_to_u64_kernel<<<cg, cb, 0, st>>>(d_n, d_n64, (uint32_t)n_reads);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(d_scan_tmp, scan_bytes, d_n64, d_off64, (int)n_reads, st));
    uint32_t first_over = 0;
    if ((rc = d2h_staged(ctx, st, {DevSpan{d_n, n_out, n_reads * 4}, DevSpan{d_off64, out_off, n_reads * 8},
                                   DevSpan{d_misc + 1, &first_over, 4}})))
        return rc;
    const uint64_t total = out_off[n_reads - 1] + n_out[n_reads - 1];
    if (total > out_cap)
        return set_error(SWB_ERR_TOO_LARGE, std::to_string(total) + " SMEMs, more than out_cap (" +
                                                std::to_string(out_cap) + ")");
    if (total) {
        // Pack the windows in read order, then copy just those entries back.
        if ((rc = ensure_dev(ctx, ctx->d_aux, total * sizeof(swb_smem)))) return rc;
        swb_smem *d_pack = (swb_smem *)ctx->d_aux.p;
        smem_pack_kernel<<<cg, cb, 0, st>>>(d_out, d_n, d_off64, (uint32_t)n_reads, cap_per_read, d_pack);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
        if ((rc = d2h_staged(ctx, st, {DevSpan{d_pack, out, total * sizeof(swb_smem)}}))) return rc;
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) ctx->last_ms = ms;
    unsigned long long exts = 0;
    if (cudaMemcpy(&exts, ctx->d_counters + kCntSeed, sizeof(exts), cudaMemcpyDeviceToHost) == cudaSuccess)
        ctx->last_cells = exts;
    if (first_over != 0xFFFFFFFFu)
        return set_error(SWB_ERR_TOO_LARGE, "read " + std::to_string(first_over) + ": " +
                                                std::to_string(n_out[first_over]) + " SMEMs, more than cap_per_read (" +
                                                std::to_string(cap_per_read) + ")");
    return SWB_OK;
}

}  // extern "C"
