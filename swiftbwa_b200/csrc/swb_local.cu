// swb_local.cu -- kernel 3: local Smith-Waterman for mate rescue, bit-exact
// with LocalSWAligner.align (Sources/Alignment/LocalSWAligner.swift:42-493).
//
// The reference runs Farrar's striped algorithm on SIMD16<UInt8> (16 lanes,
// sn = ceil(qLen/16) stripes, lane l of stripe s holding query position
// s + l*sn) with a single-pass lazy-F correction and a per-stripe
// first-lane tie-break.  That is not the textbook SW recurrence, so a
// wavefront kernel would not match it.  Here a 16-thread half-warp plays
// the 16 SIMD lanes: thread l keeps lane l of every stripe's H and E in
// registers (the stripe count is a template parameter, one instantiation
// per sn, tasks binned by it), the lane shifts are __shfl_up_sync within the
// half, the position of a new column maximum is a segment minimum and a
// ballot, and the lazy-F early break is a ballot.  All arithmetic is the
// reference's u8 wrap/saturate arithmetic, its saturating steps folded into
// DPX add-max forms where that is exact.
// Tasks the reference sends to its scalar int32 fallback (qLen*A > 250,
// u8 overflow, a zero forward score, or a failed reverse pass) are
// appended to a device list and finished by a one-thread-per-task kernel
// that restates scalarAlign/scalarSWPass (:327-492).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <atomic>

#include "swb_device.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

constexpr int kLT = 128;          // threads per block, striped kernel (8 tasks)
constexpr int kST = 64;           // threads per block, scalar fallback
constexpr unsigned kFull = 0xFFFFFFFFu;

struct LocalArgs {
    DevScoring sc;
    const uint8_t *bases;
    const uint8_t *pac;
    const swb_local_task *tasks;
    swb_local_result *out;
    const uint32_t *order;
    const uint32_t *bin_start;   // 18 entries: bin 0 = scalar, bins 1..16 = stripes
    uint32_t *fallback;          // task indices for the scalar kernel
    unsigned int *fallback_n;
    unsigned long long *cells;
    uint32_t *claim;             // per-bin claim counters (zeroed per call)
};

__device__ __forceinline__ int clamp_min_sub(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }

// Profile table of one target base: byte q = UInt8(clamping: mat[t][q] + bias)
// for q in 0..4 (LocalSWAligner.swift:153-167); byte 5 = 0 for padding lanes.
__device__ __forceinline__ RowTable prof_table(const DevScoring &sc, uint32_t t, int bias) {
    auto cl = [](int v) -> uint32_t { return (uint32_t)(v < 0 ? 0 : (v > 255 ? 255 : v)); };
    const uint32_t A = cl(sc.a + bias), B = cl(-sc.b + bias), N = cl(-1 + bias);
    RowTable r;
    if (t >= 4) {
        r.lo = N * 0x01010101u;
    } else {
        r.lo = B * 0x01010101u;
        r.lo = (r.lo & ~(0xFFu << (8 * t))) | (A << (8 * t));
    }
    r.hi = N;   // byte 4 = N column, byte 5 = 0
    return r;
}

__device__ __forceinline__ int seg_min16(int v) {
    v = min(v, __shfl_xor_sync(kFull, v, 8));
    v = min(v, __shfl_xor_sync(kFull, v, 4));
    v = min(v, __shfl_xor_sync(kFull, v, 2));
    v = min(v, __shfl_xor_sync(kFull, v, 1));
    return v;
}

__device__ __forceinline__ int seg_max16(int v) {
    v = max(v, __shfl_xor_sync(kFull, v, 8));
    v = max(v, __shfl_xor_sync(kFull, v, 4));
    v = max(v, __shfl_xor_sync(kFull, v, 2));
    v = max(v, __shfl_xor_sync(kFull, v, 1));
    return v;
}

struct PassOut {
    int score, qEnd, tEnd, score2;
    bool nil;
};

// simdSWPass (:133-306) for one task per half-warp.  `act` is uniform per
// half; the loop trip counts are uniform per warp so every shuffle/vote sees
// all 32 lanes.  rev: read query/target reversed over their given lengths.
// FULL: every active task of the warp has exactly SN stripes (the forward
// pass always: tasks are binned by stripe count), so the stripe loops run
// with a constant trip count; inactive half-warps stay at zero.
template <int SN, bool FULL>
__device__ PassOut striped_pass(const LocalArgs &a, const swb_local_task &tk, bool act, int qLen, int tLen,
                                bool rev, int minSub, uint32_t *peaks, int lane, unsigned half_mask) {
    const DevScoring &sc = a.sc;
    const int bias = sc.b & 0xFF;                        // UInt8(mismatchPenalty)
    const int gOE = (sc.o_ins + sc.e_ins) & 0xFF, gE = sc.e_ins & 0xFF;
    // subs(max(subs(x, gOE), y), gE) over u8 values is max(x - gOE - gE, y - gE, 0).
    const int gOEE = gOE + gE;
    const int sn = FULL ? SN : (act ? (qLen + 15) / 16 : 0);
    int qc[SN], H[SN], E[SN];   // qc: prmt selector of the query code (byte 5 = 0 fills the upper bytes)
#pragma unroll
    for (int s = 0; s < SN; ++s) {
        const int j = s + lane * sn;
        uint32_t code = 5;
        if (act && s < sn && j < qLen)
            code = span_base(a.bases, a.pac, tk.q_off, rev ? (qLen - 1 - j) : j, tk.qlen, tk.flags, false);
        qc[s] = (int)(code | 0x5550u);
        H[s] = 0;
        E[s] = 0;
    }
    const bool trackPeaks = minSub > 0;
    int maxBase = 0;                                     // :192-199
    if (trackPeaks) {
        auto cl = [](int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); };
        maxBase = max(max(cl(sc.a + bias), cl(-sc.b + bias)), cl(-1 + bias));
        maxBase = maxBase > bias ? maxBase - bias : 0;
    }
    int maxScore = 0, maxI = -1, maxJ = -1;
    int nPeaks = 0, lastPeak = 0;                        // lastPeak = (score << 16) | col
    bool nil = false;
    const int tLenAll = max(act ? tLen : 0, __shfl_xor_sync(kFull, act ? tLen : 0, 16));
    // Target bases, 16 columns per load: lane l holds column c0 + l of its
    // half's task (c0 a multiple of 16), the next 16 are loaded a block ahead,
    // and column i is a shuffle from lane i % 16.
    auto tload = [&](int c) -> uint32_t {
        return act && c < tLen ? span_base(a.bases, a.pac, tk.t_off, rev ? (tLen - 1 - c) : c, tk.tlen, tk.flags, true)
                               : 4u;
    };
    uint32_t tcur = tload(lane), tnext = tload(16 + lane);
    for (int i = 0; i < tLenAll; ++i) {
        const bool live = act && !nil && i < tLen;
        if (i > 0 && (i & 15) == 0) {   // warp-uniform
            tcur = tnext;
            tnext = tload(i + 16 + lane);
        }
        uint32_t tb = __shfl_sync(kFull, tcur, i & 15, 16);
        if (!live) tb = 4;
        tb = min(tb, 4u);                                // :202
        const RowTable rt = prof_table(sc, tb, bias);
        int last = 0;
#pragma unroll
        for (int s = 0; s < SN; ++s)
            if (s == sn - 1) last = H[s];
        int vH = __shfl_up_sync(kFull, last, 1, 16);    // shiftRight(hArr[sn-1]) (:206)
        if (lane == 0) vH = 0;
        int f = 0;
#pragma unroll
        for (int s = 0; s < SN; ++s) {                   // :209-231
            if (s < sn) {
                const int prof = (int)prmt(rt.lo, rt.hi, (uint32_t)qc[s]);     // score + bias, one byte
                const int hRaw = (vH + prof) & 0xFF;
                const int hPrev = H[s];
                vH = hPrev;
                const int eVal = __viaddmax_s32_relu(hPrev, -gOEE, E[s] - gE);   // subs(max(subs(H, gOE), E), gE)
                E[s] = eVal;
                const int hNew = __vimax3_s32(__viaddmax_s32(hRaw, -bias, 0), eVal, f);   // max(subs(h, bias), E, F)
                H[s] = hNew;
                f = __viaddmax_s32_relu(hNew, -gOEE, f - gE);                   // subs(max(subs(H, gOE), F), gE)
            }
        }
        int corrF = __shfl_up_sync(kFull, f, 1, 16);     // lazy-F (:234-242)
        if (lane == 0) corrF = 0;
        bool going = act && sn > 0;
#pragma unroll
        for (int s = 0; s < SN; ++s) {
            if (!__any_sync(kFull, going)) break;
            going = going && s < sn;
            int newH = H[s];
            if (going) newH = max(H[s], corrF);
            const unsigned changed = __ballot_sync(kFull, going && newH != H[s]) & half_mask;
            if (going && changed == 0) going = false;
            if (going) {
                H[s] = newH;
                corrF = __viaddmax_s32_relu(newH, -gOEE, corrF - gE);
            }
        }
        int m = 0;                                       // column max (:245-263)
#pragma unroll
        for (int s = 0; s < SN; ++s)
            if (s < sn) m = max(m, H[s]);
        const int colMax = seg_max16(m);
        if (live && colMax > 250) nil = true;
        const bool need = live && !nil && colMax > maxScore;
        // The stripe walk below takes, among the stripes whose lane maximum
        // sets a new running maximum, the last one where a real (non-padding)
        // lane holds that maximum.  The last new maximum is colMax itself, at
        // the first stripe fs whose lane maximum equals it; when a real lane
        // holds colMax there, that is the answer (first such lane), found with
        // one segment minimum and one ballot.  Otherwise (colMax only in
        // padding lanes at fs) the walk runs.
        bool walk = false;
        if (__any_sync(kFull, need)) {
            int fs = SN;                                   // this lane's first stripe holding colMax
#pragma unroll
            for (int s = SN - 1; s >= 0; --s)
                if (s < sn && H[s] == colMax) fs = s;
            const int fsAll = seg_min16(fs);
            int hAt = -1;
#pragma unroll
            for (int s = 0; s < SN; ++s)
                if (s == fsAll) hAt = H[s];
            const unsigned hit = __ballot_sync(kFull, need && hAt == colMax && fsAll + lane * sn < qLen) & half_mask;
            if (need) {
                if (hit) {
                    maxScore = colMax;
                    maxI = i;
                    const int l = __ffs(hit) - 1 - ((half_mask & 1u) ? 0 : 16);
                    maxJ = fsAll + l * sn;
                } else {
                    walk = true;
                }
            }
        }
        if (__any_sync(kFull, walk)) {
#pragma unroll
            for (int s = 0; s < SN; ++s) {
                const int lm = seg_max16(s < sn ? H[s] : 0);
                const int j = s + lane * sn;
                const unsigned hit = __ballot_sync(kFull, walk && s < sn && H[s] == lm && j < qLen) & half_mask;
                if (walk && s < sn && lm > maxScore) {
                    maxScore = lm;
                    maxI = i;
                    if (hit) {
                        const int l = __ffs(hit) - 1 - ((half_mask & 1u) ? 0 : 16);
                        maxJ = s + l * sn;
                    }
                }
            }
        }
        if (live && !nil && trackPeaks && colMax >= minSub) {   // :266-286
            if (nPeaks == 0 || (lastPeak & 0xFFFF) + 1 != i) {
                lastPeak = (colMax << 16) | i;
                if (lane == 0) peaks[nPeaks] = (uint32_t)lastPeak;
                ++nPeaks;
            } else if ((lastPeak >> 16) < colMax) {
                lastPeak = (colMax << 16) | i;
                if (lane == 0) peaks[nPeaks - 1] = (uint32_t)lastPeak;
            }
        }
    }
    PassOut o{maxScore, maxJ, maxI, 0, nil || !act};
    // score2 (:290-303): all 16 lanes scan the peak list.
    __syncwarp();
    int s2 = 0;
    const bool do2 = act && !nil && trackPeaks && nPeaks > 0 && maxScore > 0 && maxBase > 0;
    if (do2) {
        const int r = (maxScore + maxBase - 1) / maxBase;
        const int low = maxI - r, high = maxI + r;
        for (int k = lane; k < nPeaks; k += 16) {
            const uint32_t e = peaks[k];
            const int col = (int)(e & 0xFFFFu), scv = (int)(e >> 16);
            if ((col < low || col > high) && scv > s2) s2 = scv;
        }
    }
    s2 = seg_max16(s2);
    o.score2 = do2 ? s2 : 0;
    return o;
}

// Five 128-thread blocks per SM (96 registers: no spills up to 10 stripes,
// 44-164 bytes per thread from 11 to 16; six blocks spill more).  The grid
// is the device's resident blocks; each
// half-warp claims its next task of the bin from the bin's counter, longest
// target first (the sort puts them last), so the launch ends with the work
// rather than on a partly filled last wave of fixed slices.
template <int SN>
__global__ void __launch_bounds__(kLT, 5) local_striped_kernel(LocalArgs a, int bin, uint32_t *peaks_base,
                                                            int peak_stride) {
    const int lane = threadIdx.x & 15;
    const unsigned half_mask = (threadIdx.x & 16) ? 0xFFFF0000u : 0x0000FFFFu;
    const uint32_t lo = a.bin_start[bin], hi = a.bin_start[bin + 1];
    const uint32_t my_half = blockIdx.x * (kLT / 16) + (threadIdx.x >> 4);
    uint32_t *peaks = peaks_base + (size_t)my_half * peak_stride;
    unsigned long long cells = 0;
    const uint32_t span = hi - lo;
    bool done = false;
    for (;;) {
        uint32_t k = 0;
        if (!done && lane == 0) k = atomicAdd(a.claim + bin, 1u);
        k = __shfl_sync(kFull, k, threadIdx.x & 16);   // the half's claim
        done = done || k >= span;
        if (__all_sync(kFull, done)) break;            // both halves of the warp go on together
        const uint32_t pos = hi - 1 - k;
        const bool act = !done;
        const uint32_t ti = act ? a.order[pos] : 0;
        swb_local_task tk{};
        if (act) tk = a.tasks[ti];
        const int minSub = clamp_min_sub(tk.min_sub_score);
        PassOut fwd = striped_pass<SN, true>(a, tk, act, tk.qlen, tk.tlen, false, minSub, peaks, lane, half_mask);
        if (act && lane == 0) cells += (unsigned long long)tk.qlen * tk.tlen;
        const bool fwd_ok = act && !fwd.nil && fwd.score > 0;
        const int revQ = fwd.qEnd + 1, revT = fwd.tEnd + 1;
        const bool do_rev = fwd_ok && revQ > 0 && revT > 0;
        const bool rev_full = __all_sync(kFull, !do_rev || (revQ + 15) / 16 == SN);
        PassOut rv = rev_full ? striped_pass<SN, true>(a, tk, do_rev, revQ, revT, true, 0, peaks, lane, half_mask)
                              : striped_pass<SN, false>(a, tk, do_rev, revQ, revT, true, 0, peaks, lane, half_mask);
        if (do_rev && lane == 0) cells += (unsigned long long)revQ * revT;
        if (act && lane == 0) {
            if (do_rev && !rv.nil) {
                a.out[ti] = swb_local_result{fwd.score, fwd.qEnd - rv.qEnd, fwd.qEnd, fwd.tEnd - rv.tEnd,
                                             fwd.tEnd, fwd.score2};
            } else {
                const unsigned slot = atomicAdd(a.fallback_n, 1u);
                a.fallback[slot] = ti;
            }
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) cells += __shfl_down_sync(kFull, cells, o);
    if ((threadIdx.x & 31) == 0 && cells) atomicAdd(a.cells + kCntLocalStriped, cells);
}

// scalarSWPass (:383-492) over spans read through span_base.
struct ScalarPass {
    int score, qEnd, tEnd, score2;
};

__device__ ScalarPass scalar_pass(const LocalArgs &a, const swb_local_task &tk, int qLen, int tLen, bool rev,
                                  int minSub, int *h, int *e, unsigned long long *peaks, size_t stride) {
    const DevScoring &sc = a.sc;
    const int gapOE = sc.o_ins + sc.e_ins, gapE = sc.e_ins;
    for (int j = 0; j <= tLen; ++j) {
        h[(size_t)j * stride] = 0;
        e[(size_t)j * stride] = 0;
    }
    int best = 0, bq = -1, bt = -1;
    const bool trackPeaks = minSub > 0;
    int nPeaks = 0;
    unsigned long long last = 0;
    int maxBase = 0;
    if (trackPeaks) maxBase = max(max((int)(int8_t)sc.a, (int)(int8_t)(-sc.b)), max(-1, 0));
    for (int i = 0; i < qLen; ++i) {
        const uint32_t qb = min(span_base(a.bases, a.pac, tk.q_off, rev ? (qLen - 1 - i) : i, tk.qlen, tk.flags, false), 4u);
        const RowTable rt = row_table(sc, qb);   // mat is symmetric: row q, column t
        int f = 0, hPrev = 0, rowMax = 0;
        for (int j = 0; j < tLen; ++j) {
            const int j1 = j + 1;
            const uint32_t tb = min(span_base(a.bases, a.pac, tk.t_off, rev ? (tLen - 1 - j) : j, tk.tlen, tk.flags, true), 4u);
            int hCur = hPrev + row_score(rt, tb);
            const int hj1 = h[(size_t)j1 * stride];
            const int fOpen = hj1 - gapOE, fExt = f - gapE;
            f = fOpen > fExt ? fOpen : fExt;
            const int eOpen = h[(size_t)j * stride] - gapOE, eExt = e[(size_t)j1 * stride] - gapE;
            const int eVal = eOpen > eExt ? eOpen : eExt;
            e[(size_t)j1 * stride] = eVal;
            hCur = hCur > f ? hCur : f;
            hCur = hCur > eVal ? hCur : eVal;
            hCur = hCur > 0 ? hCur : 0;
            hPrev = hj1;
            h[(size_t)j1 * stride] = hCur;
            if (hCur > rowMax) rowMax = hCur;
            if (hCur > best) {
                best = hCur;
                bq = i;
                bt = j;
            }
        }
        if (trackPeaks && rowMax >= minSub) {
            const unsigned long long rm = (unsigned long long)(uint32_t)rowMax, iu = (unsigned long long)(uint32_t)i;
            if (nPeaks == 0 || (int)(uint32_t)(last & 0xFFFFFFFFull) + 1 != i) {
                last = (rm << 32) | iu;
                peaks[(size_t)nPeaks * stride] = last;
                ++nPeaks;
            } else if ((last >> 32) < rm) {
                last = (rm << 32) | iu;
                peaks[(size_t)(nPeaks - 1) * stride] = last;
            }
        }
    }
    int score2 = 0;
    if (trackPeaks && nPeaks > 0 && best > 0 && maxBase > 0) {
        const int r = (best + maxBase - 1) / maxBase;
        const int low = bq - r, high = bq + r;
        for (int k = 0; k < nPeaks; ++k) {
            const unsigned long long en = peaks[(size_t)k * stride];
            const int col = (int)(uint32_t)(en & 0xFFFFFFFFull), scv = (int)(en >> 32);
            if ((col < low || col > high) && scv > score2) score2 = scv;
        }
    }
    return ScalarPass{best, bq, bt, score2};
}

__global__ void __launch_bounds__(kST) local_scalar_kernel(LocalArgs a, int *hbuf, int *ebuf,
                                                           unsigned long long *pbuf, size_t nslots) {
    const size_t slot = blockIdx.x * (size_t)kST + threadIdx.x;
    const unsigned n = *a.fallback_n;
    unsigned long long cells = 0;
    for (size_t k = slot; k < n; k += nslots) {
        const uint32_t ti = a.fallback[k];
        const swb_local_task tk = a.tasks[ti];
        swb_local_result r{0, 0, 0, 0, 0, 0};
        const int qLen = tk.qlen, tLen = tk.tlen;
        if (qLen > 0 && tLen > 0) {
            const ScalarPass fw = scalar_pass(a, tk, qLen, tLen, false, clamp_min_sub(tk.min_sub_score), hbuf + slot,
                                              ebuf + slot, pbuf + slot, nslots);
            cells += (unsigned long long)qLen * tLen;
            if (fw.score > 0) {
                const int rq = fw.qEnd + 1, rt = fw.tEnd + 1;
                const ScalarPass rv = scalar_pass(a, tk, rq, rt, true, 0, hbuf + slot, ebuf + slot, pbuf + slot, nslots);
                cells += (unsigned long long)rq * rt;
                r = swb_local_result{fw.score, fw.qEnd - rv.qEnd, fw.qEnd, fw.tEnd - rv.tEnd, fw.tEnd, fw.score2};
            }
        }
        a.out[ti] = r;
    }
    for (int o = 16; o > 0; o >>= 1) cells += __shfl_down_sync(kFull, cells, o);
    if ((threadIdx.x & 31) == 0 && cells) atomicAdd(a.cells + kCntLocalScalar, cells);
}

// Bin: 0 = scalar (qLen*A > 250 or empty), else the stripe count.
__global__ void local_keys_kernel(const swb_local_task *__restrict__ tasks, size_t n, int a_score,
                                  uint32_t *__restrict__ keys, uint32_t *__restrict__ idx) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const swb_local_task t = tasks[i];
    int bin = 0;
    if (t.qlen > 0 && t.tlen > 0 && (long long)t.qlen * a_score <= 250) bin = (t.qlen + 15) / 16;
    keys[i] = ((uint32_t)bin << 24) | (uint32_t)min(max(t.tlen, 0), 0xFFFFFF);
    idx[i] = (uint32_t)i;
}

__global__ void local_bounds_kernel(const uint32_t *__restrict__ sorted_keys, const uint32_t *__restrict__ order,
                                    size_t n, uint32_t *__restrict__ bin_start, uint32_t *__restrict__ fallback,
                                    unsigned int *__restrict__ fallback_n) {
    const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int b = (int)(sorted_keys[p] >> 24);
    const int bprev = p == 0 ? -1 : (int)(sorted_keys[p - 1] >> 24);
    for (int bb = bprev + 1; bb <= b; ++bb) bin_start[bb] = (uint32_t)p;
    if (p == n - 1)
        for (int bb = b + 1; bb <= 17; ++bb) bin_start[bb] = (uint32_t)n;
    if (b == 0) {   // scalar bin goes straight to the fallback list
        const unsigned slot = atomicAdd(fallback_n, 1u);
        fallback[slot] = order[p];
    }
}

template <int SN>
int launch_sn(swb_ctx *ctx, const LocalArgs &a, cudaStream_t st, uint32_t *peaks, int peak_stride, size_t halves_cap,
              size_t n_bin) {
    // Resident blocks per SM of this instance (the same on every device the
    // library runs on: sm_100).
    static std::atomic<int> occ{0};
    if (occ.load(std::memory_order_relaxed) == 0) {
        int b = 0;
        SWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, local_striped_kernel<SN>, kLT, 0));
        occ.store(b > 0 ? b : 1, std::memory_order_relaxed);
    }
    const size_t halves = std::min({halves_cap, n_bin, (size_t)ctx->sm_count * occ.load() * (kLT / 16)});
    const size_t grid = (halves + kLT / 16 - 1) / (kLT / 16);
    if (grid == 0) return SWB_OK;
    static const char *names[17] = {"", "local_striped_sn1", "local_striped_sn2", "local_striped_sn3",
                                    "local_striped_sn4", "local_striped_sn5", "local_striped_sn6",
                                    "local_striped_sn7", "local_striped_sn8", "local_striped_sn9",
                                    "local_striped_sn10", "local_striped_sn11", "local_striped_sn12",
                                    "local_striped_sn13", "local_striped_sn14", "local_striped_sn15",
                                    "local_striped_sn16"};
    ProfScope ps(ctx, st, names[SN], kCntLocalStriped);
    local_striped_kernel<SN><<<(unsigned)grid, kLT, 0, st>>>(a, SN, peaks, peak_stride);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    return SWB_OK;
}

}  // namespace

int launch_local(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases, const swb_local_task *d_tasks,
                 size_t n, swb_local_result *d_out, unsigned long long *d_cells, cudaStream_t st, int max_q,
                 int max_t) {
    if (n == 0) return SWB_OK;
    if (n > 0x7FFFFFF0ull) return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 tasks in one batch");
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_keys, n * 4)) || (rc = ensure_dev(ctx, ctx->d_keys2, n * 4)) ||
        (rc = ensure_dev(ctx, ctx->d_idx, n * 4)) || (rc = ensure_dev(ctx, ctx->d_idx2, n * 8)) ||
        (rc = ensure_dev(ctx, ctx->d_misc, 256)))
        return rc;
    uint32_t *keys = (uint32_t *)ctx->d_keys.p, *keys2 = (uint32_t *)ctx->d_keys2.p;
    uint32_t *idx = (uint32_t *)ctx->d_idx.p, *idx2 = (uint32_t *)ctx->d_idx2.p;
    uint32_t *fallback = idx2 + n;
    uint32_t *bin_start = (uint32_t *)ctx->d_misc.p;          // 18 words
    unsigned int *fallback_n = (unsigned int *)((char *)ctx->d_misc.p + 128);
    uint32_t *claim = (uint32_t *)((char *)ctx->d_misc.p + 160);   // 17 per-bin claim counters
    SWB_CUDA(cudaMemsetAsync(fallback_n, 0, 128, st));              // fallback count and claim counters
    local_keys_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_tasks, n, sc.a, keys, idx);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    size_t tmp = 0;
    SWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys2, idx, idx2, (int)n, 0, 32, st));
    if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp))) return rc;
    SWB_CUDA(cub::DeviceRadixSort::SortPairs(ctx->d_sort_tmp.p, tmp, keys, keys2, idx, idx2, (int)n, 0, 32, st));
    local_bounds_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(keys2, idx2, n, bin_start, fallback, fallback_n);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());

    // Peak lists (score2) live in scratch, one window of max_t entries per half-warp.
    const int peak_stride = imax(max_t, 1);
    const size_t halves_cap = (size_t)ctx->sm_count * 16 * (kLT / 16);
    const size_t nsl = (size_t)ctx->sm_count * 4 * kST;
    const size_t scalar_bytes = nsl * ((size_t)(max_t + 2) * 8 + (size_t)(max_q + 1) * 8);
    const size_t peak_bytes = halves_cap * (size_t)peak_stride * 4;
    if ((rc = ensure_dev(ctx, ctx->d_scratch, peak_bytes + scalar_bytes + 1024))) return rc;
    uint32_t *peaks = (uint32_t *)ctx->d_scratch.p;
    char *sp = (char *)ctx->d_scratch.p + ((peak_bytes + 255) & ~(size_t)255);
    int *hbuf = (int *)sp;
    int *ebuf = hbuf + (size_t)(max_t + 1) * nsl;
    unsigned long long *pbuf = (unsigned long long *)(ebuf + (size_t)(max_t + 1) * nsl);

    LocalArgs a{sc, d_bases, ctx->d_pac, d_tasks, d_out, idx2, bin_start, fallback, fallback_n, d_cells, claim};
    // Bin sizes are not known on the host; each instantiation's grid is the
    // device's resident blocks (fewer for small batches), whose half-warps
    // claim the bin's tasks and leave when it has none left.  Only stripe
    // counts that can occur for max_q are launched.
    const int max_sn = imin(16, (max_q + 15) / 16);
    using L = int (*)(swb_ctx *, const LocalArgs &, cudaStream_t, uint32_t *, int, size_t, size_t);
    static const L fns[17] = {nullptr,        launch_sn<1>,  launch_sn<2>,  launch_sn<3>,  launch_sn<4>,  launch_sn<5>,
                              launch_sn<6>,   launch_sn<7>,  launch_sn<8>,  launch_sn<9>,  launch_sn<10>, launch_sn<11>,
                              launch_sn<12>,  launch_sn<13>, launch_sn<14>, launch_sn<15>, launch_sn<16>};
    for (int sn = 1; sn <= max_sn; ++sn)
        if ((rc = fns[sn](ctx, a, st, peaks, peak_stride, halves_cap, n))) return rc;
    {
        ProfScope ps(ctx, st, "local_scalar_i32", kCntLocalScalar);
        local_scalar_kernel<<<(unsigned)(nsl / kST), kST, 0, st>>>(a, hbuf, ebuf, pbuf, nsl);
    }
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    return SWB_OK;
}

}  // namespace swb
