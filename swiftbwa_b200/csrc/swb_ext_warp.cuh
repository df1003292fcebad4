// swb_ext_warp.cuh -- BandedSWScalar.align (Sources/Alignment/BandedSWScalar.swift:21-191)
// with one warp per extension, int32 scores, exact.
//
// The reference's row loop is sequential only through F:
//     diag(j) = M(j) ? M(j) + s(j) : 0          M(j) = h[j] before the row (H of the row above, column j-1)
//     H(j)    = max(diag(j), E(j), F(j))
//     E'(j)   = max(E(j) - eDel, diag(j) - oeDel, 0)
//     F(j+1)  = max(F(j) - eIns, diag(j) - oeIns, 0),   F(beg) = 0
// diag and E' are per column, and F is a max-plus prefix scan of
// diag(k) - oeIns with a decay of eIns per column, floored at 0 (the floor
// commutes with the max).  So a row runs as: each lane takes a contiguous
// chunk of the band; pass 1 folds its chunk's diag terms into one
// aggregate; a five-step shuffle scan over the lanes (decay eIns per
// column between chunk ends) gives every chunk its incoming F; pass 2
// recomputes diag, E', F and H per column.  The row's storage is the
// reference's: slot j keeps H of column j-1 of this row and E' of column j;
// each lane writes its own slots in place and the first slot of the next
// chunk (H of its last column) after the warp has finished reading, the row
// start keeps h1 = max(h0 - oDel - eDel(i+1), 0) when beg == 0, and
// h[end] = H(end-1), e[end] = 0.  Row max (last j on ties), z-drop and band
// narrowing (first / last nonzero slot) are warp reductions.
#pragma once

#include "swb_device.cuh"
#include "swb_ext_dp.cuh"

namespace swb {
namespace {

constexpr int kWarpMaxQ = 4096;          // longest query kept in shared memory per warp
constexpr int kWarpNeg = -(1 << 29);     // "no contribution yet" in the F scan

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = v > w ? v : w;
    }
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = v < w ? v : w;
    }
    return v;
}

// One extension by the calling warp; h, e: qlen+1 int32 slots, qc: qlen
// query codes, all private to the warp.
__device__ void ext_warp_one(const ExtArgs &a, const swb_ext_task &tk, int *h, int *e, uint8_t *qc,
                             swb_ext_result &res, unsigned long long &cells) {
    const int lane = threadIdx.x & 31;
    res = swb_ext_result{0, 0, 0, 0, 0, 0};
    const int qlen = tk.qlen, tlen = tk.tlen;
    if (!(qlen > 0 && tlen > 0)) return;                                      // :33-35
    const DevScoring &sc = a.sc;
    const int oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const int oeDel = oDel + eDel, oeIns = oIns + eIns;
    const int zDrop = sc.zdrop;
    const int h0 = tk.h0;
    // Query codes and the first row from h0 (:44-50, :65-77): the loop there
    // writes h0 - oIns - eIns*j for as long as that stays positive, so
    // h[j] = max(h0 - oIns - eIns*j, 0) for j >= 1.
    for (int j = lane; j < qlen; j += 32) qc[j] = (uint8_t)span_base(a.bases, a.pac, tk.q_off, j, qlen, tk.flags, false);
    for (int j = lane; j <= qlen; j += 32) {
        h[j] = j == 0 ? h0 : (int)max(0ll, (long long)h0 - oIns - (long long)eIns * j);
        e[j] = 0;
    }
    __syncwarp();
    int w = tk.w;                                                              // :52-62
    {
        const int maxIns = (int)((double)(qlen * sc.max_mat + tk.end_bonus - oIns) / (double)eIns + 1.0);
        w = imin(w, imax(1, maxIns));
        const int maxDel = (int)((double)(qlen * sc.max_mat + tk.end_bonus - oDel) / (double)eDel + 1.0);
        w = imin(w, imax(1, maxDel));
    }
    int maxScore = h0, maxI = -1, maxJ = -1, gScore = -1, gTle = -1, maxOff = 0;
    int beg = 0, end = qlen;
    for (int i = 0; i < tlen; ++i) {                                          // :90
        const RowTable rt = row_table(sc, span_base(a.bases, a.pac, tk.t_off, i, tlen, tk.flags, true));
        if (beg < i - w) beg = i - w;                                          // :95-97
        if (end > i + w + 1) end = i + w + 1;
        if (end > qlen) end = qlen;
        const int h1init = beg == 0 ? imax(h0 - (oDel + eDel * (i + 1)), 0) : 0;   // :99-107
        const int len = end - beg;
        int rowMax = 0, rowMaxJ = -1, h1last = h1init;
        if (len > 0) {
            if (lane == 0) cells += (unsigned long long)len;
            const int K = (len + 31) >> 5;
            const int s = beg + lane * K, t = imin(end, s + K);                // this lane's columns [s, t)
            // Pass 1: the chunk's F contribution at its end.
            int agg = kWarpNeg;
            for (int j = s; j < t; ++j) {
                const int M = h[j];
                const int diag = M != 0 ? M + row_score(rt, qc[j]) : 0;
                agg = imax(imax(agg - eIns, kWarpNeg), diag - oeIns);
            }
            // Inclusive scan over the lanes (full chunks of K columns apart).
            int incl = agg;
            for (int d = 1; d < 32; d <<= 1) {
                const int o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                const long long od = (long long)o - (long long)eIns * K * d;
                if (lane >= d) incl = imax(incl, (int)max(od, (long long)kWarpNeg));
            }
            const int prev = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
            int f = lane == 0 ? 0 : imax(prev, 0);
            // Pass 2: H, E' and F per column; slot j gets H of column j-1.
            int hPrevCol = 0, bestH = -1, bestJ = -1;
            for (int j = s; j < t; ++j) {
                const int M = h[j];
                const int ev = e[j];
                const int diag = M != 0 ? M + row_score(rt, qc[j]) : 0;
                const int H = imax(imax(diag, ev), f);
                e[j] = imax(ev - eDel, imax(diag - oeDel, 0));
                if (j > s) h[j] = hPrevCol;
                hPrevCol = H;
                if (H >= bestH) {
                    bestH = H;
                    bestJ = j;
                }
                f = imax(f - eIns, imax(diag - oeIns, 0));
            }
            __syncwarp();
            // Deferred writes: the first slot of the next chunk (or h[end]),
            // and the row start.
            if (s < t) h[t] = hPrevCol;
            if (lane == 0) h[beg] = h1init;
            const int lastLane = (len - 1) / K;
            if (lane == lastLane) e[end] = 0;                                  // :145-146
            h1last = __shfl_sync(0xFFFFFFFFu, hPrevCol, lastLane);
            // Row max, last j on ties.
            const unsigned long long key =
                bestJ < 0 ? 0ull : ((unsigned long long)(unsigned)bestH << 32) | (unsigned)bestJ;
            const unsigned long long best = warp_max(key);
            rowMax = (int)(best >> 32);
            rowMaxJ = (int)(best & 0xFFFFFFFFu);
            __syncwarp();
        } else {
            if (lane == 0) {
                h[end] = h1init;                                               // :145-146
                e[end] = 0;
            }
            __syncwarp();
        }
        if (end == qlen) {                                                     // :149-152
            gTle = gScore > h1last ? gTle : i;
            gScore = gScore > h1last ? gScore : h1last;
        }
        if (rowMax == 0) break;                                                // :155
        if (rowMax > maxScore) {                                               // :158-172
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
        // Narrowing (:175-180): first nonzero slot in [beg, end), then the
        // last nonzero slot in [nb, end].
        int first = end;
        for (int j = beg + lane; j < end; j += 32)
            if (h[j] != 0 || e[j] != 0) {
                first = j;
                break;
            }
        const int nb = warp_min(first);
        int last = nb - 1;
        for (int j = nb + lane; j <= end; j += 32)
            if (h[j] != 0 || e[j] != 0) last = j;
        const int ne = warp_max(last);
        beg = nb;
        end = imin(ne + 2, qlen);
        __syncwarp();
    }
    res = swb_ext_result{maxScore, maxJ + 1, maxI + 1, gTle + 1, gScore, maxOff};   // :183-190
}

}  // namespace
}  // namespace swb
