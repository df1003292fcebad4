// swb_ext_dp.cuh -- device-side restatement of BandedSWScalar.align
// (Sources/Alignment/BandedSWScalar.swift:21-191) over a row store, shared
// by the extension kernels of swb_ext.cu and swb_noalloc.cu.
#pragma once

#include "swb_device.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

struct ExtArgs {
    DevScoring sc;
    const uint8_t *bases;
    const uint8_t *pac;
    const swb_ext_task *tasks;
    swb_ext_result *out;
    const uint32_t *order;      // sorted task indices
    const uint32_t *bin_start;  // bins + 1 entries
    unsigned long long *cells;
    uint32_t *claim = nullptr;  // per-bin claim counters (zeroed per pass)
    int ring_above = 0x7FFFFFFF;   // queries longer than this keep their band as a ring (ext_row_len)
};

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

}  // namespace
}  // namespace swb
