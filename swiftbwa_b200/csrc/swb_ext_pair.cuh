// swb_ext_pair.cuh -- BandedSWScalar.align (Sources/Alignment/BandedSWScalar.swift:21-191)
// for int16-bounded tasks, two target rows per pass.
//
// Row layout (shared memory, [column][thread]), one word per column: H of the
// previous row at the previous column (the diagonal input) in the low half,
// E into this column in the high half -- exactly the reference's h[j] / e[j]
// storage (`h[j]` holds the left neighbour's H once the row has passed it):
//   W16 = false: a 16-bit word of two bytes, for tasks whose scores are
//                bounded by 255 (three bytes per column with the query byte
//                keep ~17 one-warp blocks resident per SM at 128 columns);
//   W16 = true : a 32-bit word of two 16-bit halves, for scores bounded by
//                32000.
// One byte per column holds the query base q, from which the prmt selector
// (q, q|8, 5, 5) -- the row's score for q as a 16-bit value [s, sign, 0, 0]
// -- is formed with one multiply-add.
//
// Rows i and i+1 advance together, row i+1 one column behind row i: at step c
// row i computes column c from the word it loads, and row i+1 computes
// column c-1 from the values row i produced for column c-1 one step earlier
// (the word row i would have stored).  The two cells are independent, so they
// run as the low and high 16-bit lanes of one register through the DPX
// s16x2 forms: two shared loads (word, query byte), one 16-bit store and ~13 ALU
// operations per two cells.  Row i's words are never stored: row i+1
// consumes them from registers and overwrites the same columns.
//
// What the reference does between rows is kept exactly:
//   * row i+1 starts at max(first nonzero column of row i, i+1-w): the first
//     nonzero word of row i is known before row i+1 reaches it (it trails);
//   * row i+1 ends at min(last nonzero word of row i + 2, i+w+2, qlen); the
//     last nonzero word of row i is one past the last column where H > 0,
//     tracked per lane.  Until row i is complete, row i+1 runs on through
//     row i's zero tail; those cells see M = 0 and E = 0, so their H is F
//     decaying by eIns per column, below the last valid H of the row, and so
//     they never change the row maximum.  Once the end is known their words
//     are reset to what the reference holds there (zero), and the row-end
//     word h[end] = H(end-1), e[end] = 0 is written;
//   * rowMax == 0 and z-drop stop the task after row i before row i+1's
//     results are used; row i+1's own checks follow in order;
//   * band narrowing after row i+1: the first nonzero word by the reference's
//     scan, the last one from lane 1's last column with H > 0.
// Ring rows (RING = true, for queries longer than the largest length class):
// when the band is narrower than the query, the task keeps P = 2w + 3
// columns, column c in slot c mod P.  A row pair starting at
// row i touches only columns i-w .. i+w+2 (the band clamps, the row-end word
// and the zero tail), so a slot is reused only after its column has left the
// band for good; columns P..qlen take their first-row value (the h0 ramp) and
// query base when they enter, at the row pair whose last column reaches them.
// The lockstep loop runs in segments that end where the slot wraps.
// The diagonal's M != 0 rule is min(M + s, Mcap) relu with Mcap >= M + s
// when M > 0 and 0 when M = 0: M*128 for byte scores, a 0/1 lane mask times
// 0x7FFF for 16-bit ones.  The row max (last column on ties) is a u16x2 key
// H*256 + j for byte scores and one s32 key (H << 16) + j per row otherwise.
#pragma once

#include <type_traits>

#include "swb_device.cuh"
#include "swb_ext_dp.cuh"

namespace swb {
namespace {

// Score of query selector `sel` (low 16 bits) against a row table, as
// [s, sign(s), 0, 0] (one 16-bit lane).
__device__ __forceinline__ uint32_t lane_score(const RowTable &rt, uint32_t sel) { return prmt(rt.lo, rt.hi, sel); }

struct PairConsts {
    uint32_t negOeDel, negOeIns, negEDel, negEIns;   // replicated in both 16-bit lanes
};

// Row words: 16-bit [H byte | E byte] or 32-bit [H16 | E16].
template <bool W16>
using RowWord = typename std::conditional<W16, uint32_t, uint16_t>::type;

// Mcap of the M != 0 rule for the lanes of M (see the header).
template <bool W16>
__device__ __forceinline__ uint32_t m_cap(uint32_t M) {
    if constexpr (W16) return __vimin3_u16x2(M, 0x00010001u, 0x00010001u) * 0x7FFFu;
    else return M * 128u;
}

// One cell in the low lane only (the high lane's inputs are zero).  `w` is the
// column's word as the reference's loop reads it; returns the new word (h1
// before, E') and updates h1, f, key, lastJ.  SYM: the open costs oDel+eDel
// and oIns+eIns are equal, so E' and F' share one operand.
template <bool SYM, bool W16>
__device__ __forceinline__ uint32_t single_cell(const PairConsts &pc, const RowTable &rt, uint32_t w, uint32_t sel,
                                                int j, uint32_t &h1, uint32_t &f, uint32_t &key, uint32_t &lastJ) {
    const uint32_t s = lane_score(rt, sel);
    const uint32_t M = W16 ? __byte_perm(w, 0u, 0x4410) : __byte_perm(w, 0u, 0x4440);   // [H, 0]
    const uint32_t e = W16 ? __byte_perm(w, 0u, 0x4432) : __byte_perm(w, 0u, 0x4441);   // [E, 0]
    const uint32_t d = __viaddmin_s16x2_relu(M, s, m_cap<W16>(M));
    const uint32_t H = __vimax3_s16x2(d, e, f);
    const uint32_t tDel = __viaddmax_s16x2(d, pc.negOeDel, 0x80008000u);
    const uint32_t nE = __viaddmax_s16x2_relu(e, pc.negEDel, tDel);
    const uint32_t tIns = SYM ? tDel : __viaddmax_s16x2(d, pc.negOeIns, 0x80008000u);
    f = __viaddmax_s16x2_relu(f, pc.negEIns, tIns);
    // [h1, E'] -> the column's new word
    const uint32_t up = W16 ? __byte_perm(h1, nE, 0x5410) : __byte_perm(h1, nE, 0x0040);
    if constexpr (W16) {
        key = (uint32_t)__viaddmax_s32((int)__byte_perm(H, 0u, 0x1044), j, (int)key);   // (H << 16) + j
        const uint32_t Hz = __vimin3_u16x2(H, 0x00010001u, 0x00010001u) * 0x7FFFu;                     // 0x7FFF where H > 0
        lastJ = __vimax3_u16x2(lastJ, __vimin3_u16x2((uint32_t)j, Hz, (uint32_t)j), lastJ);
    } else {
        const uint32_t Hs = H * 256u;
        key = __viaddmax_u16x2(Hs, (uint32_t)j, key);
        lastJ = __vimax3_u16x2(lastJ, __vimin3_u16x2((uint32_t)j, Hs, (uint32_t)j), lastJ);
    }
    h1 = H;
    return up;
}

template <bool W16>
__device__ __forceinline__ void store_up(RowWord<W16> *he, int T, int j, uint32_t up) {
    he[j * T] = (RowWord<W16>)up;
}

// prmt selector (q, q|8, 5, 5) of query code q (0-4).
__device__ __forceinline__ uint32_t sel_of(uint32_t q) { return q * 0x11u + 0x5580u; }

// Row-end bookkeeping of BandedSWScalar.swift:149-172 for row `row`; returns
// false when the task stops after this row.
struct RowTrack {
    int maxScore, maxI, maxJ, gScore, gTle, maxOff;
    __device__ __forceinline__ bool finish(int row, int rowMax, int rowMaxJ, int h1, bool atEnd, int zDrop,
                                           int eDel, int eIns) {
        if (atEnd) {                                                           // :149-152
            gTle = gScore > h1 ? gTle : row;
            gScore = gScore > h1 ? gScore : h1;
        }
        if (rowMax == 0) return false;                                         // :155
        if (rowMax > maxScore) {                                               // :158-172
            maxScore = rowMax;
            maxI = row;
            maxJ = rowMaxJ;
            const int off = abs(rowMaxJ - row);
            if (off > maxOff) maxOff = off;
        } else if (zDrop > 0) {
            const int dI = row - maxI, dJ = rowMaxJ - maxJ;
            if (dI > dJ) {
                if (maxScore - rowMax - (dI - dJ) * eDel > zDrop) return false;
            } else {
                if (maxScore - rowMax - (dJ - dI) * eIns > zDrop) return false;
            }
        }
        return true;
    }
};

template <int T, bool SYM, bool W16, bool RING>
__device__ __forceinline__ void ext_pair_one(const ExtArgs &a, const swb_ext_task &tk, RowWord<W16> *__restrict__ he,
                                             uint8_t *__restrict__ qc, swb_ext_result &res,
                                             unsigned long long &cells) {
    using Word = RowWord<W16>;
    constexpr uint32_t kLoMask = W16 ? 0xFFFFu : 0xFFu;      // one score field of a word
    res = swb_ext_result{0, 0, 0, 0, 0, 0};
    const int qlen = tk.qlen, tlen = tk.tlen;
    if (!(qlen > 0 && tlen > 0)) return;                                      // :33-35
    const DevScoring &sc = a.sc;
    const int oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const int zDrop = sc.zdrop;
    const int h0 = tk.h0;
    PairConsts pc;
    pc.negOeDel = (uint32_t)(uint16_t)(-(oDel + eDel)) * 0x10001u;
    pc.negOeIns = (uint32_t)(uint16_t)(-(oIns + eIns)) * 0x10001u;
    pc.negEDel = (uint32_t)(uint16_t)(-eDel) * 0x10001u;
    pc.negEIns = (uint32_t)(uint16_t)(-eIns) * 0x10001u;

    const int w = ext_band_w(qlen, tk.w, tk.end_bonus, sc);                  // :52-62
    // Columns held: the whole query, or the band's ring of 2w + 3.
    const int P = RING && qlen > a.ring_above ? ext_row_len(qlen, w) + 1 : qlen + 1;
    int wb = 0;   // ring: a multiple of P at or below every live column
    auto sl = [&](int c) -> int {
        if constexpr (!RING) {
            return c;
        } else {
            const int r = c - wb;
            return r >= P ? r - P : r;
        }
    };
    // Query profile and the first row from h0 (:44-50, :65-77); with a ring,
    // the columns that fit it (the rest enter with the band, below).
    {
        int hv = h0;
        bool ramp = h0 > oIns + eIns;
        for (int j = 0; j < P; ++j) {
            int hj = 0;
            if (j == 0) {
                hj = h0;
            } else if (j == 1) {
                if (ramp) hj = hv = h0 - oIns - eIns;
            } else if (ramp && hv > eIns) {
                hj = hv -= eIns;
            } else {
                ramp = false;
            }
            if (j < qlen) qc[j * T] = (uint8_t)span_base(a.bases, a.pac, tk.q_off, j, qlen, tk.flags, false);
            he[j * T] = (Word)hj;
        }
    }
    const bool tref = (tk.flags & SWB_T_FROM_REF) != 0;
    const bool tcomp = (tk.flags & SWB_T_COMPLEMENT) != 0;
    const long long tstep = (tk.flags & SWB_T_REVERSE) ? -1 : 1;
    const long long tbase = (tk.flags & SWB_T_REVERSE) ? (long long)tk.t_off + tlen - 1 : (long long)tk.t_off;
    auto row_tab = [&](int i) -> RowTable {
        const unsigned long long idx = (unsigned long long)(tbase + tstep * i);
        uint32_t tb = tref ? (a.pac[idx >> 2] >> ((3u - (uint32_t)(idx & 3)) << 1)) & 3u : a.bases[idx];
        if (tcomp && tb < 4u) tb = 3u - tb;
        return row_table(sc, tb);
    };
    auto h1_init = [&](int row) -> uint32_t {                                  // :99-107
        return (uint32_t)imax(h0 - (oDel + eDel * (row + 1)), 0);
    };

    // Ring: the first-row value of a column entering the ring (:65-77).
    auto ramp = [&](int c) -> int {
        const long long v = h0 > oIns + eIns ? (long long)h0 - oIns - (long long)eIns * c : 0;
        return v > 0 ? (int)v : 0;
    };
    RowTrack tr{h0, -1, -1, -1, -1, 0};
    int beg = 0, end = qlen;
    int i = 0;
    while (i < tlen) {
        if constexpr (RING) {
            // Slide the ring's base with the band, then bring in the columns
            // this row pair reaches first: the first-row value h0 - oIns -
            // eIns*c while positive (:65-77), else 0, and the query base.
            while (i - w >= wb + P) wb += P;
            const int cHi = imin(qlen, i + w + 2);
            for (int cc = imax(P, i + w + 1); cc <= cHi; ++cc) {
                const int k = sl(cc);
                he[k * T] = (Word)ramp(cc);
                if (cc < qlen) qc[k * T] = (uint8_t)span_base(a.bases, a.pac, tk.q_off, cc, qlen, tk.flags, false);
            }
        }
        if (beg < i - w) beg = i - w;                                          // :95-97
        if (end > i + w + 1) end = i + w + 1;
        if (end > qlen) end = qlen;
        const int b0 = beg, e0 = end;
        const RowTable rt0 = row_tab(i);
        uint32_t h1 = b0 == 0 ? h1_init(i) : 0u, f = 0u, key = 0u, lastJ = 0u;
        if (e0 > b0) cells += (unsigned long long)(e0 - b0);
        const bool pair = i + 1 < tlen;
        // ---- phase A: row i alone until row i+1 may start (or the row ends)
        const int lo1 = i + 1 - w;
        int firstNz = -1;                 // first nonzero word of row i
        int c = b0;
        uint32_t hPrev = 0u, nEPrev = 0u, sPrev = 0u;   // row i's word and selector for column c-1
        bool started = false;
        for (; c < e0; ++c) {
            const int k = sl(c);
            const uint32_t wd = he[k * T];
            const uint32_t sel = sel_of(qc[k * T]);
            const uint32_t hb = h1;
            const uint32_t up = single_cell<SYM, W16>(pc, rt0, wd, sel, c, h1, f, key, lastJ);
            hPrev = hb;
            nEPrev = W16 ? up >> 16 : up >> 8;   // E' of row i at column c (the word's high field)
            sPrev = sel;
            if (firstNz < 0 && (W16 ? up : up & 0xFFFFu) != 0u) firstNz = c;
            if (pair && firstNz >= 0 && c >= lo1) {
                ++c;
                started = true;
                break;
            }
        }
        nEPrev &= kLoMask;
        // ---- phase B: rows i and i+1 in lockstep (row i at c, row i+1 at c-1)
        const int beg1 = started ? c - 1 : -1;                                 // row i+1's first column, if known
        uint32_t h1p = h1, fp = f, lastJp = lastJ;                             // lane 0 = row i, lane 1 = row i+1
        // Row-max keys: byte scores one u16x2 key for both rows; 16-bit
        // scores one s32 key per row, row i+1's counting column + 1 while in
        // lockstep (corrected below).
        uint32_t keyp = key, key1w = 0u;
        const RowTable rt1 = pair ? row_tab(i + 1) : rt0;
        if (started) {
            h1p |= (beg1 == 0 ? h1_init(i + 1) : 0u) << 16;
            uint32_t hPrevP = hPrev;    // lane 0 of h1 before the previous step
            uint32_t jp = (uint32_t)c | ((uint32_t)(c - 1) << 16);
            // One lockstep step: row i's word for column c from slot ls, row i+1's
            // word for column c-1 into slot ss.
            auto step = [&](int ls, int ss) {
                const uint32_t wd = he[ls * T];
                const uint32_t sel = sel_of(qc[ls * T]);
                const uint32_t Mp = W16 ? __byte_perm(wd, hPrevP, 0x5410) : __byte_perm(wd, hPrevP, 0x5450);   // [H(i-1,c-1), H(i,c-2)]
                const uint32_t ep = W16 ? __byte_perm(wd, nEPrev, 0x5432) : __byte_perm(wd, nEPrev, 0x5451);   // [E(i,c),     E(i+1,c-1)]
                const uint32_t sp = lane_score(rt1, sPrev) * 65536u + lane_score(rt0, sel);
                const uint32_t d = __viaddmin_s16x2_relu(Mp, sp, m_cap<W16>(Mp));
                const uint32_t H = __vimax3_s16x2(d, ep, fp);
                const uint32_t tDel = __viaddmax_s16x2(d, pc.negOeDel, 0x80008000u);
                const uint32_t nE = __viaddmax_s16x2_relu(ep, pc.negEDel, tDel);
                const uint32_t tIns = SYM ? tDel : __viaddmax_s16x2(d, pc.negOeIns, 0x80008000u);
                fp = __viaddmax_s16x2_relu(fp, pc.negEIns, tIns);
                // row i+1's word for c-1
                store_up<W16>(he, T, ss, W16 ? __byte_perm(h1p, nE, 0x7632) : __byte_perm(h1p, nE, 0x0062));
                if constexpr (W16) {
                    keyp = (uint32_t)__viaddmax_s32((int)__byte_perm(H, 0u, 0x1044), c, (int)keyp);
                    key1w = (uint32_t)__viaddmax_s32((int)(H & 0xFFFF0000u), c, (int)key1w);
                    const uint32_t Hz = __vimin3_u16x2(H, 0x00010001u, 0x00010001u) * 0x7FFFu;
                    lastJp = __vimax3_u16x2(lastJp, __vimin3_u16x2(jp, Hz, jp), lastJp);
                } else {
                    const uint32_t Hs = H * 256u;
                    keyp = __viaddmax_u16x2(Hs, jp, keyp);
                    lastJp = __vimax3_u16x2(lastJp, __vimin3_u16x2(jp, Hs, jp), lastJp);
                }
                hPrevP = h1p;
                sPrev = sel;
                nEPrev = nE;    // low field = row i's E', the high lane's upper bits never reach a word
                h1p = H;
            };
            if constexpr (!RING) {
#pragma unroll 2
                for (; c < e0; ++c, jp += 0x10001u) step(c, c - 1);
            } else {
                int cs = sl(c);
                while (c < e0) {
                    if (cs == 0) {   // column c-1 sits in the ring's last slot
                        step(0, P - 1);
                        ++c, jp += 0x10001u, cs = 1;
                        continue;
                    }
                    const int segEnd = imin(e0, c + (P - cs));
#pragma unroll 2
                    for (; c < segEnd; ++c, ++cs, jp += 0x10001u) step(cs, cs - 1);
                    if (cs == P) cs = 0;
                }
            }
            hPrev = hPrevP & 0xFFFFu;
        }
        // ---- row i complete
        const int h1i = (int)(h1p & 0xFFFFu);
        const int key0 = W16 ? (int)keyp : (int)(keyp & 0xFFFFu);
        const int rowMax0 = e0 > b0 ? (W16 ? key0 >> 16 : key0 >> 8) : 0;
        const int rowMaxJ0 = W16 ? key0 & 0xFFFF : key0 & 0xFF;
        // (the last row's words, h[end] included, are never read again)
        if (!tr.finish(i, rowMax0, rowMaxJ0, h1i, e0 == qlen, zDrop, eDel, eIns)) break;
        if (!pair) break;   // last row
        // Narrowing after row i (:175-180): first nonzero word, last nonzero word = last H > 0 column + 1.
        const int lastH = (int)(lastJp & 0xFFFFu);
        const int bn = firstNz >= 0 ? firstNz : e0;
        const int en = imin(lastH + 3, qlen);
        // Row i+1's band (:95-97).
        int b1 = bn > i + 1 - w ? bn : i + 1 - w;
        int e1 = en < i + 1 + w + 1 ? en : i + 1 + w + 1;
        if (e1 > qlen) e1 = qlen;
        if (e1 > b1) cells += (unsigned long long)(e1 - b1);
        // ---- drain: row i+1 alone for its columns past the lockstep
        int s = started ? c - 1 : b1;                                          // next column of row i+1
        uint32_t f1 = fp >> 16, k1 = W16 ? key1w - 1u : keyp >> 16, lj1 = lastJp >> 16;
        uint32_t h1b = started ? (h1p >> 16) : (b1 == 0 ? h1_init(i + 1) : 0u);
        if (!started) f1 = 0u, k1 = 0u, lj1 = 0u;
        for (; s < e1; ++s) {
            // Row i's word for column s: from registers (c-1 = e0-1), the row-end word, or untouched.
            const int k = sl(s);
            uint32_t wd = he[k * T];
            if (s == e0 - 1) wd = hPrev | ((nEPrev & kLoMask) << (W16 ? 16 : 8));
            else if (s == e0) wd = (uint32_t)h1i;
            const uint32_t up = single_cell<SYM, W16>(pc, rt1, wd, sel_of(qc[k * T]), s, h1b, f1, k1, lj1);
            store_up<W16>(he, T, k, up);
        }
        // H of row i+1's last valid column: from the register if it was the last
        // cell computed, else from the word the lockstep stored at column e1.
        int h1last = (int)(h1b & 0xFFFFu);
        const bool overran = started && e1 <= e0 - 2;
        if (overran) h1last = (int)(he[sl(e1) * T] & kLoMask);
        const int key1 = W16 ? (int)k1 : (int)(k1 & 0xFFFFu);
        const int rowMax1 = e1 > b1 ? (W16 ? key1 >> 16 : key1 >> 8) : 0;
        const int rowMaxJ1 = W16 ? key1 & 0xFFFF : key1 & 0xFF;
        // Words the reference holds after row i+1: h[e1] = H(e1-1), e[e1] = 0,
        // then row i's zero tail up to e0.
        he[sl(e1) * T] = (Word)h1last;
        for (int z = e1 + 1; z <= e0; ++z) he[sl(z) * T] = 0;
        if (!tr.finish(i + 1, rowMax1, rowMaxJ1, h1last, e1 == qlen, zDrop, eDel, eIns)) break;
        // Narrowing after row i+1 (:175-180).
        int nb = b1;
        while (nb < e1 && he[sl(nb) * T] == 0) ++nb;
        beg = nb;
        // The last nonzero word is one past the last column with H > 0 (lane 1's
        // tracker; columns past e1 computed ahead of row i's end only decay from it).
        const int ne = imin((int)(lj1 & 0xFFFFu), e1 - 1) + 1;
        end = imin(ne + 2, qlen);
        i += 2;
    }
    res = swb_ext_result{tr.maxScore, tr.maxJ + 1, tr.maxI + 1, tr.gTle + 1, tr.gScore, tr.maxOff};   // :183-190
}

}  // namespace
}  // namespace swb
