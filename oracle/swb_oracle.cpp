// swb_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// Line-for-line C++ restatement of swiftbwa's Swift CPU Alignment functions
// (paths below are relative to the swiftbwa source tree).  Used only as the
// parity checker (tests/, __graft_entry__.smoke) and as the timed CPU
// baseline in bench.py.  Compiled with -fwrapv so that Int32 arithmetic
// wraps like the reference's -Ounchecked build (Package.swift:35-44).
//
// Swift semantics mirrored: `&+`/`&-` wrap; Int32(Double) truncates toward
// zero; UInt8(clamping:) clamps to 0..255; SIMD `.replacing(with:where:)`
// is a per-lane select; `max()` over a SIMD vector is the lane maximum.

#include "swb_oracle.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

// ScoringParameters.scoringMatrix -- Sources/BWACore/ScoringParameters.swift:65-73
void scoring_matrix(const swb_scoring *sc, int8_t mat[25]) {
    for (int k = 0; k < 25; ++k) mat[k] = -1;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            mat[i * 5 + j] = (i == j) ? (int8_t)sc->a : (int8_t)(-sc->b);
}

inline uint8_t clamp_u8(int v) { return (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v)); }

// --------------------------------------------------------------------------
// BandedSWScalar.align -- Sources/Alignment/BandedSWScalar.swift:21-191
// --------------------------------------------------------------------------
void banded_sw_scalar(const uint8_t *query, int qlen, const uint8_t *target, int tlen,
                      const swb_scoring *sc, int32_t w, int32_t h0, int32_t endBonus,
                      swb_ext_result *out, uint64_t *cells_out) {
    uint64_t cells = 0;
    *out = swb_ext_result{0, 0, 0, 0, 0, 0};
    if (cells_out) *cells_out = 0;
    if (!(qlen > 0 && tlen > 0)) return;                       // :33-35
    const int m = 5;
    int8_t mat[25];
    scoring_matrix(sc, mat);                                    // :37
    const int32_t oDel = sc->o_del, eDel = sc->e_del;
    const int32_t oIns = sc->o_ins, eIns = sc->e_ins;
    const int32_t zDrop = sc->zdrop;

    std::vector<int32_t> qp((size_t)m * qlen);                  // :44-50
    for (int k = 0; k < m; ++k)
        for (int j = 0; j < qlen; ++j) qp[(size_t)k * qlen + j] = mat[k * m + query[j]];

    int32_t maxMatScore = 0;                                    // :52-58
    for (int i = 0; i < m * m; ++i)
        if (mat[i] > maxMatScore) maxMatScore = mat[i];
    {                                                           // :59-62
        int32_t maxIns = (int32_t)((double)(qlen * maxMatScore + endBonus - oIns) / (double)eIns + 1.0);
        w = std::min(w, std::max<int32_t>(1, maxIns));
        int32_t maxDel = (int32_t)((double)(qlen * maxMatScore + endBonus - oDel) / (double)eDel + 1.0);
        w = std::min(w, std::max<int32_t>(1, maxDel));
    }

    std::vector<int32_t> h(qlen + 1, 0), e(qlen + 1, 0);       // :65-66
    h[0] = h0;                                                  // :69-77
    if (h0 > oIns + eIns) {
        h[1] = h0 - oIns - eIns;
        int j = 2;
        while (j <= qlen && h[j - 1] > eIns) {
            h[j] = h[j - 1] - eIns;
            j += 1;
        }
    }

    int32_t maxScore = h0, maxI = -1, maxJ = -1;                // :79-84
    int32_t gScore = -1, gTle = -1, maxOff = 0;
    int beg = 0, end = qlen;                                    // :86-87

    for (int i = 0; i < tlen; ++i) {                            // :90
        const int qpRow = target[i] * qlen;
        if (beg < i - w) beg = i - w;                           // :95-97
        if (end > i + w + 1) end = i + w + 1;
        if (end > qlen) end = qlen;

        int32_t f = 0;                                          // :99-107
        int32_t h1;
        if (beg == 0) {
            h1 = h0 - (oDel + eDel * (i + 1));
            if (h1 < 0) h1 = 0;
        } else {
            h1 = 0;
        }
        int32_t rowMax = 0, rowMaxJ = -1;
        cells += (uint64_t)(end > beg ? end - beg : 0);

        for (int j = beg; j < end; ++j) {                       // :112-143
            const int32_t M = h[j];
            const int32_t eVal = e[j];
            h[j] = h1;
            const int32_t diag = M != 0 ? M + qp[qpRow + j] : 0;
            int32_t hVal = diag > eVal ? diag : eVal;
            hVal = hVal > f ? hVal : f;
            h1 = hVal;
            rowMaxJ = rowMax > hVal ? rowMaxJ : j;
            rowMax = rowMax > hVal ? rowMax : hVal;
            int32_t t = diag - (oDel + eDel);
            if (t < 0) t = 0;
            int32_t newE = eVal - eDel;
            if (newE < t) newE = t;
            e[j] = newE;
            t = diag - (oIns + eIns);
            if (t < 0) t = 0;
            int32_t newF = f - eIns;
            if (newF < t) newF = t;
            f = newF;
        }
        h[end] = h1;                                            // :145-146
        e[end] = 0;

        if (end == qlen) {                                      // :149-152
            gTle = gScore > h1 ? gTle : i;
            gScore = gScore > h1 ? gScore : h1;
        }
        if (rowMax == 0) break;                                 // :155

        if (rowMax > maxScore) {                                // :158-172
            maxScore = rowMax;
            maxI = i;
            maxJ = rowMaxJ;
            int32_t off = std::abs(rowMaxJ - i);
            if (off > maxOff) maxOff = off;
        } else if (zDrop > 0) {
            int32_t deltaI = i - maxI;
            int32_t deltaJ = rowMaxJ - maxJ;
            if (deltaI > deltaJ) {
                if (maxScore - rowMax - (deltaI - deltaJ) * eDel > zDrop) break;
            } else {
                if (maxScore - rowMax - (deltaJ - deltaI) * eIns > zDrop) break;
            }
        }
        int newBeg = beg;                                       // :175-180
        while (newBeg < end && h[newBeg] == 0 && e[newBeg] == 0) newBeg += 1;
        beg = newBeg;
        int newEnd = end;
        while (newEnd >= beg && h[newEnd] == 0 && e[newEnd] == 0) newEnd -= 1;
        end = std::min(newEnd + 2, qlen);
    }
    out->score = maxScore;                                      // :183-190
    out->qle = maxJ + 1;
    out->tle = maxI + 1;
    out->gtle = gTle + 1;
    out->gscore = gScore;
    out->max_off = maxOff;
    if (cells_out) *cells_out = cells;
}

// --------------------------------------------------------------------------
// BandedSW16.align -- Sources/Alignment/BandedSW16.swift:8-203
// (secondary: the dead GPU path's CPU fallback; kept to replay its tests)
// --------------------------------------------------------------------------
typedef int16_t v8[8];
inline int16_t wadd16(int16_t a, int16_t b) { return (int16_t)(uint16_t)((uint16_t)a + (uint16_t)b); }
inline int16_t wsub16(int16_t a, int16_t b) { return (int16_t)(uint16_t)((uint16_t)a - (uint16_t)b); }
inline int16_t clamp_i16(long v) { return (int16_t)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v)); }

void banded_sw16(const uint8_t *query, int qlen, const uint8_t *target, int tlen,
                 const swb_scoring *sc, int32_t w, int32_t h0, swb_ext_result *out) {
    *out = swb_ext_result{0, 0, 0, 0, 0, 0};
    if (!(qlen > 0 && tlen > 0)) return;
    int8_t mat[25];
    scoring_matrix(sc, mat);
    const int m = 5, lanes = 8;
    const int sn = (qlen + lanes - 1) / lanes;
    const int16_t oIns = (int16_t)sc->o_ins, eIns = (int16_t)sc->e_ins;
    const int16_t oDel = (int16_t)sc->o_del, eDel = (int16_t)sc->e_del;
    const int32_t zDrop = sc->zdrop;
    std::vector<int16_t> profile((size_t)m * sn * lanes, 0), H((size_t)sn * lanes, 0), E((size_t)sn * lanes, 0);
    for (int k = 0; k < m; ++k)                                  // :48-60
        for (int s = 0; s < sn; ++s)
            for (int l = 0; l < lanes; ++l) {
                int j = s + l * sn;
                if (j < qlen) profile[((size_t)k * sn + s) * lanes + l] = mat[k * m + query[j]];
            }
    for (int s = 0; s < sn; ++s)                                 // :63-73
        for (int l = 0; l < lanes; ++l) {
            int j = s + l * sn;
            if (j < qlen && j + 1 <= w) {
                long val = (long)h0 - oIns - (long)eIns * (j + 1);
                if (val > 0) H[(size_t)s * lanes + l] = clamp_i16(val);
            }
        }
    int32_t maxScore = h0, maxI = -1, maxJ = -1, gScore = -1, gTle = -1, maxOff = 0;
    for (int i = 0; i < tlen; ++i) {
        const int16_t *prof = &profile[(size_t)target[i] * sn * lanes];
        int16_t vH[8], f[8];
        for (int l = 0; l < lanes; ++l) vH[l] = l == 0 ? 0 : H[(size_t)(sn - 1) * lanes + l - 1];
        if (i == 0) vH[0] = clamp_i16(std::max<long>(0, h0));
        for (int l = 0; l < lanes; ++l) f[l] = 0;
        for (int s = 0; s < sn; ++s) {                           // :100-130
            int16_t *Hs = &H[(size_t)s * lanes], *Es = &E[(size_t)s * lanes];
            int16_t hNew[8], hPrev[8];
            for (int l = 0; l < lanes; ++l) {
                int16_t x = wadd16(vH[l], prof[s * lanes + l]);
                if (x < 0) x = 0;
                if (vH[l] == 0) x = 0;
                hNew[l] = x;
                hPrev[l] = Hs[l];
            }
            for (int l = 0; l < lanes; ++l) {
                vH[l] = hPrev[l];
                int16_t a = wsub16(hPrev[l], oIns);
                int16_t mx = a > Es[l] ? a : Es[l];
                int16_t ev = wsub16(mx, eIns);
                if (ev < 0) ev = 0;
                Es[l] = ev;
                int16_t hh = hNew[l] > ev ? hNew[l] : ev;
                hh = hh > f[l] ? hh : f[l];
                Hs[l] = hh;
                int16_t hf = wsub16(hh, oDel);
                int16_t fm = hf > f[l] ? hf : f[l];
                int16_t fv = wsub16(fm, eDel);
                if (fv < 0) fv = 0;
                f[l] = fv;
            }
        }
        int16_t corrF[8];                                        // :133-141
        for (int l = 0; l < lanes; ++l) corrF[l] = l == 0 ? 0 : f[l - 1];
        for (int s = 0; s < sn; ++s) {
            int16_t *Hs = &H[(size_t)s * lanes];
            int16_t newH[8];
            bool same = true;
            for (int l = 0; l < lanes; ++l) {
                newH[l] = corrF[l] > Hs[l] ? corrF[l] : Hs[l];
                if (newH[l] != Hs[l]) same = false;
            }
            if (same) break;
            for (int l = 0; l < lanes; ++l) {
                Hs[l] = newH[l];
                int16_t hf = wsub16(Hs[l], oDel);
                int16_t fm = hf > corrF[l] ? hf : corrF[l];
                int16_t fv = wsub16(fm, eDel);
                if (fv < 0) fv = 0;
                corrF[l] = fv;
            }
        }
        int32_t rowMax = 0, rowMaxJ = -1;                         // :144-161
        for (int s = 0; s < sn; ++s) {
            int16_t *Hs = &H[(size_t)s * lanes];
            int16_t localMax = Hs[0];
            for (int l = 1; l < lanes; ++l) localMax = std::max(localMax, Hs[l]);
            if ((int32_t)localMax > rowMax) {
                rowMax = localMax;
                for (int l = 0; l < lanes; ++l)
                    if (Hs[l] == localMax) {
                        int j = s + l * sn;
                        if (j < qlen) { rowMaxJ = j; break; }
                    }
            }
        }
        if (rowMax == 0) break;
        if (rowMax > maxScore) {
            maxScore = rowMax; maxI = i; maxJ = rowMaxJ;
            int32_t off = std::abs(rowMaxJ - i);
            if (off > maxOff) maxOff = off;
        } else if (zDrop > 0) {
            int32_t dI = i - maxI, dJ = rowMaxJ - maxJ;
            if (dI > dJ) { if (maxScore - rowMax - (dI - dJ) * sc->e_del > zDrop) break; }
            else { if (maxScore - rowMax - (dJ - dI) * sc->e_ins > zDrop) break; }
        }
        int lastJ = qlen - 1;                                     // :185-192
        int32_t hAtEnd = H[(size_t)(lastJ % sn) * lanes + lastJ / sn];
        if (hAtEnd > gScore) { gScore = hAtEnd; gTle = i; }
    }
    *out = swb_ext_result{maxScore, maxJ + 1, maxI + 1, gTle + 1, gScore, maxOff};
}

// --------------------------------------------------------------------------
// BandedSW8.align -- Sources/Alignment/BandedSW8.swift:10-213
// --------------------------------------------------------------------------
inline uint8_t satsub_u8(uint8_t a, uint8_t b) { return (uint8_t)((a > b ? a : b) - b); }  // pmax(a,b) &- b

int banded_sw8(const uint8_t *query, int qlen, const uint8_t *target, int tlen,
               const swb_scoring *sc, int32_t w, int32_t h0, swb_ext_result *out) {
    *out = swb_ext_result{0, 0, 0, 0, 0, 0};
    if (!(qlen > 0 && tlen > 0)) return 1;
    int32_t maxPossible = h0 + qlen * sc->a;                      // :24-27
    if (maxPossible > 250) return 0;
    int8_t mat[25];
    scoring_matrix(sc, mat);
    const int m = 5, lanes = 16;
    const int sn = (qlen + lanes - 1) / lanes;
    const uint8_t bias = (uint8_t)sc->b;
    const uint8_t oIns = (uint8_t)sc->o_ins, eIns = (uint8_t)sc->e_ins;
    const uint8_t oDel = (uint8_t)sc->o_del, eDel = (uint8_t)sc->e_del;
    const int32_t zDrop = sc->zdrop;
    std::vector<uint8_t> profile((size_t)m * sn * lanes, 0), H((size_t)sn * lanes, 0), E((size_t)sn * lanes, 0);
    for (int k = 0; k < m; ++k)
        for (int s = 0; s < sn; ++s)
            for (int l = 0; l < lanes; ++l) {
                int j = s + l * sn;
                if (j < qlen) profile[((size_t)k * sn + s) * lanes + l] = clamp_u8(mat[k * m + query[j]] + bias);
            }
    for (int s = 0; s < sn; ++s)
        for (int l = 0; l < lanes; ++l) {
            int j = s + l * sn;
            if (j < qlen && j + 1 <= w) {
                long val = (long)h0 - sc->o_ins - (long)sc->e_ins * (j + 1);
                if (val > 0) H[(size_t)s * lanes + l] = clamp_u8((int)std::min<long>(val, 255));
            }
        }
    uint8_t maxScore = clamp_u8(std::max(0, h0));
    int32_t maxI = -1, maxJ = -1, gScore = -1, gTle = -1, maxOff = 0;
    for (int i = 0; i < tlen; ++i) {
        const uint8_t *prof = &profile[(size_t)target[i] * sn * lanes];
        uint8_t vH[16], f[16];
        for (int l = 0; l < lanes; ++l) vH[l] = l == 0 ? 0 : H[(size_t)(sn - 1) * lanes + l - 1];
        if (i == 0) vH[0] = clamp_u8(std::max(0, h0));
        for (int l = 0; l < lanes; ++l) f[l] = 0;
        for (int s = 0; s < sn; ++s) {
            uint8_t *Hs = &H[(size_t)s * lanes], *Es = &E[(size_t)s * lanes];
            uint8_t hNew[16], hPrev[16];
            for (int l = 0; l < lanes; ++l) {
                uint8_t x = (uint8_t)(vH[l] + prof[s * lanes + l]);
                x = satsub_u8(x, bias);
                if (vH[l] == 0) x = 0;
                hNew[l] = x;
                hPrev[l] = Hs[l];
            }
            for (int l = 0; l < lanes; ++l) {
                vH[l] = hPrev[l];
                uint8_t a = satsub_u8(hPrev[l], oIns);
                uint8_t ev = a > Es[l] ? a : Es[l];
                ev = satsub_u8(ev, eIns);
                Es[l] = ev;
                uint8_t hh = hNew[l] > ev ? hNew[l] : ev;
                hh = hh > f[l] ? hh : f[l];
                Hs[l] = hh;
                uint8_t hf = satsub_u8(hh, oDel);
                uint8_t fm = hf > f[l] ? hf : f[l];
                f[l] = satsub_u8(fm, eDel);
            }
        }
        uint8_t corrF[16];
        for (int l = 0; l < lanes; ++l) corrF[l] = l == 0 ? 0 : f[l - 1];
        for (int s = 0; s < sn; ++s) {
            uint8_t *Hs = &H[(size_t)s * lanes];
            uint8_t newH[16];
            bool same = true;
            for (int l = 0; l < lanes; ++l) {
                newH[l] = corrF[l] > Hs[l] ? corrF[l] : Hs[l];
                if (newH[l] != Hs[l]) same = false;
            }
            if (same) break;
            for (int l = 0; l < lanes; ++l) {
                Hs[l] = newH[l];
                uint8_t hf = satsub_u8(Hs[l], oDel);
                uint8_t fm = hf > corrF[l] ? hf : corrF[l];
                corrF[l] = satsub_u8(fm, eDel);
            }
        }
        uint8_t rowMax = 0;
        int32_t rowMaxJ = -1;
        for (int s = 0; s < sn; ++s) {
            uint8_t *Hs = &H[(size_t)s * lanes];
            uint8_t localMax = Hs[0];
            for (int l = 1; l < lanes; ++l) localMax = std::max(localMax, Hs[l]);
            if (localMax > 250) return 0;                            // :158
            if (localMax > rowMax) {
                rowMax = localMax;
                for (int l = 0; l < lanes; ++l)
                    if (Hs[l] == localMax) {
                        int j = s + l * sn;
                        if (j < qlen) { rowMaxJ = j; break; }
                    }
            }
        }
        if (rowMax == 0) break;
        if (rowMax > maxScore) {
            maxScore = rowMax; maxI = i; maxJ = rowMaxJ;
            int32_t off = std::abs(rowMaxJ - i);
            if (off > maxOff) maxOff = off;
        } else if (zDrop > 0) {
            int32_t dI = i - maxI, dJ = rowMaxJ - maxJ;
            if (dI > dJ) { if ((int32_t)maxScore - (int32_t)rowMax - (dI - dJ) * sc->e_del > zDrop) break; }
            else { if ((int32_t)maxScore - (int32_t)rowMax - (dJ - dI) * sc->e_ins > zDrop) break; }
        }
        int lastJ = qlen - 1;
        int32_t hAtEnd = H[(size_t)(lastJ % sn) * lanes + lastJ / sn];
        if (hAtEnd > gScore) { gScore = hAtEnd; gTle = i; }
    }
    *out = swb_ext_result{(int32_t)maxScore, maxJ + 1, maxI + 1, gTle + 1, gScore, maxOff};
    return 1;
}

// --------------------------------------------------------------------------
// CIGARBuilder -- Sources/Alignment/CIGARBuilder.swift:4-37
// --------------------------------------------------------------------------
enum { OP_M = 0, OP_I = 1, OP_D = 2, OP_S = 4, OP_H = 5 };
struct CigarBuilder {
    std::vector<std::pair<uint32_t, uint32_t>> ops;  // (op, len)
    void append(uint32_t op, uint32_t len = 1) {
        if (!ops.empty() && ops.back().first == op) ops.back().second += len;
        else ops.emplace_back(op, len);
    }
    void reverse() { std::reverse(ops.begin(), ops.end()); }
    std::vector<uint32_t> build() const {
        std::vector<uint32_t> r;
        r.reserve(ops.size());
        for (auto &o : ops) r.push_back((o.second << 4) | o.first);
        return r;
    }
};

// --------------------------------------------------------------------------
// GlobalAligner.align + traceback -- Sources/Alignment/GlobalAligner.swift:19-232
// --------------------------------------------------------------------------
int global_align(const uint8_t *query, int qlen, const uint8_t *target, int tlen,
                 const swb_scoring *sc, int32_t w_in, int32_t *score_out,
                 std::vector<uint32_t> *cigar_out, uint64_t *cells_out) {
    *score_out = 0;
    cigar_out->clear();
    if (cells_out) *cells_out = 0;
    if (!(qlen > 0 && tlen > 0)) return 0;                       // :29-31
    const int m = 5;
    int8_t mat[25];
    scoring_matrix(sc, mat);
    const int32_t oDel = sc->o_del, eDel = sc->e_del;            // :37-44
    const int32_t oIns = sc->o_ins, eIns = sc->e_ins;
    const int32_t oeDel = oDel + eDel, oeIns = oIns + eIns;
    const int32_t w = std::max(w_in, std::abs(qlen - tlen));      // :47
    const int nCol = std::min<long>(qlen, 2L * w + 1);           // :48
    const int initEnd = std::min(w, qlen);                       // :81
    if (initEnd < 1) return -1;                                  // Swift `1...0` range is undefined
    const int32_t negInf = INT32_MIN / 2;                        // :52
    std::vector<int32_t> qp((size_t)m * qlen), h(qlen + 1, negInf), e(qlen + 1, negInf);
    std::vector<uint8_t> z((size_t)tlen * nCol, 0);
    for (int k = 0; k < m; ++k)                                   // :65-72
        for (int j = 0; j < qlen; ++j) qp[(size_t)k * qlen + j] = mat[k * m + query[j]];
    h[0] = 0;                                                     // :80-84
    for (int j = 1; j <= initEnd; ++j) h[j] = 0 - (oIns + eIns * j);
    uint64_t cells = 0;
    for (int i = 0; i < tlen; ++i) {                              // :89-142
        const int beg = std::max(0, i - w);
        const int end = (int)std::min<long>(qlen, (long)i + w + 1);
        const int qpRow = target[i] * qlen;
        int32_t f = negInf;
        int32_t hDiag = h[beg];
        if (beg == 0) h[beg] = 0 - (oeDel + eDel * i);
        else h[beg] = negInf;
        uint8_t *zi = z.data() + ((size_t)i * nCol) - beg;
        cells += (uint64_t)(end > beg ? end - beg : 0);
        for (int j = beg; j < end; ++j) {
            const int j1 = j + 1;
            int32_t hCur = hDiag + qp[qpRow + j];
            hDiag = h[j1];
            const int32_t eOpen = hDiag - oeDel;
            const int32_t eExtend = e[j1] - eDel;
            const uint8_t eFlag = eOpen > eExtend ? 0 : 0x01;
            const int32_t eVal = eOpen > eExtend ? eOpen : eExtend;
            e[j1] = eVal;
            const int32_t fOpen = h[j] - oeIns;
            const int32_t fExtend = f - eIns;
            const uint8_t fFlag = fOpen > fExtend ? 0 : 0x02;
            const int32_t fVal = fOpen > fExtend ? fOpen : fExtend;
            f = fVal;
            const uint8_t fromE = eVal > hCur ? 0x04 : 0;
            hCur = eVal > hCur ? eVal : hCur;
            const uint8_t fromF = fVal > hCur ? 0x08 : 0;
            hCur = fVal > hCur ? fVal : hCur;
            h[j1] = hCur;
            zi[j] = eFlag | fFlag | fromE | fromF;
        }
    }
    *score_out = h[qlen];                                         // :144
    if (cells_out) *cells_out = cells;

    CigarBuilder builder;                                         // traceback :160-232
    int i = tlen - 1, j = qlen - 1, state = 0;
    while (i >= 0 || j >= 0) {
        if (i < 0) { builder.append(OP_I); j -= 1; continue; }
        if (j < 0) { builder.append(OP_D); i -= 1; continue; }
        const int beg = std::max(0, i - w);
        const int col = j - beg;
        if (!(col >= 0 && col < nCol)) break;
        const uint8_t d = z[(size_t)i * nCol + col];
        switch (state) {
        case 0: {
            const int hDir = (d >> 2) & 0x03;
            if (hDir == 0) { builder.append(OP_M); i -= 1; j -= 1; }
            else if (hDir == 1) state = 1;
            else state = 2;
            break;
        }
        case 1:
            builder.append(OP_D);
            if ((d & 0x01) == 0) state = 0;
            i -= 1;
            break;
        case 2:
            builder.append(OP_I);
            if ((d & 0x02) == 0) state = 0;
            j -= 1;
            break;
        default: break;
        }
    }
    builder.reverse();
    *cigar_out = builder.build();
    return 0;
}

// GlobalAligner.computeNM -- GlobalAligner.swift:235-273
int32_t compute_nm_global(const uint32_t *cigar, int n, const uint8_t *q, int qlen, const uint8_t *t, int tlen) {
    int32_t nm = 0;
    long qi = 0, ti = 0;
    for (int k = 0; k < n; ++k) {
        const uint32_t op = cigar[k] & 0xF;
        const long len = cigar[k] >> 4;
        switch (op) {
        case OP_M:
            for (long x = 0; x < len; ++x)
                if (qi < qlen && ti < tlen) {
                    if (q[qi] != t[ti]) nm += 1;
                    qi += 1; ti += 1;
                }
            break;
        case OP_I: nm += (int32_t)len; qi += len; break;
        case OP_D: nm += (int32_t)len; ti += len; break;
        case OP_S: qi += len; break;
        default: break;
        }
    }
    return nm;
}

// --------------------------------------------------------------------------
// CIGARGenerator -- Sources/Alignment/CIGARGenerator.swift
// --------------------------------------------------------------------------
// inferBandWidth (:147-170)
int32_t infer_band_width(int32_t queryLen, int32_t refLen, int32_t score, const swb_scoring *sc) {
    const int32_t maxLen = std::max(queryLen, refLen), minLen = std::min(queryLen, refLen);
    const int32_t diff = maxLen - minLen;
    const int32_t expectedScore = minLen * sc->a;
    if (score >= expectedScore) return diff + 3;
    const int32_t deficit = expectedScore - score;
    const int32_t gapCost = sc->o_ins + sc->e_ins;
    const int32_t mmDelta = sc->a + sc->b;
    const int32_t estimatedErrors = deficit / std::min(gapCost, mmDelta);
    return std::max(diff + 3, estimatedErrors);
}

// computeNMFromCigar (:173-210)
int32_t nm_from_cigar(const std::vector<uint32_t> &cigar, const uint8_t *q, int qlen,
                      const uint8_t *t, int tlen, long targetOffset) {
    int32_t nm = 0;
    long qi = 0, ti = targetOffset;
    for (uint32_t c : cigar) {
        const uint32_t op = c & 0xF;
        const long len = c >> 4;
        switch (op) {
        case OP_M:
            for (long x = 0; x < len; ++x)
                if (qi < qlen && ti < tlen) {
                    if (q[qi] != t[ti]) nm += 1;
                    qi += 1; ti += 1;
                }
            break;
        case OP_I: nm += (int32_t)len; qi += len; break;
        case OP_D: nm += (int32_t)len; ti += len; break;
        default: break;
        }
    }
    return nm;
}

// baseChar (:323-331)
const char *base_char(uint8_t b) {
    switch (b) { case 0: return "A"; case 1: return "C"; case 2: return "G"; case 3: return "T"; default: return "N"; }
}

// generateMD (:219-268)
std::string generate_md(const std::vector<uint32_t> &cigar, const uint8_t *q, int qlen,
                        const uint8_t *t, int tlen, long targetOffset) {
    std::string md;
    long matchCount = 0, qi = 0, ti = targetOffset;
    for (uint32_t c : cigar) {
        const uint32_t op = c & 0xF;
        const long len = c >> 4;
        switch (op) {
        case OP_M:
            for (long x = 0; x < len; ++x)
                if (qi < qlen && ti < tlen) {
                    if (q[qi] == t[ti]) matchCount += 1;
                    else {
                        md += std::to_string(matchCount);
                        md += base_char(t[ti]);
                        matchCount = 0;
                    }
                    qi += 1; ti += 1;
                }
            break;
        case OP_I: qi += len; break;
        case OP_D:
            md += std::to_string(matchCount);
            md += "^";
            for (long x = 0; x < len; ++x)
                if (ti < tlen) { md += base_char(t[ti]); ti += 1; }
            matchCount = 0;
            break;
        default: break;
        }
    }
    md += std::to_string(matchCount);
    return md;
}

// squeezeDeletions (:272-295)
void squeeze_deletions(std::vector<uint32_t> &cigar, int64_t *posAdj, long *refOffset) {
    *posAdj = 0;
    *refOffset = 0;
    while (!cigar.empty()) {
        if ((cigar[0] & 0xF) == OP_D) {
            const long len = cigar[0] >> 4;
            *posAdj += len;
            *refOffset += len;
            cigar.erase(cigar.begin());
        } else break;
    }
    while (!cigar.empty()) {
        if ((cigar.back() & 0xF) == OP_D) cigar.pop_back();
        else break;
    }
}

// addSoftClips (:298-320)
void add_soft_clips(std::vector<uint32_t> &cigar, int32_t qb, int32_t qe, int readLength, bool isReverse) {
    const long intQb = qb, intQe = qe;
    if (isReverse) {
        const long clip5 = readLength - intQe, clip3 = intQb;
        if (clip5 > 0) cigar.insert(cigar.begin(), ((uint32_t)clip5 << 4) | OP_S);
        if (clip3 > 0) cigar.push_back(((uint32_t)clip3 << 4) | OP_S);
    } else {
        if (intQb > 0) cigar.insert(cigar.begin(), ((uint32_t)intQb << 4) | OP_S);
        if (intQe < readLength) cigar.push_back(((uint32_t)(readLength - intQe) << 4) | OP_S);
    }
}

int copy_out(const std::vector<uint32_t> &cigar, const std::string &md, uint32_t *cigar_buf,
             int32_t *n_cigar, char *md_buf, int32_t md_cap) {
    if ((long)cigar.size() > *n_cigar || (long)md.size() + 1 > md_cap) return -1;
    std::copy(cigar.begin(), cigar.end(), cigar_buf);
    *n_cigar = (int32_t)cigar.size();
    std::memcpy(md_buf, md.c_str(), md.size() + 1);
    return 0;
}

// --------------------------------------------------------------------------
// LocalSWAligner -- Sources/Alignment/LocalSWAligner.swift
// --------------------------------------------------------------------------
struct PassResult { int32_t score, qEnd, tEnd, score2; };
typedef uint8_t V16[16];

inline void shift_right16(const uint8_t *v, uint8_t *r) {   // shiftRight (:316-323)
    r[0] = 0;
    for (int l = 1; l < 16; ++l) r[l] = v[l - 1];
}

// simdSWPass (:133-306).  Returns false for nil (8-bit overflow).
bool simd_sw_pass(const uint8_t *query, int qLen, const uint8_t *target, int tLen,
                  const int8_t *mat, int32_t gapOE, int32_t gapE, uint8_t bias,
                  uint8_t minSubScore, PassResult *res) {
    const int lanes = 16;
    // A reverse pass with revQLen == 0 would read hArr[-1] in the Swift code
    // (possible only if the forward maximum sat in a padding lane); both this
    // oracle and the CUDA kernel define it as nil, i.e. the scalar fallback.
    if (qLen <= 0) return false;
    const int sn = (qLen + lanes - 1) / lanes;
    std::vector<uint8_t> profile((size_t)5 * sn * lanes, 0), hArr((size_t)sn * lanes, 0), eArr((size_t)sn * lanes, 0);
    for (int k = 0; k < 5; ++k)                                   // :153-167
        for (int s = 0; s < sn; ++s)
            for (int l = 0; l < lanes; ++l) {
                const int j = s + l * sn;
                if (j < qLen) profile[((size_t)k * sn + s) * lanes + l] = clamp_u8((int)mat[k * 5 + query[j]] + (int)bias);
            }
    const uint8_t gOE = (uint8_t)gapOE, gE = (uint8_t)gapE;      // :175-177
    uint8_t maxScore = 0;
    int32_t maxI = -1, maxJ = -1;
    std::vector<uint64_t> peaks;                                  // :185-189
    const bool trackPeaks = minSubScore > 0;
    uint8_t maxBaseScore = 0;                                     // :192-199
    if (trackPeaks) {
        for (int k = 0; k < 25; ++k) {
            uint8_t v = clamp_u8((int)mat[k] + (int)bias);
            if (v > maxBaseScore) maxBaseScore = v;
        }
        maxBaseScore = maxBaseScore > bias ? (uint8_t)(maxBaseScore - bias) : 0;
    }
    for (int i = 0; i < tLen; ++i) {                              // :201
        const int tBase = std::min<int>(target[i], 4);
        const uint8_t *prof = &profile[(size_t)tBase * sn * lanes];
        uint8_t vH[16], f[16];
        shift_right16(&hArr[(size_t)(sn - 1) * lanes], vH);       // :206
        std::memset(f, 0, 16);
        for (int s = 0; s < sn; ++s) {                            // :209-231
            uint8_t *H = &hArr[(size_t)s * lanes], *E = &eArr[(size_t)s * lanes];
            for (int l = 0; l < lanes; ++l) {
                uint8_t hNew = (uint8_t)(vH[l] + prof[s * lanes + l]);
                hNew = satsub_u8(hNew, bias);
                const uint8_t hPrev = H[l];
                vH[l] = hPrev;
                const uint8_t eOpen = satsub_u8(hPrev, gOE);
                uint8_t eVal = eOpen > E[l] ? eOpen : E[l];
                eVal = satsub_u8(eVal, gE);
                E[l] = eVal;
                hNew = hNew > eVal ? hNew : eVal;
                hNew = hNew > f[l] ? hNew : f[l];
                H[l] = hNew;
                const uint8_t fOpen = satsub_u8(H[l], gOE);
                uint8_t fv = fOpen > f[l] ? fOpen : f[l];
                f[l] = satsub_u8(fv, gE);
            }
        }
        uint8_t corrF[16];                                        // :234-242
        shift_right16(f, corrF);
        for (int s = 0; s < sn; ++s) {
            uint8_t *H = &hArr[(size_t)s * lanes];
            uint8_t newH[16];
            bool same = true;
            for (int l = 0; l < lanes; ++l) {
                newH[l] = corrF[l] > H[l] ? corrF[l] : H[l];
                if (newH[l] != H[l]) same = false;
            }
            if (same) break;
            for (int l = 0; l < lanes; ++l) {
                H[l] = newH[l];
                const uint8_t fOpen = satsub_u8(H[l], gOE);
                uint8_t cf = fOpen > corrF[l] ? fOpen : corrF[l];
                corrF[l] = satsub_u8(cf, gE);
            }
        }
        uint8_t colMax = 0;                                       // :245-263
        for (int s = 0; s < sn; ++s) {
            const uint8_t *H = &hArr[(size_t)s * lanes];
            uint8_t localMax = H[0];
            for (int l = 1; l < lanes; ++l) localMax = std::max(localMax, H[l]);
            if (localMax > 250) return false;
            if (localMax > colMax) colMax = localMax;
            if (localMax > maxScore) {
                maxScore = localMax;
                maxI = i;
                for (int l = 0; l < lanes; ++l)
                    if (H[l] == localMax) {
                        const int j = s + l * sn;
                        if (j < qLen) { maxJ = j; break; }
                    }
            }
        }
        if (trackPeaks && colMax >= minSubScore) {                // :266-286
            const uint64_t cm = colMax;
            if (peaks.empty() || (int32_t)(peaks.back() & 0xFFFFFFFFull) + 1 != i) {
                peaks.push_back((cm << 32) | (uint64_t)(uint32_t)i);
            } else if ((peaks.back() >> 32) < cm) {
                peaks.back() = (cm << 32) | (uint64_t)(uint32_t)i;
            }
        }
    }
    int32_t score2 = 0;                                           // :290-303
    if (trackPeaks && !peaks.empty() && maxScore > 0 && maxBaseScore > 0) {
        const int32_t r = ((int32_t)maxScore + (int32_t)maxBaseScore - 1) / (int32_t)maxBaseScore;
        const int32_t low = maxI - r, high = maxI + r;
        for (uint64_t entry : peaks) {
            const int32_t col = (int32_t)(uint32_t)(entry & 0xFFFFFFFFull);
            const int32_t scv = (int32_t)(entry >> 32);
            if ((col < low || col > high) && scv > score2) score2 = scv;
        }
    }
    *res = PassResult{(int32_t)maxScore, maxJ, maxI, score2};
    return true;
}

// scalarSWPass (:383-492)
PassResult scalar_sw_pass(const uint8_t *query, int qLen, const uint8_t *target, int tLen,
                          const int8_t *mat, int32_t gapOE, int32_t gapE, int32_t minSubScore) {
    std::vector<int32_t> h(tLen + 1, 0), e(tLen + 1, 0);
    int32_t bestScore = 0, bestQEnd = -1, bestTEnd = -1;
    const bool trackPeaks = minSubScore > 0;
    std::vector<uint64_t> peaks;
    int32_t maxBaseScore = 0;
    if (trackPeaks)
        for (int k = 0; k < 25; ++k)
            if (mat[k] > maxBaseScore) maxBaseScore = mat[k];
    for (int i = 0; i < qLen; ++i) {
        const int qBase = std::min<int>(query[i], 4);
        const int8_t *matRow = mat + qBase * 5;
        int32_t f = 0, hPrev = 0, rowMax = 0;
        for (int j = 0; j < tLen; ++j) {
            const int j1 = j + 1;
            const int tBase = std::min<int>(target[j], 4);
            int32_t hCur = hPrev + (int32_t)matRow[tBase];
            const int32_t fOpen = h[j1] - gapOE, fExt = f - gapE;
            f = fOpen > fExt ? fOpen : fExt;
            const int32_t eOpen = h[j] - gapOE, eExt = e[j1] - gapE;
            const int32_t eVal = eOpen > eExt ? eOpen : eExt;
            e[j1] = eVal;
            hCur = hCur > f ? hCur : f;
            hCur = hCur > eVal ? hCur : eVal;
            hCur = hCur > 0 ? hCur : 0;
            hPrev = h[j1];
            h[j1] = hCur;
            if (hCur > rowMax) rowMax = hCur;
            if (hCur > bestScore) { bestScore = hCur; bestQEnd = i; bestTEnd = j; }
        }
        if (trackPeaks && rowMax >= minSubScore) {
            const uint64_t rm = (uint64_t)(uint32_t)rowMax, iu = (uint64_t)(uint32_t)i;
            if (peaks.empty() || (int32_t)(peaks.back() & 0xFFFFFFFFull) + 1 != i) peaks.push_back((rm << 32) | iu);
            else if ((peaks.back() >> 32) < rm) peaks.back() = (rm << 32) | iu;
        }
    }
    int32_t score2 = 0;
    if (trackPeaks && !peaks.empty() && bestScore > 0 && maxBaseScore > 0) {
        const int32_t r = (bestScore + maxBaseScore - 1) / maxBaseScore;
        const int32_t low = bestQEnd - r, high = bestQEnd + r;
        for (uint64_t entry : peaks) {
            const int32_t col = (int32_t)(uint32_t)(entry & 0xFFFFFFFFull);
            const int32_t scv = (int32_t)(entry >> 32);
            if ((col < low || col > high) && scv > score2) score2 = scv;
        }
    }
    return PassResult{bestScore, bestQEnd, bestTEnd, score2};
}

// LocalSWAligner.align (:42-79) with simdLocalSW (:85-125) and scalarAlign (:327-381)
bool local_align(const uint8_t *query, int qLen, const uint8_t *target, int tLen,
                 const swb_scoring *sc, uint8_t minSubScore, swb_local_result *out,
                 uint64_t *cells, int *path) {
    *out = swb_local_result{0, 0, 0, 0, 0, 0};
    uint64_t c = 0;
    if (path) *path = 0;
    if (!(qLen > 0 && tLen > 0)) { if (cells) *cells = 0; return false; }
    int8_t mat[25];
    scoring_matrix(sc, mat);
    const int32_t gapOE = sc->o_ins + sc->e_ins, gapE = sc->e_ins;
    const uint8_t bias = (uint8_t)sc->b;
    const int32_t maxPossibleScore = qLen * sc->a;
    if (maxPossibleScore <= 250) {
        PassResult fwd;
        c += (uint64_t)qLen * tLen;
        if (simd_sw_pass(query, qLen, target, tLen, mat, gapOE, gapE, bias, minSubScore, &fwd) && fwd.score > 0) {
            const int revQLen = fwd.qEnd + 1, revTLen = fwd.tEnd + 1;
            std::vector<uint8_t> revQ(std::max(revQLen, 0)), revT(std::max(revTLen, 0));
            for (int k = 0; k < revQLen; ++k) revQ[k] = query[revQLen - 1 - k];
            for (int k = 0; k < revTLen; ++k) revT[k] = target[revTLen - 1 - k];
            PassResult rev;
            c += (uint64_t)std::max(revQLen, 0) * std::max(revTLen, 0);
            if (simd_sw_pass(revQ.data(), revQLen, revT.data(), revTLen, mat, gapOE, gapE, bias, 0, &rev)) {
                *out = swb_local_result{fwd.score, fwd.qEnd - rev.qEnd, fwd.qEnd,
                                        fwd.tEnd - rev.tEnd, fwd.tEnd, fwd.score2};
                if (cells) *cells = c;
                return true;
            }
        }
    }
    if (path) *path = 1;                                          // scalar fallback (:74-78)
    c += (uint64_t)qLen * tLen;
    PassResult fr = scalar_sw_pass(query, qLen, target, tLen, mat, gapOE, gapE, (int32_t)minSubScore);
    if (!(fr.score > 0)) { if (cells) *cells = c; return false; }
    const int revQLen = fr.qEnd + 1, revTLen = fr.tEnd + 1;
    std::vector<uint8_t> revQ(revQLen), revT(revTLen);
    for (int k = 0; k < revQLen; ++k) revQ[k] = query[revQLen - 1 - k];
    for (int k = 0; k < revTLen; ++k) revT[k] = target[revTLen - 1 - k];
    c += (uint64_t)revQLen * revTLen;
    PassResult rr = scalar_sw_pass(revQ.data(), revQLen, revT.data(), revTLen, mat, gapOE, gapE, 0);
    *out = swb_local_result{fr.score, fr.qEnd - rr.qEnd, fr.qEnd, fr.tEnd - rr.tEnd, fr.tEnd, fr.score2};
    if (cells) *cells = c;
    return true;
}

// --------------------------------------------------------------------------
// PackedReference.base -- Sources/FMIndex/PackedReference.swift:34-38
// FMIndex.getReference(at:length:into:) -- Sources/FMIndex/FMIndex.swift:147-170
// --------------------------------------------------------------------------
inline uint8_t pac_base(const uint8_t *pac, int64_t pos) {
    const int shift = (3 - (int)(pos & 3)) << 1;
    return (uint8_t)((pac[pos >> 2] >> shift) & 3);
}

int32_t get_reference(const uint8_t *pac, int64_t gl, int64_t pos, int32_t length, uint8_t *buffer) {
    if (pos >= gl) {
        const int64_t fwdEnd = 2 * gl - pos;
        const int64_t fwdStart = fwdEnd - length;
        const int64_t safeStart = std::max<int64_t>(0, fwdStart);
        const int64_t safeEnd = std::min(fwdEnd, gl);
        const int64_t safeLen = safeEnd - safeStart;
        if (!(safeLen > 0)) return 0;
        for (int64_t i = 0; i < safeLen; ++i) buffer[i] = pac_base(pac, safeStart + i);
        std::reverse(buffer, buffer + safeLen);
        for (int64_t i = 0; i < safeLen; ++i) buffer[i] = (uint8_t)(3 - buffer[i]);
        return (int32_t)safeLen;
    } else {
        const int64_t safeLen = std::min<int64_t>(length, gl - pos);
        if (!(safeLen > 0 && pos >= 0)) return 0;
        for (int64_t i = 0; i < safeLen; ++i) buffer[i] = pac_base(pac, pos + i);
        return (int32_t)safeLen;
    }
}

// --------------------------------------------------------------------------
// ExtensionAligner.extend -- Sources/Alignment/ExtensionAligner.swift:114-346
// --------------------------------------------------------------------------
long cal_max_gap(long queryLen, const swb_scoring *sc) {      // :352-363
    const long a = sc->a, oDel = sc->o_del, eDel = sc->e_del, oIns = sc->o_ins, eIns = sc->e_ins;
    const long lDel = eDel > 0 ? (queryLen * a - oDel) / eDel + 1 : 1;
    const long lIns = eIns > 0 ? (queryLen * a - oIns) / eIns + 1 : 1;
    long l = std::max(lDel, lIns);
    l = std::max(l, 1L);
    return std::min(l, (long)sc->band_width << 1);
}

// Task target/query materialisation shared by the batch drivers.
void load_span(const uint8_t *bases, const uint8_t *pac, uint64_t off, int len, uint32_t flags,
               bool is_target, uint8_t *dst) {
    const bool rev = is_target ? (flags & SWB_T_REVERSE) : (flags & SWB_Q_REVERSE);
    const bool comp = is_target && (flags & SWB_T_COMPLEMENT);
    const bool from_ref = is_target && (flags & SWB_T_FROM_REF);
    for (int k = 0; k < len; ++k) {
        const uint64_t idx = off + (uint64_t)(rev ? (len - 1 - k) : k);
        uint8_t b = from_ref ? pac_base(pac, (int64_t)idx) : bases[idx];
        if (comp && b < 4) b = (uint8_t)(3 - b);   // N stays N
        dst[k] = b;
    }
}

template <class F>
void parallel_for(size_t n, int n_threads, F fn) {
    if (n_threads <= 1 || n < 64) { fn(0, n, 0); return; }
    std::vector<std::thread> th;
    const size_t chunk = (n + n_threads - 1) / n_threads;
    for (int t = 0; t < n_threads; ++t) {
        const size_t lo = t * chunk, hi = std::min(n, lo + chunk);
        if (lo >= hi) break;
        th.emplace_back(fn, lo, hi, t);
    }
    for (auto &x : th) x.join();
}

}  // namespace

// ============================================================== extern "C"
extern "C" {

void orc_scoring_matrix(const swb_scoring *sc, int8_t mat[25]) { scoring_matrix(sc, mat); }

void orc_banded_sw_scalar(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                          const swb_scoring *sc, int32_t w, int32_t h0, int32_t end_bonus,
                          swb_ext_result *out, uint64_t *cells) {
    banded_sw_scalar(q, qlen, t, tlen, sc, w, h0, end_bonus, out, cells);
}

void orc_banded_sw16(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                     const swb_scoring *sc, int32_t w, int32_t h0, swb_ext_result *out) {
    banded_sw16(q, qlen, t, tlen, sc, w, h0, out);
}

int orc_banded_sw8(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                   const swb_scoring *sc, int32_t w, int32_t h0, swb_ext_result *out) {
    return banded_sw8(q, qlen, t, tlen, sc, w, h0, out);
}

int orc_global_align(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                     const swb_scoring *sc, int32_t w, int32_t *score,
                     uint32_t *cigar, int32_t *n_cigar, uint64_t *cells) {
    std::vector<uint32_t> c;
    if (global_align(q, qlen, t, tlen, sc, w, score, &c, cells) != 0) return -1;
    if ((long)c.size() > *n_cigar) return -1;
    std::copy(c.begin(), c.end(), cigar);
    *n_cigar = (int32_t)c.size();
    return 0;
}

int32_t orc_compute_nm(const uint32_t *cigar, int32_t n, const uint8_t *q, int32_t qlen,
                       const uint8_t *t, int32_t tlen) {
    return compute_nm_global(cigar, n, q, qlen, t, tlen);
}

int32_t orc_infer_band_width(int32_t qlen, int32_t rlen, int32_t score, const swb_scoring *sc) {
    return infer_band_width(qlen, rlen, score, sc);
}

// CIGARGenerator.generate -- CIGARGenerator.swift:30-111
int orc_cigar_generate(const uint8_t *qseg, int32_t qlen, const uint8_t *rseg, int32_t rlen,
                       int32_t qb, int32_t qe, int32_t read_len, int32_t is_rev,
                       int32_t true_score, int32_t initial_w, const swb_scoring *sc,
                       int64_t ref_pos, uint32_t *cigar_buf, int32_t *n_cigar,
                       int32_t *nm_out, char *md_buf, int32_t md_cap, int32_t *score_out,
                       int64_t *pos_out, uint64_t *cells, int32_t *used_dp) {
    int32_t w = infer_band_width(qe - qb, rlen, true_score, sc);   // :44-50
    w = std::max(w, initial_w);
    int retries = 0;
    const int maxRetries = 3;
    const int32_t minIndelCost = sc->o_ins + sc->e_ins + sc->o_del + sc->e_del;  // :63-67
    const int32_t deficit = qlen * sc->a - true_score;
    if (cells) *cells = 0;
    if (used_dp) *used_dp = 0;
    if (qlen == rlen && qlen > 0 && deficit < minIndelCost) {      // :69-80
        std::vector<uint32_t> cigar{((uint32_t)qlen << 4) | OP_M};
        const int32_t nm = nm_from_cigar(cigar, qseg, qlen, rseg, rlen, 0);
        const std::string md = generate_md(cigar, qseg, qlen, rseg, rlen, 0);
        add_soft_clips(cigar, qb, qe, read_len, is_rev != 0);
        *nm_out = nm;
        *score_out = true_score;
        *pos_out = ref_pos;
        return copy_out(cigar, md, cigar_buf, n_cigar, md_buf, md_cap);
    }
    if (used_dp) *used_dp = 1;
    int32_t score;
    std::vector<uint32_t> raw;
    uint64_t c1 = 0, total = 0;
    if (global_align(qseg, qlen, rseg, rlen, sc, w, &score, &raw, &c1) != 0) return -1;  // :82-86
    total += c1;
    while (score < true_score && retries < maxRetries) {          // :88-96
        w *= 2;
        retries += 1;
        if (global_align(qseg, qlen, rseg, rlen, sc, w, &score, &raw, &c1) != 0) return -1;
        total += c1;
    }
    if (cells) *cells = total;
    int64_t posAdj;
    long refOffset;
    squeeze_deletions(raw, &posAdj, &refOffset);                  // :98-101
    const int32_t nm = nm_from_cigar(raw, qseg, qlen, rseg, rlen, refOffset);
    const std::string md = generate_md(raw, qseg, qlen, rseg, rlen, refOffset);
    add_soft_clips(raw, qb, qe, read_len, is_rev != 0);
    *nm_out = nm;
    *score_out = score;
    *pos_out = ref_pos + posAdj;
    return copy_out(raw, md, cigar_buf, n_cigar, md_buf, md_cap);
}

// CIGARGenerator.postProcess -- CIGARGenerator.swift:118-142
int orc_cigar_postprocess(const uint32_t *raw_in, int32_t n_raw, int32_t score,
                          const uint8_t *qseg, int32_t qlen, const uint8_t *rseg, int32_t rlen,
                          int32_t qb, int32_t qe, int32_t read_len, int32_t is_rev, int64_t ref_pos,
                          uint32_t *cigar_buf, int32_t *n_cigar, int32_t *nm_out,
                          char *md_buf, int32_t md_cap, int32_t *score_out, int64_t *pos_out) {
    std::vector<uint32_t> cigar(raw_in, raw_in + n_raw);
    int64_t posAdj;
    long refOffset;
    squeeze_deletions(cigar, &posAdj, &refOffset);
    const int32_t nm = nm_from_cigar(cigar, qseg, qlen, rseg, rlen, refOffset);
    const std::string md = generate_md(cigar, qseg, qlen, rseg, rlen, refOffset);
    add_soft_clips(cigar, qb, qe, read_len, is_rev != 0);
    *nm_out = nm;
    *score_out = score;
    *pos_out = ref_pos + posAdj;
    return copy_out(cigar, md, cigar_buf, n_cigar, md_buf, md_cap);
}

int orc_local_align(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                    const swb_scoring *sc, int32_t min_sub_score,
                    swb_local_result *out, uint64_t *cells, int32_t *path) {
    int p = 0;
    const bool ok = local_align(q, qlen, t, tlen, sc, clamp_u8(min_sub_score), out, cells, &p);
    if (path) *path = p;
    return ok ? 1 : 0;
}

uint8_t orc_pac_base(const uint8_t *pac, int64_t pos) { return pac_base(pac, pos); }

int32_t orc_get_reference(const uint8_t *pac, int64_t genome_len, int64_t pos, int32_t len, uint8_t *buf) {
    return get_reference(pac, genome_len, pos, len, buf);
}

int orc_extend(const orc_seed *seeds, int32_t n_seeds, int32_t rid,
               const uint8_t *read, int32_t read_len,
               const uint8_t *ref, int64_t ref_len, int32_t ref_mode,
               const swb_scoring *sc, orc_region *out, int32_t cap,
               uint64_t *sw_calls, uint64_t *cells_out) {
    uint64_t calls = 0, cells = 0;
    std::vector<orc_region> regions;
    auto getReference = [&](int64_t pos, int length, uint8_t *buf) -> int {
        if (ref_mode == 0) {   // the tests' closure: start = max(0,pos), end = min(count, start+len)
            const int64_t start = std::max<int64_t>(0, pos);
            const int64_t end = std::min<int64_t>(ref_len, start + length);
            if (start >= end) return 0;
            std::memcpy(buf, ref + start, (size_t)(end - start));
            return (int)(end - start);
        }
        return get_reference(ref, ref_len, pos, length, buf);
    };
    if (n_seeds <= 0) { if (sw_calls) *sw_calls = 0; if (cells_out) *cells_out = 0; return 0; }
    const int32_t readLen = read_len;
    const int32_t bandWidth = sc->band_width;
    const long lQuery = readLen;
    std::vector<uint8_t> queryBuf(std::max(read_len, 1)), targetBuf(10200);

    int64_t rmax0 = INT64_MAX, rmax1 = 0;                            // :134-144
    for (int i = 0; i < n_seeds; ++i) {
        const orc_seed &t = seeds[i];
        const int64_t b = t.rbeg - (int64_t)((long)t.qbeg + cal_max_gap(t.qbeg, sc));
        const long remaining = lQuery - t.qbeg - t.len;
        const int64_t e = t.rbeg + t.len + (int64_t)(remaining + cal_max_gap(remaining, sc));
        if (b < rmax0) rmax0 = b;
        if (e > rmax1) rmax1 = e;
    }
    if (rmax0 < 0) rmax0 = 0;
    const int32_t tmp = std::max(sc->a + sc->b, std::max(sc->o_ins + sc->e_ins, sc->o_del + sc->e_del));  // :146-150

    std::vector<int> seedOrder(n_seeds);                               // :155-158 (stable)
    for (int i = 0; i < n_seeds; ++i) seedOrder[i] = i;
    if (n_seeds > 1)
        std::stable_sort(seedOrder.begin(), seedOrder.end(),
                         [&](int x, int y) { return seeds[x].score > seeds[y].score; });

    for (int sortedIdx : seedOrder) {
        const int32_t seedQbeg = seeds[sortedIdx].qbeg, seedLen = seeds[sortedIdx].len;
        const int64_t seedRbeg = seeds[sortedIdx].rbeg;
        const int32_t seedScore = seeds[sortedIdx].score;
        const int32_t seedQEnd = seedQbeg + seedLen;
        const int64_t seedREnd = seedRbeg + seedLen;

        int coveringRegIdx = -1;                                        // :172-189
        for (size_t idx = 0; idx < regions.size(); ++idx)
            if (seedQbeg >= regions[idx].qb && seedQEnd <= regions[idx].qe) { coveringRegIdx = (int)idx; break; }
        if (coveringRegIdx >= 0) {
            const int32_t seedAlnScore = seedLen * sc->a;
            orc_region &r = regions[coveringRegIdx];
            if (seedAlnScore > r.sub) r.sub = seedAlnScore;
            if (seedAlnScore >= r.score - tmp) r.sub_n += 1;
            continue;
        }
        orc_region reg{};
        reg.w = bandWidth;
        reg.rid = rid;
        reg.seed_cov = seedLen;
        reg.seed_len0 = seedLen;
        int32_t accumulatedH0 = seedScore;

        int32_t leftScore = 0, leftQLen = 0, leftTLen = 0;               // :202-262
        if (seedQbeg > 0) {
            const int queryLeftLen = seedQbeg;
            for (int i = 0; i < queryLeftLen; ++i) queryBuf[i] = read[queryLeftLen - 1 - i];
            const int targetLeftLen = (int)std::min<int64_t>(seedRbeg - rmax0, 10000);
            if (targetLeftLen > 0) {
                const int64_t targetStart = seedRbeg - targetLeftLen;
                const int actual = getReference(targetStart, targetLeftLen, targetBuf.data());
                std::reverse(targetBuf.begin(), targetBuf.begin() + std::max(actual, 0));
                int32_t w = bandWidth, prevScore = seedScore;
                swb_ext_result lr{};
                for (int32_t tryIdx = 0; tryIdx < 2; ++tryIdx) {
                    uint64_t c = 0;
                    banded_sw_scalar(queryBuf.data(), queryLeftLen, targetBuf.data(), actual, sc, w,
                                     seedScore, sc->pen_clip5, &lr, &c);
                    calls += 1; cells += c;
                    if (lr.score == prevScore || lr.max_off < (w >> 1) + (w >> 2) || tryIdx == 1) break;
                    prevScore = lr.score;
                    w = w << 1;
                }
                accumulatedH0 = lr.score;
                reg.w = std::max(reg.w, w);
                if (lr.gscore <= 0 || lr.gscore <= lr.score - sc->pen_clip5) {
                    leftQLen = lr.qle; leftTLen = lr.tle; leftScore = lr.score;
                } else {
                    leftQLen = seedQbeg; leftTLen = lr.gtle; leftScore = lr.gscore;
                }
            }
        }
        int32_t rightScore = 0, rightQLen = 0, rightTLen = 0;            // :265-316
        if (seedQEnd < readLen) {
            const int queryRightLen = read_len - seedQEnd;
            for (int i = 0; i < queryRightLen; ++i) queryBuf[i] = read[seedQEnd + i];
            const int targetRightLen = (int)std::min<int64_t>(rmax1 - seedREnd, 10000);
            if (targetRightLen > 0) {
                const int actual = getReference(seedREnd, targetRightLen, targetBuf.data());
                int32_t w = bandWidth, prevScore = accumulatedH0;
                swb_ext_result rr{};
                for (int32_t tryIdx = 0; tryIdx < 2; ++tryIdx) {
                    uint64_t c = 0;
                    banded_sw_scalar(queryBuf.data(), queryRightLen, targetBuf.data(), actual, sc, w,
                                     accumulatedH0, sc->pen_clip3, &rr, &c);
                    calls += 1; cells += c;
                    if (rr.score == prevScore || rr.max_off < (w >> 1) + (w >> 2) || tryIdx == 1) break;
                    prevScore = rr.score;
                    w = w << 1;
                }
                reg.w = std::max(reg.w, w);
                if (rr.gscore <= 0 || rr.gscore <= rr.score - sc->pen_clip3) {
                    rightQLen = rr.qle; rightTLen = rr.tle; rightScore = rr.score;
                } else {
                    rightQLen = readLen - seedQEnd; rightTLen = rr.gtle; rightScore = rr.gscore;
                }
            }
        }
        reg.qb = seedQbeg - leftQLen;                                    // :318-331
        reg.qe = seedQEnd + rightQLen;
        reg.rb = seedRbeg - leftTLen;
        reg.re = seedREnd + rightTLen;
        int32_t trueScore = seedLen * sc->a;
        if (leftScore > 0) trueScore = leftScore;
        if (rightScore > 0) trueScore += rightScore - accumulatedH0;
        reg.score = trueScore;
        reg.true_score = trueScore;
        int32_t seedCov = 0;                                             // :333 (computeSeedCov :36-70)
        for (int i = 0; i < n_seeds; ++i)
            if (seeds[i].qbeg >= reg.qb && seeds[i].qbeg + seeds[i].len <= reg.qe &&
                seeds[i].rbeg >= reg.rb && seeds[i].rbeg + seeds[i].len <= reg.re)
                seedCov += seeds[i].len;
        reg.seed_cov = seedCov;
        regions.push_back(reg);
    }
    const int32_t subThreshold = sc->min_seed_len * sc->a;               // :338-343
    for (auto &r : regions)
        if (r.sub > 0 && r.sub < subThreshold) r.sub = 0;
    if (sw_calls) *sw_calls = calls;
    if (cells_out) *cells_out = cells;
    if ((int)regions.size() > cap) return -1;
    std::copy(regions.begin(), regions.end(), out);
    return (int)regions.size();
}

int orc_ext_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                  uint64_t ref_bases, const swb_ext_task *tasks, size_t n,
                  swb_ext_result *out, int n_threads, uint64_t *cells) {
    (void)ref_bases;
    std::vector<uint64_t> per(std::max(n_threads, 1), 0);
    parallel_for(n, n_threads, [&](size_t lo, size_t hi, int tid) {
        std::vector<uint8_t> q, t;
        uint64_t acc = 0;
        for (size_t k = lo; k < hi; ++k) {
            const swb_ext_task &tk = tasks[k];
            q.resize(std::max(tk.qlen, 1));
            t.resize(std::max(tk.tlen, 1));
            load_span(bases, pac, tk.q_off, tk.qlen, tk.flags, false, q.data());
            load_span(bases, pac, tk.t_off, tk.tlen, tk.flags, true, t.data());
            uint64_t c = 0;
            banded_sw_scalar(q.data(), tk.qlen, t.data(), tk.tlen, sc, tk.w, tk.h0, tk.end_bonus, &out[k], &c);
            acc += c;
        }
        per[tid] += acc;
    });
    if (cells) { *cells = 0; for (auto v : per) *cells += v; }
    return 0;
}

int orc_global_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                     uint64_t ref_bases, const swb_global_task *tasks, size_t n,
                     swb_global_result *results, uint32_t *cigar_out, size_t cigar_cap,
                     int n_threads, uint64_t *cells) {
    (void)ref_bases;
    std::vector<uint64_t> offs(n + 1, 0);
    for (size_t k = 0; k < n; ++k) offs[k + 1] = offs[k] + (uint64_t)std::max(tasks[k].qlen, 0) + std::max(tasks[k].tlen, 0);
    if (offs[n] > cigar_cap) return -1;
    std::vector<uint64_t> per(std::max(n_threads, 1), 0);
    std::vector<int> bad(std::max(n_threads, 1), 0);
    parallel_for(n, n_threads, [&](size_t lo, size_t hi, int tid) {
        std::vector<uint8_t> q, t;
        std::vector<uint32_t> cig;
        uint64_t acc = 0;
        for (size_t k = lo; k < hi; ++k) {
            const swb_global_task &tk = tasks[k];
            q.resize(std::max(tk.qlen, 1));
            t.resize(std::max(tk.tlen, 1));
            load_span(bases, pac, tk.q_off, tk.qlen, tk.flags, false, q.data());
            load_span(bases, pac, tk.t_off, tk.tlen, tk.flags, true, t.data());
            int32_t w = tk.w, score = 0, attempts = 1;
            uint64_t c = 0;
            if (global_align(q.data(), tk.qlen, t.data(), tk.tlen, sc, w, &score, &cig, &c) != 0) { bad[tid] = 1; continue; }
            acc += c;
            if (tk.flags & SWB_GLB_RETRY) {
                int retries = 0;
                while (score < tk.true_score && retries < 3) {
                    w *= 2;
                    retries += 1;
                    attempts += 1;
                    if (global_align(q.data(), tk.qlen, t.data(), tk.tlen, sc, w, &score, &cig, &c) != 0) { bad[tid] = 1; break; }
                    acc += c;
                }
            }
            results[k].score = score;
            results[k].n_cigar = (int32_t)cig.size();
            results[k].w_used = w;
            results[k].attempts = attempts;
            results[k].cigar_off = offs[k];
            std::copy(cig.begin(), cig.end(), cigar_out + offs[k]);
        }
        per[tid] += acc;
    });
    if (cells) { *cells = 0; for (auto v : per) *cells += v; }
    for (int b : bad) if (b) return -1;
    return 0;
}

// CIGARGenerator.generate (CIGARGenerator.swift:30-111) over a batch of
// swb_cigar_task, host threads over static task ranges.  Task k writes its
// CIGAR at cigar_out + sum_{j<k}(qlen_j + rlen_j + 2) and its MD string
// (NUL-terminated) at md_out + sum_{j<k}(6*(qlen_j + rlen_j) + 8), the
// fixed-capacity layout of swb_cigar_batch's header.
int orc_cigar_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                    const swb_cigar_task *tasks, size_t n, swb_cigar_result *results,
                    uint32_t *cigar_out, size_t cigar_cap, char *md_out, size_t md_cap,
                    int n_threads, uint64_t *cells) {
    std::vector<uint64_t> coff(n + 1, 0), moff(n + 1, 0);
    for (size_t k = 0; k < n; ++k) {
        const uint64_t qr = (uint64_t)std::max(tasks[k].qlen, 0) + (uint64_t)std::max(tasks[k].rlen, 0);
        coff[k + 1] = coff[k] + qr + 2;
        moff[k + 1] = moff[k] + 6 * qr + 8;
    }
    if (coff[n] > cigar_cap || moff[n] > md_cap) return -1;
    std::vector<uint64_t> per(std::max(n_threads, 1), 0);
    std::vector<int> bad(std::max(n_threads, 1), 0);
    parallel_for(n, n_threads, [&](size_t lo, size_t hi, int tid) {
        std::vector<uint8_t> q, r;
        uint64_t acc = 0;
        for (size_t k = lo; k < hi; ++k) {
            const swb_cigar_task &tk = tasks[k];
            q.resize(std::max(tk.qlen, 1));
            r.resize(std::max(tk.rlen, 1));
            load_span(bases, pac, tk.q_off, tk.qlen, tk.flags, false, q.data());
            load_span(bases, pac, tk.t_off, tk.rlen, tk.flags, true, r.data());
            swb_cigar_result &res = results[k];
            int32_t ncig = (int32_t)(coff[k + 1] - coff[k]), nm = 0, score = 0, used = 0;
            int64_t pos = 0;
            uint64_t c = 0;
            if (orc_cigar_generate(q.data(), tk.qlen, r.data(), tk.rlen, tk.qb, tk.qe, tk.read_len, tk.is_reverse,
                                   tk.true_score, tk.initial_w, sc, tk.ref_pos, cigar_out + coff[k], &ncig, &nm,
                                   md_out + moff[k], (int32_t)(moff[k + 1] - moff[k]), &score, &pos, &c,
                                   &used) != 0) {
                bad[tid] = 1;
                continue;
            }
            acc += c;
            res.score = score;
            res.nm = nm;
            res.n_cigar = ncig;
            res.md_len = (int32_t)std::strlen(md_out + moff[k]);
            res.pos = pos;
            res.cigar_off = coff[k];
            res.md_off = moff[k];
            res.used_dp = used;
            res.reserved = 0;
        }
        per[tid] += acc;
    });
    if (cells) { *cells = 0; for (auto v : per) *cells += v; }
    for (int b : bad) if (b) return -1;
    return 0;
}

int orc_local_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                    uint64_t ref_bases, const swb_local_task *tasks, size_t n,
                    swb_local_result *out, int n_threads, uint64_t *cells) {
    (void)ref_bases;
    std::vector<uint64_t> per(std::max(n_threads, 1), 0);
    parallel_for(n, n_threads, [&](size_t lo, size_t hi, int tid) {
        std::vector<uint8_t> q, t;
        uint64_t acc = 0;
        for (size_t k = lo; k < hi; ++k) {
            const swb_local_task &tk = tasks[k];
            q.resize(std::max(tk.qlen, 1));
            t.resize(std::max(tk.tlen, 1));
            load_span(bases, pac, tk.q_off, tk.qlen, tk.flags, false, q.data());
            load_span(bases, pac, tk.t_off, tk.tlen, tk.flags, true, t.data());
            uint64_t c = 0;
            local_align(q.data(), tk.qlen, t.data(), tk.tlen, sc, clamp_u8(tk.min_sub_score), &out[k], &c, nullptr);
            acc += c;
        }
        per[tid] += acc;
    });
    if (cells) { *cells = 0; for (auto v : per) *cells += v; }
    return 0;
}

}  // extern "C"

int orc_extend_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac, int64_t genome_len,
                     const swb_seed *seeds, const swb_chain *chains, size_t n_chains,
                     swb_region *out, uint32_t *n_regions, int n_threads, uint64_t *cells) {
    static_assert(sizeof(orc_region) == sizeof(swb_region), "region layouts differ");
    static_assert(sizeof(orc_seed) == sizeof(swb_seed), "seed layouts differ");
    std::vector<uint64_t> per(std::max(n_threads, 1), 0);
    std::atomic<int> bad{0};
    parallel_for(n_chains, n_threads, [&](size_t lo, size_t hi, int tid) {
        for (size_t c = lo; c < hi; ++c) {
            const swb_chain &ch = chains[c];
            uint64_t calls = 0, cl = 0;
            const int n = orc_extend(reinterpret_cast<const orc_seed *>(seeds + ch.seed_off), (int32_t)ch.n_seeds,
                                     ch.rid, bases + ch.read_off, ch.read_len, pac, genome_len, 1, sc,
                                     reinterpret_cast<orc_region *>(out + ch.seed_off), (int32_t)ch.n_seeds, &calls, &cl);
            if (n < 0) bad = 1;
            n_regions[c] = (uint32_t)std::max(n, 0);
            per[tid] += cl;
        }
    });
    if (cells) { *cells = 0; for (auto v : per) *cells += v; }
    return bad ? -1 : 0;
}

// --------------------------------------------------------------------------
// MateRescue.rescue -- Sources/BWAMem/MateRescue.swift:29-171, with
// hasMateHit (:319-346), PackedReference.fetchSequence
// (Sources/FMIndex/PackedReference.swift:73-121) and
// ReferenceMetadata.sequenceID (Sources/BWACore/ReferenceMetadata.swift:77-89).
// --------------------------------------------------------------------------
namespace {

int32_t sequence_id(const int64_t *off, size_t n, int64_t pos) {   // ReferenceMetadata.swift:77-89
    long lo = 0, hi = (long)n - 1;
    while (lo < hi) {
        const long mid = (lo + hi + 1) / 2;
        if (off[mid] <= pos) lo = mid; else hi = mid - 1;
    }
    return (int32_t)lo;
}

struct Fetched {
    std::vector<uint8_t> bases;
    int64_t clamped_begin = 0;
    int32_t rid = 0;
};

bool fetch_sequence(const uint8_t *pac, int64_t bwtBegin, int64_t bwtEnd, int64_t gl, const int64_t *off,
                    const int32_t *len, size_t n, Fetched &f) {         // PackedReference.swift:73-121
    if (!(bwtBegin < bwtEnd)) return false;
    const bool isReverse = bwtBegin >= gl;
    if (!isReverse) {
        const int32_t rid = sequence_id(off, n, bwtBegin);
        const int64_t chromEnd = off[rid] + (int64_t)len[rid];
        const int64_t cb = std::max(bwtBegin, off[rid]), ce = std::min(bwtEnd, chromEnd);
        if (!(cb < ce)) return false;
        f.bases.resize((size_t)(ce - cb));
        for (int64_t i = 0; i < ce - cb; ++i) f.bases[(size_t)i] = pac_base(pac, cb + i);
        f.clamped_begin = cb;
        f.rid = rid;
    } else {
        const int64_t fwdBegin = 2 * gl - bwtEnd, fwdEnd = 2 * gl - bwtBegin;
        const int32_t rid = sequence_id(off, n, fwdBegin);
        const int64_t chromEnd = off[rid] + (int64_t)len[rid];
        const int64_t cb = std::max(fwdBegin, off[rid]), ce = std::min(fwdEnd, chromEnd);
        if (!(cb < ce)) return false;
        f.bases.resize((size_t)(ce - cb));
        for (int64_t i = 0; i < ce - cb; ++i) f.bases[(size_t)i] = pac_base(pac, cb + i);
        std::reverse(f.bases.begin(), f.bases.end());
        for (auto &b : f.bases) b = (uint8_t)(3 - b);
        f.clamped_begin = 2 * gl - ce;
        f.rid = rid;
    }
    return true;
}

bool has_mate_hit(const swb_anchor *mregs, uint32_t nm, const swb_anchor &t, int dir, const swb_orientation &st,
                  int64_t gl) {                                         // MateRescue.swift:319-346
    for (uint32_t k = 0; k < nm; ++k) {
        const swb_anchor &m = mregs[k];
        if (m.rid != t.rid) continue;
        const bool sameStrand = (t.rb >= gl) == (m.rb >= gl);
        const int64_t p2 = sameStrand ? m.rb : (2 * gl - 1 - m.rb);
        const int bwaDir = (sameStrand ? 0 : 1) ^ (p2 > t.rb ? 0 : 3);
        if (bwaDir != dir) continue;
        const int64_t d = p2 > t.rb ? p2 - t.rb : t.rb - p2;
        if (d >= st.proper_low && d <= st.proper_high) return true;
    }
    return false;
}

}  // namespace

int orc_mate_rescue_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac, int64_t gl,
                          const swb_rescue_job *jobs, size_t n_jobs, const swb_anchor *templates,
                          const swb_anchor *mate_regions, const swb_orientation *stats, int32_t primary,
                          const int64_t *coff, const int32_t *clen, size_t n_contigs,
                          swb_rescued *out, uint32_t *n_out, uint32_t *n_cand, int n_threads, uint64_t *cells) {
    std::vector<uint64_t> per(std::max(n_threads, 1), 0);
    parallel_for(n_jobs, n_threads, [&](size_t lo, size_t hi, int tid) {
        std::vector<uint8_t> fwd, rev;
        Fetched f;
        for (size_t j = lo; j < hi; ++j) {
            const swb_rescue_job &jb = jobs[j];
            uint32_t nout = 0, ncand = 0;
            swb_rescued *o = out + 4 * (size_t)jb.tmpl_off;
            if (jb.n_tmpl > 0 && !stats[primary].failed) {                // :40-44
                const int64_t mateLen = jb.mate_len;
                const int32_t minScore = sc->min_seed_len * sc->a;
                fwd.assign(bases + jb.mate_off, bases + jb.mate_off + jb.mate_len);
                rev.resize(fwd.size());
                for (size_t k = 0; k < fwd.size(); ++k) {                  // ReadSequence.reverseComplement
                    const uint8_t b = fwd[fwd.size() - 1 - k];
                    rev[k] = b < 4 ? (uint8_t)(3 - b) : 4;
                }
                for (uint32_t ti = 0; ti < jb.n_tmpl; ++ti) {
                    const swb_anchor &a = templates[jb.tmpl_off + ti];
                    bool allSatisfied = true;
                    for (int r = 0; r < 4; ++r) {
                        const swb_orientation &os = stats[r];
                        if (os.failed) continue;
                        if (has_mate_hit(mate_regions + jb.mreg_off, jb.n_mreg, a, r, os, gl)) continue;
                        allSatisfied = false;
                        const bool isRev = (r >> 1) != (r & 1), isLarger = (r >> 1) == 0;   // :70-73
                        int64_t rb, re;
                        if (!isRev) {
                            if (isLarger) { rb = a.rb + os.proper_low; re = a.rb + os.proper_high + mateLen; }
                            else { rb = a.rb - os.proper_high - mateLen; re = a.rb - os.proper_low; }
                        } else {
                            if (isLarger) { rb = a.rb + os.proper_low - mateLen; re = a.rb + os.proper_high; }
                            else { rb = a.rb - os.proper_high; re = a.rb - os.proper_low + mateLen; }
                        }
                        rb = std::max<int64_t>(rb, 0);                     // :104-106
                        re = std::min<int64_t>(re, 2 * gl);
                        if (!(rb < re)) continue;
                        if (!fetch_sequence(pac, rb, re, gl, coff, clen, n_contigs, f)) continue;
                        if (f.rid != a.rid) continue;
                        const std::vector<uint8_t> &q = isRev ? rev : fwd;
                        swb_local_result sw;
                        uint64_t c = 0;
                        ++ncand;
                        local_align(q.data(), (int)q.size(), f.bases.data(), (int)f.bases.size(), sc,
                                    clamp_u8(minScore), &sw, &c, nullptr);
                        per[tid] += c;
                        if (sw.score == 0) continue;                         // nil
                        if (!(sw.score >= minScore)) continue;
                        swb_rescued g{};
                        g.score = sw.score;
                        g.true_score = sw.score;
                        g.csub = sw.score2;
                        g.rid = a.rid;
                        const int64_t tb = sw.tb, te = sw.te;
                        if (!isRev) {                                       // :146-158
                            g.rb = f.clamped_begin + tb;
                            g.re = f.clamped_begin + te + 1;
                            g.qb = sw.qb;
                            g.qe = sw.qe + 1;
                        } else {
                            g.rb = 2 * gl - (f.clamped_begin + te + 1);
                            g.re = 2 * gl - (f.clamped_begin + tb);
                            g.qb = (int32_t)mateLen - (sw.qe + 1);
                            g.qe = (int32_t)mateLen - sw.qb;
                        }
                        const int64_t refSpan = te - tb + 1, querySpan = (int64_t)(sw.qe - sw.qb + 1);
                        g.seed_cov = (int32_t)(std::min(refSpan, querySpan) / 2);
                        o[nout++] = g;
                    }
                    if (allSatisfied) break;
                }
            }
            n_out[j] = nout;
            if (n_cand) n_cand[j] = ncand;
        }
    });
    if (cells) { *cells = 0; for (auto v : per) *cells += v; }
    return 0;
}

// --------------------------------------------------------------------------
// FM index and SMEM finding -- Sources/FMIndex/BWT.swift, BackwardSearch.swift,
// SMEMFinder.swift (bwa-mem2 FMI_search.cpp's backwardExt and
// getSMEMsOnePosOneThread / getSMEMsAllPosOneThread).
// --------------------------------------------------------------------------
namespace {

struct OrcBwt {
    const swb_bwt_checkpoint *cp;
    int64_t count[5];
    int64_t length, sentinel;
    // BWT.occ (BWT.swift:68-84): checkpoint count plus the set bits of the
    // block before position y (oneHotMaskArray[y] = the top y bits).
    int64_t occ(int64_t pos, int c) const {
        const swb_bwt_checkpoint &k = cp[pos >> 6];
        const int y = (int)(pos & 63);
        const uint64_t mask = y == 0 ? 0ull : ~(~0ull >> y);
        return k.counts[c] + (int64_t)__builtin_popcountll(k.bits[c] & mask);
    }
};

struct Intv {
    int64_t k, l, s;
};

// BackwardSearch.backwardExt (BackwardSearch.swift:21-77).
Intv backward_ext(const OrcBwt &b, int64_t k, int64_t l, int64_t s, int a) {
    if (a >= 4) return {0, 0, 0};
    const int64_t sp = k, ep = k + s;
    int64_t kAll[4], sAll[4], lAll[4];
    for (int c = 0; c < 4; ++c) {
        const int64_t occSP = b.occ(sp, c), occEP = b.occ(ep, c);
        kAll[c] = b.count[c] + occSP;
        sAll[c] = occEP - occSP;
    }
    const int64_t sentinelOffset = (sp <= b.sentinel && ep > b.sentinel) ? 1 : 0;
    lAll[3] = l + sentinelOffset;
    lAll[2] = lAll[3] + sAll[3];
    lAll[1] = lAll[2] + sAll[2];
    lAll[0] = lAll[1] + sAll[1];
    return {kAll[a], lAll[a], sAll[a]};
}

// SMEMFinder.BidiInterval (SMEMFinder.swift:67-73).
struct Bidi {
    int64_t k, l, s;
    int32_t m, n;
};

// SMEMFinder.findSMEMsAtPosition (SMEMFinder.swift:89-268); returns nextPos.
int find_smems_at(const OrcBwt &b, const uint8_t *query, int readLength, int startPos, int32_t minSeedLen,
                  int64_t minIntv, std::vector<swb_smem> &smems, std::vector<Bidi> &prev) {
    int nextPos = startPos + 1;
    const int a = query[startPos];
    if (a >= 4) return nextPos;                                              // :104-107
    Bidi smem{b.count[a], b.count[3 - a], b.count[a + 1] - b.count[a], startPos, startPos};   // :111-117
    prev.clear();
    int numPrev = 0;
    int j = startPos + 1;                                                    // :124-157
    while (j < readLength) {
        const int base = query[j];
        nextPos = j + 1;
        if (base >= 4) break;
        const Intv ext = backward_ext(b, smem.l, smem.k, smem.s, 3 - base);   // swapped k/l, complement base
        const Bidi newSmem{ext.l, ext.k, ext.s, smem.m, (int32_t)j};
        if (newSmem.s != smem.s) {
            prev.push_back(smem);
            numPrev += 1;
        }
        if (newSmem.s < minIntv) {
            nextPos = j;
            break;
        }
        smem = newSmem;
        j += 1;
    }
    if (smem.s >= minIntv) {                                                 // :160-163
        prev.push_back(smem);
        numPrev += 1;
    }
    std::reverse(prev.begin(), prev.end());                                  // :166
    for (int bj = startPos - 1; bj >= 0; --bj) {                             // :169-250
        const int base = query[bj];
        if (base >= 4) break;
        int numCurr = 0;
        int64_t currS = -1;
        int p = 0;
        while (p < numPrev) {
            const Bidi iv = prev[p];
            const Intv ext = backward_ext(b, iv.k, iv.l, iv.s, base);
            const Bidi ni{ext.k, ext.l, ext.s, (int32_t)bj, iv.n};
            if (ni.s < minIntv && (iv.n - iv.m + 1) >= minSeedLen) {          // condition 1
                smems.push_back(swb_smem{iv.k, iv.k + iv.s - 1, iv.m, iv.n + 1});
                break;
            }
            if (ni.s >= minIntv && ni.s != currS) {                          // condition 2
                currS = ni.s;
                if (numCurr < (int)prev.size()) prev[numCurr] = ni;
                else prev.push_back(ni);
                numCurr += 1;
                break;
            }
            p += 1;
        }
        p += 1;
        while (p < numPrev) {
            const Bidi iv = prev[p];
            const Intv ext = backward_ext(b, iv.k, iv.l, iv.s, base);
            const Bidi ni{ext.k, ext.l, ext.s, (int32_t)bj, iv.n};
            if (ni.s >= minIntv && ni.s != currS) {
                currS = ni.s;
                if (numCurr < (int)prev.size()) prev[numCurr] = ni;
                else prev.push_back(ni);
                numCurr += 1;
            }
            p += 1;
        }
        numPrev = numCurr;
        if (numCurr == 0) break;
    }
    if (numPrev != 0) {                                                      // :253-265
        const Bidi iv = prev[0];
        if ((iv.n - iv.m + 1) >= minSeedLen) smems.push_back(swb_smem{iv.k, iv.k + iv.s - 1, iv.m, iv.n + 1});
    }
    return nextPos;
}

// SMEMFinder.findAllSMEMs (SMEMFinder.swift:28-63): every start position in
// turn, then sorted by query begin, longer first.
void find_all_smems(const OrcBwt &b, const uint8_t *query, int readLength, int32_t minSeedLen, int64_t minIntv,
                    std::vector<swb_smem> &out) {
    out.clear();
    std::vector<Bidi> prev;
    int pos = 0;
    while (pos < readLength) pos = find_smems_at(b, query, readLength, pos, minSeedLen, minIntv, out, prev);
    std::stable_sort(out.begin(), out.end(), [](const swb_smem &x, const swb_smem &y) {
        if (x.qb != y.qb) return x.qb < y.qb;
        return (x.qe - x.qb) > (y.qe - y.qb);
    });
}

}  // namespace

// FM index of a forward strand (codes 0-3) in the layout the reference
// loads (BWT.swift, CheckpointOCC.swift): the text is the strand followed by
// its reverse complement, then '$'; SA by prefix doubling; BWT[i] =
// text[SA[i]-1] ('$' where SA[i] = 0: the sentinel position); count[c] =
// 1 + the characters below c; a checkpoint per 64 BWT positions.  Test
// infrastructure: builds the indexes of the synthetic references.
int orc_bwt_build(const uint8_t *codes, int64_t n, swb_bwt_checkpoint *cp, int64_t n_cp, int64_t count_out[5],
                  int64_t *length_out, int64_t *sentinel_out, int n_threads) {
    (void)n_threads;
    const int64_t N = 2 * n + 1;
    if (n_cp < (N >> 6) + 1) return -1;
    std::vector<uint8_t> T((size_t)N);
    for (int64_t i = 0; i < n; ++i) {
        if (codes[i] > 3) return -2;
        T[(size_t)i] = (uint8_t)(codes[i] + 1);
        T[(size_t)(n + i)] = (uint8_t)(3 - codes[n - 1 - i] + 1);
    }
    T[(size_t)(2 * n)] = 0;                                   // '$', smallest
    // Prefix doubling: rank by the first h characters, h = 1, 2, 4, ...
    std::vector<int32_t> sa((size_t)N), rank((size_t)N), tmp((size_t)N);
    for (int64_t i = 0; i < N; ++i) { sa[(size_t)i] = (int32_t)i; rank[(size_t)i] = T[(size_t)i]; }
    for (int64_t h = 1;; h <<= 1) {
        auto key = [&](int32_t i) -> std::pair<int32_t, int32_t> {
            return {rank[(size_t)i], i + h < N ? rank[(size_t)(i + h)] : -1};
        };
        std::sort(sa.begin(), sa.end(), [&](int32_t x, int32_t y) { return key(x) < key(y); });
        tmp[(size_t)sa[0]] = 0;
        for (int64_t r = 1; r < N; ++r)
            tmp[(size_t)sa[(size_t)r]] = tmp[(size_t)sa[(size_t)(r - 1)]] + (key(sa[(size_t)(r - 1)]) < key(sa[(size_t)r]) ? 1 : 0);
        rank.swap(tmp);
        if (rank[(size_t)sa[(size_t)(N - 1)]] == N - 1) break;
    }
    int64_t cnt[5] = {0, 0, 0, 0, 0};
    for (int64_t i = 0; i < 2 * n; ++i) cnt[T[(size_t)i]] += 1;        // cnt[c+1] = occurrences of base c
    count_out[0] = 1;
    for (int c = 1; c <= 4; ++c) count_out[c] = count_out[c - 1] + cnt[c];
    int64_t run[4] = {0, 0, 0, 0};
    int64_t sentinel = -1;
    for (int64_t b = 0; b < n_cp; ++b) {
        for (int c = 0; c < 4; ++c) { cp[b].counts[c] = run[c]; cp[b].bits[c] = 0; }
        for (int y = 0; y < 64; ++y) {
            const int64_t i = b * 64 + y;
            if (i >= N) break;
            const int32_t s = sa[(size_t)i];
            if (s == 0) { sentinel = i; continue; }
            const int c = T[(size_t)(s - 1)] - 1;
            cp[b].bits[c] |= 1ull << (63 - y);
            run[c] += 1;
        }
    }
    *length_out = N;
    *sentinel_out = sentinel;
    return 0;
}

// BWAMemAligner.internalReseed (BWAMemAligner.swift:259-305, the arena form
// alignReadPhase1to3 calls): every SMEM of the first pass at least split_len
// long with at most split_width occurrences is searched again from its
// midpoint with minIntv = its count + 1; the new SMEMs are appended and the
// list re-sorted.
void internal_reseed(const OrcBwt &b, const uint8_t *query, int readLength, int32_t minSeedLen, int32_t splitLen,
                     int32_t splitWidth, std::vector<swb_smem> &smems) {
    const size_t originalCount = smems.size();
    std::vector<swb_smem> added;
    std::vector<Bidi> prev;
    for (size_t i = 0; i < originalCount; ++i) {
        const swb_smem sm = smems[i];
        const int len = sm.qe - sm.qb;
        const int64_t cnt = sm.l - sm.k + 1;
        if (len < splitLen || cnt > (int64_t)splitWidth) continue;
        const int midpoint = (sm.qb + sm.qe) / 2;
        find_smems_at(b, query, readLength, midpoint, minSeedLen, cnt + 1, added, prev);
    }
    if (added.empty()) return;
    smems.insert(smems.end(), added.begin(), added.end());
    std::stable_sort(smems.begin(), smems.end(), [](const swb_smem &x, const swb_smem &y) {
        if (x.qb != y.qb) return x.qb < y.qb;
        return (x.qe - x.qb) > (y.qe - y.qb);
    });
}

// findAllSMEMs (and, when split_len > 0, internalReseed) over a batch of
// reads (host threads); the output layout of swb_smem_batch: read r's SMEMs
// at out[r * cap ..+ n_out[r]] (the first cap kept when there are more).
// Returns the number of reads with more than cap.
int64_t orc_smem_batch(const swb_bwt_checkpoint *cp, const int64_t count[5], int64_t length, int64_t sentinel,
                       const uint8_t *bases, const uint64_t *read_off, const int32_t *read_len, size_t n_reads,
                       int32_t min_seed_len, int64_t min_intv, int32_t split_len, int32_t split_width, uint32_t cap,
                       swb_smem *out, uint32_t *n_out, int n_threads) {
    OrcBwt b{cp, {count[0], count[1], count[2], count[3], count[4]}, length, sentinel};
    std::atomic<int64_t> over{0};
    parallel_for(n_reads, n_threads, [&](size_t lo, size_t hi, int) {
        std::vector<swb_smem> v;
        for (size_t r = lo; r < hi; ++r) {
            find_all_smems(b, bases + read_off[r], read_len[r], min_seed_len, min_intv, v);
            if (split_len > 0) internal_reseed(b, bases + read_off[r], read_len[r], min_seed_len, split_len, split_width, v);
            n_out[r] = (uint32_t)v.size();
            if (v.size() > cap) over += 1;
            std::copy(v.begin(), v.begin() + std::min<size_t>(v.size(), cap), out + r * (size_t)cap);
        }
    });
    return over.load();
}
