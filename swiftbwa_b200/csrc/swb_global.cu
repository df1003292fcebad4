// swb_global.cu -- kernel 2: banded global alignment with CIGAR traceback,
// bit-exact with GlobalAligner.align (Sources/Alignment/GlobalAligner.swift:19-232)
// and, per task flag, CIGARGenerator.generate's band-doubling retry
// (Sources/Alignment/CIGARGenerator.swift:88-96).
//
// One thread owns one alignment.  Alignments are sorted by row width, then
// largest shape first; queries up to 256 run global_smem_kernel (H/E rows in
// shared memory, int16 where every value provably fits, else int32), whose
// warps claim 32 sorted alignments at a time; longer queries run
// global_kernel over rows in global scratch.  The 4-bit backpointers go to
// global memory [row][word][slot], eight columns per word, so a warp's
// threads touch adjacent words.  The backpointer matrix of the last attempt
// is walked by the same thread; ops are written in traceback order into the
// task's CIGAR window, merged into runs on the fly, and reversed in place at
// the end (CIGARBuilder.swift).
#include <type_traits>

#include "swb_device.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

constexpr int kGT = 64;   // threads per block
constexpr int kNegInf = INT32_MIN / 2;   // GlobalAligner.swift:52

// CIGARGenerator.generate repeats the DP with the band doubled while the
// score is below the true score, at most three times (CIGARGenerator.swift:
// 88-96).  Once the band covers the whole matrix (every row spans all qlen
// columns: w >= max(qlen, tlen) - 1) a wider band computes the same matrix,
// score and backpointers, so the attempts left are accounted for -- width,
// attempt count and their qlen * tlen cells each -- instead of recomputed.
// Returns true when it did so (the caller stops retrying).
__device__ __forceinline__ bool nw_skip_covered_retries(int qlen, int tlen, int w, int retries, int &w0,
                                                        swb_global_result &r, unsigned long long &cells) {
    if (w < imax(qlen, tlen) - 1) return false;
    const int left = 3 - retries;
    w0 *= 1 << left;
    r.attempts += left;
    cells += (unsigned long long)left * (unsigned long long)qlen * (unsigned long long)tlen;
    return true;
}

struct GlobalArgs {
    DevScoring sc;
    const uint8_t *bases;
    const uint8_t *pac;
    const swb_global_task *tasks;
    swb_global_result *res;
    uint32_t *cigar;
    const unsigned long long *cigar_off;   // per task
    unsigned long long *cells;
    size_t n;
    int qsplit;   // tasks with qlen <= qsplit belong to the shared-memory kernel
};

struct Scratch {
    int *h, *e;
    uint8_t *q, *t, *z;
    size_t nslots, slot;
    int qmax, tmax;
    __device__ __forceinline__ int &H(int j) const { return h[(size_t)j * nslots + slot]; }
    __device__ __forceinline__ int &E(int j) const { return e[(size_t)j * nslots + slot]; }
    __device__ __forceinline__ uint8_t Q(int j) const { return q[(size_t)j * nslots + slot]; }
    __device__ __forceinline__ uint8_t T(int i) const { return t[(size_t)i * nslots + slot]; }
    __device__ __forceinline__ uint8_t &Z(int i, int col) const {
        return z[((size_t)i * qmax + col) * nslots + slot];
    }
};

// One DP attempt (GlobalAligner.swift:26-144); returns h[qlen].
__device__ int global_dp(const DevScoring &sc, const Scratch &s, int qlen, int tlen, int w,
                         int nCol, unsigned long long &cells) {
    const int oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const int oeDel = oDel + eDel, oeIns = oIns + eIns;
    for (int j = 0; j <= qlen; ++j) {                                       // :75-76
        s.H(j) = kNegInf;
        s.E(j) = kNegInf;
    }
    s.H(0) = 0;                                                             // :80-84
    const int initEnd = imin(w, qlen);
    for (int j = 1; j <= initEnd; ++j) s.H(j) = 0 - (oIns + eIns * j);
    for (int i = 0; i < tlen; ++i) {                                        // :89-142
        const int beg = imax(0, i - w);
        const int end = (int)min((long long)qlen, (long long)i + w + 1);
        const RowTable rt = row_table(sc, s.T(i));
        int f = kNegInf;
        int hDiag = s.H(beg);
        s.H(beg) = beg == 0 ? 0 - (oeDel + eDel * i) : kNegInf;
        if (end > beg) cells += (unsigned long long)(end - beg);
        int hLeft = s.H(beg);   // h[j] for the first column of the row
        for (int j = beg; j < end; ++j) {
            const int j1 = j + 1;
            int hCur = hDiag + row_score(rt, s.Q(j));
            hDiag = s.H(j1);
            const int eOpen = hDiag - oeDel;
            const int eExtend = s.E(j1) - eDel;
            const uint32_t eFlag = eOpen > eExtend ? 0u : 1u;
            const int eVal = eOpen > eExtend ? eOpen : eExtend;
            s.E(j1) = eVal;
            const int fOpen = hLeft - oeIns;
            const int fExtend = f - eIns;
            const uint32_t fFlag = fOpen > fExtend ? 0u : 2u;
            const int fVal = fOpen > fExtend ? fOpen : fExtend;
            f = fVal;
            const uint32_t fromE = eVal > hCur ? 4u : 0u;
            hCur = eVal > hCur ? eVal : hCur;
            const uint32_t fromF = fVal > hCur ? 8u : 0u;
            hCur = fVal > hCur ? fVal : hCur;
            s.H(j1) = hCur;
            hLeft = hCur;
            s.Z(i, j - beg) = (uint8_t)(eFlag | fFlag | fromE | fromF);
        }
    }
    (void)nCol;
    return s.H(qlen);                                                       // :144
}

// Run-length CIGAR writer in traceback (reverse) order.
struct CigarOut {
    uint32_t *p;
    int n = 0;
    uint32_t op = 0xFFFFFFFFu, len = 0;
    __device__ __forceinline__ void append(uint32_t o) {
        if (o == op) {
            ++len;
        } else {
            if (len) p[n++] = (len << 4) | op;
            op = o;
            len = 1;
        }
    }
    __device__ __forceinline__ void finish() {
        if (len) p[n++] = (len << 4) | op;
        for (int a = 0, b = n - 1; a < b; ++a, --b) {                       // builder.reverse()
            const uint32_t x = p[a];
            p[a] = p[b];
            p[b] = x;
        }
    }
};

// Traceback (GlobalAligner.swift:160-232); zat(i, col) is the 4-bit
// direction code of row i, band column col.
template <class ZAt>
__device__ int global_traceback(ZAt zat, int qlen, int tlen, int w, int nCol, uint32_t *out) {
    CigarOut c{out};
    int i = tlen - 1, j = qlen - 1, state = 0;
    while (i >= 0 || j >= 0) {
        if (i < 0) { c.append(1u); --j; continue; }
        if (j < 0) { c.append(2u); --i; continue; }
        const int beg = imax(0, i - w);
        const int col = j - beg;
        if (!(col >= 0 && col < nCol)) break;
        const uint32_t d = zat(i, col);
        if (state == 0) {
            const uint32_t hDir = (d >> 2) & 3u;
            if (hDir == 0) { c.append(0u); --i; --j; }
            else if (hDir == 1) state = 1;
            else state = 2;
        } else if (state == 1) {
            c.append(2u);
            if ((d & 1u) == 0) state = 0;
            --i;
        } else {
            c.append(1u);
            if ((d & 2u) == 0) state = 0;
            --j;
        }
    }
    c.finish();
    return c.n;
}

__global__ void __launch_bounds__(kGT) global_kernel(GlobalArgs a, Scratch base) {
    Scratch s = base;
    s.slot = blockIdx.x * (size_t)kGT + threadIdx.x;
    unsigned long long cells = 0;
    const size_t iters = (a.n + s.nslots - 1) / s.nslots;
    for (size_t it = 0; it < iters; ++it) {
        const size_t k = it * s.nslots + s.slot;
        if (k >= a.n) continue;
        const swb_global_task tk = a.tasks[k];
        if (tk.qlen <= a.qsplit) continue;
        swb_global_result r{0, 0, tk.w, 1, a.cigar_off[k]};
        const int qlen = tk.qlen, tlen = tk.tlen;
        if (qlen > 0 && tlen > 0) {                                          // :29-31
            for (int j = 0; j < qlen; ++j) s.q[(size_t)j * s.nslots + s.slot] =
                (uint8_t)span_base(a.bases, a.pac, tk.q_off, j, qlen, tk.flags, false);
            for (int i = 0; i < tlen; ++i) s.t[(size_t)i * s.nslots + s.slot] =
                (uint8_t)span_base(a.bases, a.pac, tk.t_off, i, tlen, tk.flags, true);
            int w0 = tk.w;
            int w = imax(w0, abs(qlen - tlen));                               // :47
            int nCol = (int)min((long long)qlen, 2ll * w + 1);               // :48
            int score = global_dp(a.sc, s, qlen, tlen, w, nCol, cells);
            if (tk.flags & SWB_GLB_RETRY) {                                  // CIGARGenerator.swift:88-96
                int retries = 0;
                while (score < tk.true_score && retries < 3) {
                    if (nw_skip_covered_retries(qlen, tlen, w, retries, w0, r, cells)) break;
                    w0 *= 2;
                    ++retries;
                    r.attempts++;
                    w = imax(w0, abs(qlen - tlen));
                    nCol = (int)min((long long)qlen, 2ll * w + 1);
                    score = global_dp(a.sc, s, qlen, tlen, w, nCol, cells);
                }
            }
            r.score = score;
            r.w_used = w0;
            r.n_cigar = global_traceback([&](int i, int col) -> uint32_t { return s.Z(i, col); }, qlen, tlen, w, nCol,
                                             a.cigar + r.cigar_off);
        }
        a.res[k] = r;
    }
    for (int o = 16; o > 0; o >>= 1) cells += __shfl_down_sync(0xFFFFFFFFu, cells, o);
    if ((threadIdx.x & 31) == 0 && cells) atomicAdd(a.cells, cells);
}

// ------------------------------------------------------------------------
// Shared-memory variant for queries of up to kGlbSmemMaxQ bases: the H/E
// row of each thread's alignment lives in shared memory ([column][thread],
// 8 bytes per column), the query codes beside it, and the 4-bit direction
// codes go to global memory packed 8 per word, laid out
// [row][word][slot] so a warp's stores of one word index are contiguous.
// Same recurrences, sentinels and traceback as above.
constexpr int kGlbSmemMaxQ = kGlobalSmemMaxQ;

struct ZPacked {
    uint32_t *z;      // this slot's first word
    size_t nslots;
    int ncw;          // words per row for this attempt
    int w = 0;        // band of this attempt (absolute layout)
    bool absolute = false;   // nibble of absolute column j (not of band column j - beg)
    __device__ __forceinline__ uint32_t operator()(int i, int col) const {
        const int j = absolute ? col + imax(0, i - w) : col;
        return (z[((size_t)i * ncw + (j >> 3)) * nslots] >> ((j & 7) << 2)) & 0xFu;
    }
};

// Row stores of the shared-memory kernel, [column][thread].
//   RowI32: H and E as int32 (the reference's types, sentinel -2^30).
//   RowI16: H and E as the two int16 halves of one word, with -16384 standing
//   in for the sentinel.  Exact when fits_i16() holds: every real H/E/F lies
//   in [-(q+t+2)P, a(q+t)] (P = the largest cost of one step), every value
//   derived from the sentinel stays within (q+t+2)(a+P) of it, so real values
//   still exceed all sentinel-derived ones, and sentinel-derived values keep
//   their order (they differ from the reference's only by the same shift).
//   A sentinel-derived final score is shifted back.
struct RowI32 {
    int2 *he;
    int T;
    static constexpr int kNeg = kNegInf;
    __device__ __forceinline__ void load(int j, int &h, int &e) const {
        const int2 v = he[j * T];
        h = v.x;
        e = v.y;
    }
    __device__ __forceinline__ void store(int j, int h, int e) const { he[j * T] = make_int2(h, e); }
    __device__ __forceinline__ int getH(int j) const { return he[j * T].x; }
    __device__ __forceinline__ void setH(int j, int h) const { he[j * T].x = h; }
    __device__ __forceinline__ int final_score(int s, int) const { return s; }
};

//   The int16 rows are computed two target rows at a time (global_dp_pair16).
struct RowI16 {
    uint32_t *he;
    int T;
    static constexpr int kNeg = -16384;
    // thr: every real value is above it, every sentinel-derived one at or below.
    __device__ __forceinline__ int final_score(int s, int thr) const { return s <= thr ? kNegInf + (s - kNeg) : s; }
};

__device__ __forceinline__ int step_cost(const DevScoring &sc) {
    return nw_i16_cost(sc.a, sc.b, sc.o_del, sc.e_del, sc.o_ins, sc.e_ins) - sc.a;
}

__device__ __forceinline__ bool fits_i16(const DevScoring &sc, int qlen, int tlen) {
    return nw_fits_i16(qlen, tlen, nw_i16_cost(sc.a, sc.b, sc.o_del, sc.e_del, sc.o_ins, sc.e_ins));
}

template <class Row>
__device__ int global_dp_smem(const DevScoring &sc, const Row &row, const uint8_t *qs, int T, const GlobalArgs &a,
                              const swb_global_task &tk, int w, const ZPacked &zp, unsigned long long &cells) {
    constexpr int kNeg = Row::kNeg;
    const int qlen = tk.qlen, tlen = tk.tlen;
    const int oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const int oeDel = oDel + eDel, oeIns = oIns + eIns;
    for (int j = 0; j <= qlen; ++j) row.store(j, kNeg, kNeg);                    // :75-76
    row.setH(0, 0);                                                              // :80-84
    const int initEnd = imin(w, qlen);
    for (int j = 1; j <= initEnd; ++j) row.setH(j, 0 - (oIns + eIns * j));
    const size_t rstride = (size_t)zp.ncw * zp.nslots;
    for (int i = 0; i < tlen; ++i) {                                             // :89-142
        const int beg = imax(0, i - w);
        const int end = (int)min((long long)qlen, (long long)i + w + 1);
        const RowTable rt = row_table(sc, span_base(a.bases, a.pac, tk.t_off, i, tlen, tk.flags, true));
        int f = kNeg;
        int hDiag = row.getH(beg);
        const int hBeg = beg == 0 ? 0 - (oeDel + eDel * i) : kNeg;
        row.setH(beg, hBeg);
        if (end > beg) cells += (unsigned long long)(end - beg);
        int hLeft = hBeg;
        uint32_t *zrow = zp.z + (size_t)i * rstride;
        // One cell: H, E, F and its 4-bit backpointer code (bit 0: E extends,
        // 1: F extends, 2: H from E, 3: H from F; ties as the reference).
        // __vibmax_s32(a, b, &p) gives max(a, b) and p = (a >= b).
        auto cell = [&](int j) -> uint32_t {
            int vh, ve;
            row.load(j + 1, vh, ve);
            int hCur = hDiag + row_score(rt, qs[j * T]);
            hDiag = vh;
            bool eExt, fExt, hKeepE, hKeepF;
            const int eVal = __vibmax_s32(ve - eDel, vh - oeDel, &eExt);          // extend unless open > extend
            const int fVal = __vibmax_s32(f - eIns, hLeft - oeIns, &fExt);
            f = fVal;
            hCur = __vibmax_s32(hCur, eVal, &hKeepE);                              // from E when E > H
            hCur = __vibmax_s32(hCur, fVal, &hKeepF);                              // from F when F > H
            row.store(j + 1, hCur, eVal);
            hLeft = hCur;
            return (eExt ? 1u : 0u) | (fExt ? 2u : 0u) | (hKeepE ? 0u : 4u) | (hKeepF ? 0u : 8u);
        };
        // Eight columns per backpointer word, with constant shifts.
        int j = beg;
        size_t zo = 0;
        for (; j + 8 <= end; j += 8, zo += zp.nslots) {
            uint32_t word = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) word |= cell(j + k) << (4 * k);
            zrow[zo] = word;
        }
        if (j < end) {
            uint32_t word = 0;
            for (int k = 0; j < end; ++j, ++k) word |= cell(j) << (4 * k);
            zrow[zo] = word;
        }
    }
    const int thr = -(qlen + tlen + 2) * step_cost(sc) - 1;
    return row.final_score(row.getH(qlen), thr);                                 // :144
}

// ------------------------------------------------------------------------
// int16-row instance, two target rows per pass.  Row i's cell at column c
// and row i+1's at column c-1 are the low and high 16-bit lanes of one
// register and go through the DPX s16x2 forms together: vibmax_s16x2 gives
// each lane's max and its comparison, so the reference's tie rules and
// backpointer bits come out of the same operation.  Row i+1 takes row i's H
// and E of column c-1 from registers (one step old) and its diagonal, H of
// row i at column c-2, from two steps back; only row i+1's words reach
// shared memory, so a row pair costs one word load and one word store per
// column.  Row i's band [beg0, end0) and row i+1's [beg1, end1) differ by at
// most one column at each end (GlobalAligner.swift:90-91), so a pair runs
// row i alone for one or two columns, both rows together, then row i+1
// alone for one or two columns.  Backpointer codes are addressed by absolute
// column (word j/8 of the row, nibble j%8).  Values are those of RowI16.
__device__ __forceinline__ uint32_t rep16(int v) { return (uint32_t)(uint16_t)(int16_t)v * 0x10001u; }
// Lane-wise a + b (no lane leaves int16 here: see RowI16).
__device__ __forceinline__ uint32_t padd16(uint32_t a, uint32_t b) { return __viaddmax_s16x2(a, b, 0x80008000u); }
// prmt selector (q, q|8, 5, 5) of query code q: score as one 16-bit lane.
__device__ __forceinline__ uint32_t nw_sel(uint32_t q) { return q * 0x11u + 0x5580u; }

struct NwPairConsts {
    uint32_t negOeDel, negEDel, negOeIns, negEIns;
};

// One step of both lanes: DG/UH/UE are the diagonal H, the H and E above,
// S the scores; h, f are the previous step's H and F (the left neighbours),
// e receives E.  code0/code1: the 4-bit backpointers of lanes 0/1
// (GlobalAligner.swift:112-140: bit 0 E extends, 1 F extends, 2 H from E, 3 H from F).
__device__ __forceinline__ void nw_pair_step(const NwPairConsts &k, uint32_t DG, uint32_t UH, uint32_t UE, uint32_t S,
                                             uint32_t &h, uint32_t &e, uint32_t &f, uint32_t &code0,
                                             uint32_t &code1) {
    bool eh, el, fh, fl, keh, kel, kfh, kfl;
    uint32_t hc = padd16(DG, S);
    const uint32_t ev = __vibmax_s16x2(padd16(UE, k.negEDel), padd16(UH, k.negOeDel), &eh, &el);
    const uint32_t fv = __vibmax_s16x2(padd16(f, k.negEIns), padd16(h, k.negOeIns), &fh, &fl);
    hc = __vibmax_s16x2(hc, ev, &keh, &kel);
    hc = __vibmax_s16x2(hc, fv, &kfh, &kfl);
    code0 = (el ? 1u : 0u) | (fl ? 2u : 0u) | (kel ? 0u : 4u) | (kfl ? 0u : 8u);
    code1 = (eh ? 1u : 0u) | (fh ? 2u : 0u) | (keh ? 0u : 4u) | (kfh ? 0u : 8u);
    f = fv;
    h = hc;
    e = ev;
}

// Backpointer word of one row: codes are or-ed in at nibble j%8 and the
// word is stored when its last column is done.
struct ZRow {
    uint32_t *z;      // word 0 of this row and slot
    size_t nslots;
    uint32_t acc = 0;
    __device__ __forceinline__ void put(int j, uint32_t code, int last) {
        acc |= code << ((j & 7) << 2);
        if ((j & 7) == 7 || j == last) {
            z[(size_t)(j >> 3) * nslots] = acc;
            acc = 0;
        }
    }
};

// One lockstep step at column c (both lanes): row i at c, row i+1 at c-1.
// Returns the two backpointer codes; stores row i+1's word c.
struct NwLane2 {
    uint32_t h, hp2, e, f, wdp, selp;
};
__device__ __forceinline__ void nw_both(const NwPairConsts &k, const RowTable &rt0, const RowTable &rt1,
                                        uint32_t *__restrict__ he, const uint8_t *__restrict__ qs, int T, int c,
                                        NwLane2 &st, uint32_t &code0, uint32_t &code1) {
    const uint32_t wd = he[(c + 1) * T];                          // [H(i-1,c) | E(i-1,c)]
    const uint32_t sel = nw_sel(qs[c * T]);
    const uint32_t DG = __byte_perm(st.wdp, st.hp2, 0x5410);      // [H(i-1,c-1), H(i,c-2)]
    const uint32_t UH = __byte_perm(wd, st.h, 0x5410);            // [H(i-1,c),   H(i,c-1)]
    const uint32_t UE = __byte_perm(wd, st.e, 0x5432);            // [E(i-1,c),   E(i,c-1)]
    const uint32_t S = prmt(rt1.lo, rt1.hi, st.selp) * 65536u + prmt(rt0.lo, rt0.hi, sel);
    st.hp2 = st.h;
    nw_pair_step(k, DG, UH, UE, S, st.h, st.e, st.f, code0, code1);
    he[c * T] = __byte_perm(st.h, st.e, 0x7632);                  // row i+1's word c: H, E of column c-1
    st.wdp = wd;
    st.selp = sel;
}

__device__ int global_dp_pair16(const DevScoring &sc, uint32_t *__restrict__ he, const uint8_t *__restrict__ qs,
                                int T, const GlobalArgs &a, const swb_global_task &tk, int w, const ZPacked &zp,
                                unsigned long long &cells) {
    constexpr int kNeg = RowI16::kNeg;
    const int qlen = tk.qlen, tlen = tk.tlen;
    const int oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const int oeDel = oDel + eDel, oeIns = oIns + eIns;
    const NwPairConsts k{rep16(-oeDel), rep16(-eDel), rep16(-oeIns), rep16(-eIns)};
    const uint32_t negHi = (uint32_t)(uint16_t)kNeg << 16;
    // First row (GlobalAligner.swift:75-84): h[0] = 0, h[j] = -(oIns + eIns*j) up to w, E = -inf.
    const int initEnd = imin(w, qlen);
    for (int j = 0; j <= qlen; ++j) {
        const int hv = j == 0 ? 0 : (j <= initEnd ? 0 - (oIns + eIns * j) : kNeg);
        he[j * T] = ((uint32_t)hv & 0xFFFFu) | negHi;
    }
    const size_t rstride = (size_t)zp.ncw * zp.nslots;
    const size_t ns = zp.nslots;
    for (int i = 0; i < tlen; i += 2) {                                          // :89-142, two rows at a time
        const bool pair = i + 1 < tlen;
        const int beg0 = imax(0, i - w), end0 = imin(qlen, i + w + 1);
        const int beg1 = imax(0, i + 1 - w), end1 = pair ? imin(qlen, i + w + 2) : beg1;
        const RowTable rt0 = row_table(sc, span_base(a.bases, a.pac, tk.t_off, i, tlen, tk.flags, true));
        const RowTable rt1 = pair ? row_table(sc, span_base(a.bases, a.pac, tk.t_off, i + 1, tlen, tk.flags, true)) : rt0;
        const int hBeg0 = beg0 == 0 ? 0 - (oeDel + eDel * i) : kNeg;
        const int hBeg1 = beg1 == 0 ? 0 - (oeDel + eDel * (i + 1)) : kNeg;
        cells += (unsigned long long)(end0 - beg0) + (unsigned long long)(end1 - beg1);
        uint32_t *z0w = zp.z + (size_t)i * rstride, *z1w = z0w + rstride;
        ZRow z0{z0w, ns}, z1{z1w, ns};
        // Lane 0 state: H of row i at column beg0-1 is hBeg0 (the reference's h[beg0]); F starts at -inf.
        NwLane2 st{(uint32_t)hBeg0 & 0xFFFFu, (uint32_t)hBeg0 & 0xFFFFu, 0u, (uint32_t)(uint16_t)kNeg,
                   he[beg0 * T], 0u};
        uint32_t code0, code1;
        if (!pair) {                                   // the last row alone: it stores its own words
            for (int c = beg0; c < end0; ++c) {
                const uint32_t wd = he[(c + 1) * T];
                const uint32_t sel = nw_sel(qs[c * T]);
                const uint32_t DG = __byte_perm(st.wdp, st.hp2, 0x5410);
                const uint32_t UH = __byte_perm(wd, st.h, 0x5410);
                const uint32_t UE = __byte_perm(wd, st.e, 0x5432);
                st.hp2 = st.h;
                nw_pair_step(k, DG, UH, UE, prmt(rt0.lo, rt0.hi, sel), st.h, st.e, st.f, code0, code1);
                he[(c + 1) * T] = __byte_perm(st.h, st.e, 0x5410);
                z0.put(c, code0, end0 - 1);
                st.wdp = wd;
            }
            continue;
        }
        // Row i alone up to column beg1 (lane 1 starts at column beg1, step beg1 + 1).
        int c = beg0;
        const int aEnd = imin(beg1, end0 - 1);
        for (; c <= aEnd; ++c) {
            nw_both(k, rt0, rt1, he, qs, T, c, st, code0, code1);
            z0.put(c, code0, end0 - 1);
        }
        // Lane 1: H at beg1-1 is hBeg1, F is -inf; the reference's h[beg1] = hBeg1.
        st.h = (st.h & 0xFFFFu) | ((uint32_t)hBeg1 << 16);
        st.f = (st.f & 0xFFFFu) | negHi;
        reinterpret_cast<int16_t *>(he + beg1 * T)[0] = (int16_t)hBeg1;
        // Both rows, columns c .. end0-1 (row i+1 at c-1): first up to a multiple of 8.
        for (; c < end0 && (c & 7); ++c) {
            nw_both(k, rt0, rt1, he, qs, T, c, st, code0, code1);
            z0.put(c, code0, end0 - 1);
            z1.put(c - 1, code1, end1 - 1);
        }
        // Blocks of 8 aligned columns: row i fills word c/8 (nibbles 0..7), row i+1
        // completes word c/8 - 1 (nibble 7, column c-1) then fills nibbles 0..6 of word c/8.
        for (; c + 8 <= end0; c += 8) {
            uint32_t w0 = 0, w1;
            nw_both(k, rt0, rt1, he, qs, T, c, st, code0, code1);
            w0 |= code0;
            z1w[(size_t)((c >> 3) - 1) * ns] = z1.acc | (code1 << 28);
            w1 = 0;
#pragma unroll
            for (int s2 = 1; s2 < 8; ++s2) {
                nw_both(k, rt0, rt1, he, qs, T, c + s2, st, code0, code1);
                w0 |= code0 << (4 * s2);
                w1 |= code1 << (4 * (s2 - 1));
            }
            z0w[(size_t)(c >> 3) * ns] = w0;
            z1.acc = w1;
        }
        for (; c < end0; ++c) {
            nw_both(k, rt0, rt1, he, qs, T, c, st, code0, code1);
            z0.put(c, code0, end0 - 1);
            z1.put(c - 1, code1, end1 - 1);
        }
        // Row i+1 alone for its columns past row i's band (c = end0 .. end1).
        // Row i's H at end0-1 (or hBeg0) is its diagonal at column end0.
        const uint32_t hLast0 = st.h & 0xFFFFu, eLast0 = st.e & 0xFFFFu, hLast0p = st.hp2 & 0xFFFFu;
        for (c = imax(end0, beg1 + 1); c <= end1; ++c) {
            const uint32_t sel = nw_sel(qs[(c - 1) * T]);
            uint32_t DG, UH, UE;
            if (c - 1 < end0) {             // column end0-1: row i's values from registers
                DG = hLast0p << 16;
                UH = hLast0 << 16;
                UE = eLast0 << 16;
            } else {                        // column end0: diagonal H(i, end0-1), stale word above
                const uint32_t wd = he[c * T];
                DG = hLast0 << 16;
                UH = wd << 16;
                UE = wd & 0xFFFF0000u;
            }
            nw_pair_step(k, DG, UH, UE, prmt(rt1.lo, rt1.hi, sel) * 65536u, st.h, st.e, st.f, code0, code1);
            he[c * T] = __byte_perm(st.h, st.e, 0x7632);
            z1.put(c - 1, code1, end1 - 1);
        }
    }
    const int thr = -(qlen + tlen + 2) * step_cost(sc) - 1;
    return RowI16{he, T}.final_score((int)(int16_t)(he[qlen * T] & 0xFFFFu), thr);     // :144
}

// Sort key: shared-memory tasks first, then by query length, target length
// and band, so the threads of a warp align tasks of the same shape.
// Sort key: the shared-memory kernels' int16-row alignments first, then
// their int32-row ones, then the long queries; within a class the largest
// shapes first (they are claimed first and overlap the rest), and equal
// shapes together so a warp's 32 alignments walk similar matrices.
__global__ void global_keys_kernel(const swb_global_task *__restrict__ tasks, size_t n, DevScoring sc,
                                   uint32_t *__restrict__ keys, uint32_t *__restrict__ idx) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const swb_global_task t = tasks[i];
    const uint32_t big = t.qlen > kGlbSmemMaxQ ? 1u : 0u;
    const uint32_t wide = !big && !fits_i16(sc, t.qlen, t.tlen) ? 1u : 0u;
    keys[i] = (big << 31) | (wide << 30) | ((2047u - (uint32_t)min(max(t.qlen, 0), 2047)) << 19) |
              ((4095u - (uint32_t)min(max(t.tlen, 0), 4095)) << 7) | (127u - (uint32_t)min(max(t.w, 0), 127));
    idx[i] = (uint32_t)i;
}

// Sorted tasks order[begin, begin + count) of one row width (all with
// qlen <= qcap).  Each warp claims the next 32 from `claim`, so warps that
// draw large matrices never hold the launch up.
template <bool I16>
__global__ void __launch_bounds__(256) global_smem_kernel(GlobalArgs a, const uint32_t *__restrict__ order,
                                                          size_t begin, uint32_t count, uint32_t *claim,
                                                          uint32_t *z, size_t nslots, int qcap) {
    extern __shared__ int2 smem[];
    const int T = blockDim.x;
    const size_t row_bytes = (size_t)(qcap + 1) * T * (I16 ? 4 : 8);
    using Row = typename std::conditional<I16, RowI16, RowI32>::type;
    Row row;
    row.T = T;
    if constexpr (I16) row.he = reinterpret_cast<uint32_t *>(smem) + threadIdx.x;
    else row.he = smem + threadIdx.x;
    uint8_t *qs = reinterpret_cast<uint8_t *>(smem) + row_bytes + threadIdx.x;
    const size_t slot = blockIdx.x * (size_t)T + threadIdx.x;
    const int lane = threadIdx.x & 31;
    unsigned long long cells = 0;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(claim, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= count) break;
        if (base + (uint32_t)lane >= count) continue;
        const size_t k = order[begin + base + lane];
        const swb_global_task tk = a.tasks[k];
        if (tk.qlen > qcap) continue;                                    // (never: sorted by class)
        swb_global_result r{0, 0, tk.w, 1, a.cigar_off[k]};
        const int qlen = tk.qlen, tlen = tk.tlen;
        if (qlen > 0 && tlen > 0) {                                      // :29-31
            for (int j = 0; j < qlen; ++j) qs[j * T] = (uint8_t)span_base(a.bases, a.pac, tk.q_off, j, qlen, tk.flags, false);
            int w0 = tk.w;
            int w = imax(w0, abs(qlen - tlen));                          // :47
            int nCol = (int)min((long long)qlen, 2ll * w + 1);           // :48
            // int16 rows: backpointers by absolute column, qlen/8 words per row.
            ZPacked zp{z + slot, nslots, I16 ? (qlen + 7) >> 3 : (nCol + 7) >> 3, w, I16};
            auto dp = [&]() -> int {
                if constexpr (I16) return global_dp_pair16(a.sc, row.he, qs, T, a, tk, w, zp, cells);
                else return global_dp_smem(a.sc, row, qs, T, a, tk, w, zp, cells);
            };
            int score = dp();
            if (tk.flags & SWB_GLB_RETRY) {                              // CIGARGenerator.swift:88-96
                int retries = 0;
                while (score < tk.true_score && retries < 3) {
                    if (nw_skip_covered_retries(qlen, tlen, w, retries, w0, r, cells)) break;
                    w0 *= 2;
                    ++retries;
                    r.attempts++;
                    w = imax(w0, abs(qlen - tlen));
                    nCol = (int)min((long long)qlen, 2ll * w + 1);
                    if (!I16) zp.ncw = (nCol + 7) >> 3;
                    zp.w = w;
                    score = dp();
                }
            }
            r.score = score;
            r.w_used = w0;
            r.n_cigar = global_traceback(zp, qlen, tlen, w, nCol, a.cigar + r.cigar_off);
        }
        a.res[k] = r;
    }
    for (int o = 16; o > 0; o >>= 1) cells += __shfl_down_sync(0xFFFFFFFFu, cells, o);
    if ((threadIdx.x & 31) == 0 && cells) atomicAdd(a.cells, cells);
}

__global__ void cigar_offsets_kernel(const swb_global_task *__restrict__ tasks, size_t n,
                                     unsigned long long *__restrict__ lens) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) lens[i] = (unsigned long long)max(tasks[i].qlen, 0) + (unsigned long long)max(tasks[i].tlen, 0);
}

}  // namespace
}  // namespace swb

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace swb {

int launch_global(swb_ctx *ctx, const DevScoring &sc, const uint8_t *d_bases,
                  const swb_global_task *d_tasks, size_t n, swb_global_result *d_res,
                  uint32_t *d_cigar, unsigned long long *d_cells, cudaStream_t st, const GlobalShape &shape) {
    if (n == 0) return SWB_OK;
    int rc;
    // Per-task CIGAR windows: exclusive prefix sum of (qlen + tlen).
    if ((rc = ensure_dev(ctx, ctx->d_keys, n * 8)) || (rc = ensure_dev(ctx, ctx->d_keys2, n * 8))) return rc;
    unsigned long long *lens = (unsigned long long *)ctx->d_keys.p, *offs = (unsigned long long *)ctx->d_keys2.p;
    cigar_offsets_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_tasks, n, lens);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    size_t tmp = 0;
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, lens, offs, (int)n, st));
    if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp))) return rc;
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(ctx->d_sort_tmp.p, tmp, lens, offs, (int)n, st));
    // Shape order (the scan is done with `lens`, so its buffer holds the keys).
    if ((rc = ensure_dev(ctx, ctx->d_idx, n * 4)) || (rc = ensure_dev(ctx, ctx->d_idx2, n * 4))) return rc;
    uint32_t *skeys = (uint32_t *)ctx->d_keys.p, *skeys2 = skeys + n;
    uint32_t *sidx = (uint32_t *)ctx->d_idx.p, *order = (uint32_t *)ctx->d_idx2.p;
    global_keys_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_tasks, n, sc, skeys, sidx);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    SWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, skeys, skeys2, sidx, order, (int)n, 0, 32, st));
    if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp))) return rc;
    SWB_CUDA(cub::DeviceRadixSort::SortPairs(ctx->d_sort_tmp.p, tmp, skeys, skeys2, sidx, order, (int)n, 0, 32, st));
    GlobalArgs a{sc, d_bases, ctx->d_pac, d_tasks, d_res, d_cigar, offs, d_cells + kCntGlobal, n, kGlbSmemMaxQ};
    const size_t avail0 = ctx->budget > ctx->allocated ? (ctx->budget - ctx->allocated) / 2 : 0;

    // Shared-memory kernels (int16 rows where exact, int32 rows otherwise):
    // block size and blocks per SM that keep the most threads resident.
    struct SmemCfg {
        int T = 0, grid = 0;
        size_t smem = 0, nslots = 0;
    } cfg[2];   // [0] int32 rows, [1] int16 rows
    size_t z_bytes = 0;
    int qcap = 0;
    const size_t n_small_of[2] = {shape.n_small - shape.n_small16, shape.n_small16};
    if (shape.n_small > 0) {
        qcap = imax(shape.small_q, 1);
        int sm_bytes = 0, blk_bytes = 0;
        SWB_CUDA(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
        SWB_CUDA(cudaDeviceGetAttribute(&blk_bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
        const size_t per_slot = (size_t)imax(shape.small_t, 1) * (size_t)((qcap + 7) >> 3) * 4;
        size_t max_slots = 0;
        for (int v = 0; v < 2; ++v) {
            if (n_small_of[v] == 0) continue;
            const size_t per_thread = (size_t)(qcap + 1) * (v ? 4 : 8) + (size_t)((qcap + 7) & ~7);
            int best = 0, T = 0;
            for (int t = 32; t <= 256; t += 32) {
                const size_t b = (size_t)t * per_thread;
                if (b > (size_t)blk_bytes) break;
                const int blocks = imin((int)((size_t)sm_bytes / (b + 1024)), 2048 / t);
                if (blocks * t > best) {
                    best = blocks * t;
                    T = t;
                }
            }
            if (T == 0) return set_error(SWB_ERR_TOO_LARGE, "global alignment rows do not fit shared memory");
            SmemCfg &c = cfg[v];
            c.T = T;
            c.smem = (size_t)T * per_thread;
            c.grid = (int)std::min<size_t>((size_t)ctx->sm_count * (best / T), (n_small_of[v] + T - 1) / T);
            while (c.grid > 1 && (size_t)c.grid * T * per_slot > avail0) c.grid /= 2;
            c.nslots = (size_t)c.grid * T;
            max_slots = std::max(max_slots, c.nslots);
            if (v) SWB_CUDA(cudaFuncSetAttribute(global_smem_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem));
            else SWB_CUDA(cudaFuncSetAttribute(global_smem_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem));
        }
        z_bytes = (max_slots * per_slot + 1023) & ~(size_t)1023;
        if (z_bytes > avail0) return set_error(SWB_ERR_OOM, "global alignment scratch does not fit the memory budget");
    }
    // Global-scratch kernel for longer queries.
    Scratch s{};
    size_t big_bytes = 0, grid_b = 0;
    if (shape.n_big > 0) {
        const int qmax = imax(shape.big_q, 1), tmax = imax(shape.big_t, 1);
        const size_t per_slot = (size_t)(qmax + 1) * 8 + (size_t)qmax + (size_t)tmax + (size_t)tmax * qmax;
        size_t nslots = std::min((size_t)ctx->sm_count * 8 * kGT, ((shape.n_big + kGT - 1) / kGT) * kGT);
        const size_t avail = avail0 > z_bytes ? avail0 - z_bytes : 0;
        while (nslots > kGT && nslots * per_slot > avail) nslots /= 2;
        nslots = (nslots / kGT) * kGT;
        if (nslots == 0 || nslots * per_slot > avail)
            return set_error(SWB_ERR_OOM, "global alignment scratch does not fit the memory budget");
        grid_b = nslots / kGT;
        big_bytes = nslots * per_slot + 1024;
        s.nslots = nslots;
        s.qmax = qmax;
        s.tmax = tmax;
    }
    if ((rc = ensure_dev(ctx, ctx->d_scratch, z_bytes + big_bytes + 256))) return rc;
    uint32_t *claim = (uint32_t *)((char *)ctx->d_scratch.p + z_bytes + big_bytes);   // one counter per row width
    SWB_CUDA(cudaMemsetAsync(claim, 0, 2 * sizeof(uint32_t), st));
    ProfScope ps(ctx, st, "global_nw_traceback", kCntGlobal);
    // The sorted order holds the int16-row alignments, then the int32-row ones.
    const size_t begin_of[2] = {shape.n_small16, 0};
    for (int v = 1; v >= 0; --v) {
        if (n_small_of[v] == 0) continue;
        const SmemCfg &c = cfg[v];
        if (v)
            global_smem_kernel<true><<<(unsigned)c.grid, c.T, c.smem, st>>>(
                a, order, begin_of[v], (uint32_t)n_small_of[v], claim + v, (uint32_t *)ctx->d_scratch.p, c.nslots, qcap);
        else
            global_smem_kernel<false><<<(unsigned)c.grid, c.T, c.smem, st>>>(
                a, order, begin_of[v], (uint32_t)n_small_of[v], claim + v, (uint32_t *)ctx->d_scratch.p, c.nslots, qcap);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    if (shape.n_big > 0) {
        // The big kernel visits every task and skips those of the shared-memory kernel.
        char *p = (char *)ctx->d_scratch.p + z_bytes;
        s.slot = 0;
        s.h = (int *)p;
        p += (size_t)(s.qmax + 1) * s.nslots * 4;
        s.e = (int *)p;
        p += (size_t)(s.qmax + 1) * s.nslots * 4;
        s.q = (uint8_t *)p;
        p += (size_t)s.qmax * s.nslots;
        s.t = (uint8_t *)p;
        p += (size_t)s.tmax * s.nslots;
        s.z = (uint8_t *)p;
        a.qsplit = shape.n_small > 0 ? qcap : 0;
        global_kernel<<<(unsigned)grid_b, kGT, 0, st>>>(a, s);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    return SWB_OK;
}

}  // namespace swb
