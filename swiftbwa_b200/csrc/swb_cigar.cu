// swb_cigar.cu -- CIGARGenerator.generate for a batch
// (Sources/Alignment/CIGARGenerator.swift:30-111): the band inference and the
// pure-M fast path on the host, the banded global alignments with their
// band-doubling retries on the device (kernel 2), then the reference's
// post-processing -- deletion squeeze, NM, MD and soft clips -- on host
// threads, exactly as the reference's own GPU path post-processes on the CPU
// (CIGARGenerator.postProcess, :118-142).
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "swb_internal.h"

namespace swb {
namespace {

enum : uint32_t { kOpM = 0, kOpI = 1, kOpD = 2, kOpS = 4 };

inline uint8_t pac_base(const uint8_t *pac, uint64_t p) { return (uint8_t)((pac[p >> 2] >> ((3u - (p & 3)) << 1)) & 3u); }

// A task span materialised on the host (same flags semantics as the kernels).
void load_span(const uint8_t *bases, const uint8_t *pac, uint64_t off, int len, uint32_t flags, bool target,
               std::vector<uint8_t> &dst) {
    dst.resize((size_t)std::max(len, 0));
    const bool rev = target ? (flags & SWB_T_REVERSE) : (flags & SWB_Q_REVERSE);
    const bool comp = target && (flags & SWB_T_COMPLEMENT);
    const bool ref = target && (flags & SWB_T_FROM_REF);
    for (int k = 0; k < len; ++k) {
        const uint64_t i = off + (uint64_t)(rev ? len - 1 - k : k);
        uint8_t b = ref ? pac_base(pac, i) : bases[i];
        if (comp && b < 4) b = (uint8_t)(3 - b);
        dst[(size_t)k] = b;
    }
}

// inferBandWidth (:147-170)
int32_t infer_band_width(int32_t qlen, int32_t rlen, int32_t score, const swb_scoring &sc) {
    const int32_t maxLen = std::max(qlen, rlen), minLen = std::min(qlen, rlen);
    const int32_t diff = maxLen - minLen;
    const int32_t expected = minLen * sc.a;
    if (score >= expected) return diff + 3;
    const int32_t deficit = expected - score;
    const int32_t est = deficit / std::min(sc.o_ins + sc.e_ins, sc.a + sc.b);
    return std::max(diff + 3, est);
}

const char kBaseChar[5] = {'A', 'C', 'G', 'T', 'N'};

// Squeeze, NM, MD and soft clips of one alignment (:98-108, :118-142).
void post_process(std::vector<uint32_t> cigar, const std::vector<uint8_t> &q, const std::vector<uint8_t> &r,
                  const swb_cigar_task &t, int32_t score, bool squeeze, swb_cigar_result &res, uint32_t *cig_out,
                  char *md_out) {
    int64_t pos_adj = 0;
    size_t ref_off = 0;
    if (squeeze) {                                               // squeezeDeletions (:272-295)
        size_t lead = 0;
        while (lead < cigar.size() && (cigar[lead] & 0xF) == kOpD) {
            pos_adj += cigar[lead] >> 4;
            ref_off += cigar[lead] >> 4;
            ++lead;
        }
        cigar.erase(cigar.begin(), cigar.begin() + (long)lead);
        while (!cigar.empty() && (cigar.back() & 0xF) == kOpD) cigar.pop_back();
    }
    // NM (:173-210) and MD (:219-268) in one walk.
    const size_t qn = q.size(), rn = r.size();
    size_t qi = 0, ti = ref_off;
    int32_t nm = 0;
    long match = 0;
    std::string md;
    for (uint32_t c : cigar) {
        const uint32_t op = c & 0xF;
        const size_t len = c >> 4;
        if (op == kOpM) {
            for (size_t x = 0; x < len; ++x)
                if (qi < qn && ti < rn) {
                    if (q[qi] == r[ti]) {
                        ++match;
                    } else {
                        ++nm;
                        md += std::to_string(match);
                        md += kBaseChar[std::min<int>(r[ti], 4)];
                        match = 0;
                    }
                    ++qi;
                    ++ti;
                }
        } else if (op == kOpI) {
            nm += (int32_t)len;
            qi += len;
        } else if (op == kOpD) {
            nm += (int32_t)len;
            md += std::to_string(match);
            md += '^';
            for (size_t x = 0; x < len; ++x)
                if (ti < rn) md += kBaseChar[std::min<int>(r[ti++], 4)];
            match = 0;
        }
    }
    md += std::to_string(match);
    // addSoftClips (:298-320)
    std::vector<uint32_t> out;
    out.reserve(cigar.size() + 2);
    long front = 0, back = 0;
    if (t.is_reverse) {
        front = (long)t.read_len - t.qe;
        back = t.qb;
    } else {
        front = t.qb;
        back = (long)t.read_len - t.qe;
    }
    if (front > 0) out.push_back(((uint32_t)front << 4) | kOpS);
    out.insert(out.end(), cigar.begin(), cigar.end());
    if (back > 0) out.push_back(((uint32_t)back << 4) | kOpS);
    std::copy(out.begin(), out.end(), cig_out);
    std::memcpy(md_out, md.c_str(), md.size() + 1);
    res.score = score;
    res.nm = nm;
    res.n_cigar = (int32_t)out.size();
    res.md_len = (int32_t)md.size();
    res.pos = t.ref_pos + pos_adj;
}

template <class F>
void parallel(size_t n, F fn) {
    const size_t nth = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), (n + 4095) / 4096);
    if (nth <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (n + nth - 1) / nth;
    for (size_t k = 0; k < nth; ++k) th.emplace_back([&, k] { fn(k * per, std::min(n, (k + 1) * per)); });
    for (auto &x : th) x.join();
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" int swb_cigar_batch(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                               const swb_cigar_task *tasks, size_t n_tasks, swb_cigar_result *results,
                               uint32_t *cigar_out, size_t cigar_cap, char *md_out, size_t md_cap) {
    if (!ctx || !sc || (!tasks && n_tasks) || (!results && n_tasks) || (!bases && n_bases) ||
        (!cigar_out && n_tasks) || (!md_out && n_tasks))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    if (n_tasks == 0) return SWB_OK;
    // Offsets, validation and the fast-path decision (:44-80).
    std::vector<uint64_t> coff(n_tasks + 1, 0), moff(n_tasks + 1, 0);
    for (size_t i = 0; i < n_tasks; ++i) {
        const swb_cigar_task &t = tasks[i];
        if (t.qlen < 0 || t.rlen < 0) return set_error(SWB_ERR_INVALID_ARG, "task " + std::to_string(i) + ": negative length");
        if (t.qlen > kMaxLen || t.rlen > kMaxLen) return set_error(SWB_ERR_TOO_LARGE, "task " + std::to_string(i) + ": length above 65535");
        if (t.qlen > 0 && t.q_off + (uint64_t)t.qlen > n_bases)
            return set_error(SWB_ERR_INVALID_ARG, "task " + std::to_string(i) + ": query span outside bases");
        if (t.rlen > 0) {
            if (t.flags & SWB_T_FROM_REF) {
                if (ctx->h_pac.empty()) return set_error(SWB_ERR_NO_REFERENCE, "task reads the reference but none is uploaded");
                if (t.t_off + (uint64_t)t.rlen > ctx->ref_bases)
                    return set_error(SWB_ERR_INVALID_ARG, "task " + std::to_string(i) + ": reference span outside reference");
            } else if (t.t_off + (uint64_t)t.rlen > n_bases) {
                return set_error(SWB_ERR_INVALID_ARG, "task " + std::to_string(i) + ": reference span outside bases");
            }
        }
        coff[i + 1] = coff[i] + (uint64_t)t.qlen + (uint64_t)t.rlen + 2;
        moff[i + 1] = moff[i] + 6ull * ((uint64_t)t.qlen + (uint64_t)t.rlen) + 8;
    }
    if (coff[n_tasks] > cigar_cap) return set_error(SWB_ERR_INVALID_ARG, "cigar_cap below sum of (qlen + rlen + 2)");
    if (moff[n_tasks] > md_cap) return set_error(SWB_ERR_INVALID_ARG, "md_cap below sum of (6*(qlen+rlen)+8)");
    const int32_t min_indel = sc->o_ins + sc->e_ins + sc->o_del + sc->e_del;
    std::vector<uint8_t> fast(n_tasks, 0);
    std::vector<swb_global_task> dp;
    std::vector<size_t> dp_of;
    for (size_t i = 0; i < n_tasks; ++i) {
        const swb_cigar_task &t = tasks[i];
        int32_t w = infer_band_width(t.qe - t.qb, t.rlen, t.true_score, *sc);
        w = std::max(w, t.initial_w);
        const int32_t deficit = t.qlen * sc->a - t.true_score;
        if (t.qlen == t.rlen && t.qlen > 0 && deficit < min_indel) {
            fast[i] = 1;
        } else {
            dp.push_back(swb_global_task{t.q_off, t.t_off, t.qlen, t.rlen, w, t.true_score,
                                         (t.flags & (SWB_Q_REVERSE | SWB_T_REVERSE | SWB_T_COMPLEMENT | SWB_T_FROM_REF)) |
                                             SWB_GLB_RETRY,
                                         0});
            dp_of.push_back(i);
        }
    }
    // Device DP for the rest (the ABI's global batch: DP, retries, traceback).
    std::vector<swb_global_result> dres(dp.size());
    std::vector<uint32_t> dcig;
    if (!dp.empty()) {
        size_t need = 0;
        for (const auto &g : dp) need += (size_t)g.qlen + (size_t)g.tlen;
        dcig.resize(std::max<size_t>(need, 1));
        const int rc = swb_global_batch(ctx, sc, bases, n_bases, dp.data(), dp.size(), dres.data(), dcig.data(), dcig.size());
        if (rc) return rc;
    }
    std::vector<int64_t> dp_index(n_tasks, -1);
    for (size_t k = 0; k < dp_of.size(); ++k) dp_index[dp_of[k]] = (int64_t)k;
    const uint8_t *hpac = ctx->h_pac.empty() ? nullptr : ctx->h_pac.data();
    parallel(n_tasks, [&](size_t lo, size_t hi) {
        std::vector<uint8_t> q, r;
        for (size_t i = lo; i < hi; ++i) {
            const swb_cigar_task &t = tasks[i];
            load_span(bases, hpac, t.q_off, t.qlen, t.flags, false, q);
            load_span(bases, hpac, t.t_off, t.rlen, t.flags, true, r);
            swb_cigar_result &res = results[i];
            res = swb_cigar_result{};
            res.cigar_off = coff[i];
            res.md_off = moff[i];
            if (fast[i]) {                                             // :69-80
                post_process({((uint32_t)t.qlen << 4) | kOpM}, q, r, t, t.true_score, false, res, cigar_out + coff[i],
                             md_out + moff[i]);
                res.used_dp = 0;
            } else {                                                   // :82-110
                const swb_global_result &g = dres[(size_t)dp_index[i]];
                std::vector<uint32_t> raw(dcig.begin() + (long)g.cigar_off, dcig.begin() + (long)(g.cigar_off + (uint64_t)g.n_cigar));
                post_process(std::move(raw), q, r, t, g.score, true, res, cigar_out + coff[i], md_out + moff[i]);
                res.used_dp = 1;
            }
        }
    });
    return SWB_OK;
}
