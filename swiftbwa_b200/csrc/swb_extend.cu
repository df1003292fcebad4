// swb_extend.cu -- ExtensionAligner.extend for many chains at once
// (Sources/Alignment/ExtensionAligner.swift:114-346).
//
// Within one chain the reference is sequential: seeds run in descending
// score order, a seed inside an earlier region of the chain is only
// counted (sub/subN), the left extension may be retried once with a doubled
// band, the right extension starts from the left score (h0), and may be
// retried too.  Across chains everything is independent.  So each chain is
// a small host state machine, and the GPU work is gathered in rounds: every
// round collects the one pending extension of every active chain into a
// single batch (one sort + binned pass over the device-resident reads),
// then feeds each result back to its chain, which either emits its next
// extension (retry, right side, next seed) or finishes.
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "swb_internal.h"

namespace swb {
int ext_big_max_q(const swb_ext_task *tasks, size_t n, int max_mat);
}

using namespace swb;

namespace {

// calMaxGap (ExtensionAligner.swift:352-363)
long cal_max_gap(long qlen, const swb_scoring &sc) {
    const long a = sc.a, oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const long lDel = eDel > 0 ? (qlen * a - oDel) / eDel + 1 : 1;
    const long lIns = eIns > 0 ? (qlen * a - oIns) / eIns + 1 : 1;
    long l = std::max(std::max(lDel, lIns), 1L);
    return std::min(l, (long)sc.band_width << 1);
}

// FMIndex.getReference(at:length:) as a span of the resident forward strand
// (FMIndex.swift:147-170): forward positions read directly, reverse-strand
// positions as the reverse complement of the mirrored forward window.
struct RefSpan {
    uint64_t off = 0;
    int32_t len = 0;
    bool rc = false;   // reverse-complemented
};

RefSpan get_reference(int64_t pos, long length, int64_t gl) {
    RefSpan r;
    if (pos >= gl) {
        const int64_t fwdEnd = 2 * gl - pos, fwdStart = fwdEnd - length;
        const int64_t s = std::max<int64_t>(0, fwdStart), e = std::min(fwdEnd, gl);
        if (e - s > 0) {
            r.off = (uint64_t)s;
            r.len = (int32_t)(e - s);
            r.rc = true;
        }
    } else {
        const int64_t n = std::min<int64_t>(length, gl - pos);
        if (n > 0 && pos >= 0) {
            r.off = (uint64_t)pos;
            r.len = (int32_t)n;
        }
    }
    return r;
}

enum Phase { kSeed, kLeft, kRight, kDone };

struct Chain {
    const swb_chain *ch = nullptr;
    const swb_seed *seeds = nullptr;   // this chain's seeds
    std::vector<uint32_t> order;
    int64_t rmax0 = 0, rmax1 = 0;
    int32_t tmp = 0;
    size_t k = 0;
    Phase phase = kSeed;
    // current seed
    int32_t qbeg = 0, len = 0, score = 0, qend = 0;
    int64_t rbeg = 0, rend = 0;
    swb_region reg{};
    int32_t accH0 = 0, w = 0, prev = 0, tryIdx = 0;
    int32_t lScore = 0, lQ = 0, lT = 0, rScore = 0, rQ = 0, rT = 0;
    swb_ext_task task{};
    std::vector<swb_region> regions;
};

struct Driver {
    const swb_scoring &sc;
    int64_t gl;
    std::vector<Chain> &chains;

    // Left extension task of the current seed, or none (:206-216).
    bool left_task(Chain &c) {
        if (c.qbeg <= 0) return false;
        const long tl = std::min<int64_t>(c.rbeg - c.rmax0, 10000);
        if (tl <= 0) return false;
        const RefSpan t = get_reference(c.rbeg - tl, tl, gl);
        // The fetched window is reversed (:219-224): a forward window reads
        // backwards, a reverse-complement window becomes the plain complement.
        const uint32_t tf = SWB_T_FROM_REF | (t.rc ? SWB_T_COMPLEMENT : SWB_T_REVERSE);
        c.w = sc.band_width;
        c.prev = c.score;
        c.tryIdx = 0;
        c.task = swb_ext_task{c.ch->read_off, t.off, c.qbeg, t.len, c.w, c.score, sc.pen_clip5, SWB_Q_REVERSE | tf};
        c.phase = kLeft;
        return true;
    }

    // Right extension task (:269-279).
    bool right_task(Chain &c) {
        if (c.qend >= c.ch->read_len) return false;
        const long tl = std::min<int64_t>(c.rmax1 - c.rend, 10000);
        if (tl <= 0) return false;
        const RefSpan t = get_reference(c.rend, tl, gl);
        const uint32_t tf = SWB_T_FROM_REF | (t.rc ? (SWB_T_REVERSE | SWB_T_COMPLEMENT) : 0u);
        c.w = sc.band_width;
        c.prev = c.accH0;
        c.tryIdx = 0;
        c.task = swb_ext_task{c.ch->read_off + (uint64_t)c.qend, t.off, c.ch->read_len - c.qend, t.len, c.w, c.accH0,
                              sc.pen_clip3, tf};
        c.phase = kRight;
        return true;
    }

    // Region assembly (:318-335).
    void finish_seed(Chain &c) {
        c.reg.qb = c.qbeg - c.lQ;
        c.reg.qe = c.qend + c.rQ;
        c.reg.rb = c.rbeg - c.lT;
        c.reg.re = c.rend + c.rT;
        int32_t trueScore = c.len * sc.a;
        if (c.lScore > 0) trueScore = c.lScore;
        if (c.rScore > 0) trueScore += c.rScore - c.accH0;
        c.reg.score = trueScore;
        c.reg.true_score = trueScore;
        int32_t cov = 0;                                            // computeSeedCov (:36-70)
        for (uint32_t i = 0; i < c.ch->n_seeds; ++i) {
            const swb_seed &s = c.seeds[i];
            if (s.qbeg >= c.reg.qb && s.qbeg + s.len <= c.reg.qe && s.rbeg >= c.reg.rb && s.rbeg + s.len <= c.reg.re)
                cov += s.len;
        }
        c.reg.seed_cov = cov;
        c.regions.push_back(c.reg);
        ++c.k;
        c.phase = kSeed;
    }

    // Advances a chain on the host until it needs a GPU extension or is done.
    void advance(Chain &c) {
        while (c.phase == kSeed) {
            if (c.k == c.order.size()) {                            // :338-343
                const int32_t thr = sc.min_seed_len * sc.a;
                for (auto &r : c.regions)
                    if (r.sub > 0 && r.sub < thr) r.sub = 0;
                c.phase = kDone;
                return;
            }
            const swb_seed &s = c.seeds[c.order[c.k]];
            c.qbeg = s.qbeg;
            c.len = s.len;
            c.score = s.score;
            c.rbeg = s.rbeg;
            c.qend = s.qbeg + s.len;
            c.rend = s.rbeg + s.len;
            int cover = -1;                                          // :172-189
            for (size_t i = 0; i < c.regions.size(); ++i)
                if (c.qbeg >= c.regions[i].qb && c.qend <= c.regions[i].qe) {
                    cover = (int)i;
                    break;
                }
            if (cover >= 0) {
                swb_region &r = c.regions[(size_t)cover];
                const int32_t aln = c.len * sc.a;
                if (aln > r.sub) r.sub = aln;
                if (aln >= r.score - c.tmp) r.sub_n += 1;
                ++c.k;
                continue;
            }
            c.reg = swb_region{};                                    // :191-199
            c.reg.w = sc.band_width;
            c.reg.rid = c.ch->rid;
            c.reg.seed_cov = c.len;
            c.reg.seed_len0 = c.len;
            c.accH0 = c.score;
            c.lScore = c.lQ = c.lT = c.rScore = c.rQ = c.rT = 0;
            if (left_task(c)) return;
            if (right_task(c)) return;
            finish_seed(c);
        }
    }

    // Feeds one extension result back (:233-260 and :288-314).
    void feed(Chain &c, const swb_ext_result &r) {
        const bool stop = r.score == c.prev || r.max_off < (c.w >> 1) + (c.w >> 2) || c.tryIdx == 1;
        if (!stop) {
            c.prev = r.score;
            c.w <<= 1;
            c.tryIdx = 1;
            c.task.w = c.w;
            return;                                                  // same task, doubled band
        }
        if (c.phase == kLeft) {
            c.accH0 = r.score;
            c.reg.w = std::max(c.reg.w, c.w);
            if (r.gscore <= 0 || r.gscore <= r.score - sc.pen_clip5) {
                c.lQ = r.qle;
                c.lT = r.tle;
                c.lScore = r.score;
            } else {
                c.lQ = c.qbeg;
                c.lT = r.gtle;
                c.lScore = r.gscore;
            }
            c.phase = kSeed;
            if (right_task(c)) return;
            finish_seed(c);
        } else {
            c.reg.w = std::max(c.reg.w, c.w);
            if (r.gscore <= 0 || r.gscore <= r.score - sc.pen_clip3) {
                c.rQ = r.qle;
                c.rT = r.tle;
                c.rScore = r.score;
            } else {
                c.rQ = c.ch->read_len - c.qend;
                c.rT = r.gtle;
                c.rScore = r.gscore;
            }
            finish_seed(c);
        }
        advance(c);
    }
};

}  // namespace

extern "C" int swb_extend_chains(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                                 const swb_seed *seeds, size_t n_seeds, const swb_chain *chains, size_t n_chains,
                                 uint64_t genome_len, swb_region *out, uint32_t *n_regions, uint32_t *rounds) {
    if (!ctx || !sc || (!bases && n_bases) || (!seeds && n_seeds) || (!chains && n_chains) ||
        (!out && n_seeds) || (!n_regions && n_chains))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    if (sc->e_ins <= 0 || sc->e_del <= 0 || sc->a < 0 || sc->b < 0 || sc->a > 127 || sc->b > 128)
        return set_error(SWB_ERR_INVALID_ARG, "scoring out of range");
    if (rounds) *rounds = 0;
    if (n_chains == 0) return SWB_OK;
    if (!ctx->d_pac || genome_len > ctx->ref_bases)
        return set_error(SWB_ERR_NO_REFERENCE, "the forward strand (genome_len bases) must be uploaded first");
    // Chain set-up (:126-158).
    std::vector<Chain> cs(n_chains);
    for (size_t i = 0; i < n_chains; ++i) {
        const swb_chain &ch = chains[i];
        if ((uint64_t)ch.seed_off + ch.n_seeds > n_seeds || ch.read_len < 0 || ch.read_len > kMaxLen ||
            ch.read_off + (uint64_t)ch.read_len > n_bases)
            return set_error(SWB_ERR_INVALID_ARG, "chain " + std::to_string(i) + ": seeds or read outside the inputs");
        Chain &c = cs[i];
        c.ch = &ch;
        c.seeds = seeds + ch.seed_off;
        for (uint32_t k = 0; k < ch.n_seeds; ++k) {
            const swb_seed &s = c.seeds[k];
            if (s.qbeg < 0 || s.len < 0 || s.qbeg + s.len > ch.read_len || s.rbeg < 0 || s.rbeg + s.len > 2 * (int64_t)genome_len)
                return set_error(SWB_ERR_INVALID_ARG, "chain " + std::to_string(i) + ": seed " + std::to_string(k) + " out of range");
        }
        c.rmax0 = INT64_MAX;
        c.rmax1 = 0;
        const long lq = ch.read_len;
        for (uint32_t k = 0; k < ch.n_seeds; ++k) {
            const swb_seed &t = c.seeds[k];
            const int64_t b = t.rbeg - (int64_t)((long)t.qbeg + cal_max_gap(t.qbeg, *sc));
            const long remaining = lq - t.qbeg - t.len;
            const int64_t e = t.rbeg + t.len + (int64_t)(remaining + cal_max_gap(remaining, *sc));
            c.rmax0 = std::min(c.rmax0, b);
            c.rmax1 = std::max(c.rmax1, e);
        }
        if (c.rmax0 < 0) c.rmax0 = 0;
        c.tmp = std::max(sc->a + sc->b, std::max(sc->o_ins + sc->e_ins, sc->o_del + sc->e_del));
        c.order.resize(ch.n_seeds);
        for (uint32_t k = 0; k < ch.n_seeds; ++k) c.order[k] = k;
        std::stable_sort(c.order.begin(), c.order.end(),
                         [&](uint32_t x, uint32_t y) { return c.seeds[x].score > c.seeds[y].score; });
    }
    Driver drv{*sc, (int64_t)genome_len, cs};
    for (Chain &c : cs) drv.advance(c);

    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    const DevScoring dsc = make_dev_scoring(*sc);
    const size_t bases_bytes = (std::max<size_t>(n_bases, 1) + 255) & ~(size_t)255;
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_bases, bases_bytes))) return rc;
    SWB_CUDA(cudaMemcpyAsync(ctx->d_bases.p, bases, std::max<size_t>(n_bases, 1), cudaMemcpyHostToDevice, ctx->stream));
    SWB_CUDA(cudaMemsetAsync(ctx->d_counters, 0, sizeof(unsigned long long) * kNumCounters, ctx->stream));
    std::vector<swb_ext_task> batch;
    std::vector<size_t> owner;
    std::vector<swb_ext_result> res;
    uint32_t nround = 0;
    for (;;) {
        batch.clear();
        owner.clear();
        for (size_t i = 0; i < cs.size(); ++i)
            if (cs[i].phase == kLeft || cs[i].phase == kRight) {
                batch.push_back(cs[i].task);
                owner.push_back(i);
            }
        if (batch.empty()) break;
        const size_t n = batch.size();
        res.resize(n);
        if ((rc = ensure_dev(ctx, ctx->d_tasks, n * sizeof(swb_ext_task))) ||
            (rc = ensure_dev(ctx, ctx->d_out, n * sizeof(swb_ext_result))))
            return rc;
        SWB_CUDA(cudaMemcpyAsync(ctx->d_tasks.p, batch.data(), n * sizeof(swb_ext_task), cudaMemcpyHostToDevice, ctx->stream));
        if ((rc = launch_ext(ctx, dsc, (const uint8_t *)ctx->d_bases.p, (const swb_ext_task *)ctx->d_tasks.p, n,
                             (swb_ext_result *)ctx->d_out.p, ctx->d_counters, ctx->stream,
                             ext_big_max_q(batch.data(), n, dsc.max_mat))))
            return rc;
        SWB_CUDA(cudaMemcpyAsync(res.data(), ctx->d_out.p, n * sizeof(swb_ext_result), cudaMemcpyDeviceToHost, ctx->stream));
        SWB_CUDA(cudaStreamSynchronize(ctx->stream));
        ++nround;
        for (size_t k = 0; k < n; ++k) drv.feed(cs[owner[k]], res[k]);
    }
    unsigned long long c[kNumCounters] = {0};
    if (cudaMemcpy(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) {
        unsigned long long sum = 0;
        for (int k = 0; k < kNumCounters; ++k) sum += c[k];
        ctx->last_cells = sum;
    }
    for (size_t i = 0; i < cs.size(); ++i) {
        n_regions[i] = (uint32_t)cs[i].regions.size();
        std::copy(cs[i].regions.begin(), cs[i].regions.end(), out + chains[i].seed_off);
    }
    if (rounds) *rounds = nround;
    return SWB_OK;
}
