// swb_extend.cu -- ExtensionAligner.extend for many chains at once
// (Sources/Alignment/ExtensionAligner.swift:114-346).
//
// Within one chain the reference is sequential: seeds run in descending
// score order (stable), a seed inside an earlier region of the chain is only
// counted (sub/subN), the left extension may be retried once with a doubled
// band, the right extension starts from the left score (h0) and may be
// retried too.  Across chains everything is independent.  So every chain is
// a small state machine held in device memory (one thread per chain), and
// the extensions are gathered in rounds:
//
//   seed order     one segmented stable sort of all seeds by score
//   init           rmax0/rmax1 per chain, then advance to the first task
//   per round      compact the live chains, gather their pending task into a
//                  dense batch, run the binned extension pass (launch_ext),
//                  then feed each result back: the chain either emits its
//                  next task (retry, right side, next seed) or finishes.
//
// The host only reads one count per round.  Regions are written in place
// (chain c's at out[seed_off ...]) and copied back once at the end.
#include <algorithm>
#include <thread>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_segmented_sort.cuh>
#include <cub/device/device_select.cuh>

#include "swb_device.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

enum : int32_t { kSeed = 0, kLeft = 1, kRight = 2, kDone = 3 };

struct ChainState {
    int64_t rmax0, rmax1, rbeg, rend;
    swb_region reg;                       // region of the current seed
    int32_t k, phase, qbeg, len, score, qend, accH0, w, prev, try_idx;
    int32_t l_score, l_q, l_t, r_score, r_q, r_t, nreg, tmp;
};

struct ChainArgs {
    DevScoring sc;
    int64_t gl;
    const swb_chain *chains;
    const swb_seed *seeds;
    const uint32_t *order;   // per chain, its seeds' global indices in descending score order
    ChainState *state;
    swb_ext_task *task;      // pending task per chain
    swb_region *regions;     // chain c's at seed_off
    uint32_t n_chains;
};

// calMaxGap (ExtensionAligner.swift:352-363)
__device__ long cal_max_gap(long qlen, const DevScoring &sc) {
    const long a = sc.a, oDel = sc.o_del, eDel = sc.e_del, oIns = sc.o_ins, eIns = sc.e_ins;
    const long lDel = eDel > 0 ? (qlen * a - oDel) / eDel + 1 : 1;
    const long lIns = eIns > 0 ? (qlen * a - oIns) / eIns + 1 : 1;
    long l = lDel > lIns ? lDel : lIns;
    l = l > 1 ? l : 1;
    const long cap = (long)sc.band_width << 1;
    return l < cap ? l : cap;
}

// FMIndex.getReference(at:length:) as a span of the resident forward strand
// (FMIndex.swift:147-170): forward positions directly, reverse-strand
// positions as the reverse complement of the mirrored forward window.
struct RefSpan {
    uint64_t off;
    int32_t len;
    bool rc;
};

__device__ RefSpan get_reference(int64_t pos, int64_t length, int64_t gl) {
    RefSpan r{0, 0, false};
    if (pos >= gl) {
        const int64_t fwdEnd = 2 * gl - pos, fwdStart = fwdEnd - length;
        const int64_t s = fwdStart > 0 ? fwdStart : 0, e = fwdEnd < gl ? fwdEnd : gl;
        if (e - s > 0) r = RefSpan{(uint64_t)s, (int32_t)(e - s), true};
    } else {
        const int64_t n = length < gl - pos ? length : gl - pos;
        if (n > 0 && pos >= 0) r = RefSpan{(uint64_t)pos, (int32_t)n, false};
    }
    return r;
}

struct Chain {
    const ChainArgs &a;
    const swb_chain ch;
    ChainState &c;
    swb_ext_task &task;
    swb_region *regs;

    // Left extension of the current seed, if any (:202-216).  The fetched
    // window is used reversed (:219-224): a forward window reads backwards,
    // a reverse-complement window becomes the plain complement.
    __device__ bool left_task() {
        if (c.qbeg <= 0) return false;
        const int64_t d = c.rbeg - c.rmax0;
        const int64_t tl = d < 10000 ? d : 10000;
        if (tl <= 0) return false;
        const RefSpan t = get_reference(c.rbeg - tl, tl, a.gl);
        c.w = a.sc.band_width;
        c.prev = c.score;
        c.try_idx = 0;
        task = swb_ext_task{ch.read_off, t.off, c.qbeg, t.len, c.w, c.score, a.sc.pen_clip5,
                            SWB_Q_REVERSE | SWB_T_FROM_REF | (t.rc ? SWB_T_COMPLEMENT : SWB_T_REVERSE)};
        c.phase = kLeft;
        return true;
    }

    // Right extension (:265-279).
    __device__ bool right_task() {
        if (c.qend >= ch.read_len) return false;
        const int64_t d = c.rmax1 - c.rend;
        const int64_t tl = d < 10000 ? d : 10000;
        if (tl <= 0) return false;
        const RefSpan t = get_reference(c.rend, tl, a.gl);
        c.w = a.sc.band_width;
        c.prev = c.accH0;
        c.try_idx = 0;
        task = swb_ext_task{ch.read_off + (uint64_t)c.qend, t.off, ch.read_len - c.qend, t.len, c.w, c.accH0,
                            a.sc.pen_clip3, SWB_T_FROM_REF | (t.rc ? (SWB_T_REVERSE | SWB_T_COMPLEMENT) : 0u)};
        c.phase = kRight;
        return true;
    }

    // Region assembly and seed coverage (:318-335, computeSeedCov :36-70).
    __device__ void finish_seed() {
        swb_region &r = c.reg;
        r.qb = c.qbeg - c.l_q;
        r.qe = c.qend + c.r_q;
        r.rb = c.rbeg - c.l_t;
        r.re = c.rend + c.r_t;
        int32_t trueScore = c.len * a.sc.a;
        if (c.l_score > 0) trueScore = c.l_score;
        if (c.r_score > 0) trueScore += c.r_score - c.accH0;
        r.score = trueScore;
        r.true_score = trueScore;
        int32_t cov = 0;
        const swb_seed *sd = a.seeds + ch.seed_off;
        for (uint32_t i = 0; i < ch.n_seeds; ++i) {
            const swb_seed s = sd[i];
            if (s.qbeg >= r.qb && s.qbeg + s.len <= r.qe && s.rbeg >= r.rb && s.rbeg + s.len <= r.re) cov += s.len;
        }
        r.seed_cov = cov;
        regs[c.nreg++] = r;
        ++c.k;
        c.phase = kSeed;
    }

    // Runs the chain on until it needs an extension or is done.
    __device__ void advance() {
        while (c.phase == kSeed) {
            if ((uint32_t)c.k == ch.n_seeds) {                          // :338-343
                const int32_t thr = a.sc.min_seed_len * a.sc.a;
                for (int i = 0; i < c.nreg; ++i)
                    if (regs[i].sub > 0 && regs[i].sub < thr) regs[i].sub = 0;
                c.phase = kDone;
                return;
            }
            const swb_seed s = a.seeds[a.order[ch.seed_off + (uint32_t)c.k]];
            c.qbeg = s.qbeg;
            c.len = s.len;
            c.score = s.score;
            c.rbeg = s.rbeg;
            c.qend = s.qbeg + s.len;
            c.rend = s.rbeg + s.len;
            int cover = -1;                                             // :172-189
            for (int i = 0; i < c.nreg; ++i)
                if (c.qbeg >= regs[i].qb && c.qend <= regs[i].qe) {
                    cover = i;
                    break;
                }
            if (cover >= 0) {
                swb_region &r = regs[cover];
                const int32_t aln = c.len * a.sc.a;
                if (aln > r.sub) r.sub = aln;
                if (aln >= r.score - c.tmp) r.sub_n += 1;
                ++c.k;
                continue;
            }
            c.reg = swb_region{};                                       // :191-199
            c.reg.w = a.sc.band_width;
            c.reg.rid = ch.rid;
            c.reg.seed_cov = c.len;
            c.reg.seed_len0 = c.len;
            c.accH0 = c.score;
            c.l_score = c.l_q = c.l_t = c.r_score = c.r_q = c.r_t = 0;
            if (left_task()) return;
            if (right_task()) return;
            finish_seed();
        }
    }

    // One extension result (:233-260 left, :288-314 right).
    __device__ void feed(const swb_ext_result &r) {
        if (!(r.score == c.prev || r.max_off < (c.w >> 1) + (c.w >> 2) || c.try_idx == 1)) {
            c.prev = r.score;                                           // retry with a doubled band
            c.w <<= 1;
            c.try_idx = 1;
            task.w = c.w;
            return;
        }
        c.reg.w = c.reg.w > c.w ? c.reg.w : c.w;
        if (c.phase == kLeft) {
            c.accH0 = r.score;
            if (r.gscore <= 0 || r.gscore <= r.score - a.sc.pen_clip5) {
                c.l_q = r.qle;
                c.l_t = r.tle;
                c.l_score = r.score;
            } else {
                c.l_q = c.qbeg;
                c.l_t = r.gtle;
                c.l_score = r.gscore;
            }
            c.phase = kSeed;
            if (right_task()) return;
            finish_seed();
        } else {
            if (r.gscore <= 0 || r.gscore <= r.score - a.sc.pen_clip3) {
                c.r_q = r.qle;
                c.r_t = r.tle;
                c.r_score = r.score;
            } else {
                c.r_q = ch.read_len - c.qend;
                c.r_t = r.gtle;
                c.r_score = r.gscore;
            }
            finish_seed();
        }
        advance();
    }
};

__global__ void seed_keys_kernel(const swb_seed *__restrict__ seeds, size_t n_seeds, const swb_chain *__restrict__ chains,
                                 uint32_t n_chains, int32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                 uint32_t *__restrict__ beg, uint32_t *__restrict__ end) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n_seeds) {
        keys[i] = seeds[i].score;
        vals[i] = (uint32_t)i;
    }
    if (i < n_chains) {
        beg[i] = chains[i].seed_off;
        end[i] = chains[i].seed_off + chains[i].n_seeds;
    }
}

// Chain set-up (:126-158) and the first advance; live[c] = chain c has a task.
__global__ void chain_init_kernel(ChainArgs a, uint32_t *__restrict__ ids, uint8_t *__restrict__ live) {
    const uint32_t ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= a.n_chains) return;
    const swb_chain ch = a.chains[ci];
    ChainState c{};
    const long lq = ch.read_len;
    c.rmax0 = INT64_MAX;
    c.rmax1 = 0;
    const swb_seed *sd = a.seeds + ch.seed_off;
    for (uint32_t k = 0; k < ch.n_seeds; ++k) {
        const swb_seed t = sd[k];
        const int64_t b = t.rbeg - (int64_t)((long)t.qbeg + cal_max_gap(t.qbeg, a.sc));
        const long remaining = lq - t.qbeg - t.len;
        const int64_t e = t.rbeg + t.len + (int64_t)(remaining + cal_max_gap(remaining, a.sc));
        c.rmax0 = b < c.rmax0 ? b : c.rmax0;
        c.rmax1 = e > c.rmax1 ? e : c.rmax1;
    }
    if (c.rmax0 < 0) c.rmax0 = 0;
    c.tmp = imax(a.sc.a + a.sc.b, imax(a.sc.o_ins + a.sc.e_ins, a.sc.o_del + a.sc.e_del));
    c.phase = kSeed;
    swb_ext_task task{};
    Chain{a, ch, c, task, a.regions + ch.seed_off}.advance();
    a.state[ci] = c;
    a.task[ci] = task;
    ids[ci] = ci;
    live[ci] = c.phase != kDone;
}

// Feeds round results back; live[k] = active chain k still has a task.
__global__ void chain_feed_kernel(ChainArgs a, const uint32_t *__restrict__ active, uint32_t n,
                                  const swb_ext_result *__restrict__ res, uint8_t *__restrict__ live) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t ci = active[k];
    const swb_chain ch = a.chains[ci];
    ChainState c = a.state[ci];
    swb_ext_task task = a.task[ci];
    Chain{a, ch, c, task, a.regions + ch.seed_off}.feed(res[k]);
    a.state[ci] = c;
    a.task[ci] = task;
    live[k] = c.phase != kDone;
}

// Dense batch of the live chains' tasks (count read on the device).
__global__ void gather_tasks_kernel(const uint32_t *__restrict__ active, const uint32_t *__restrict__ n_active,
                                    const swb_ext_task *__restrict__ task, swb_ext_task *__restrict__ out, uint32_t cap) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < cap && k < *n_active) out[k] = task[active[k]];
}

__global__ void region_counts_kernel(const ChainState *__restrict__ st, uint32_t n, uint32_t *__restrict__ counts) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) counts[k] = (uint32_t)st[k].nreg;
}

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" int swb_extend_chains(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                                 const swb_seed *seeds, size_t n_seeds, const swb_chain *chains, size_t n_chains,
                                 uint64_t genome_len, swb_region *out, uint32_t *n_regions, uint32_t *rounds) {
    if (!ctx || (!bases && n_bases) || (!seeds && n_seeds) || (!chains && n_chains) || (!out && n_seeds) ||
        (!n_regions && n_chains))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    if (rounds) *rounds = 0;
    if (n_chains == 0) return SWB_OK;
    if (n_chains > 0x7FFFFFF0ull || n_seeds > 0x7FFFFFF0ull)
        return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 chains or seeds");
    if (!ctx->d_pac || genome_len > ctx->ref_bases)
        return set_error(SWB_ERR_NO_REFERENCE, "the forward strand (genome_len bases) must be uploaded first");
    // Validation: spans inside the inputs, seed ranges of different chains
    // disjoint (regions are written at each chain's seed_off).  Host threads
    // check ranges of chains; the first failing chain is reported.
    const size_t nth = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()),
                                        std::max<size_t>(1, n_chains / 16384));
    struct Part {
        size_t bad = SIZE_MAX;
        std::string msg;
        int max_read = 0;
        bool sorted = true;
        uint64_t first_off = UINT64_MAX, max_end = 0;
    };
    std::vector<Part> parts(nth);
    const size_t per = (n_chains + nth - 1) / nth;
    auto check = [&](size_t t) {
        Part &pt = parts[t];
        const size_t lo = std::min(n_chains, t * per), hi = std::min(n_chains, lo + per);
        for (size_t i = lo; i < hi; ++i) {
            const swb_chain &ch = chains[i];
            if ((uint64_t)ch.seed_off + ch.n_seeds > n_seeds || ch.read_len < 0 || ch.read_len > kMaxLen ||
                ch.read_off + (uint64_t)ch.read_len > n_bases) {
                pt.bad = i;
                pt.msg = "chain " + std::to_string(i) + ": seeds or read outside the inputs";
                return;
            }
            pt.max_read = std::max(pt.max_read, ch.read_len);
            for (uint32_t k = 0; k < ch.n_seeds; ++k) {
                const swb_seed &sd = seeds[ch.seed_off + k];
                if (sd.qbeg < 0 || sd.len < 0 || sd.qbeg + sd.len > ch.read_len || sd.rbeg < 0 ||
                    sd.rbeg + sd.len > 2 * (int64_t)genome_len) {
                    pt.bad = i;
                    pt.msg = "chain " + std::to_string(i) + ": seed " + std::to_string(k) + " out of range";
                    return;
                }
            }
            if (ch.n_seeds) {
                if (pt.first_off == UINT64_MAX) pt.first_off = ch.seed_off;
                if (ch.seed_off < pt.max_end) pt.sorted = false;
                pt.max_end = std::max<uint64_t>(pt.max_end, (uint64_t)ch.seed_off + ch.n_seeds);
            }
        }
    };
    if (nth == 1) {
        check(0);
    } else {
        std::vector<std::thread> th;
        for (size_t t = 0; t < nth; ++t) th.emplace_back(check, t);
        for (auto &x : th) x.join();
    }
    int max_read = 0;
    bool sorted = true;
    uint64_t prev_end = 0;
    for (const Part &pt : parts) {
        if (pt.bad != SIZE_MAX) return set_error(SWB_ERR_INVALID_ARG, pt.msg);
        max_read = std::max(max_read, pt.max_read);
        sorted = sorted && pt.sorted && (pt.first_off == UINT64_MAX || pt.first_off >= prev_end);
        prev_end = std::max(prev_end, pt.max_end);
    }
    if (!sorted) {
        std::vector<std::pair<uint32_t, uint32_t>> r;
        for (size_t i = 0; i < n_chains; ++i)
            if (chains[i].n_seeds) r.emplace_back(chains[i].seed_off, chains[i].n_seeds);
        std::sort(r.begin(), r.end());
        for (size_t i = 1; i < r.size(); ++i)
            if ((uint64_t)r[i - 1].first + r[i - 1].second > r[i].first)
                return set_error(SWB_ERR_INVALID_ARG, "chains' seed ranges overlap");
    }

    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const DevScoring dsc = make_dev_scoring(*sc);
    const size_t nc = n_chains, ns = std::max<size_t>(n_seeds, 1);
    // Device layout of the chain buffer.
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off += al256(bytes);
        return o;
    };
    const size_t o_seeds = carve(ns * sizeof(swb_seed)), o_chains = carve(nc * sizeof(swb_chain));
    const size_t o_state = carve(nc * sizeof(ChainState)), o_task = carve(nc * sizeof(swb_ext_task));
    const size_t o_reg = carve(ns * sizeof(swb_region)), o_act0 = carve(nc * 4), o_act1 = carve(nc * 4);
    const size_t o_live = carve(nc), o_num = carve(8), o_counts = carve(nc * 4);
    const size_t o_keys = carve(ns * 4), o_keys2 = carve(ns * 4), o_vals = carve(ns * 4), o_order = carve(ns * 4);
    const size_t o_beg = carve(nc * 4), o_end = carve(nc * 4);
    if ((rc = ensure_dev(ctx, ctx->d_chain, off))) return rc;
    char *base = (char *)ctx->d_chain.p;
    swb_seed *d_seeds = (swb_seed *)(base + o_seeds);
    swb_chain *d_chains = (swb_chain *)(base + o_chains);
    uint32_t *act[2] = {(uint32_t *)(base + o_act0), (uint32_t *)(base + o_act1)};
    uint8_t *d_live = (uint8_t *)(base + o_live);
    uint32_t *d_num = (uint32_t *)(base + o_num);
    swb_region *d_reg = (swb_region *)(base + o_reg);
    ChainState *d_state = (ChainState *)(base + o_state);
    const size_t bases_bytes = std::max<size_t>(n_bases, 1);
    if ((rc = ensure_dev(ctx, ctx->d_bases, al256(bases_bytes))) ||
        (rc = ensure_dev(ctx, ctx->d_tasks, nc * sizeof(swb_ext_task))) ||
        (rc = ensure_dev(ctx, ctx->d_out, nc * sizeof(swb_ext_result))))
        return rc;

    SWB_CUDA(cudaMemsetAsync(ctx->d_counters, 0, sizeof(unsigned long long) * kNumCounters, st));
    SWB_CUDA(cudaEventRecord(ctx->ev_start, st));
    // Inputs: straight from the caller's buffers when they are pinned, else
    // through the context's pinned staging buffer (host threads copy, then
    // one transfer for the bases and one for the seeds and chains, which sit
    // together at the start of the chain buffer).
    if ((n_bases == 0 || is_pinned(bases)) && (n_seeds == 0 || is_pinned(seeds)) && is_pinned(chains)) {
        if (n_bases) SWB_CUDA(cudaMemcpyAsync(ctx->d_bases.p, bases, n_bases, cudaMemcpyHostToDevice, st));
        if (n_seeds)
            SWB_CUDA(cudaMemcpyAsync(base + o_seeds, seeds, n_seeds * sizeof(swb_seed), cudaMemcpyHostToDevice, st));
        SWB_CUDA(cudaMemcpyAsync(base + o_chains, chains, nc * sizeof(swb_chain), cudaMemcpyHostToDevice, st));
    } else {
        const size_t sc_bytes = o_chains + nc * sizeof(swb_chain);
        if ((rc = ensure_host(ctx, ctx->h_in, al256(n_bases) + sc_bytes))) return rc;
        char *stage = (char *)ctx->h_in.p, *stage_sc = stage + al256(n_bases);
        par_copy(stage, bases, n_bases);
        par_copy(stage_sc + o_seeds, seeds, n_seeds * sizeof(swb_seed));
        par_copy(stage_sc + o_chains, chains, nc * sizeof(swb_chain));
        if (n_bases) SWB_CUDA(cudaMemcpyAsync(ctx->d_bases.p, stage, n_bases, cudaMemcpyHostToDevice, st));
        SWB_CUDA(cudaMemcpyAsync(base, stage_sc, sc_bytes, cudaMemcpyHostToDevice, st));
    }
    SWB_CUDA(cudaMemsetAsync(d_reg, 0, ns * sizeof(swb_region), st));

    // Seed order: stable descending sort of each chain's seeds by score (:155-158).
    uint32_t *order = (uint32_t *)(base + o_order);
    const unsigned tb = 256;
    {
        const size_t m = std::max(ns, nc);
        ProfScope ps(ctx, st, "chain_seed_order", -1);
        seed_keys_kernel<<<(unsigned)((m + tb - 1) / tb), tb, 0, st>>>(
            d_seeds, n_seeds, d_chains, (uint32_t)nc, (int32_t *)(base + o_keys), (uint32_t *)(base + o_vals),
            (uint32_t *)(base + o_beg), (uint32_t *)(base + o_end));
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
        if (n_seeds) {
            size_t tmp = 0;
            SWB_CUDA(cub::DeviceSegmentedSort::StableSortPairsDescending(
                nullptr, tmp, (const int32_t *)(base + o_keys), (int32_t *)(base + o_keys2),
                (const uint32_t *)(base + o_vals), order, (int)n_seeds, (int)nc, (const uint32_t *)(base + o_beg),
                (const uint32_t *)(base + o_end), st));
            if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp))) return rc;
            SWB_CUDA(cub::DeviceSegmentedSort::StableSortPairsDescending(
                ctx->d_sort_tmp.p, tmp, (const int32_t *)(base + o_keys), (int32_t *)(base + o_keys2),
                (const uint32_t *)(base + o_vals), order, (int)n_seeds, (int)nc, (const uint32_t *)(base + o_beg),
                (const uint32_t *)(base + o_end), st));
        }
    }
    ChainArgs ca{dsc, (int64_t)genome_len, d_chains, d_seeds, order, d_state,
                 (swb_ext_task *)(base + o_task), d_reg, (uint32_t)nc};
    {
        ProfScope ps(ctx, st, "chain_step", -1);
        chain_init_kernel<<<(unsigned)((nc + tb - 1) / tb), tb, 0, st>>>(ca, act[1], d_live);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    // act[1] lists the chains of the last step with their live flags; each
    // round compacts it into act[0], then the two swap.
    uint32_t n_prev = (uint32_t)nc, nround = 0;
    swb_ext_task *d_batch = (swb_ext_task *)ctx->d_tasks.p;
    swb_ext_result *d_res = (swb_ext_result *)ctx->d_out.p;
    for (;;) {
        size_t tmp = 0;
        SWB_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, act[1], d_live, act[0], d_num, (int)n_prev, st));
        if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp))) return rc;
        SWB_CUDA(cub::DeviceSelect::Flagged(ctx->d_sort_tmp.p, tmp, act[1], d_live, act[0], d_num, (int)n_prev, st));
        gather_tasks_kernel<<<(n_prev + tb - 1) / tb, tb, 0, st>>>(act[0], d_num, ca.task, d_batch, n_prev);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
        uint32_t n = 0;
        SWB_CUDA(cudaMemcpyAsync(&n, d_num, sizeof(n), cudaMemcpyDeviceToHost, st));
        SWB_CUDA(cudaStreamSynchronize(st));
        if (n == 0) break;
        if ((rc = launch_ext(ctx, dsc, (const uint8_t *)ctx->d_bases.p, d_batch, n, d_res, ctx->d_counters, st,
                             max_read)))
            return rc;
        ++nround;
        {
            ProfScope ps(ctx, st, "chain_step", -1);
            chain_feed_kernel<<<(n + tb - 1) / tb, tb, 0, st>>>(ca, act[0], n, d_res, d_live);
            ctx->launches++;
            SWB_CUDA(cudaGetLastError());
        }
        std::swap(act[0], act[1]);
        n_prev = n;
    }
    uint32_t *d_counts = (uint32_t *)(base + o_counts);
    region_counts_kernel<<<(unsigned)((nc + tb - 1) / tb), tb, 0, st>>>(d_state, (uint32_t)nc, d_counts);
    ctx->launches++;
    SWB_CUDA(cudaGetLastError());
    if ((rc = d2h_staged(ctx, st, {DevSpan{d_reg, out, n_seeds * sizeof(swb_region)},
                                   DevSpan{d_counts, n_regions, nc * sizeof(uint32_t)}}, ctx->ev_stop)))
        return rc;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) ctx->last_ms = ms;
    unsigned long long c[kNumCounters] = {0};
    if (cudaMemcpy(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) {
        unsigned long long sum = 0;
        for (int k = 0; k < kNumCounters; ++k) sum += c[k];
        ctx->last_cells = sum;
    }
    if (rounds) *rounds = nround;
    return SWB_OK;
}
