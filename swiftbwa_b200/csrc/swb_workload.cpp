// swb_workload.cpp -- seeded synthetic workloads for the benchmark configs
// (host C++, built into libswb_workload.so; no CUDA).
//
// The reference ships no benchmark data for this path, so the configs are
// synthetic: a uniform random ACGT reference (optionally with inserted
// tandem-repeat blocks), reads sampled from it with substitutions, 1-3 bp
// indels and N bases, and the extension / global / local-SW tasks derived
// from them exactly as the configs describe.  Generation is split into
// fixed-size chunks with per-chunk seeds, so the output depends only on the
// seed, never on the thread count.
//
// PRNG: xoshiro256** (Blackman & Vigna) seeded through splitmix64.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/swb_cuda.h"

namespace {

inline uint64_t splitmix64(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto &v : s) v = splitmix64(x);
    }
    static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    inline uint64_t next() {
        const uint64_t result = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return result;
    }
    inline double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    inline uint64_t below(uint64_t n) { return n ? next() % n : 0; }
    inline int64_t range(int64_t lo, int64_t hi) { return lo + (int64_t)below((uint64_t)(hi - lo + 1)); }   // inclusive
    inline uint8_t base() { return (uint8_t)(next() >> 62); }
    inline double normal() {   // Box-Muller
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

template <class F>
void chunked(size_t n, size_t chunk, F fn) {
    const size_t nchunks = (n + chunk - 1) / chunk;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (unsigned t = 0; t < hw; ++t)
        th.emplace_back([&, t] {
            for (size_t c = t; c < nchunks; c += hw) fn(c, c * chunk, std::min(n, (c + 1) * chunk));
        });
    for (auto &x : th) x.join();
}

inline uint64_t chunk_seed(uint64_t seed, uint64_t c) {
    uint64_t x = seed ^ (0xA5A5A5A5ull + c * 0x100000001B3ull);
    return splitmix64(x);
}

// One simulated read copied from ref[start...] with errors.  clean[k] marks
// read bases that are exact copies of ref[rpos[k]] with no event before them.
struct ReadSim {
    std::vector<uint8_t> bases;
    std::vector<int64_t> rpos;
    std::vector<uint8_t> clean;
    int64_t ref_end = 0;
    int n_sub = 0, n_indel = 0, indel_bases = 0;
};

void simulate_read(Rng &r, const uint8_t *ref, int64_t ref_len, int64_t start, int len, double sub,
                   double indel, double n_rate, ReadSim &out) {
    out.bases.clear();
    out.rpos.clear();
    out.clean.clear();
    out.n_sub = out.n_indel = out.indel_bases = 0;
    int64_t p = start;
    while ((int)out.bases.size() < len && p < ref_len) {
        const double u = r.uniform();
        if (u < indel * 0.5) {                                   // deletion of 1-3 reference bases
            const int d = (int)r.range(1, 3);
            p += d;
            out.n_indel++;
            out.indel_bases += d;
            if (!out.clean.empty()) out.clean.back() = 0;
            continue;
        }
        if (u < indel) {                                         // insertion of 1-3 read bases
            const int ins = (int)r.range(1, 3);
            out.n_indel++;
            out.indel_bases += ins;
            for (int k = 0; k < ins && (int)out.bases.size() < len; ++k) {
                out.bases.push_back(r.base());
                out.rpos.push_back(p);
                out.clean.push_back(0);
            }
            continue;
        }
        uint8_t b = ref[p];
        bool ok = true;
        const double v = r.uniform();
        if (v < sub) {
            b = (uint8_t)((b + r.range(1, 3)) & 3);
            ok = false;
            out.n_sub++;
        } else if (v < sub + n_rate) {
            b = 4;
            ok = false;
            out.n_sub++;
        }
        out.bases.push_back(b);
        out.rpos.push_back(p);
        out.clean.push_back(ok ? 1 : 0);
        ++p;
    }
    while ((int)out.bases.size() < len) {   // ran off the reference end: pad with random bases
        out.bases.push_back(r.base());
        out.rpos.push_back(ref_len);
        out.clean.push_back(0);
    }
    out.ref_end = p;
}

// First (or a random) run of `seed_len` clean read bases on consecutive
// reference positions; returns the read offset or -1.
int find_seed(Rng &r, const ReadSim &rs, int seed_len, bool random_start) {
    const int L = (int)rs.bases.size();
    std::vector<int> starts;
    int run = 0;
    for (int k = 0; k < L; ++k) {
        const bool cont = rs.clean[k] && (run == 0 || rs.rpos[k] == rs.rpos[k - 1] + 1);
        run = cont ? run + 1 : (rs.clean[k] ? 1 : 0);
        if (run >= seed_len) {
            const int s = k - seed_len + 1;
            if (!random_start) return s;
            starts.push_back(s);
        }
    }
    if (starts.empty()) return -1;
    return starts[r.below(starts.size())];
}

}  // namespace

extern "C" {

// Uniform random reference of n bases (codes 0-3) with optional tandem
// blocks (period 2-6, length 1-5 kbp) covering ~tandem_frac of it.  Writes
// codes (if non-NULL) and the .pac layout (bits 7-6 first).  Returns the
// number of tandem blocks (their [start, len) go to blocks, up to max_blocks).
int64_t swbw_reference(uint64_t seed, uint64_t n, double tandem_frac, uint8_t *codes, uint8_t *pac,
                       int64_t *blocks, int64_t max_blocks) {
    std::vector<uint8_t> local;
    uint8_t *c = codes;
    if (!c) {
        local.resize(n);
        c = local.data();
    }
    chunked(n, 1 << 20, [&](size_t ci, size_t lo, size_t hi) {
        Rng r(chunk_seed(seed, ci));
        size_t i = lo;
        for (; i + 32 <= hi; i += 32) {
            uint64_t x = r.next();
            for (int k = 0; k < 32; ++k) c[i + k] = (uint8_t)((x >> (2 * k)) & 3);
        }
        for (; i < hi; ++i) c[i] = r.base();
    });
    int64_t nb = 0;
    if (tandem_frac > 0 && n > 10000) {
        Rng r(seed ^ 0x7A9D3E5Bull);
        uint64_t covered = 0;
        const uint64_t want = (uint64_t)(tandem_frac * (double)n);
        while (covered < want && nb < max_blocks) {
            const int64_t len = r.range(1000, 5000);
            const int64_t start = (int64_t)r.below(n - (uint64_t)len);
            const int period = (int)r.range(2, 6);
            uint8_t unit[6];
            for (int k = 0; k < period; ++k) unit[k] = r.base();
            for (int64_t k = 0; k < len; ++k) c[start + k] = unit[k % period];
            if (blocks) {
                blocks[2 * nb] = start;
                blocks[2 * nb + 1] = len;
            }
            ++nb;
            covered += (uint64_t)len;
        }
    }
    if (pac) {
        chunked((n + 3) / 4, 1 << 20, [&](size_t, size_t lo, size_t hi) {
            for (size_t b = lo; b < hi; ++b) {
                uint8_t v = 0;
                for (int k = 0; k < 4; ++k) {
                    const uint64_t p = 4 * b + k;
                    v = (uint8_t)(v | ((p < n ? (c[p] & 3) : 0) << (6 - 2 * k)));
                }
                pac[b] = v;
            }
        });
    }
    return nb;
}

// Reads and extension tasks (configs 0 and 1).  For each read: simulate it
// from a uniform position (or, with probability tandem_read_frac, from a
// tandem block), find an error-free seed_len-mer (the first, or a random
// one), and emit the right extension (query = read suffix after the seed,
// target = reference [seedEnd, seedEnd+qlen+w) clamped) and, when `left`,
// the left extension (query = reversed prefix, target = reversed reference
// window ending at the seed).  Targets are read from the resident reference
// (SWB_T_FROM_REF).  Tasks are written contiguously per read (left first);
// reads without a seed produce no tasks.  read_info[4*i..] = {ref_start,
// ref_end, n_sub, n_indel_bases}.  Returns the number of tasks.
int64_t swbw_ext_tasks(uint64_t seed, const uint8_t *ref, int64_t ref_len, const int64_t *blocks,
                       int64_t n_blocks, double tandem_read_frac, int64_t n_reads, int read_len,
                       double sub, double indel, double n_rate, int seed_len, int random_seed_pos,
                       int w, int h0, int end_bonus5, int end_bonus3, int left,
                       uint8_t *reads_out, swb_ext_task *tasks_out, int64_t *read_info) {
    const size_t chunk = 16384;
    const int per_read = left ? 2 : 1;
    std::vector<int64_t> counts((n_reads + chunk - 1) / chunk, 0);
    // Tasks of read i go to slots [per_read*i, per_read*i + per_read); unused
    // slots are compacted afterwards.
    std::vector<uint8_t> used((size_t)n_reads * per_read, 0);
    chunked((size_t)n_reads, chunk, [&](size_t ci, size_t lo, size_t hi) {
        Rng r(chunk_seed(seed, ci));
        ReadSim rs;
        for (size_t i = lo; i < hi; ++i) {
            int64_t start;
            if (n_blocks > 0 && r.uniform() < tandem_read_frac) {
                const int64_t b = (int64_t)r.below((uint64_t)n_blocks);
                const int64_t bs = blocks[2 * b], bl = blocks[2 * b + 1];
                start = bs + (int64_t)r.below((uint64_t)std::max<int64_t>(1, bl - read_len / 2));
                start = std::min<int64_t>(start, ref_len - read_len - 16);
            } else {
                start = (int64_t)r.below((uint64_t)std::max<int64_t>(1, ref_len - read_len - 16));
            }
            simulate_read(r, ref, ref_len, start, read_len, sub, indel, n_rate, rs);
            uint8_t *rd = reads_out + i * (size_t)read_len;
            std::memcpy(rd, rs.bases.data(), (size_t)read_len);
            if (read_info) {
                read_info[4 * i] = start;
                read_info[4 * i + 1] = rs.ref_end;
                read_info[4 * i + 2] = rs.n_sub;
                read_info[4 * i + 3] = rs.indel_bases;
            }
            const int s = find_seed(r, rs, seed_len, random_seed_pos != 0);
            if (s < 0) continue;
            const int64_t rbeg = rs.rpos[s], rend = rbeg + seed_len;
            const int qe = s + seed_len;
            swb_ext_task *slot = tasks_out + i * per_read;
            if (left && s > 0) {
                const int qlen = s;
                int64_t tl = std::min<int64_t>((int64_t)qlen + w, rbeg);
                swb_ext_task t{i * (uint64_t)read_len, (uint64_t)(rbeg - tl), qlen, (int32_t)tl, w, h0, end_bonus5,
                               SWB_Q_REVERSE | SWB_T_REVERSE | SWB_T_FROM_REF};
                slot[0] = t;
                used[i * per_read] = 1;
            }
            if (qe < read_len) {
                const int qlen = read_len - qe;
                int64_t tl = std::min<int64_t>((int64_t)qlen + w, ref_len - rend);
                swb_ext_task t{i * (uint64_t)read_len + qe, (uint64_t)rend, qlen, (int32_t)std::max<int64_t>(tl, 0), w, h0,
                               end_bonus3, SWB_T_FROM_REF};
                slot[per_read - 1] = t;
                used[i * per_read + per_read - 1] = 1;
            }
        }
    });
    int64_t k = 0;
    for (size_t i = 0; i < used.size(); ++i)
        if (used[i]) tasks_out[k++] = tasks_out[i];
    return k;
}

// Uneven extension tasks (config 2 / the serving mix): query length
// log-uniform in [qmin, qmax] (or drawn from `mix` lengths when n_mix > 0),
// w uniform in [wmin, wmax], h0 uniform in [h0min, h0max]; the query is a
// mutated copy of a random reference window and the target is the
// reference window [pos, pos + qlen + w) (SWB_T_FROM_REF).  Queries are
// written back to back into bases_out (capacity n * qmax).  Returns bases used.
int64_t swbw_uneven_tasks(uint64_t seed, const uint8_t *ref, int64_t ref_len, int64_t n, int qmin, int qmax,
                          const int *mix, int n_mix, int wmin, int wmax, int h0min, int h0max, double sub,
                          double indel, int end_bonus, uint8_t *bases_out, swb_ext_task *tasks_out) {
    // Every task owns a qmax-sized window in bases_out, compacted afterwards.
    chunked((size_t)n, 16384, [&](size_t ci, size_t lo, size_t hi) {
        Rng r(chunk_seed(seed, ci));
        ReadSim rs;
        const double lmin = std::log((double)qmin), lmax = std::log((double)qmax + 1.0);
        for (size_t i = lo; i < hi; ++i) {
            int qlen;
            if (n_mix > 0) {
                qlen = mix[r.below((uint64_t)n_mix)];
            } else {
                qlen = (int)std::floor(std::exp(lmin + (lmax - lmin) * r.uniform()));
                qlen = std::min(std::max(qlen, qmin), qmax);
            }
            const int w = (int)r.range(wmin, wmax);
            const int h0 = (int)r.range(h0min, h0max);
            const int64_t pos = (int64_t)r.below((uint64_t)std::max<int64_t>(1, ref_len - qlen - w - 16));
            simulate_read(r, ref, ref_len, pos, qlen, sub, indel, 0.0, rs);
            std::memcpy(bases_out + i * (size_t)qmax, rs.bases.data(), (size_t)qlen);
            const int64_t tl = std::min<int64_t>((int64_t)qlen + w, ref_len - pos);
            tasks_out[i] = swb_ext_task{i * (uint64_t)qmax, (uint64_t)pos, qlen, (int32_t)tl, w, h0, end_bonus,
                                        SWB_T_FROM_REF};
        }
    });
    uint64_t off = 0;
    for (int64_t i = 0; i < n; ++i) {
        const uint64_t src = tasks_out[i].q_off;
        if (src != off) std::memmove(bases_out + off, bases_out + src, (size_t)tasks_out[i].qlen);
        tasks_out[i].q_off = off;
        off += (uint64_t)tasks_out[i].qlen;
    }
    return (int64_t)off;
}

// Mate-rescue tasks (config 3): per pair a mate of mate_len bases with
// `sub` substitutions, a reference window of win_len bases from the
// resident reference, and the mate placed at an insert offset drawn from
// N(insert_mean, insert_sd) inside it; a fraction no_hit_frac of mates are
// random (no true hit).  Mates go to bases_out (n * mate_len).
void swbw_rescue_tasks(uint64_t seed, const uint8_t *ref, int64_t ref_len, int64_t n, int mate_len, int win_len,
                       double insert_mean, double insert_sd, double sub, double no_hit_frac, int min_sub_score,
                       uint8_t *bases_out, swb_local_task *tasks_out) {
    chunked((size_t)n, 16384, [&](size_t ci, size_t lo, size_t hi) {
        Rng r(chunk_seed(seed, ci));
        for (size_t i = lo; i < hi; ++i) {
            const int64_t wpos = (int64_t)r.below((uint64_t)std::max<int64_t>(1, ref_len - win_len - 1));
            uint8_t *m = bases_out + i * (size_t)mate_len;
            if (r.uniform() < no_hit_frac) {
                for (int k = 0; k < mate_len; ++k) m[k] = r.base();
            } else {
                // window covers [mean - 4sd, mean + 4sd] of insert offsets; place the mate by its drawn offset.
                double ins = insert_mean + insert_sd * r.normal();
                double lo_ins = insert_mean - 4 * insert_sd;
                int64_t off = (int64_t)std::llround(ins - lo_ins) + (win_len - mate_len - (int64_t)(8 * insert_sd)) / 2;
                off = std::min<int64_t>(std::max<int64_t>(off, 0), win_len - mate_len);
                for (int k = 0; k < mate_len; ++k) {
                    uint8_t b = ref[wpos + off + k];
                    if (r.uniform() < sub) b = (uint8_t)((b + r.range(1, 3)) & 3);
                    m[k] = b;
                }
            }
            tasks_out[i] = swb_local_task{i * (uint64_t)mate_len, (uint64_t)wpos, mate_len, win_len, min_sub_score,
                                          SWB_T_FROM_REF};
        }
    });
}

// Seed chains for ExtensionAligner.extend: n reads of read_len bases, each
// from a random position of either strand of the genome (BWT coordinates,
// [0, 2*gl): positions >= gl read the reverse complement), with errors.  A
// chain's seeds are the clean runs of at least min_seed bases at the read's
// true location (up to max_seeds, in read order, score = len * a), plus with
// probability spurious_frac one extra seed of the read placed at a random
// offset of up to +-200 bases.  Reads go to bases_out (n * read_len); seeds
// are compacted in chain order.  Returns the number of seeds.
int64_t swbw_chains(uint64_t seed, const uint8_t *ref, int64_t gl, int64_t n, int read_len, double sub, double indel,
                    double n_rate, int min_seed, int max_seeds, int a, double spurious_frac, uint8_t *bases_out,
                    swb_seed *seeds_out, swb_chain *chains_out) {
    std::vector<uint32_t> cnt((size_t)n, 0);
    chunked((size_t)n, 4096, [&](size_t ci, size_t lo, size_t hi) {
        Rng r(chunk_seed(seed, ci));
        ReadSim rs;
        std::vector<uint8_t> win;
        const int span = read_len + 64;
        for (size_t i = lo; i < hi; ++i) {
            const bool rev = r.uniform() < 0.5;
            const int64_t fpos = (int64_t)r.below((uint64_t)std::max<int64_t>(1, gl - span));
            int64_t p0;                                         // BWT coordinate of win[0]
            win.resize((size_t)span);
            if (!rev) {
                p0 = fpos;
                std::memcpy(win.data(), ref + fpos, (size_t)span);
            } else {                                            // reverse complement of ref[fpos, fpos+span)
                p0 = 2 * gl - (fpos + span);
                for (int k = 0; k < span; ++k) win[(size_t)k] = (uint8_t)(3 - ref[fpos + span - 1 - k]);
            }
            simulate_read(r, win.data(), span, 0, read_len, sub, indel, n_rate, rs);
            std::memcpy(bases_out + i * (size_t)read_len, rs.bases.data(), (size_t)read_len);
            swb_seed *sd = seeds_out + i * (size_t)(max_seeds + 1);
            uint32_t m = 0;
            int run = 0;
            for (int k = 0; k <= read_len; ++k) {
                const bool ok = k < read_len && rs.clean[(size_t)k] && rs.rpos[(size_t)k] < span &&
                                (run == 0 || rs.rpos[(size_t)k] == rs.rpos[(size_t)k - 1] + 1);
                if (ok) {
                    ++run;
                    continue;
                }
                if (run >= min_seed && (int)m < max_seeds) {
                    const int qb = k - run;
                    sd[m++] = swb_seed{p0 + rs.rpos[(size_t)qb], qb, run, run * a, 0};
                }
                run = (k < read_len && rs.clean[(size_t)k] && rs.rpos[(size_t)k] < span) ? 1 : 0;
            }
            if (m > 0 && r.uniform() < spurious_frac) {
                const swb_seed &b = sd[r.below(m)];
                int64_t rb = b.rbeg + r.range(-200, 200);
                const int64_t lo_b = rev ? gl : 0, hi_b = rev ? 2 * gl - b.len : gl - b.len;
                rb = std::min(std::max(rb, lo_b), hi_b);
                sd[m++] = swb_seed{rb, b.qbeg, b.len, b.len * a, 0};
            }
            cnt[i] = m;
            chains_out[i] = swb_chain{i * (uint64_t)read_len, read_len, (int32_t)(i & 0x7fffffff), 0, m};
        }
    });
    uint64_t off = 0;
    for (int64_t i = 0; i < n; ++i) {
        const swb_seed *src = seeds_out + (size_t)i * (size_t)(max_seeds + 1);
        if (src != seeds_out + off) std::memmove(seeds_out + off, src, cnt[(size_t)i] * sizeof(swb_seed));
        chains_out[i].seed_off = (uint32_t)off;
        off += cnt[(size_t)i];
    }
    return (int64_t)off;
}

// Mate-rescue jobs: n mates of mate_len bases.  Each job has 1-3 template
// regions on a random strand (BWT coordinates); the first one is the true
// anchor: in the template's strand the mate's reverse complement lies at
// [rb + ins - mate_len, rb + ins), ins ~ N(ins_mean, ins_sd) (an FR pair),
// with `sub` substitutions.  A fraction no_hit_frac of mates are random.
// With probability hit_frac the mate already has a region consistent with
// FR (so that direction is skipped), plus 0-2 unrelated mate regions.  The
// template's rid is the contig of its forward position.  Mates go to
// bases_out (n * mate_len); templates / mate regions are compacted; returns
// (n_templates << 32) | n_mate_regions.
uint64_t swbw_rescue_jobs(uint64_t seed, const uint8_t *ref, int64_t gl, const int64_t *coff, int64_t n_contigs,
                          int64_t n, int mate_len, double ins_mean, double ins_sd, double sub, double no_hit_frac,
                          double hit_frac, uint8_t *bases_out, swb_rescue_job *jobs, swb_anchor *tmpl,
                          swb_anchor *mreg) {
    auto full = [&](int64_t p) -> uint8_t { return p < gl ? ref[p] : (uint8_t)(3 - ref[2 * gl - 1 - p]); };
    auto rid_of = [&](int64_t bwt) -> int32_t {   // contig of the forward position
        const int64_t f = bwt < gl ? bwt : 2 * gl - 1 - bwt;
        int64_t lo = 0, hi = n_contigs - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (coff[mid] <= f) lo = mid; else hi = mid - 1;
        }
        return (int32_t)lo;
    };
    std::vector<uint32_t> nt((size_t)n), nm((size_t)n);
    chunked((size_t)n, 4096, [&](size_t ci, size_t lo, size_t hi) {
        Rng r(chunk_seed(seed, ci));
        for (size_t i = lo; i < hi; ++i) {
            uint8_t *m = bases_out + i * (size_t)mate_len;
            swb_anchor *t = tmpl + i * 3;
            swb_anchor *mr = mreg + i * 3;
            const int64_t rb = (int64_t)r.below((uint64_t)(2 * gl - mate_len));
            const int64_t ins = (int64_t)std::llround(ins_mean + ins_sd * r.normal());
            if (r.uniform() < no_hit_frac) {
                for (int k = 0; k < mate_len; ++k) m[k] = r.base();
            } else {
                // mate = reverse complement of full[rb + ins - mate_len, rb + ins)
                for (int k = 0; k < mate_len; ++k) {
                    const int64_t p = rb + ins - 1 - k;
                    uint8_t b = (p >= 0 && p < 2 * gl) ? (uint8_t)(3 - full(p)) : r.base();
                    if (r.uniform() < sub) b = (uint8_t)((b + r.range(1, 3)) & 3);
                    m[k] = b;
                }
            }
            uint32_t a = 0;
            t[a++] = swb_anchor{rb, rid_of(rb), 0};
            const int extra = (int)r.below(3);
            for (int k = 0; k < extra; ++k) {
                const int64_t x = (int64_t)r.below((uint64_t)(2 * gl));
                t[a++] = swb_anchor{x, rid_of(x), 0};
            }
            uint32_t b = 0;
            if (r.uniform() < hit_frac) {
                // opposite strand at FR distance ins: p2 = rb + ins, m.rb = 2gl - 1 - p2
                const int64_t p2 = rb + ins;
                const int64_t mrb = 2 * gl - 1 - p2;
                if (mrb >= 0 && mrb < 2 * gl) mr[b++] = swb_anchor{mrb, rid_of(mrb), 0};
            }
            const int decoys = (int)r.below(3);
            for (int k = 0; k < decoys; ++k) {
                const int64_t x = (int64_t)r.below((uint64_t)(2 * gl));
                if (b < 3) mr[b++] = swb_anchor{x, rid_of(x), 0};
            }
            nt[i] = a;
            nm[i] = b;
            jobs[i] = swb_rescue_job{i * (uint64_t)mate_len, mate_len, 0, 0, a, 0, b};
        }
    });
    uint64_t to = 0, mo = 0;
    for (int64_t i = 0; i < n; ++i) {
        const swb_anchor *ts = tmpl + (size_t)i * 3, *ms = mreg + (size_t)i * 3;
        if (ts != tmpl + to) std::memmove(tmpl + to, ts, nt[(size_t)i] * sizeof(swb_anchor));
        if (ms != mreg + mo) std::memmove(mreg + mo, ms, nm[(size_t)i] * sizeof(swb_anchor));
        jobs[i].tmpl_off = (uint32_t)to;
        jobs[i].mreg_off = (uint32_t)mo;
        to += nt[(size_t)i];
        mo += nm[(size_t)i];
    }
    return (to << 32) | mo;
}

}  // extern "C"
