// swb_cigar.cu -- CIGARGenerator.generate for a batch
// (Sources/Alignment/CIGARGenerator.swift:30-111), device-resident:
//
//   host     band inference (inferBandWidth) and the pure-M fast-path test
//            per task; the tasks needing DP become banded global tasks
//   kernel 2 the banded global alignments with the band-doubling retries
//            (launch_global), raw CIGARs in device scratch
//   measure  per task: deletion squeeze, NM, MD and soft clips walked once to
//            size the final CIGAR and MD (CIGARGenerator.postProcess :118-142)
//   scan     exclusive sums of the sizes give compact output offsets
//   emit     the same walk again, writing the CIGAR words and MD bytes
//
// Only the results and the compact CIGAR / MD bytes come back to the host.
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "swb_device.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

enum : uint32_t { kOpM = 0, kOpI = 1, kOpD = 2, kOpS = 4 };

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

struct PostArgs {
    const uint8_t *bases;
    const uint8_t *pac;
    const swb_cigar_task *tasks;
    const int32_t *dp_index;              // -1: fast path
    const swb_global_result *gres;
    const uint32_t *raw;                  // raw CIGARs of the DP tasks
    swb_cigar_result *res;
    unsigned long long *cig_len, *md_len; // measure: sizes; emit: compact offsets (after the scans)
    uint32_t *cig_out;
    char *md_out;
    size_t n;
};

__device__ const char kBaseChar[5] = {'A', 'C', 'G', 'T', 'N'};

// Decimal digits of v (v >= 0), written at p when EMIT.
template <bool EMIT>
__device__ __forceinline__ int put_uint(char *p, unsigned long long v) {
    char tmp[20];
    int n = 0;
    do {
        tmp[n++] = (char)('0' + (int)(v % 10));
        v /= 10;
    } while (v);
    if (EMIT)
        for (int i = 0; i < n; ++i) p[i] = tmp[n - 1 - i];
    return n;
}

// Squeeze (squeezeDeletions :272-295), NM (:173-210), MD (:219-268) and
// soft clips (addSoftClips :298-320) of one task.
template <bool EMIT>
__global__ void cigar_post_kernel(PostArgs a) {
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const swb_cigar_task t = a.tasks[k];
    const int32_t di = a.dp_index[k];
    uint32_t one = ((uint32_t)t.qlen << 4) | kOpM;   // fast path: a single M run (:69-80)
    const uint32_t *ops = &one;
    int n_ops = 1, score = t.true_score;
    long lead = 0, trail = 0;
    int64_t pos_adj = 0;
    if (di >= 0) {
        const swb_global_result g = a.gres[di];
        ops = a.raw + g.cigar_off;
        n_ops = g.n_cigar;
        score = g.score;
        while (lead < n_ops && (ops[lead] & 0xF) == kOpD) pos_adj += ops[lead++] >> 4;
        while (n_ops - trail > lead && (ops[n_ops - 1 - trail] & 0xF) == kOpD) ++trail;
    }
    const size_t ref_off = (size_t)pos_adj;
    const int qn = t.qlen, rn = t.rlen;
    uint32_t *cig = nullptr;
    char *md = nullptr;
    if (EMIT) {
        cig = a.cig_out + a.cig_len[k];
        md = a.md_out + a.md_len[k];
    }
    long front, back;
    if (t.is_reverse) {
        front = (long)t.read_len - t.qe;
        back = t.qb;
    } else {
        front = t.qb;
        back = (long)t.read_len - t.qe;
    }
    int nc = 0;
    if (front > 0) {
        if (EMIT) cig[nc] = ((uint32_t)front << 4) | kOpS;
        ++nc;
    }
    size_t qi = 0, ti = ref_off;
    int32_t nm = 0;
    unsigned long long match = 0;
    long mdn = 0;
    for (long o = lead; o < n_ops - trail; ++o) {
        const uint32_t c = ops[o];
        if (EMIT) cig[nc] = c;
        ++nc;
        const uint32_t op = c & 0xF;
        const size_t len = c >> 4;
        if (op == kOpM) {
            for (size_t x = 0; x < len; ++x)
                if (qi < (size_t)qn && ti < (size_t)rn) {
                    const uint32_t qb = span_base(a.bases, a.pac, t.q_off, (int)qi, qn, t.flags, false);
                    const uint32_t rb = span_base(a.bases, a.pac, t.t_off, (int)ti, rn, t.flags, true);
                    if (qb == rb) {
                        ++match;
                    } else {
                        ++nm;
                        mdn += put_uint<EMIT>(md + (EMIT ? mdn : 0), match);
                        if (EMIT) md[mdn] = kBaseChar[rb < 4 ? rb : 4];
                        ++mdn;
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
            mdn += put_uint<EMIT>(md + (EMIT ? mdn : 0), match);
            if (EMIT) md[mdn] = '^';
            ++mdn;
            for (size_t x = 0; x < len; ++x)
                if (ti < (size_t)rn) {
                    if (EMIT) {
                        const uint32_t rb = span_base(a.bases, a.pac, t.t_off, (int)ti, rn, t.flags, true);
                        md[mdn] = kBaseChar[rb < 4 ? rb : 4];
                    }
                    ++mdn;
                    ++ti;
                }
            match = 0;
        }
    }
    mdn += put_uint<EMIT>(md + (EMIT ? mdn : 0), match);
    if (back > 0) {
        if (EMIT) cig[nc] = ((uint32_t)back << 4) | kOpS;
        ++nc;
    }
    if (EMIT) {
        md[mdn] = '\0';
        swb_cigar_result r{};
        r.score = score;
        r.nm = nm;
        r.n_cigar = nc;
        r.md_len = (int32_t)mdn;
        r.pos = t.ref_pos + pos_adj;
        r.cigar_off = a.cig_len[k];
        r.md_off = a.md_len[k];
        r.used_dp = di >= 0;
        a.res[k] = r;
    } else {
        a.cig_len[k] = (unsigned long long)nc;
        a.md_len[k] = (unsigned long long)mdn + 1;
    }
}

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" int swb_cigar_batch(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                               const swb_cigar_task *tasks, size_t n_tasks, swb_cigar_result *results,
                               uint32_t *cigar_out, size_t cigar_cap, char *md_out, size_t md_cap) {
    if (!ctx || !sc || (!tasks && n_tasks) || (!results && n_tasks) || (!bases && n_bases) ||
        (!cigar_out && n_tasks) || (!md_out && n_tasks))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    if (n_tasks == 0) return SWB_OK;
    if (n_tasks > 0x7FFFFFF0ull) return set_error(SWB_ERR_TOO_LARGE, "more than 2^31-16 tasks in one batch");
    // One pass per host thread over a contiguous range: validation, the
    // capacity rule, the fast-path decision (:44-80) and, for the tasks that
    // need DP, the inferred band (:82-96), the band rule and the DP shapes.
    const size_t nth = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()),
                                        std::max<size_t>(1, n_tasks / 4096));
    struct Range {
        size_t lo = 0, hi = 0, nd = 0, dp0 = 0, raw = 0;
        int code = 0;
        std::string msg;
        size_t band_bad = SIZE_MAX;   // first task breaking the band rule
        unsigned long long cc = 0, cm = 0;
        GlobalShape shape;
    };
    std::vector<Range> rg(nth);
    std::vector<uint8_t> fast(n_tasks, 0);
    const int32_t min_indel = sc->o_ins + sc->e_ins + sc->o_del + sc->e_del;
    const bool have_ref = ctx->d_pac != nullptr;
    const int cost16 = nw_i16_cost(sc->a, sc->b, sc->o_del, sc->e_del, sc->o_ins, sc->e_ins);
    auto band_of = [&](const swb_cigar_task &t) {
        return std::max(infer_band_width(t.qe - t.qb, t.rlen, t.true_score, *sc), t.initial_w);
    };
    auto parallel = [&](auto &&fn) {
        if (nth == 1) return fn((size_t)0);
        std::vector<std::thread> th;
        for (size_t w = 0; w < nth; ++w) th.emplace_back(fn, w);
        for (auto &x : th) x.join();
    };
    {
        const size_t per = (n_tasks + nth - 1) / nth;
        parallel([&](size_t w) {
            Range &r = rg[w];
            r.lo = std::min(n_tasks, w * per);
            r.hi = std::min(n_tasks, r.lo + per);
            for (size_t i = r.lo; i < r.hi; ++i) {
                const swb_cigar_task &t = tasks[i];
                const char *why = nullptr;
                int code = SWB_ERR_INVALID_ARG;
                if (t.qlen < 0 || t.rlen < 0) why = "negative length";
                else if (t.qlen > kMaxLen || t.rlen > kMaxLen) why = "length above 65535", code = SWB_ERR_TOO_LARGE;
                else if (t.qlen > 0 && t.q_off + (uint64_t)t.qlen > n_bases) why = "query span outside bases";
                else if (t.rlen > 0 && (t.flags & SWB_T_FROM_REF) && !have_ref)
                    why = "task reads the reference but none is uploaded", code = SWB_ERR_NO_REFERENCE;
                else if (t.rlen > 0 && (t.flags & SWB_T_FROM_REF) && t.t_off + (uint64_t)t.rlen > ctx->ref_bases)
                    why = "reference span outside reference";
                else if (t.rlen > 0 && !(t.flags & SWB_T_FROM_REF) && t.t_off + (uint64_t)t.rlen > n_bases)
                    why = "reference span outside bases";
                if (why) {
                    r.code = code;
                    r.msg = "task " + std::to_string(i) + ": " + why;
                    return;
                }
                r.cc += (unsigned long long)t.qlen + (unsigned long long)t.rlen + 2;
                r.cm += 6ull * ((unsigned long long)t.qlen + (unsigned long long)t.rlen) + 8;
                const int32_t deficit = t.qlen * sc->a - t.true_score;
                fast[i] = t.qlen == t.rlen && t.qlen > 0 && deficit < min_indel;
                if (fast[i]) continue;
                if (r.band_bad == SIZE_MAX && t.qlen > 0 && t.rlen > 0 && std::max(band_of(t), std::abs(t.qlen - t.rlen)) < 1)
                    r.band_bad = i;
                ++r.nd;
                r.raw += (size_t)t.qlen + (size_t)t.rlen;
                r.shape.add(t.qlen, t.rlen, cost16);
            }
        });
    }
    unsigned long long need_c = 0, need_m = 0;
    for (const Range &r : rg) {
        if (r.code) return set_error(r.code, r.msg);
        need_c += r.cc;
        need_m += r.cm;
    }
    if (need_c > cigar_cap) return set_error(SWB_ERR_INVALID_ARG, "cigar_cap below sum of (qlen + rlen + 2)");
    if (need_m > md_cap) return set_error(SWB_ERR_INVALID_ARG, "md_cap below sum of (6*(qlen+rlen)+8)");
    size_t nd = 0, raw_words = 0;
    GlobalShape shape;
    for (Range &r : rg) {
        if (r.band_bad != SIZE_MAX)
            return set_error(SWB_ERR_INVALID_ARG, "task " + std::to_string(r.band_bad) + ": band width below 1 with equal lengths");
        r.dp0 = nd;
        nd += r.nd;
        raw_words += r.raw;
        shape.n_small += r.shape.n_small;
        shape.n_small16 += r.shape.n_small16;
        shape.n_big += r.shape.n_big;
        shape.small_q = std::max(shape.small_q, r.shape.small_q);
        shape.small_t = std::max(shape.small_t, r.shape.small_t);
        shape.big_q = std::max(shape.big_q, r.shape.big_q);
        shape.big_t = std::max(shape.big_t, r.shape.big_t);
    }

    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->last_ms = 0;
    ctx->last_cells = 0;
    SWB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t n = n_tasks;
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off += al256(bytes);
        return o;
    };
    const size_t o_bases = carve(std::max<size_t>(n_bases, 1)), o_tasks = carve(n * sizeof(swb_cigar_task));
    const size_t o_dpi = carve(n * 4), o_dp = carve(std::max<size_t>(nd, 1) * sizeof(swb_global_task));
    const size_t o_gres = carve(std::max<size_t>(nd, 1) * sizeof(swb_global_result));
    const size_t o_res = carve(n * sizeof(swb_cigar_result));
    const size_t o_cl = carve(n * 8), o_ml = carve(n * 8), o_co = carve(n * 8), o_mo = carve(n * 8);
    if ((rc = ensure_dev(ctx, ctx->d_chain, off)) ||
        (rc = ensure_dev(ctx, ctx->d_cigar, std::max<size_t>(raw_words, 1) * sizeof(uint32_t))) ||
        (rc = ensure_host(ctx, ctx->h_in, o_gres)))
        return rc;
    char *base = (char *)ctx->d_chain.p;
    unsigned long long *d_cl = (unsigned long long *)(base + o_cl), *d_ml = (unsigned long long *)(base + o_ml);
    unsigned long long *d_co = (unsigned long long *)(base + o_co), *d_mo = (unsigned long long *)(base + o_mo);
    // Inputs staged in pinned memory in the device layout (bases, tasks, DP
    // index, DP tasks) by the host threads, then one copy.  Bases and tasks
    // the caller already holds in pinned memory are copied from there
    // directly instead.
    const bool direct = n_bases > 0 && is_pinned(bases) && is_pinned(tasks);
    char *stage = (char *)ctx->h_in.p;
    {
        const size_t bper = (n_bases + nth - 1) / nth;
        parallel([&](size_t w) {
            const Range &r = rg[w];
            const size_t b0 = std::min(n_bases, w * bper), b1 = std::min(n_bases, b0 + bper);
            if (!direct && b1 > b0) std::memcpy(stage + o_bases + b0, bases + b0, b1 - b0);
            if (!direct && r.hi > r.lo)
                std::memcpy(stage + o_tasks + r.lo * sizeof(swb_cigar_task), tasks + r.lo,
                            (r.hi - r.lo) * sizeof(swb_cigar_task));
            int32_t *dpi = (int32_t *)(stage + o_dpi);
            swb_global_task *dp = (swb_global_task *)(stage + o_dp);
            size_t k = r.dp0;
            for (size_t i = r.lo; i < r.hi; ++i) {
                if (fast[i]) {
                    dpi[i] = -1;
                    continue;
                }
                const swb_cigar_task &t = tasks[i];
                dpi[i] = (int32_t)k;
                dp[k++] = swb_global_task{t.q_off, t.t_off, t.qlen, t.rlen, band_of(t), t.true_score,
                                          (t.flags & (SWB_Q_REVERSE | SWB_T_REVERSE | SWB_T_COMPLEMENT | SWB_T_FROM_REF)) |
                                              SWB_GLB_RETRY,
                                          0};
            }
        });
    }
    SWB_CUDA(cudaMemsetAsync(ctx->d_counters, 0, sizeof(unsigned long long) * kNumCounters, st));
    SWB_CUDA(cudaEventRecord(ctx->ev_start, st));
    if (direct) {
        SWB_CUDA(cudaMemcpyAsync(base + o_bases, bases, n_bases, cudaMemcpyHostToDevice, st));
        SWB_CUDA(cudaMemcpyAsync(base + o_tasks, tasks, n * sizeof(swb_cigar_task), cudaMemcpyHostToDevice, st));
        SWB_CUDA(cudaMemcpyAsync(base + o_dpi, stage + o_dpi, o_dp - o_dpi + nd * sizeof(swb_global_task),
                                 cudaMemcpyHostToDevice, st));
    } else {
        SWB_CUDA(cudaMemcpyAsync(base, stage, o_dp + nd * sizeof(swb_global_task), cudaMemcpyHostToDevice, st));
    }
    if (nd) {
        if ((rc = launch_global(ctx, make_dev_scoring(*sc), (const uint8_t *)(base + o_bases),
                                (const swb_global_task *)(base + o_dp), nd, (swb_global_result *)(base + o_gres),
                                (uint32_t *)ctx->d_cigar.p, ctx->d_counters, st, shape)))
            return rc;
    }
    PostArgs pa{(const uint8_t *)(base + o_bases), ctx->d_pac, (const swb_cigar_task *)(base + o_tasks),
                (const int32_t *)(base + o_dpi), (const swb_global_result *)(base + o_gres),
                (const uint32_t *)ctx->d_cigar.p, (swb_cigar_result *)(base + o_res), d_cl, d_ml, nullptr, nullptr, n};
    const unsigned tb = 128;
    const unsigned grid = (unsigned)((n + tb - 1) / tb);
    {
        ProfScope ps(ctx, st, "cigar_post_measure", -1);
        cigar_post_kernel<false><<<grid, tb, 0, st>>>(pa);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    // Compact offsets: exclusive sums of the sizes; each total is the last
    // offset plus the last size.
    size_t tmp = 0, tmp2 = 0;
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_cl, d_co, (int)n, st));
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, d_ml, d_mo, (int)n, st));
    if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, std::max(tmp, tmp2)))) return rc;
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(ctx->d_sort_tmp.p, tmp, d_cl, d_co, (int)n, st));
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(ctx->d_sort_tmp.p, tmp2, d_ml, d_mo, (int)n, st));
    unsigned long long last[4];
    SWB_CUDA(cudaMemcpyAsync(&last[0], d_co + (n - 1), 8, cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaMemcpyAsync(&last[1], d_cl + (n - 1), 8, cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaMemcpyAsync(&last[2], d_mo + (n - 1), 8, cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaMemcpyAsync(&last[3], d_ml + (n - 1), 8, cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaStreamSynchronize(st));
    const size_t tot_c = (size_t)(last[0] + last[1]), tot_m = (size_t)(last[2] + last[3]);
    if ((rc = ensure_dev(ctx, ctx->d_aux, al256(tot_c * 4) + al256(tot_m)))) return rc;
    uint32_t *d_cig = (uint32_t *)ctx->d_aux.p;
    char *d_md = (char *)ctx->d_aux.p + al256(tot_c * 4);
    pa.cig_len = d_co;
    pa.md_len = d_mo;
    pa.cig_out = d_cig;
    pa.md_out = d_md;
    {
        ProfScope ps(ctx, st, "cigar_post_emit", -1);
        cigar_post_kernel<true><<<grid, tb, 0, st>>>(pa);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    // Results, CIGAR words and MD bytes back: straight into the caller's
    // buffers when they are pinned, else through pinned staging and host
    // threads.
    const size_t r_bytes = n * sizeof(swb_cigar_result), c_bytes = tot_c * 4;
    const bool direct_out = is_pinned(results) && (tot_c == 0 || is_pinned(cigar_out)) && (tot_m == 0 || is_pinned(md_out));
    if (direct_out) {
        SWB_CUDA(cudaMemcpyAsync(results, base + o_res, r_bytes, cudaMemcpyDeviceToHost, st));
        if (tot_c) SWB_CUDA(cudaMemcpyAsync(cigar_out, d_cig, c_bytes, cudaMemcpyDeviceToHost, st));
        if (tot_m) SWB_CUDA(cudaMemcpyAsync(md_out, d_md, tot_m, cudaMemcpyDeviceToHost, st));
        SWB_CUDA(cudaEventRecord(ctx->ev_stop, st));
        SWB_CUDA(cudaStreamSynchronize(st));
    } else {
        if ((rc = ensure_host(ctx, ctx->h_out, al256(r_bytes) + al256(c_bytes) + al256(tot_m)))) return rc;
        char *back = (char *)ctx->h_out.p;
        SWB_CUDA(cudaMemcpyAsync(back, base + o_res, r_bytes, cudaMemcpyDeviceToHost, st));
        if (tot_c) SWB_CUDA(cudaMemcpyAsync(back + al256(r_bytes), d_cig, c_bytes, cudaMemcpyDeviceToHost, st));
        if (tot_m) SWB_CUDA(cudaMemcpyAsync(back + al256(r_bytes) + al256(c_bytes), d_md, tot_m, cudaMemcpyDeviceToHost, st));
        SWB_CUDA(cudaEventRecord(ctx->ev_stop, st));
        SWB_CUDA(cudaStreamSynchronize(st));
        parallel([&](size_t w) {
            auto part = [&](void *dst, const char *src, size_t bytes) {
                const size_t per = (bytes + nth - 1) / nth, a0 = std::min(bytes, w * per), a1 = std::min(bytes, a0 + per);
                if (a1 > a0) std::memcpy((char *)dst + a0, src + a0, a1 - a0);
            };
            part(results, back, r_bytes);
            part(cigar_out, back + al256(r_bytes), c_bytes);
            part(md_out, back + al256(r_bytes) + al256(c_bytes), tot_m);
        });
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) ctx->last_ms = ms;
    unsigned long long c[kNumCounters] = {0};
    if (cudaMemcpy(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) {
        unsigned long long sum = 0;
        for (int k = 0; k < kNumCounters; ++k) sum += c[k];
        ctx->last_cells = sum;
    }
    return SWB_OK;
}
