// swb_rescue.cu -- MateRescue.rescue for many mates
// (Sources/BWAMem/MateRescue.swift:29-171), device-resident:
//
//   rc       reverse complement of every mate (ReadSequence.reverseComplement)
//   count    one thread per job walks its templates x 4 orientations exactly
//            as the reference (failed orientation, hasMateHit, window,
//            clamp, fetchSequence's contig clamp, rid check, the
//            all-directions-satisfied break) and counts the local alignments
//   scan     exclusive sum of the counts = each job's first dense task
//   emit     the same walk writes the local-SW tasks (the window as a span of
//            the resident reference, reversed + complemented for the reverse
//            strand) and each task's coordinate mapping
//   kernel 3 the striped local SW with score2 (launch_local)
//   apply    one thread per job keeps the hits >= min_seed_len * a and maps
//            them back to BWT coordinates (:133-163), in candidate order.
#include <algorithm>
#include <string>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "swb_device.cuh"
#include "swb_internal.h"

namespace swb {
namespace {

struct CandMeta {
    int64_t clamped_begin;   // fetchSequence's clampedBegin (BWT coordinate)
    int32_t is_rev, rid;
};

struct RescueArgs {
    const swb_rescue_job *jobs;
    const swb_anchor *tmpl, *mreg;
    const int64_t *coff;
    const int32_t *clen;
    int n_contigs;
    swb_orientation st[4];
    int primary;
    int64_t gl;
    uint64_t rc_base;        // offset of the reverse-complemented mates in the bases buffer
    int32_t min_score;
    size_t n_jobs;
    uint32_t *n_cand;        // count pass: per job; emit pass: read
    const unsigned long long *cand_base;
    swb_local_task *tasks;
    CandMeta *meta;
};

__device__ int32_t sequence_id(const int64_t *off, int n, int64_t pos) {     // ReferenceMetadata.swift:77-89
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (off[mid] <= pos) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ bool has_mate_hit(const swb_anchor *m, uint32_t nm, const swb_anchor &t, int dir,
                             const swb_orientation &st, int64_t gl) {        // MateRescue.swift:319-346
    for (uint32_t k = 0; k < nm; ++k) {
        const swb_anchor r = m[k];
        if (r.rid != t.rid) continue;
        const bool same = (t.rb >= gl) == (r.rb >= gl);
        const int64_t p2 = same ? r.rb : (2 * gl - 1 - r.rb);
        const int bwaDir = (same ? 0 : 1) ^ (p2 > t.rb ? 0 : 3);
        if (bwaDir != dir) continue;
        const int64_t d = p2 > t.rb ? p2 - t.rb : t.rb - p2;
        if (d >= st.proper_low && d <= st.proper_high) return true;
    }
    return false;
}

template <bool EMIT>
__global__ void rescue_cand_kernel(RescueArgs a) {
    const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (j >= a.n_jobs) return;
    const swb_rescue_job jb = a.jobs[j];
    uint32_t c = 0;
    const unsigned long long base = EMIT ? a.cand_base[j] : 0ull;
    if (jb.n_tmpl > 0 && !a.st[a.primary].failed) {                          // :40-44
        const int64_t mateLen = jb.mate_len;
        for (uint32_t ti = 0; ti < jb.n_tmpl; ++ti) {
            const swb_anchor t = a.tmpl[jb.tmpl_off + ti];
            bool allSatisfied = true;
            for (int r = 0; r < 4; ++r) {
                const swb_orientation os = a.st[r];
                if (os.failed) continue;
                if (has_mate_hit(a.mreg + jb.mreg_off, jb.n_mreg, t, r, os, a.gl)) continue;
                allSatisfied = false;
                const bool isRev = (r >> 1) != (r & 1), isLarger = (r >> 1) == 0;   // :70-99
                int64_t rb, re;
                if (!isRev) {
                    if (isLarger) {
                        rb = t.rb + os.proper_low;
                        re = t.rb + os.proper_high + mateLen;
                    } else {
                        rb = t.rb - os.proper_high - mateLen;
                        re = t.rb - os.proper_low;
                    }
                } else {
                    if (isLarger) {
                        rb = t.rb + os.proper_low - mateLen;
                        re = t.rb + os.proper_high;
                    } else {
                        rb = t.rb - os.proper_high;
                        re = t.rb - os.proper_low + mateLen;
                    }
                }
                rb = rb > 0 ? rb : 0;                                           // :104-106
                re = re < 2 * a.gl ? re : 2 * a.gl;
                if (!(rb < re)) continue;
                // fetchSequence (PackedReference.swift:73-121)
                const bool rev_strand = rb >= a.gl;
                const int64_t fb = rev_strand ? 2 * a.gl - re : rb, fe = rev_strand ? 2 * a.gl - rb : re;
                const int32_t rid = sequence_id(a.coff, a.n_contigs, fb);
                const int64_t chromEnd = a.coff[rid] + (int64_t)a.clen[rid];
                const int64_t cb = fb > a.coff[rid] ? fb : a.coff[rid], ce = fe < chromEnd ? fe : chromEnd;
                if (!(cb < ce)) continue;
                if (rid != t.rid) continue;
                if (EMIT) {
                    const unsigned long long k = base + c;
                    a.tasks[k] = swb_local_task{isRev ? a.rc_base + jb.mate_off : jb.mate_off, (uint64_t)cb,
                                                jb.mate_len, (int32_t)(ce - cb), a.min_score,
                                                SWB_T_FROM_REF | (rev_strand ? (SWB_T_REVERSE | SWB_T_COMPLEMENT) : 0u)};
                    a.meta[k] = CandMeta{rev_strand ? 2 * a.gl - ce : cb, isRev ? 1 : 0, t.rid};
                }
                ++c;
            }
            if (allSatisfied) break;
        }
    }
    if (!EMIT) a.n_cand[j] = c;
}

__global__ void rescue_rc_kernel(const swb_rescue_job *__restrict__ jobs, size_t n_jobs, uint8_t *bases,
                                 uint64_t rc_base) {
    const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (j >= n_jobs) return;
    const swb_rescue_job jb = jobs[j];
    const uint8_t *src = bases + jb.mate_off;
    uint8_t *dst = bases + rc_base + jb.mate_off;
    for (int k = 0; k < jb.mate_len; ++k) {
        const uint8_t b = src[jb.mate_len - 1 - k];
        dst[k] = b < 4 ? (uint8_t)(3 - b) : (uint8_t)4;
    }
}

__global__ void rescue_apply_kernel(RescueArgs a, const swb_local_result *__restrict__ res, swb_rescued *__restrict__ out,
                                    uint32_t *__restrict__ n_out) {
    const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (j >= a.n_jobs) return;
    const swb_rescue_job jb = a.jobs[j];
    const unsigned long long base = a.cand_base[j];
    const uint32_t nc = a.n_cand[j];
    swb_rescued *o = out + 4 * (size_t)jb.tmpl_off;
    uint32_t k = 0;
    for (uint32_t c = 0; c < nc; ++c) {
        const swb_local_result sw = res[base + c];
        if (sw.score == 0 || !(sw.score >= a.min_score)) continue;              // nil, then :130
        const CandMeta m = a.meta[base + c];
        swb_rescued g{};
        g.score = sw.score;
        g.true_score = sw.score;
        g.csub = sw.score2;
        g.rid = m.rid;
        const int64_t tb = sw.tb, te = sw.te;
        if (!m.is_rev) {                                                          // :146-158
            g.rb = m.clamped_begin + tb;
            g.re = m.clamped_begin + te + 1;
            g.qb = sw.qb;
            g.qe = sw.qe + 1;
        } else {
            g.rb = 2 * a.gl - (m.clamped_begin + te + 1);
            g.re = 2 * a.gl - (m.clamped_begin + tb);
            g.qb = jb.mate_len - (sw.qe + 1);
            g.qe = jb.mate_len - sw.qb;
        }
        const int64_t refSpan = te - tb + 1, querySpan = (int64_t)(sw.qe - sw.qb + 1);   // :161-163
        g.seed_cov = (int32_t)((refSpan < querySpan ? refSpan : querySpan) / 2);
        o[k++] = g;
    }
    n_out[j] = k;
}

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" int swb_mate_rescue(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                               const swb_rescue_job *jobs, size_t n_jobs, const swb_anchor *templates,
                               size_t n_templates, const swb_anchor *mate_regions, size_t n_mate_regions,
                               const swb_orientation stats[4], int32_t primary, const int64_t *contig_offsets,
                               const int32_t *contig_lengths, size_t n_contigs, uint64_t genome_len, swb_rescued *out,
                               uint32_t *n_out, uint32_t *n_cand) {
    if (!ctx || (!bases && n_bases) || (!jobs && n_jobs) || (!templates && n_templates) ||
        (!mate_regions && n_mate_regions) || !stats || (!out && n_templates) || (!n_out && n_jobs))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    if (n_jobs == 0) return SWB_OK;
    if (primary < 0 || primary > 3) return set_error(SWB_ERR_INVALID_ARG, "primary orientation outside 0..3");
    if (n_contigs == 0 || n_contigs > 0x7FFFFFFF || !contig_offsets || !contig_lengths)
        return set_error(SWB_ERR_INVALID_ARG, "need at least one contig");
    for (size_t i = 0; i < n_contigs; ++i)
        if (contig_lengths[i] < 0 || (i && contig_offsets[i] <= contig_offsets[i - 1]) || contig_offsets[i] < 0)
            return set_error(SWB_ERR_INVALID_ARG, "contig offsets must ascend and lengths be >= 0");
    if (!ctx->d_pac || genome_len > ctx->ref_bases)
        return set_error(SWB_ERR_NO_REFERENCE, "the forward strand (genome_len bases) must be uploaded first");
    if ((uint64_t)contig_offsets[n_contigs - 1] + (uint64_t)contig_lengths[n_contigs - 1] > genome_len)
        return set_error(SWB_ERR_INVALID_ARG, "contigs run past genome_len");
    if (4 * (uint64_t)n_templates > 0x7FFFFFF0ull || n_jobs > 0x7FFFFFF0ull)
        return set_error(SWB_ERR_TOO_LARGE, "more than 2^29 template regions or 2^31 jobs");
    int max_q = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        const swb_rescue_job &jb = jobs[j];
        if (jb.mate_len < 0 || jb.mate_len > kMaxLen || jb.mate_off + (uint64_t)jb.mate_len > n_bases ||
            (uint64_t)jb.tmpl_off + jb.n_tmpl > n_templates || (uint64_t)jb.mreg_off + jb.n_mreg > n_mate_regions)
            return set_error(SWB_ERR_INVALID_ARG, "job " + std::to_string(j) + ": ranges outside the inputs");
        max_q = std::max(max_q, jb.mate_len);
    }
    // Longest window: proper_high - proper_low + mate length over the orientations in use.
    int64_t max_win = 0;
    for (int r = 0; r < 4; ++r)
        if (!stats[r].failed) {
            if (stats[r].proper_high < stats[r].proper_low)
                return set_error(SWB_ERR_INVALID_ARG, "orientation with proper_high < proper_low");
            max_win = std::max<int64_t>(max_win, stats[r].proper_high - stats[r].proper_low + max_q);
        }
    if (max_win > kMaxLen) return set_error(SWB_ERR_TOO_LARGE, "rescue window longer than 65535 bases");

    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t nj = n_jobs, nt = std::max<size_t>(n_templates, 1), nmr = std::max<size_t>(n_mate_regions, 1);
    const uint64_t rc_base = al256(std::max<size_t>(n_bases, 1));
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off += al256(bytes);
        return o;
    };
    const size_t o_jobs = carve(nj * sizeof(swb_rescue_job)), o_tmpl = carve(nt * sizeof(swb_anchor));
    const size_t o_mreg = carve(nmr * sizeof(swb_anchor)), o_coff = carve(n_contigs * 8), o_clen = carve(n_contigs * 4);
    const size_t o_ncand = carve(nj * 8), o_cbase = carve(nj * 8), o_nout = carve(nj * 4);
    const size_t o_out = carve(4 * nt * sizeof(swb_rescued));
    if ((rc = ensure_dev(ctx, ctx->d_chain, off)) || (rc = ensure_dev(ctx, ctx->d_bases, 2 * rc_base))) return rc;
    char *base = (char *)ctx->d_chain.p;
    uint8_t *d_b = (uint8_t *)ctx->d_bases.p;
    SWB_CUDA(cudaMemsetAsync(ctx->d_counters, 0, sizeof(unsigned long long) * kNumCounters, st));
    SWB_CUDA(cudaEventRecord(ctx->ev_start, st));
    if (n_bases) SWB_CUDA(cudaMemcpyAsync(d_b, bases, n_bases, cudaMemcpyHostToDevice, st));
    SWB_CUDA(cudaMemcpyAsync(base + o_jobs, jobs, nj * sizeof(swb_rescue_job), cudaMemcpyHostToDevice, st));
    if (n_templates)
        SWB_CUDA(cudaMemcpyAsync(base + o_tmpl, templates, n_templates * sizeof(swb_anchor), cudaMemcpyHostToDevice, st));
    if (n_mate_regions)
        SWB_CUDA(cudaMemcpyAsync(base + o_mreg, mate_regions, n_mate_regions * sizeof(swb_anchor), cudaMemcpyHostToDevice,
                                 st));
    SWB_CUDA(cudaMemcpyAsync(base + o_coff, contig_offsets, n_contigs * 8, cudaMemcpyHostToDevice, st));
    SWB_CUDA(cudaMemcpyAsync(base + o_clen, contig_lengths, n_contigs * 4, cudaMemcpyHostToDevice, st));

    RescueArgs ra{};
    ra.jobs = (const swb_rescue_job *)(base + o_jobs);
    ra.tmpl = (const swb_anchor *)(base + o_tmpl);
    ra.mreg = (const swb_anchor *)(base + o_mreg);
    ra.coff = (const int64_t *)(base + o_coff);
    ra.clen = (const int32_t *)(base + o_clen);
    ra.n_contigs = (int)n_contigs;
    for (int r = 0; r < 4; ++r) ra.st[r] = stats[r];
    ra.primary = primary;
    ra.gl = (int64_t)genome_len;
    ra.rc_base = rc_base;
    ra.min_score = sc->min_seed_len * sc->a;
    ra.n_jobs = nj;
    uint32_t *d_ncand32 = (uint32_t *)(base + o_ncand);
    unsigned long long *d_cbase = (unsigned long long *)(base + o_cbase);
    ra.n_cand = d_ncand32;
    ra.cand_base = d_cbase;
    const unsigned tb = 128, grid = (unsigned)((nj + tb - 1) / tb);
    {
        ProfScope ps(ctx, st, "rescue_candidates", -1);
        rescue_rc_kernel<<<grid, tb, 0, st>>>(ra.jobs, nj, d_b, rc_base);
        rescue_cand_kernel<false><<<grid, tb, 0, st>>>(ra);
        ctx->launches += 2;
        SWB_CUDA(cudaGetLastError());
    }
    size_t tmp = 0;
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_ncand32, d_cbase, (int)nj, st));
    if ((rc = ensure_dev(ctx, ctx->d_sort_tmp, tmp))) return rc;
    SWB_CUDA(cub::DeviceScan::ExclusiveSum(ctx->d_sort_tmp.p, tmp, d_ncand32, d_cbase, (int)nj, st));
    unsigned long long last_base = 0;
    uint32_t last_n = 0;
    SWB_CUDA(cudaMemcpyAsync(&last_base, d_cbase + (nj - 1), 8, cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaMemcpyAsync(&last_n, d_ncand32 + (nj - 1), 4, cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaStreamSynchronize(st));
    const size_t n_tasks = (size_t)last_base + last_n;
    const size_t nn = std::max<size_t>(n_tasks, 1);
    if ((rc = ensure_dev(ctx, ctx->d_tasks, nn * sizeof(swb_local_task) + al256(nn * sizeof(CandMeta)) + 256)) ||
        (rc = ensure_dev(ctx, ctx->d_out, nn * sizeof(swb_local_result))))
        return rc;
    ra.tasks = (swb_local_task *)ctx->d_tasks.p;
    ra.meta = (CandMeta *)((char *)ctx->d_tasks.p + al256(nn * sizeof(swb_local_task)));
    if (n_tasks) {
        {
            ProfScope ps(ctx, st, "rescue_candidates", -1);
            rescue_cand_kernel<true><<<grid, tb, 0, st>>>(ra);
            ctx->launches++;
            SWB_CUDA(cudaGetLastError());
        }
        if ((rc = launch_local(ctx, make_dev_scoring(*sc), d_b, ra.tasks, n_tasks, (swb_local_result *)ctx->d_out.p,
                               ctx->d_counters, st, std::max(max_q, 1), (int)std::max<int64_t>(max_win, 1))))
            return rc;
    }
    swb_rescued *d_out = (swb_rescued *)(base + o_out);
    uint32_t *d_nout = (uint32_t *)(base + o_nout);
    {
        ProfScope ps(ctx, st, "rescue_apply", -1);
        rescue_apply_kernel<<<grid, tb, 0, st>>>(ra, (const swb_local_result *)ctx->d_out.p, d_out, d_nout);
        ctx->launches++;
        SWB_CUDA(cudaGetLastError());
    }
    if (n_templates) SWB_CUDA(cudaMemcpyAsync(out, d_out, 4 * n_templates * sizeof(swb_rescued), cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaMemcpyAsync(n_out, d_nout, nj * 4, cudaMemcpyDeviceToHost, st));
    if (n_cand) SWB_CUDA(cudaMemcpyAsync(n_cand, d_ncand32, nj * 4, cudaMemcpyDeviceToHost, st));
    SWB_CUDA(cudaEventRecord(ctx->ev_stop, st));
    SWB_CUDA(cudaStreamSynchronize(st));
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
