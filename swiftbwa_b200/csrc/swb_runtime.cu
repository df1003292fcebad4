// swb_runtime.cu -- context, device memory, staging and the C ABI of
// libswb_cuda.so (include/swb_cuda.h).
//
// Synchronous batch calls: each host array (bases, tasks) is copied straight
// from the caller's buffer with one cudaMemcpyAsync (full PCIe rate when the
// caller's memory is pinned), processed on the context's stream, and the
// results come back with one copy into the caller's output array.  Device
// buffers are grow-only and reused across calls; the context's budget caps
// what it may hold on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>

#include "swb_internal.h"

namespace swb {

int ext_big_max_q_range(const swb_ctx *ctx, const swb_ext_task *tasks, size_t lo, size_t hi, const DevScoring &sc);

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int check_cuda(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return set_error(SWB_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    }
    return set_error(SWB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int ensure_dev(swb_ctx *ctx, DevBuf &b, size_t bytes) {
    if (bytes <= b.cap) return SWB_OK;
    size_t want = std::max(bytes, b.cap + b.cap / 2);
    want = (want + 4095) & ~(size_t)4095;
    const size_t after = ctx->allocated - b.cap + want;
    if (after > ctx->budget) {
        want = (bytes + 4095) & ~(size_t)4095;
        if (ctx->allocated - b.cap + want > ctx->budget)
            return set_error(SWB_ERR_OOM, "device memory budget exceeded (" + std::to_string(ctx->allocated - b.cap + want) +
                                              " > " + std::to_string(ctx->budget) + " bytes)");
    }
    if (b.p) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(b.p);
        ctx->allocated -= b.cap;
        b.p = nullptr;
        b.cap = 0;
    }
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return check_cuda(e, "cudaMalloc");
    }
    b.cap = want;
    ctx->allocated += want;
    return SWB_OK;
}

int ensure_host(swb_ctx *ctx, HostBuf &b, size_t bytes) {
    (void)ctx;
    if (bytes <= b.cap) return SWB_OK;
    size_t want = std::max(bytes, b.cap + b.cap / 2);
    want = (want + 4095) & ~(size_t)4095;
    if (b.p) {
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    cudaError_t e = cudaMallocHost(&b.p, want);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return check_cuda(e, "cudaMallocHost");
    }
    b.cap = want;
    return SWB_OK;
}

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static void free_buf(swb_ctx *ctx, DevBuf &b) {
    if (b.p) cudaFree(b.p);
    ctx->allocated -= b.cap;
    b.p = nullptr;
    b.cap = 0;
}

int validate_scoring(const swb_scoring *sc) {
    if (!sc) return set_error(SWB_ERR_INVALID_ARG, "scoring is NULL");
    if (sc->e_ins <= 0 || sc->e_del <= 0 || sc->o_ins < 0 || sc->o_del < 0 || sc->a < 0 || sc->b < 0 ||
        sc->a > 127 || sc->b > 128)
        return set_error(SWB_ERR_INVALID_ARG,
                         "scoring: need e_ins, e_del > 0, o_* >= 0 and 0 <= a <= 127, 0 <= b <= 128");
    return SWB_OK;
}

// Checks spans against the bases buffer / reference and lengths against the
// caps; large batches are checked by several host threads.
template <class Task>
static int validate_range(const swb_ctx *ctx, const Task *tasks, size_t lo, size_t hi, size_t n_bases,
                          int *max_q, int *max_t, std::string *err, int *code) {
    int mq = 0, mt = 0;
    for (size_t i = lo; i < hi; ++i) {
        const Task &t = tasks[i];
        const char *why = nullptr;
        int c = SWB_ERR_INVALID_ARG;
        if (t.qlen < 0 || t.tlen < 0) {
            why = "negative length";
        } else if (t.qlen > kMaxLen || t.tlen > kMaxLen) {
            why = "length above 65535";
            c = SWB_ERR_TOO_LARGE;
        } else if (t.qlen > 0 && (t.q_off > n_bases || t.q_off + (uint64_t)t.qlen > n_bases)) {
            why = "query span outside bases";
        } else if (t.tlen > 0) {
            if (t.flags & SWB_T_FROM_REF) {
                if (!ctx->d_pac) {
                    why = "task reads the reference but none is uploaded";
                    c = SWB_ERR_NO_REFERENCE;
                } else if (t.t_off > ctx->ref_bases || t.t_off + (uint64_t)t.tlen > ctx->ref_bases) {
                    why = "target span outside reference";
                }
            } else if (t.t_off > n_bases || t.t_off + (uint64_t)t.tlen > n_bases) {
                why = "target span outside bases";
            }
        }
        if (why) {
            *err = "task " + std::to_string(i) + ": " + why;
            *code = c;
            return c;
        }
        mq = std::max(mq, t.qlen);
        mt = std::max(mt, t.tlen);
    }
    *max_q = mq;
    *max_t = mt;
    return SWB_OK;
}

template <class Task>
static int validate_spans(const swb_ctx *ctx, const Task *tasks, size_t n, size_t n_bases, int *max_q,
                          int *max_t) {
    const size_t kChunk = 1 << 18;
    const size_t nth = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), (n + kChunk - 1) / kChunk);
    std::vector<int> mq(nth, 0), mt(nth, 0), codes(nth, 0);
    std::vector<std::string> errs(nth);
    if (nth <= 1) {
        codes[0] = validate_range(ctx, tasks, 0, n, n_bases, &mq[0], &mt[0], &errs[0], &codes[0]);
    } else {
        std::vector<std::thread> th;
        const size_t per = (n + nth - 1) / nth;
        for (size_t k = 0; k < nth; ++k)
            th.emplace_back([&, k] {
                const size_t lo = k * per, hi = std::min(n, lo + per);
                if (lo < hi) codes[k] = validate_range(ctx, tasks, lo, hi, n_bases, &mq[k], &mt[k], &errs[k], &codes[k]);
            });
        for (auto &t : th) t.join();
    }
    for (size_t k = 0; k < nth; ++k)
        if (codes[k]) return set_error(codes[k], errs[k]);
    if (max_q) *max_q = *std::max_element(mq.begin(), mq.end());
    if (max_t) *max_t = *std::max_element(mt.begin(), mt.end());
    return SWB_OK;
}

// Copies each part straight from the caller's buffer (pinned or pageable)
// into one device region, one cudaMemcpyAsync per part; returns the device
// pointer of each part.
struct Part {
    const void *src;
    size_t bytes;
    void **dev;
};

}  // namespace swb

// Host memcpy on several host threads for large copies.
void swb::par_copy(void *dst, const void *src, size_t bytes) {
    const size_t kPart = 8u << 20;
    const size_t nth = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), bytes / kPart);
    if (nth <= 1) {
        if (bytes) std::memcpy(dst, src, bytes);
        return;
    }
    const size_t per = (bytes + nth - 1) / nth;
    std::vector<std::thread> th;
    for (size_t t = 0; t < nth; ++t)
        th.emplace_back([=] {
            const size_t a = std::min(bytes, t * per), b = std::min(bytes, a + per);
            if (b > a) std::memcpy((char *)dst + a, (const char *)src + a, b - a);
        });
    for (auto &x : th) x.join();
}

bool swb::is_pinned(const void *p) {
    if (!p) return false;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Parts whose destination is pinned are copied there directly; the rest go
// through the context's pinned staging buffer and host threads.
int swb::d2h_staged(swb_ctx *ctx, cudaStream_t st, std::initializer_list<DevSpan> parts, cudaEvent_t after_copies) {
    size_t total = 0;
    std::vector<bool> direct;
    for (const DevSpan &p : parts) {
        direct.push_back(p.bytes > 0 && is_pinned(p.dst));
        if (!direct.back()) total += align256(p.bytes);
    }
    int rc;
    if ((rc = ensure_host(ctx, ctx->h_out, std::max<size_t>(total, 256)))) return rc;
    char *stage = (char *)ctx->h_out.p;
    size_t off = 0, k = 0;
    for (const DevSpan &p : parts) {
        if (direct[k++]) {
            SWB_CUDA(cudaMemcpyAsync(p.dst, p.dev, p.bytes, cudaMemcpyDeviceToHost, st));
            continue;
        }
        if (p.bytes) SWB_CUDA(cudaMemcpyAsync(stage + off, p.dev, p.bytes, cudaMemcpyDeviceToHost, st));
        off += align256(p.bytes);
    }
    if (after_copies) SWB_CUDA(cudaEventRecord(after_copies, st));
    SWB_CUDA(cudaStreamSynchronize(st));
    off = 0, k = 0;
    for (const DevSpan &p : parts) {
        if (direct[k++]) continue;
        par_copy(p.dst, stage + off, p.bytes);
        off += align256(p.bytes);
    }
    return SWB_OK;
}

namespace swb {

// Inputs of one call into the context's device buffer.
static int stage_in(swb_ctx *ctx, std::initializer_list<Part> parts) {
    size_t total = 0;
    for (const Part &p : parts) total += align256(p.bytes);
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_bases, total + 256))) return rc;
    size_t off = 0;
    for (const Part &p : parts) {
        *p.dev = (char *)ctx->d_bases.p + off;
        if (p.bytes) SWB_CUDA(cudaMemcpyAsync(*p.dev, p.src, p.bytes, cudaMemcpyHostToDevice, ctx->stream));
        off += align256(p.bytes);
    }
    return SWB_OK;
}

struct Timer {
    swb_ctx *ctx;
    unsigned long long *d_cells;
    int begin() {
        d_cells = ctx->d_counters;
        SWB_CUDA(cudaMemsetAsync(d_cells, 0, sizeof(unsigned long long) * kNumCounters, ctx->stream));
        SWB_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
        return SWB_OK;
    }
    int end() {
        SWB_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
        return SWB_OK;
    }
    // After the stream synchronised.
    void collect() {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) ctx->last_ms = ms;
        unsigned long long c[kNumCounters] = {0};
        if (cudaMemcpy(c, d_cells, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) {
            unsigned long long sum = 0;
            for (int k = 0; k < kNumCounters; ++k) sum += c[k];
            ctx->last_cells = sum;
        }
    }
};

static cudaEvent_t pooled_event(swb_ctx *ctx) {
    if (ctx->ev_used == ctx->ev_pool.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        ctx->ev_pool.push_back(e);
    }
    return ctx->ev_pool[ctx->ev_used++];
}

ProfScope::ProfScope(swb_ctx *c, cudaStream_t st, const char *name, int counter) : ctx(c), s(st) {
    if (!ctx->prof_on || !name) return;
    cudaEvent_t a = pooled_event(ctx), b = pooled_event(ctx);
    if (!a || !b) return;
    ctx->prof.push_back(swb_ctx::ProfRec{name, counter, a, b});
    idx = (int)ctx->prof.size() - 1;
    cudaEventRecord(a, s);
}

ProfScope::~ProfScope() {
    if (idx >= 0) cudaEventRecord(ctx->prof[idx].b, s);
}

}  // namespace swb

using namespace swb;

namespace {

// Candidate length-class sets for a batch: the defaults, uniform steps, and
// quantiles of the shared-memory bins' row lengths (the query length, or for
// queries above 256 bases min(qlen, 2w+2) after the band clamp, ext_row_len)
// by task count and by estimated cells
// (qlen * min(tlen, 2w+1)), 6 to 15 classes, bounds rounded up to multiples
// of 8 and the last one covering the longest such row.
std::vector<ExtBins> ext_bin_candidates(const swb_ext_task *tasks, size_t n, const DevScoring &sc) {
    std::vector<ExtBins> out;
    auto add = [&](std::vector<int> q) {
        std::sort(q.begin(), q.end());
        q.erase(std::unique(q.begin(), q.end()), q.end());
        if (q.empty() || (int)q.size() > kMaxLenClasses) return;
        ExtBins b;
        b.n = (int)q.size();
        for (int k = 0; k < b.n; ++k) b.q[k] = q[k];
        for (const ExtBins &o : out)
            if (o.n == b.n && std::equal(o.q, o.q + o.n, b.q)) return;
        out.push_back(b);
    };
    const ExtBins dflt;
    add(std::vector<int>(dflt.q, dflt.q + dflt.n));
    std::vector<int> s16, s32;
    for (int q = 32; q <= kExtSmemMaxQ; q += 16) s16.push_back(q);
    for (int q = 32; q <= kExtSmemMaxQ; q += 32) s32.push_back(q);
    add(s16);
    add(s32);
    const bool pair_ok = sc.o_del + sc.e_del <= 32767 && sc.o_ins + sc.e_ins <= 32767;
    std::vector<std::pair<int, uint64_t>> ql;   // (row length, estimated cells) of the shared-memory bins' tasks
    const size_t step = std::max<size_t>(1, n / 200000);
    for (size_t i = 0; i < n; i += step) {
        const swb_ext_task &t = tasks[i];
        if (t.qlen <= 0 || t.tlen <= 0 || !pair_ok || t.qlen > kMaxLen || !fits16(t.qlen, t.h0, sc.max_mat)) continue;
        const int len = t.qlen <= kExtSmemMaxQ ? t.qlen : ext_row_len(t.qlen, ext_band_w(t.qlen, t.w, t.end_bonus, sc));
        if (len > kExtSmemMaxQ) continue;
        const uint64_t band = 2 * (uint64_t)std::max(t.w, 0) + 1;
        ql.push_back({len, (uint64_t)t.qlen * std::min<uint64_t>((uint64_t)t.tlen, band)});
    }
    if (ql.empty()) return out;
    std::sort(ql.begin(), ql.end());
    auto up8 = [](int q) { return std::min(kExtSmemMaxQ, std::max(16, (q + 7) / 8 * 8)); };
    const int top = up8(ql.back().first);
    uint64_t total = 0;
    for (auto &x : ql) total += x.second;
    for (int k : {6, 10, 15}) {
        std::vector<int> by_n, by_c;
        for (int j = 1; j < k; ++j) by_n.push_back(up8(ql[ql.size() * j / k].first));
        uint64_t acc = 0;
        int j = 1;
        for (auto &x : ql) {
            acc += x.second;
            while (j < k && acc * (uint64_t)k >= total * (uint64_t)j) {
                by_c.push_back(up8(x.first));
                ++j;
            }
        }
        by_n.push_back(top);
        by_c.push_back(top);
        add(by_n);
        add(by_c);
    }
    return out;
}

}  // namespace

extern "C" {

void swb_scoring_default(swb_scoring *s) {
    if (!s) return;
    *s = swb_scoring{1, 4, 6, 1, 6, 1, 100, 5, 5, 100, 19};
}

const char *swb_strerror(int status) {
    switch (status) {
    case SWB_OK: return "ok";
    case SWB_ERR_INVALID_ARG: return "invalid argument";
    case SWB_ERR_NO_DEVICE: return "no usable CUDA device";
    case SWB_ERR_CUDA: return "CUDA runtime error";
    case SWB_ERR_OOM: return "out of device memory or over budget";
    case SWB_ERR_TOO_LARGE: return "task exceeds the supported size";
    case SWB_ERR_NO_REFERENCE: return "no resident reference uploaded";
    case SWB_ERR_TIMEOUT: return "device wait timed out";
    case SWB_ERR_NOT_FOUND: return "unknown ticket";
    case SWB_ERR_KERNEL: return "kernel reported an internal check failure";
    default: return "unknown status";
    }
}

const char *swb_last_error_message(void) { return g_last_error.c_str(); }

int swb_init(int device, size_t mem_budget_bytes, swb_ctx **out) {
    if (!out) return set_error(SWB_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(SWB_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0 || device >= ndev) return set_error(SWB_ERR_INVALID_ARG, "device index out of range");
    cudaDeviceProp prop;
    SWB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return set_error(SWB_ERR_NO_DEVICE, std::string("device ") + prop.name + " is not sm_100 (built for sm_100a)");
    SWB_CUDA(cudaSetDevice(device));
    swb_ctx *ctx = new swb_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    ctx->budget = mem_budget_bytes ? mem_budget_bytes : free_b / 4 * 3;
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_counters, sizeof(unsigned long long) * kNumCounters);
    if (e == cudaSuccess) e = cudaMemset(ctx->d_counters, 0, sizeof(unsigned long long) * kNumCounters);
    for (int k = 0; k < kSideStreams && e == cudaSuccess; ++k) {
        e = cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->join_ev[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking);
    for (int k = 0; k < kMaxChunks && e == cudaSuccess; ++k) {
        e = cudaEventCreateWithFlags(&ctx->chunk_in[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->chunk_done[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_start);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_stop);
    if (e != cudaSuccess) {
        swb_destroy(ctx);
        return check_cuda(e, "stream/event create");
    }
    *out = ctx;
    return SWB_OK;
}

void swb_destroy(swb_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    DevBuf *bufs[] = {&ctx->d_bases, &ctx->d_tasks, &ctx->d_out, &ctx->d_keys, &ctx->d_keys2, &ctx->d_idx,
                      &ctx->d_idx2, &ctx->d_sort_tmp, &ctx->d_misc, &ctx->d_scratch, &ctx->d_cigar, &ctx->d_aux, &ctx->d_chain,
                      &ctx->d_bwt, &ctx->d_seed};
    for (DevBuf *b : bufs) free_buf(ctx, *b);
    if (ctx->d_pac && ctx->pac_owned) cudaFree(ctx->d_pac);
    if (ctx->d_counters) cudaFree(ctx->d_counters);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->h_in.p) cudaFreeHost(ctx->h_in.p);
    if (ctx->h_out.p) cudaFreeHost(ctx->h_out.p);
    if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
    if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
    for (int k = 0; k < kSideStreams; ++k) {
        if (ctx->side[k]) {
            cudaStreamSynchronize(ctx->side[k]);
            cudaStreamDestroy(ctx->side[k]);
        }
        if (ctx->join_ev[k]) cudaEventDestroy(ctx->join_ev[k]);
    }
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    for (cudaStream_t st : {ctx->h2d, ctx->d2h})
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    for (int k = 0; k < kMaxChunks; ++k) {
        if (ctx->chunk_in[k]) cudaEventDestroy(ctx->chunk_in[k]);
        if (ctx->chunk_done[k]) cudaEventDestroy(ctx->chunk_done[k]);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int swb_upload_reference(swb_ctx *ctx, const uint8_t *pac, uint64_t n_bases) {
    if (!ctx || (!pac && n_bases)) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)((n_bases + 3) / 4);
    if (ctx->d_pac) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->d_pac);
        ctx->allocated -= ctx->pac_bytes;
        ctx->d_pac = nullptr;
        ctx->pac_bytes = 0;
        ctx->ref_bases = 0;
    }
    if (n_bases == 0) return SWB_OK;
    if (ctx->allocated + bytes + 16 > ctx->budget) return set_error(SWB_ERR_OOM, "reference exceeds the memory budget");
    SWB_CUDA(cudaMalloc(&ctx->d_pac, bytes + 16));
    ctx->pac_bytes = bytes + 16;
    ctx->allocated += ctx->pac_bytes;
    SWB_CUDA(cudaMemcpy(ctx->d_pac, pac, bytes, cudaMemcpyHostToDevice));
    ctx->ref_bases = n_bases;
    return SWB_OK;
}

int swb_ext_batch(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                  const swb_ext_task *tasks, size_t n_tasks, swb_ext_result *out) {
    if (!ctx || (!tasks && n_tasks) || (!out && n_tasks) || (!bases && n_bases))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->last_ms = 0;
    ctx->last_cells = 0;
    if (n_tasks == 0) return SWB_OK;
    SWB_CUDA(cudaSetDevice(ctx->device));
    const DevScoring dsc = make_dev_scoring(*sc);

    // Large batches (8M tasks and up): chunks that grow by half from 1/32 of
    // the batch, so each chunk's copy (≈2.6 ns per config-1 task) ends within
    // the kernels of the one before (≈3.6 ns per task) and the GPU waits only
    // for the first, then two short chunks (6 % and 3 %) so that the last
    // pass and its copy back are short.  Smaller batches: up to eight equal
    // chunks of at least 512K tasks.  The host checks chunk k (spans, the
    // bases prefix it needs, the longest query of the int32 bin) while the
    // GPU works on the chunks before it; chunk k starts once the prefix of
    // `bases` its tasks reference is on the device.
    const size_t kMinChunk = 1u << 19;
    std::vector<size_t> cb{0};   // chunk k is tasks[cb[k], cb[k + 1])
    {
        static const double kGrow[] = {1.0 / 32, 0.078, 0.148, 0.254, 0.412, 0.65, 0.91, 0.97};   // cumulative
        if (n_tasks / 16 >= kMinChunk) {
            for (double f : kGrow) cb.push_back((size_t)(f * (double)n_tasks));
            cb.push_back(n_tasks);
        } else {
            const size_t m = std::min<size_t>(8, std::max<size_t>(1, n_tasks / kMinChunk)), p = (n_tasks + m - 1) / m;
            for (size_t k = 1; k <= m; ++k) cb.push_back(std::min(n_tasks, k * p));
        }
    }
    static_assert(kMaxChunks >= 9, "chunk events");
    const size_t nchunks = cb.size() - 1;
    size_t per = 0;   // the largest chunk (sizes the scratch sets)
    for (size_t k = 0; k < nchunks; ++k) per = std::max(per, cb[k + 1] - cb[k]);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    struct Part {
        int code = 0, big_q = 0;
        size_t need = 0;
        std::string err;
    };
    std::vector<Part> parts(hw);
    auto scan_chunk = [&](size_t lo, size_t hi, size_t &need, int &big_q) -> int {
        const size_t nth = std::min<size_t>(hw, std::max<size_t>(1, (hi - lo) / 16384));
        const size_t sub = (hi - lo + nth - 1) / nth;
        auto work = [&](size_t t) {
            Part &pt = parts[t];
            pt = Part{};
            const size_t a = lo + t * sub, b = std::min(hi, a + sub);
            if (a >= b) return;
            int mq, mt;
            if ((pt.code = validate_range(ctx, tasks, a, b, n_bases, &mq, &mt, &pt.err, &pt.code))) return;
            pt.big_q = ext_big_max_q_range(ctx, tasks, a, b, dsc);
            size_t m = 0;
            for (size_t i = a; i < b; ++i) {
                const swb_ext_task &tk = tasks[i];
                if (tk.qlen > 0) m = std::max<size_t>(m, tk.q_off + (size_t)tk.qlen);
                if (tk.tlen > 0 && !(tk.flags & SWB_T_FROM_REF)) m = std::max<size_t>(m, tk.t_off + (size_t)tk.tlen);
            }
            pt.need = m;
        };
        if (nth == 1) {
            work(0);
        } else {
            std::vector<std::thread> th;
            for (size_t t = 0; t < nth; ++t) th.emplace_back(work, t);
            for (auto &x : th) x.join();
        }
        for (size_t t = 0; t < nth; ++t) {
            if (parts[t].code) return set_error(parts[t].code, parts[t].err);
            need = std::max(need, parts[t].need);
            big_q = std::max(big_q, parts[t].big_q);
        }
        return SWB_OK;
    };
    const size_t bases_bytes = align256(std::max<size_t>(n_bases, 1));
    if ((rc = ensure_dev(ctx, ctx->d_bases, bases_bytes + align256(n_tasks * sizeof(swb_ext_task)) + 256))) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_out, n_tasks * sizeof(swb_ext_result)))) return rc;
    uint8_t *d_b = (uint8_t *)ctx->d_bases.p;
    swb_ext_task *d_t = (swb_ext_task *)((char *)ctx->d_bases.p + bases_bytes);
    swb_ext_result *d_o = (swb_ext_result *)ctx->d_out.p;
    // Sort and bin scratch for two chunks in flight, sized before the first
    // launch (growing a buffer synchronizes).
    if ((rc = ext_reserve(ctx, per))) return rc;
    Timer tm{ctx, nullptr};
    if ((rc = tm.begin())) return rc;
    // Copies must not overtake work still using these buffers.
    SWB_CUDA(cudaEventRecord(ctx->fork_ev, ctx->stream));
    SWB_CUDA(cudaStreamWaitEvent(ctx->h2d, ctx->fork_ev, 0));
    SWB_CUDA(cudaStreamWaitEvent(ctx->d2h, ctx->fork_ev, 0));
    size_t copied = 0, need = 0, last = 0;
    for (size_t k = 0; k < nchunks; ++k) {
        const size_t lo = cb[k], hi = cb[k + 1];
        if (lo >= hi) break;
        int big_q = 0;
        if ((rc = scan_chunk(lo, hi, need, big_q))) {
            // Let the chunks already queued finish before reporting (they write `out`).
            cudaStreamSynchronize(ctx->d2h);
            cudaStreamSynchronize(ctx->stream);
            return rc;
        }
        if (need > copied) {
            SWB_CUDA(cudaMemcpyAsync(d_b + copied, bases + copied, need - copied, cudaMemcpyHostToDevice, ctx->h2d));
            copied = need;
        }
        SWB_CUDA(cudaMemcpyAsync(d_t + lo, tasks + lo, (hi - lo) * sizeof(swb_ext_task), cudaMemcpyHostToDevice, ctx->h2d));
        SWB_CUDA(cudaEventRecord(ctx->chunk_in[k], ctx->h2d));
        SWB_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->chunk_in[k], 0));
        // Chunk k reuses chunk k-2's scratch set: its bins must be done.  Chunk
        // k-1's bins may still run while chunk k sorts and starts its own.
        if (k >= 2) SWB_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->chunk_done[k - 2], 0));
        const ExtPipe pipe{(int)(k & 1), per, ctx->d2h};
        // Small batches take the one-launch form: with too few tasks to fill
        // the GPU, the sort and the per-bin launches cost more than they save.
        rc = n_tasks <= kExtPlainMaxTasks
                 ? launch_ext_plain(ctx, dsc, d_b, d_t + lo, hi - lo, d_o + lo, tm.d_cells, ctx->stream)
                 : launch_ext(ctx, dsc, d_b, d_t + lo, hi - lo, d_o + lo, tm.d_cells, ctx->stream, big_q, 0, &pipe);
        if (rc) {
            cudaStreamSynchronize(ctx->d2h);
            cudaStreamSynchronize(ctx->stream);
            return rc;
        }
        if (n_tasks <= kExtPlainMaxTasks) {   // the plain launch ran on the launching stream
            SWB_CUDA(cudaEventRecord(ctx->fork_ev, ctx->stream));
            SWB_CUDA(cudaStreamWaitEvent(ctx->d2h, ctx->fork_ev, 0));
        }
        // The D2H stream has waited for every bin of chunk k.
        SWB_CUDA(cudaEventRecord(ctx->chunk_done[k], ctx->d2h));
        SWB_CUDA(cudaMemcpyAsync(out + lo, d_o + lo, (hi - lo) * sizeof(swb_ext_result), cudaMemcpyDeviceToHost, ctx->d2h));
        last = k;
    }
    SWB_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->chunk_done[last], 0));
    if ((rc = tm.end())) return rc;
    SWB_CUDA(cudaStreamSynchronize(ctx->d2h));
    SWB_CUDA(cudaStreamSynchronize(ctx->stream));
    tm.collect();
    return SWB_OK;
}

int swb_set_ext_bins(swb_ctx *ctx, const int32_t *qmax, int n) {
    if (!ctx || !qmax) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    if (n < 1 || n > kMaxLenClasses)
        return set_error(SWB_ERR_INVALID_ARG, "between 1 and " + std::to_string(kMaxLenClasses) + " length classes");
    ExtBins b;
    b.n = n;
    for (int k = 0; k < n; ++k) {
        if (qmax[k] < 8 || qmax[k] > kExtSmemMaxQ || (k > 0 && qmax[k] <= qmax[k - 1]))
            return set_error(SWB_ERR_INVALID_ARG, "length classes must ascend strictly within [8, 256]");
        b.q[k] = qmax[k];
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->ext_bins = b;
    return SWB_OK;
}

int swb_get_ext_bins(swb_ctx *ctx, int32_t *qmax, int cap, int *n) {
    if (!ctx || !n || (!qmax && cap > 0)) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    *n = ctx->ext_bins.n;
    for (int k = 0; k < std::min(cap, ctx->ext_bins.n); ++k) qmax[k] = ctx->ext_bins.q[k];
    return SWB_OK;
}

int swb_tune_ext_bins(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                      const swb_ext_task *tasks, size_t n_tasks, int32_t *qmax_out, int cap, int *n_out,
                      float *best_ms, float *default_ms) {
    if (!ctx || !sc || (!tasks && n_tasks) || (!bases && n_bases)) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    {
        int mq = 0, mt = 0, code = 0;
        std::string err;
        if ((rc = validate_range(ctx, tasks, 0, n_tasks, n_bases, &mq, &mt, &err, &code))) return set_error(rc, err);
    }
    const DevScoring dsc = make_dev_scoring(*sc);
    const std::vector<ExtBins> cand = ext_bin_candidates(tasks, n_tasks, dsc);
    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    const ExtBins keep = ctx->ext_bins;
    // Any early return (a failed CUDA call) puts the caller's classes back.
    struct Restore {
        swb_ctx *c;
        ExtBins b;
        bool on = true;
        ~Restore() {
            if (on) c->ext_bins = b;
        }
    } restore{ctx, keep};
    float t_best = 0.f, t_default = 0.f;
    ExtBins best = keep;
    if (n_tasks > 0) {
        const size_t bases_bytes = align256(std::max<size_t>(n_bases, 1));
        if ((rc = ensure_dev(ctx, ctx->d_bases, bases_bytes + align256(n_tasks * sizeof(swb_ext_task)) + 256)) ||
            (rc = ensure_dev(ctx, ctx->d_out, n_tasks * sizeof(swb_ext_result))))
            return rc;
        uint8_t *d_b = (uint8_t *)ctx->d_bases.p;
        swb_ext_task *d_t = (swb_ext_task *)((char *)ctx->d_bases.p + bases_bytes);
        if (n_bases) SWB_CUDA(cudaMemcpyAsync(d_b, bases, n_bases, cudaMemcpyHostToDevice, ctx->stream));
        SWB_CUDA(cudaMemcpyAsync(d_t, tasks, n_tasks * sizeof(swb_ext_task), cudaMemcpyHostToDevice, ctx->stream));
        t_best = 1e30f;
        for (size_t c = 0; c < cand.size(); ++c) {
            ctx->ext_bins = cand[c];
            const int hint = ext_big_max_q_range(ctx, tasks, 0, n_tasks, dsc);
            float ms = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {   // a warm-up run, then the better of two
                float t = 0.f;
                SWB_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
                rc = launch_ext(ctx, dsc, d_b, d_t, n_tasks, (swb_ext_result *)ctx->d_out.p, ctx->d_counters, ctx->stream,
                                hint);
                if (rc) return rc;
                SWB_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
                SWB_CUDA(cudaEventSynchronize(ctx->ev_stop));
                SWB_CUDA(cudaEventElapsedTime(&t, ctx->ev_start, ctx->ev_stop));
                if (rep > 0 && t < ms) ms = t;
            }
            if (c == 0) t_default = ms;
            if (ms < t_best) {
                t_best = ms;
                best = cand[c];
            }
        }
        // Another set replaces the defaults only for a gain above the
        // run-to-run spread (2 %).
        if (!(t_best < 0.98f * t_default)) {
            best = cand.front();
            t_best = t_default;
        }
    }
    restore.on = false;
    ctx->ext_bins = best;
    if (n_out) *n_out = best.n;
    for (int k = 0; k < std::min(cap, best.n) && qmax_out; ++k) qmax_out[k] = best.q[k];
    if (best_ms) *best_ms = t_best;
    if (default_ms) *default_ms = t_default;
    return SWB_OK;
}

int swb_ext_batch_device(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *d_bases,
                         const swb_ext_task *d_tasks, size_t n_tasks, swb_ext_result *d_out,
                         void *stream) {
    if (!ctx || (!d_tasks && n_tasks) || (!d_out && n_tasks)) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (n_tasks == 0) return SWB_OK;
    SWB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    return launch_ext(ctx, make_dev_scoring(*sc), d_bases, d_tasks, n_tasks, d_out, ctx->d_counters, s, -1);
}

int swb_ext_batch_plain_device(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *d_bases,
                               const swb_ext_task *d_tasks, size_t n_tasks, swb_ext_result *d_out, void *stream) {
    if (!ctx || (!d_tasks && n_tasks) || (!d_out && n_tasks)) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (n_tasks == 0) return SWB_OK;
    SWB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    return launch_ext_plain(ctx, make_dev_scoring(*sc), d_bases, d_tasks, n_tasks, d_out, ctx->d_counters, s);
}

int swb_global_batch(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                     const swb_global_task *tasks, size_t n_tasks, swb_global_result *results,
                     uint32_t *cigar_out, size_t cigar_cap) {
    if (!ctx || (!tasks && n_tasks) || (!results && n_tasks) || (!bases && n_bases) || (!cigar_out && n_tasks))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->last_ms = 0;
    ctx->last_cells = 0;
    if (n_tasks == 0) return SWB_OK;
    int max_q = 0, max_t = 0;
    if ((rc = validate_spans(ctx, tasks, n_tasks, n_bases, &max_q, &max_t))) return rc;
    size_t need = 0;
    GlobalShape shape;
    const int cost16 = nw_i16_cost(sc->a, sc->b, sc->o_del, sc->e_del, sc->o_ins, sc->e_ins);
    for (size_t i = 0; i < n_tasks; ++i) {
        need += (size_t)tasks[i].qlen + (size_t)tasks[i].tlen;
        const swb_global_task &t = tasks[i];
        shape.add(t.qlen, t.tlen, cost16);
        if (t.qlen > 0 && t.tlen > 0 && std::max(t.w, std::abs(t.qlen - t.tlen)) < 1)
            return set_error(SWB_ERR_INVALID_ARG, "task " + std::to_string(i) + ": band width below 1 with equal lengths");
    }
    if (need > cigar_cap) return set_error(SWB_ERR_INVALID_ARG, "cigar_cap below sum of (qlen + tlen)");
    SWB_CUDA(cudaSetDevice(ctx->device));
    const DevScoring dsc = make_dev_scoring(*sc);
    void *d_b = nullptr, *d_t = nullptr;
    if ((rc = stage_in(ctx, {Part{bases, n_bases, &d_b}, Part{tasks, n_tasks * sizeof(swb_global_task), &d_t}}))) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_out, n_tasks * sizeof(swb_global_result)))) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_cigar, std::max<size_t>(need, 1) * sizeof(uint32_t)))) return rc;
    Timer tm{ctx, nullptr};
    if ((rc = tm.begin())) return rc;
    if ((rc = launch_global(ctx, dsc, (const uint8_t *)d_b, (const swb_global_task *)d_t, n_tasks,
                            (swb_global_result *)ctx->d_out.p, (uint32_t *)ctx->d_cigar.p, tm.d_cells,
                            ctx->stream, shape)))
        return rc;
    if ((rc = tm.end())) return rc;
    SWB_CUDA(cudaMemcpyAsync(results, ctx->d_out.p, n_tasks * sizeof(swb_global_result), cudaMemcpyDeviceToHost, ctx->stream));
    SWB_CUDA(cudaMemcpyAsync(cigar_out, ctx->d_cigar.p, std::max<size_t>(need, 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             ctx->stream));
    SWB_CUDA(cudaStreamSynchronize(ctx->stream));
    tm.collect();
    return SWB_OK;
}

int swb_local_batch(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                    const swb_local_task *tasks, size_t n_tasks, swb_local_result *out) {
    if (!ctx || (!tasks && n_tasks) || (!out && n_tasks) || (!bases && n_bases))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = validate_scoring(sc))) return rc;
    if (sc->o_ins + sc->e_ins > 255 || sc->e_ins > 255)
        return set_error(SWB_ERR_INVALID_ARG, "local SW: gap penalties must fit in 8 bits (UInt8(gapOE))");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->last_ms = 0;
    ctx->last_cells = 0;
    if (n_tasks == 0) return SWB_OK;
    int max_q = 0, max_t = 0;
    if ((rc = validate_spans(ctx, tasks, n_tasks, n_bases, &max_q, &max_t))) return rc;
    SWB_CUDA(cudaSetDevice(ctx->device));
    const DevScoring dsc = make_dev_scoring(*sc);
    void *d_b = nullptr, *d_t = nullptr;
    if ((rc = stage_in(ctx, {Part{bases, n_bases, &d_b}, Part{tasks, n_tasks * sizeof(swb_local_task), &d_t}}))) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_out, n_tasks * sizeof(swb_local_result)))) return rc;
    Timer tm{ctx, nullptr};
    if ((rc = tm.begin())) return rc;
    if ((rc = launch_local(ctx, dsc, (const uint8_t *)d_b, (const swb_local_task *)d_t, n_tasks,
                           (swb_local_result *)ctx->d_out.p, tm.d_cells, ctx->stream, max_q, max_t)))
        return rc;
    if ((rc = tm.end())) return rc;
    SWB_CUDA(cudaMemcpyAsync(out, ctx->d_out.p, n_tasks * sizeof(swb_local_result), cudaMemcpyDeviceToHost, ctx->stream));
    SWB_CUDA(cudaStreamSynchronize(ctx->stream));
    tm.collect();
    return SWB_OK;
}

int swb_banded_sw_align(swb_ctx *ctx, const uint8_t *query, int32_t qlen, const uint8_t *target,
                        int32_t tlen, const swb_scoring *sc, int32_t w, int32_t h0, int32_t end_bonus,
                        swb_ext_result *out) {
    if (!out || qlen < 0 || tlen < 0 || (!query && qlen) || (!target && tlen))
        return set_error(SWB_ERR_INVALID_ARG, "bad argument");
    std::string buf((size_t)qlen + (size_t)tlen + 1, '\0');
    if (qlen) std::memcpy(&buf[0], query, (size_t)qlen);
    if (tlen) std::memcpy(&buf[(size_t)qlen], target, (size_t)tlen);
    swb_ext_task t{0, (uint64_t)qlen, qlen, tlen, w, h0, end_bonus, 0u};
    return swb_ext_batch(ctx, sc, (const uint8_t *)buf.data(), buf.size(), &t, 1, out);
}

int swb_global_align(swb_ctx *ctx, const uint8_t *query, int32_t qlen, const uint8_t *target, int32_t tlen,
                     const swb_scoring *sc, int32_t w, int32_t *score, uint32_t *cigar, int32_t *n_cigar) {
    if (!score || !n_cigar || qlen < 0 || tlen < 0 || (!query && qlen) || (!target && tlen))
        return set_error(SWB_ERR_INVALID_ARG, "bad argument");
    if (*n_cigar < qlen + tlen || (!cigar && *n_cigar))
        return set_error(SWB_ERR_INVALID_ARG, "cigar capacity below qlen + tlen");
    std::string buf((size_t)qlen + (size_t)tlen + 1, '\0');
    if (qlen) std::memcpy(&buf[0], query, (size_t)qlen);
    if (tlen) std::memcpy(&buf[(size_t)qlen], target, (size_t)tlen);
    swb_global_task t{0, (uint64_t)qlen, qlen, tlen, w, 0, 0u, 0};
    swb_global_result r{};
    std::vector<uint32_t> tmp((size_t)qlen + (size_t)tlen + 1);
    int rc = swb_global_batch(ctx, sc, (const uint8_t *)buf.data(), buf.size(), &t, 1, &r, tmp.data(), tmp.size());
    if (rc) return rc;
    *score = r.score;
    std::copy(tmp.begin(), tmp.begin() + r.n_cigar, cigar);
    *n_cigar = r.n_cigar;
    return SWB_OK;
}

int swb_local_align(swb_ctx *ctx, const uint8_t *query, int32_t qlen, const uint8_t *target, int32_t tlen,
                    const swb_scoring *sc, int32_t min_sub_score, swb_local_result *out) {
    if (!out || qlen < 0 || tlen < 0 || (!query && qlen) || (!target && tlen))
        return set_error(SWB_ERR_INVALID_ARG, "bad argument");
    std::string buf((size_t)qlen + (size_t)tlen + 1, '\0');
    if (qlen) std::memcpy(&buf[0], query, (size_t)qlen);
    if (tlen) std::memcpy(&buf[(size_t)qlen], target, (size_t)tlen);
    swb_local_task t{0, (uint64_t)qlen, qlen, tlen, min_sub_score, 0u};
    return swb_local_batch(ctx, sc, (const uint8_t *)buf.data(), buf.size(), &t, 1, out);
}

uint64_t swb_kernel_launches(const swb_ctx *ctx) { return ctx ? ctx->launches : 0; }

int swb_profile(swb_ctx *ctx, int enable) {
    if (!ctx) return set_error(SWB_ERR_INVALID_ARG, "ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->prof_on = enable != 0;
    return SWB_OK;
}

int swb_profile_reset(swb_ctx *ctx) {
    if (!ctx) return set_error(SWB_ERR_INVALID_ARG, "ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    SWB_CUDA(cudaDeviceSynchronize());
    ctx->prof.clear();
    ctx->ev_used = 0;
    SWB_CUDA(cudaMemset(ctx->d_counters, 0, sizeof(unsigned long long) * kNumCounters));
    return SWB_OK;
}

int swb_profile_read(swb_ctx *ctx, swb_kernel_stat *stats, int cap, int *n_stats) {
    if (!ctx || !n_stats || (!stats && cap > 0)) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    SWB_CUDA(cudaDeviceSynchronize());
    unsigned long long c[kNumCounters] = {0};
    SWB_CUDA(cudaMemcpy(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    std::vector<swb_kernel_stat> out;
    std::vector<int> counters;
    for (const auto &r : ctx->prof) {
        float ms = 0.f;
        SWB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        int k = 0;
        while (k < (int)out.size() && std::strcmp(out[k].name, r.name) != 0) ++k;
        if (k == (int)out.size()) {
            swb_kernel_stat st{};
            std::strncpy(st.name, r.name, sizeof(st.name) - 1);
            out.push_back(st);
            counters.push_back(r.counter);
        }
        out[k].launches++;
        out[k].total_ms += ms;
    }
    for (size_t k = 0; k < out.size(); ++k)
        out[k].cells = counters[k] >= 0 ? c[counters[k]] : 0;
    *n_stats = (int)out.size();
    for (int k = 0; k < (int)out.size() && k < cap; ++k) stats[k] = out[k];
    return SWB_OK;
}

int swb_last_batch_stats(const swb_ctx *ctx, double *kernel_ms, uint64_t *cells) {
    if (!ctx) return set_error(SWB_ERR_INVALID_ARG, "ctx is NULL");
    if (kernel_ms) *kernel_ms = ctx->last_ms;
    if (cells) *cells = ctx->last_cells;
    return SWB_OK;
}

}  // extern "C"
