// swb_serve.cu -- continuous-batching request loop for extension batches.
//
// Requests (each: a bases buffer, extension tasks over it, an output array)
// are submitted from any host thread and answered asynchronously by ticket.
// One worker thread:
//   * admits requests in arrival order, staging each request's bases once
//     into a device arena (first-fit, arena_bytes), which is the admission
//     budget: a request whose bases do not fit waits until earlier ones free
//     their space;
//   * forms waves of at most max_wave_tasks tasks, taking requests by least
//     remaining work (those waiting longer than 50 ms first, by arrival) and
//     splitting large requests across waves, so that short requests do not
//     wait behind the waves of long ones;
//   * copies each piece of a wave straight from the caller's buffers when
//     they are pinned (the task offsets are then rebased into the arena by a
//     small kernel), or through a pinned bounce buffer when they are not;
//   * runs a wave as one sort + binned extension pass over all its tasks
//     (the launch sequence of swb_ext_batch), rotating over three lanes
//     -- internal contexts with their own streams and buffers sharing the
//     resident reference -- so one wave's copies overlap the other's kernels;
//   * copies each request's slice of a wave's results back (directly into a
//     pinned output, through a bounce buffer otherwise) and completes the
//     request when its last slice has landed.
// plain = 1 is the baseline of the same kernels: one request at a time, copy
// in, compute, copy out, synchronise.  plain = 2 also swaps the binned pass
// for the plain one-launch-per-batch kernel (launch_ext_plain: the same
// two-row code over the request in input order, no sort or bins).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>
#include <vector>

#include "swb_internal.h"

using namespace swb;

namespace {

constexpr int kMaxPieces = 4096;   // pieces (request slices) per wave
constexpr int kLanes = 3;          // waves in flight at once
constexpr uint64_t kAgeNs = 50'000'000;   // a request waiting longer than this is served in arrival order

inline size_t align_up256(size_t x) { return (x + 255) & ~(size_t)255; }

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Req {
    uint64_t ticket = 0;
    const uint8_t *bases = nullptr;
    size_t n_bases = 0;
    uint64_t origin = 0;
    const swb_ext_task *tasks = nullptr;
    size_t n = 0;
    swb_ext_result *out = nullptr;
    bool tasks_pinned = false, out_pinned = false;
    int max_q = 0;                       // longest query (sizes the int32 bin's scratch)
    size_t dispatched = 0, completed = 0;
    bool staged = false;
    size_t arena_off = 0, arena_len = 0;
    int status = SWB_OK;
    bool done = false;
    uint64_t t_submit = 0, t_done = 0;
};

struct Piece {
    Req *r;
    size_t lo, hi, woff;
};

// Device-side rebase of one piece of a wave: q_off and explicit t_off += delta.
struct RebasePiece {
    unsigned long long woff, n, delta;
};

__global__ void rebase_kernel(swb_ext_task *__restrict__ t, const RebasePiece *__restrict__ pieces) {
    const RebasePiece p = pieces[blockIdx.y];
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < p.n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        swb_ext_task &x = t[p.woff + i];
        x.q_off += p.delta;
        if (!(x.flags & SWB_T_FROM_REF)) x.t_off += p.delta;
    }
}

// First-fit allocator over the device arena (offsets, 256-byte granules).
struct Arena {
    size_t cap = 0;
    std::map<size_t, size_t> free_;   // offset -> length
    void init(size_t c) {
        cap = c;
        free_.clear();
        free_[0] = c;
    }
    bool alloc(size_t len, size_t *off) {
        len = align_up256(len);
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= len) {
                *off = it->first;
                const size_t rest = it->second - len, o = it->first + len;
                free_.erase(it);
                if (rest) free_[o] = rest;
                return true;
            }
        return false;
    }
    void release(size_t off, size_t len) {
        len = align_up256(len);
        auto it = free_.emplace(off, len).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Lane {
    swb_ctx *ctx = nullptr;
    swb_ext_task *h_stage = nullptr;        // pinned bounce buffer for pageable tasks
    swb_ext_result *h_out = nullptr;        // pinned bounce buffer for pageable outputs
    RebasePiece *h_pieces = nullptr;        // pinned piece table
    RebasePiece *d_pieces = nullptr;
    unsigned long long *h_cells = nullptr;  // pinned copy of the wave's cell counters
    cudaEvent_t ev_done = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    bool busy = false;
    std::vector<Piece> pieces;
    int launch_rc = SWB_OK;
};

}  // namespace

struct swb_server {
    swb_ctx *parent = nullptr;
    swb_scoring sc{};
    DevScoring dsc{};
    int plain = 0;
    size_t max_wave = 1u << 20;
    uint32_t latency_cells = 0;
    uint8_t *d_arena = nullptr;
    Arena arena;
    Lane lanes[kLanes];
    int next_lane = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> queue;
    std::unordered_map<uint64_t, Req *> reqs;
    uint64_t next_ticket = 1;
    bool stopping = false, paused = false;
    swb_server_stats stats{};
};

namespace {

void complete_wave(swb_server *s, Lane &L) {
    // Called with s->mu held, after L.ev_done completed.
    float ms = 0.f;
    cudaEventElapsedTime(&ms, L.ev_t0, L.ev_t1);
    s->stats.busy_ms += ms;
    unsigned long long cells = 0;
    for (int k = 0; k < kNumCounters; ++k) cells += L.h_cells[k];
    s->stats.cells += cells;
    s->stats.waves++;
    const uint64_t t = now_ns();
    for (const Piece &p : L.pieces) {
        Req *r = p.r;
        if (L.launch_rc != SWB_OK) r->status = L.launch_rc;
        if (!r->out_pinned && L.launch_rc == SWB_OK)
            std::memcpy(r->out + p.lo, L.h_out + p.woff, (p.hi - p.lo) * sizeof(swb_ext_result));
        r->completed += p.hi - p.lo;
        s->stats.tasks_completed += p.hi - p.lo;
        if (r->completed == r->n) {
            r->done = true;
            r->t_done = t;
            s->stats.completed++;
            if (r->staged && r->arena_len) s->arena.release(r->arena_off, r->arena_len);
            r->staged = false;
        }
    }
    L.pieces.clear();
    L.busy = false;
    s->cv_done.notify_all();
}

// Forms and launches one wave on lane L.  Called with s->mu held; returns
// false when nothing could be dispatched.
bool launch_wave(swb_server *s, Lane &L) {
    swb_ctx *c = L.ctx;
    // One copy stream for both lanes: a request split across waves on both
    // lanes has its bases copied once, and every later wave's task copy (and
    // so its kernels) is ordered after that copy.
    cudaStream_t h2d = s->lanes[0].ctx->h2d, st = c->stream, d2h = c->d2h;
    if (ensure_dev(c, c->d_tasks, s->max_wave * sizeof(swb_ext_task)) ||
        ensure_dev(c, c->d_out, s->max_wave * sizeof(swb_ext_result)))
        return false;
    swb_ext_task *d_tasks = (swb_ext_task *)c->d_tasks.p;
    swb_ext_result *d_out = (swb_ext_result *)c->d_out.p;
    size_t wn = 0;
    int npin = 0;
    bool host_staged = false;
    // Wave order: requests that have waited longer than kAgeNs first, by
    // arrival; then the others by least remaining work (so a short request
    // does not queue behind the waves of a long one).  Plain mode keeps the
    // arrival order, one request per wave.
    std::vector<Req *> order;
    order.reserve(s->queue.size());
    for (Req *r : s->queue)
        if (r->dispatched < r->n) order.push_back(r);
    if (!s->plain) {
        const uint64_t now = now_ns();
        std::stable_sort(order.begin(), order.end(), [&](const Req *x, const Req *y) {
            const bool ox = now - x->t_submit > kAgeNs, oy = now - y->t_submit > kAgeNs;
            if (ox != oy) return ox;
            if (ox) return false;   // both old: arrival order (the queue's)
            return x->n - x->dispatched < y->n - y->dispatched;
        });
    }
    for (Req *r : order) {
        if (wn >= s->max_wave || (int)L.pieces.size() >= kMaxPieces) break;
        if (r->dispatched == r->n) continue;
        if (!r->staged) {
            size_t off = 0;
            if (!s->arena.alloc(std::max<size_t>(r->n_bases, 1), &off)) break;   // admission: wait for space
            r->arena_off = off;
            r->arena_len = std::max<size_t>(r->n_bases, 1);
            r->staged = true;
            if (r->n_bases) cudaMemcpyAsync(s->d_arena + off, r->bases, r->n_bases, cudaMemcpyHostToDevice, h2d);
        }
        const size_t take = std::min(r->n - r->dispatched, s->max_wave - wn);
        const unsigned long long delta = (unsigned long long)r->arena_off - (unsigned long long)r->origin;
        if (r->tasks_pinned) {
            cudaMemcpyAsync(d_tasks + wn, r->tasks + r->dispatched, take * sizeof(swb_ext_task), cudaMemcpyHostToDevice, h2d);
            L.h_pieces[npin++] = RebasePiece{wn, take, delta};
        } else {
            for (size_t k = 0; k < take; ++k) {
                swb_ext_task t = r->tasks[r->dispatched + k];
                t.q_off += delta;
                if (!(t.flags & SWB_T_FROM_REF)) t.t_off += delta;
                L.h_stage[wn + k] = t;
            }
            host_staged = true;
        }
        L.pieces.push_back(Piece{r, r->dispatched, r->dispatched + take, wn});
        r->dispatched += take;
        wn += take;
        if (s->plain) break;
    }
    if (wn == 0) return false;
    int rc = SWB_OK;
    if (host_staged)
        for (const Piece &p : L.pieces)
            if (!p.r->tasks_pinned &&
                cudaMemcpyAsync(d_tasks + p.woff, L.h_stage + p.woff, (p.hi - p.lo) * sizeof(swb_ext_task),
                                cudaMemcpyHostToDevice, h2d) != cudaSuccess)
                rc = SWB_ERR_CUDA;
    if (!rc && npin) {
        cudaMemcpyAsync(L.d_pieces, L.h_pieces, npin * sizeof(RebasePiece), cudaMemcpyHostToDevice, h2d);
        size_t maxn = 0;
        for (int k = 0; k < npin; ++k) maxn = std::max<size_t>(maxn, L.h_pieces[k].n);
        const dim3 grid((unsigned)std::min<size_t>((maxn + 255) / 256, 1024), (unsigned)npin);
        rebase_kernel<<<grid, 256, 0, h2d>>>(d_tasks, L.d_pieces);
        c->launches++;
        if (cudaGetLastError() != cudaSuccess) rc = SWB_ERR_CUDA;
    }
    if (!rc && cudaEventRecord(c->chunk_in[0], h2d) != cudaSuccess) rc = SWB_ERR_CUDA;
    if (!rc && cudaStreamWaitEvent(st, c->chunk_in[0], 0) != cudaSuccess) rc = SWB_ERR_CUDA;
    if (!rc) cudaMemsetAsync(c->d_counters, 0, sizeof(unsigned long long) * kNumCounters, st);
    if (!rc) cudaEventRecord(L.ev_t0, st);
    if (!rc) {
        if (s->plain == 2) {
            // The plain launch reads the request's shape back (a stream
            // synchronisation): submitters and waiters need not wait for it.
            // Only this worker thread touches the lanes and the dispatched
            // requests meanwhile.
            s->mu.unlock();
            rc = launch_ext_plain(c, s->dsc, s->d_arena, d_tasks, wn, d_out, c->d_counters, st);
            s->mu.lock();
        } else {
            // The int32 bin's scratch is sized from the longest query of the
            // wave's requests (an upper bound of the bin's), known since submit.
            int max_q = 0;
            for (const Piece &p : L.pieces) max_q = std::max(max_q, p.r->max_q);
            rc = launch_ext(c, s->dsc, s->d_arena, d_tasks, wn, d_out, c->d_counters, st, max_q, s->latency_cells);
        }
    }
    if (!rc) cudaEventRecord(L.ev_t1, st);
    if (!rc && cudaEventRecord(c->chunk_done[0], st) != cudaSuccess) rc = SWB_ERR_CUDA;
    if (!rc && cudaStreamWaitEvent(d2h, c->chunk_done[0], 0) != cudaSuccess) rc = SWB_ERR_CUDA;
    if (!rc) {
        for (const Piece &p : L.pieces)
            cudaMemcpyAsync(p.r->out_pinned ? p.r->out + p.lo : L.h_out + p.woff, d_out + p.woff,
                            (p.hi - p.lo) * sizeof(swb_ext_result), cudaMemcpyDeviceToHost, d2h);
        cudaMemcpyAsync(L.h_cells, c->d_counters, sizeof(unsigned long long) * kNumCounters, cudaMemcpyDeviceToHost, d2h);
    }
    L.launch_rc = rc;
    cudaEventRecord(L.ev_done, rc ? st : d2h);
    L.busy = true;
    s->queue.erase(std::remove_if(s->queue.begin(), s->queue.end(), [](const Req *r) { return r->dispatched == r->n; }),
                   s->queue.end());
    return true;
}

void worker_loop(swb_server *s) {
    cudaSetDevice(s->parent->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progressed = false;
        for (Lane &L : s->lanes)
            if (L.busy && cudaEventQuery(L.ev_done) == cudaSuccess) {
                complete_wave(s, L);
                progressed = true;
            }
        const bool have_work = !s->paused && std::any_of(s->queue.begin(), s->queue.end(),
                                                          [](Req *r) { return r->dispatched < r->n; });
        if (have_work) {
            const int nl = s->plain ? 1 : kLanes;
            for (int k = 0; k < nl; ++k) {
                Lane &L = s->lanes[(s->next_lane + k) % nl];
                if (!L.busy) {
                    if (launch_wave(s, L)) {
                        s->next_lane = (s->next_lane + k + 1) % nl;
                        progressed = true;
                    }
                    break;
                }
            }
        }
        const bool inflight = std::any_of(std::begin(s->lanes), std::end(s->lanes), [](const Lane &L) { return L.busy; });
        if (s->stopping && !inflight && !have_work) break;
        if (!progressed) {
            if (inflight) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(20));
                lk.lock();
            } else {
                s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            }
        }
    }
}

}  // namespace

extern "C" {

int swb_server_start(swb_ctx *ctx, const swb_scoring *sc, const swb_server_opts *opts, swb_server **out) {
    if (!ctx || !sc || !out) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    if (sc->e_ins <= 0 || sc->e_del <= 0 || sc->o_ins < 0 || sc->o_del < 0 || sc->a < 0 || sc->b < 0 || sc->a > 127 ||
        sc->b > 128)
        return set_error(SWB_ERR_INVALID_ARG, "scoring: need e_ins, e_del > 0, o_* >= 0 and 0 <= a <= 127, 0 <= b <= 128");
    *out = nullptr;
    swb_server_opts o{};
    if (opts) o = *opts;
    if (o.plain < 0 || o.plain > 2) return set_error(SWB_ERR_INVALID_ARG, "plain must be 0, 1 or 2");
    auto *s = new swb_server();
    s->parent = ctx;
    s->sc = *sc;
    s->dsc = make_dev_scoring(*sc);
    s->plain = o.plain;
    s->paused = o.start_paused != 0;
    s->max_wave = o.max_wave_tasks ? o.max_wave_tasks : (1u << 20);
    s->latency_cells = o.latency_cells;
    const size_t arena = o.arena_bytes ? o.arena_bytes : ((size_t)1 << 30);
    SWB_CUDA(cudaSetDevice(ctx->device));
    int rc = SWB_OK;
    if (ctx->allocated + arena > ctx->budget) rc = set_error(SWB_ERR_OOM, "server arena exceeds the context's memory budget");
    if (!rc && cudaMalloc(&s->d_arena, arena) != cudaSuccess) rc = check_cuda(cudaGetLastError(), "cudaMalloc(arena)");
    if (!rc) s->arena.init(arena);
    for (Lane &L : s->lanes) {
        if (rc) break;
        rc = swb_init(ctx->device, ctx->budget, &L.ctx);
        if (rc) break;
        L.ctx->d_pac = ctx->d_pac;            // shared resident reference (not owned)
        L.ctx->pac_owned = false;
        L.ctx->ref_bases = ctx->ref_bases;
        if (cudaMallocHost(&L.h_stage, s->max_wave * sizeof(swb_ext_task)) != cudaSuccess ||
            cudaMallocHost(&L.h_out, s->max_wave * sizeof(swb_ext_result)) != cudaSuccess ||
            cudaMallocHost(&L.h_pieces, kMaxPieces * sizeof(RebasePiece)) != cudaSuccess ||
            cudaMalloc(&L.d_pieces, kMaxPieces * sizeof(RebasePiece)) != cudaSuccess ||
            cudaMallocHost(&L.h_cells, sizeof(unsigned long long) * kNumCounters) != cudaSuccess ||
            cudaEventCreateWithFlags(&L.ev_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&L.ev_t0) != cudaSuccess || cudaEventCreate(&L.ev_t1) != cudaSuccess)
            rc = check_cuda(cudaGetLastError(), "server lane set-up");
    }
    if (rc) {
        for (Lane &L : s->lanes) {
            if (L.h_stage) cudaFreeHost(L.h_stage);
            if (L.h_out) cudaFreeHost(L.h_out);
            if (L.h_pieces) cudaFreeHost(L.h_pieces);
            if (L.d_pieces) cudaFree(L.d_pieces);
            if (L.h_cells) cudaFreeHost(L.h_cells);
            if (L.ctx) swb_destroy(L.ctx);
        }
        if (s->d_arena) cudaFree(s->d_arena);
        delete s;
        return rc;
    }
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return SWB_OK;
}

int swb_server_submit(swb_server *s, const uint8_t *bases, size_t n_bases, uint64_t span_origin,
                      const swb_ext_task *tasks, size_t n_tasks, swb_ext_result *out, uint64_t *ticket) {
    if (!s || !ticket || (!bases && n_bases) || (!tasks && n_tasks) || (!out && n_tasks))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    if (align_up256(std::max<size_t>(n_bases, 1)) > s->arena.cap)
        return set_error(SWB_ERR_TOO_LARGE, "request bases exceed the server arena");
    // Span validation against the request's own buffer and the reference.
    const uint64_t lo = span_origin, hi = span_origin + n_bases;
    int max_q = 0;
    for (size_t i = 0; i < n_tasks; ++i) {
        const swb_ext_task &t = tasks[i];
        max_q = std::max(max_q, t.qlen);
        const bool bad_len = t.qlen < 0 || t.tlen < 0 || t.qlen > kMaxLen || t.tlen > kMaxLen;
        const bool bad_q = t.qlen > 0 && (t.q_off < lo || t.q_off + (uint64_t)t.qlen > hi);
        const bool bad_t = t.tlen > 0 && ((t.flags & SWB_T_FROM_REF)
                                              ? (!s->parent->d_pac || t.t_off + (uint64_t)t.tlen > s->parent->ref_bases)
                                              : (t.t_off < lo || t.t_off + (uint64_t)t.tlen > hi));
        if (bad_len || bad_q || bad_t)
            return set_error(bad_len ? SWB_ERR_TOO_LARGE : SWB_ERR_INVALID_ARG, "task " + std::to_string(i) + ": bad span or length");
    }
    auto *r = new Req();
    r->bases = bases;
    r->n_bases = n_bases;
    r->origin = span_origin;
    r->tasks = tasks;
    r->n = n_tasks;
    r->out = out;
    r->max_q = max_q;
    r->tasks_pinned = is_pinned(tasks);
    r->out_pinned = is_pinned(out);
    r->t_submit = now_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) {
            delete r;
            return set_error(SWB_ERR_INVALID_ARG, "server is stopping");
        }
        r->ticket = s->next_ticket++;
        s->reqs[r->ticket] = r;
        s->stats.submitted++;
        if (n_tasks == 0) {
            r->done = true;
            r->t_done = r->t_submit;
            s->stats.completed++;
        } else {
            s->queue.push_back(r);
        }
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return SWB_OK;
}

int swb_server_poll(swb_server *s, uint64_t ticket, int *done, int *status) {
    if (!s || !done) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_error(SWB_ERR_NOT_FOUND, "unknown ticket " + std::to_string(ticket));
    *done = it->second->done ? 1 : 0;
    if (status) *status = it->second->status;
    return SWB_OK;
}

int swb_server_wait(swb_server *s, uint64_t ticket, int timeout_ms, int *status, uint64_t *submit_ns, uint64_t *done_ns) {
    if (!s) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_error(SWB_ERR_NOT_FOUND, "unknown ticket " + std::to_string(ticket));
    Req *r = it->second;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(std::max(timeout_ms, 0));
    while (!r->done)
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !r->done)
            return set_error(SWB_ERR_TIMEOUT, "ticket " + std::to_string(ticket) + " not done after " +
                                                  std::to_string(timeout_ms) + " ms");
    if (status) *status = r->status;
    if (submit_ns) *submit_ns = r->t_submit;
    if (done_ns) *done_ns = r->t_done;
    s->reqs.erase(it);
    delete r;
    return SWB_OK;
}

int swb_server_resume(swb_server *s) {
    if (!s) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->paused = false;
    }
    s->cv_work.notify_one();
    return SWB_OK;
}

int swb_server_stats_get(swb_server *s, swb_server_stats *st) {
    if (!s || !st) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->stats;
    return SWB_OK;
}

int swb_server_stop(swb_server *s) {
    if (!s) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->paused = false;
    }
    s->cv_work.notify_one();
    if (s->worker.joinable()) s->worker.join();
    for (Lane &L : s->lanes) {
        if (L.ctx) {
            cudaStreamSynchronize(L.ctx->stream);
            cudaStreamSynchronize(L.ctx->d2h);
            cudaStreamSynchronize(L.ctx->h2d);
        }
        if (L.ev_done) cudaEventDestroy(L.ev_done);
        if (L.ev_t0) cudaEventDestroy(L.ev_t0);
        if (L.ev_t1) cudaEventDestroy(L.ev_t1);
        if (L.h_stage) cudaFreeHost(L.h_stage);
        if (L.h_out) cudaFreeHost(L.h_out);
        if (L.h_pieces) cudaFreeHost(L.h_pieces);
        if (L.d_pieces) cudaFree(L.d_pieces);
        if (L.h_cells) cudaFreeHost(L.h_cells);
        if (L.ctx) swb_destroy(L.ctx);
    }
    if (s->d_arena) cudaFree(s->d_arena);
    for (auto &kv : s->reqs) delete kv.second;
    delete s;
    return SWB_OK;
}

}  // extern "C"
