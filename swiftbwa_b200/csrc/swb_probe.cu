// swb_probe.cu -- integer ALU throughput probe: the roofline denominator
// for the SW kernels, which are bound by int32 issue, not by HBM or tensor
// cores.  Each thread runs 8 independent add/max chains (the two
// operations of the DP recurrences), so the measured rate is the SM's
// sustained int32 add/max rate at the clocks of the moment.
#include "swb_internal.h"

namespace swb {
namespace {

__global__ void __launch_bounds__(256) alu_probe_kernel(int iters, int seed, int *sink) {
    int x[8], y[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = seed + k + threadIdx.x;
        y[k] = (seed ^ (k * 7919)) + blockIdx.x;
    }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                x[k] = max(x[k] + y[k], y[k] - u);   // add + max
                y[k] = max(y[k] - x[k], x[k] + k);   // add + max
            }
        }
    }
    int acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc ^= x[k] ^ y[k];
    if (acc == 0x7FFFFFFF) sink[0] = acc;   // keeps the chains live
}

// The same chains on packed 16-bit lanes: one DPX add+max per statement,
// two lanes per instruction (the form the shared-memory extension kernels
// compute their two target rows in).
__global__ void __launch_bounds__(256) alu16x2_probe_kernel(int iters, int seed, int *sink) {
    uint32_t x[8], y[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = (uint32_t)(seed + k + threadIdx.x) * 0x10001u;
        y[k] = (uint32_t)((seed ^ (k * 7919)) + blockIdx.x) * 0x10001u;
    }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                x[k] = __viaddmax_s16x2(x[k], y[k], y[k]);   // add + max, both lanes
                y[k] = __viaddmax_s16x2(y[k], x[k], x[k]);   // add + max, both lanes
            }
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc ^= x[k] ^ y[k];
    if (acc == 0x7FFFFFFFu) sink[0] = (int)acc;   // keeps the chains live
}

// Best of three timed launches (after one warm-up) of a probe kernel.
template <class Launch>
int time_probe(swb_ctx *ctx, Launch launch, float *best_ms) {
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        SWB_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
        launch(rep);
        SWB_CUDA(cudaGetLastError());
        SWB_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
        SWB_CUDA(cudaEventSynchronize(ctx->ev_stop));
        float ms = 0.f;
        SWB_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
        if (rep > 0 && ms < best) best = ms;
    }
    *best_ms = best;
    return SWB_OK;
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" int swb_int_alu_peak(swb_ctx *ctx, double *ops_per_s) {
    if (!ctx || !ops_per_s) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_aux, 64))) return rc;
    const int blocks = ctx->sm_count * 8, threads = 256, iters = 2000;
    // Source-level int ops per thread: iters * 16 unrolled * 8 chains *
    // 2 statements * 3 ops (two adds and a max each), the same way the DP
    // kernels' ops per cell are counted.
    const double ops = (double)blocks * threads * iters * 16 * 8 * 2 * 3;
    float best = 0.f;
    int *sink = (int *)ctx->d_aux.p;
    if ((rc = time_probe(ctx, [&](int rep) { alu_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(iters, rep, sink); },
                         &best)))
        return rc;
    *ops_per_s = ops / (best * 1e-3);
    return SWB_OK;
}

extern "C" int swb_int16x2_alu_peak(swb_ctx *ctx, double *lane_ops_per_s) {
    if (!ctx || !lane_ops_per_s) return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    SWB_CUDA(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_aux, 64))) return rc;
    const int blocks = ctx->sm_count * 8, threads = 256, iters = 2000;
    // 16-bit lane operations: iters * 16 * 8 chains * 2 statements * 2 lanes
    // * 2 ops (an add and a max each).
    const double ops = (double)blocks * threads * iters * 16 * 8 * 2 * 2 * 2;
    float best = 0.f;
    int *sink = (int *)ctx->d_aux.p;
    if ((rc = time_probe(ctx, [&](int rep) { alu16x2_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(iters, rep, sink); },
                         &best)))
        return rc;
    *lane_ops_per_s = ops / (best * 1e-3);
    return SWB_OK;
}
