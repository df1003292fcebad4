// swb_noalloc.cu -- a banded-extension entry point that allocates nothing.
//
// Some callers cannot let the library call cudaMalloc: a server that has
// handed all free HBM to its own arena (the resident reference plus request
// buffers admitted against a memory budget) has nothing left for the
// library to take, and a continuous-batching loop cannot afford
// cudaMalloc/cudaFree, which may synchronise the device and stall the other
// requests' streams.  swb_ext_batch_static serves them: the caller passes
// device inputs and outputs, and the only working memory is the
// file-scope array below.  The driver places it on a GPU when this file's
// device code is loaded there -- with CUDA's default lazy module loading,
// at the first call on that GPU (a call with zero tasks is enough) -- and
// keeps it until the process exits.  That first call also does the
// one-time set-up below, so a caller makes it before any stream capture,
// and before it gives the free HBM to its own arena.
//
// It runs the same device code as swb_ext_batch_device (swb_ext_dp.cuh),
// without the sort/binning pass: tasks are taken in input order by the
// shared-memory kernel (queries up to 256 bases with int16-safe scores),
// and the remaining tasks by the int32 kernel whose rows live in the static
// array, 2048 tasks at a time, queries up to 1024 bases.
#include <mutex>

#include "swb_ext_dp.cuh"

namespace swb {
namespace {

constexpr int kStaticT = 64;                     // threads per block, both kernels
constexpr int kStaticSmemQ = 256;                // shared-memory row length
constexpr int kStaticSlots = 2048;               // int32-path tasks in flight
constexpr int kStaticMaxQ = 1024;                // longest query the int32 path accepts here
constexpr size_t kStaticCols = kStaticMaxQ + 1;
constexpr size_t kStatusBytes = 256;             // error code, offending task index
constexpr size_t kStaticScratchBytes =
    kStatusBytes + kStaticCols * kStaticSlots * (2 * sizeof(int) + 1);   // 18.9 MB

// The working memory of swb_ext_batch_static.  Host code must not use this
// name as a device address; the set-up below asks the runtime for it.
static __device__ __align__(256) unsigned char g_ext_static_scratch[kStaticScratchBytes];

__device__ __forceinline__ bool static_smem_task(const swb_ext_task &t, int max_mat) {
    return t.qlen <= 0 || t.tlen <= 0 || (t.qlen <= kStaticSmemQ && fits16(t.qlen, t.h0, max_mat));
}

__global__ void __launch_bounds__(kStaticT) ext_static_smem_kernel(ExtArgs a, size_t n) {
    extern __shared__ uint32_t sm[];
    Smem16<kStaticT> st{sm, sm + (kStaticSmemQ + 1) * kStaticT, (int)threadIdx.x};
    unsigned long long cells = 0;
    const size_t per_iter = (size_t)gridDim.x * kStaticT;
    for (size_t pos = blockIdx.x * (size_t)kStaticT + threadIdx.x; pos < n; pos += per_iter) {
        const swb_ext_task tk = a.tasks[pos];
        if (!static_smem_task(tk, a.sc.max_mat)) continue;
        swb_ext_result r;
        ext_one(a, tk, st, r, cells);
        a.out[pos] = r;
    }
}

__global__ void __launch_bounds__(kStaticT) ext_static_global_kernel(ExtArgs a, size_t n, unsigned char *scratch) {
    int *status = (int *)scratch;                 // [0] error code, [1] first offending task
    int *h = (int *)(scratch + kStatusBytes);
    int *e = h + kStaticCols * kStaticSlots;
    uint8_t *q = (uint8_t *)(e + kStaticCols * kStaticSlots);
    const size_t slot = blockIdx.x * (size_t)kStaticT + threadIdx.x;
    Global32 st{h, e, q, (size_t)kStaticSlots, slot};
    unsigned long long cells = 0;
    for (size_t pos = slot; pos < n; pos += kStaticSlots) {
        const swb_ext_task tk = a.tasks[pos];
        if (static_smem_task(tk, a.sc.max_mat)) continue;
        if (tk.qlen > kStaticMaxQ) {
            atomicCAS(&status[0], 0, SWB_ERR_TOO_LARGE);
            atomicMin((unsigned int *)&status[1], (unsigned int)pos);
            a.out[pos] = swb_ext_result{0, 0, 0, 0, 0, 0};
            continue;
        }
        swb_ext_result r;
        ext_one(a, tk, st, r, cells);
        a.out[pos] = r;
    }
}

struct DeviceState {
    bool ready = false;
    unsigned char *scratch = nullptr;   // device address of g_ext_static_scratch
    int sm_count = 0;
    int smem_blocks = 1;
    std::mutex call_mu;                 // one call at a time per device in this process
};

std::mutex g_state_mu;
DeviceState g_state[64];

constexpr size_t kStaticSmemBytes = (size_t)((kStaticSmemQ + 1) + kStaticSmemQ / 4) * kStaticT * sizeof(uint32_t);

// One-time set-up per device, with that device current: look up the
// array's device address and size the shared-memory kernel.  Allocates
// nothing.
int device_state(int dev, DeviceState **out) {
    if (dev < 0 || dev >= 64) return set_error(SWB_ERR_NO_DEVICE, "device index above 63");
    std::lock_guard<std::mutex> lk(g_state_mu);
    DeviceState &st = g_state[dev];
    if (!st.ready) {
        int major = 0;
        SWB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
        if (major < 10) return set_error(SWB_ERR_NO_DEVICE, "current device is not sm_100 (built for sm_100a)");
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_ext_static_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return set_error(SWB_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
        }
        SWB_CUDA(cudaDeviceGetAttribute(&st.sm_count, cudaDevAttrMultiProcessorCount, dev));
        SWB_CUDA(cudaFuncSetAttribute(ext_static_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kStaticSmemBytes));
        SWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&st.smem_blocks, ext_static_smem_kernel, kStaticT,
                                                               kStaticSmemBytes));
        if (st.smem_blocks < 1) st.smem_blocks = 1;
        st.scratch = (unsigned char *)p;
        st.ready = true;
    }
    *out = &st;
    return SWB_OK;
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" int swb_ext_batch_static(const swb_scoring *sc, const uint8_t *d_bases, const uint8_t *d_pac,
                                    const swb_ext_task *d_tasks, size_t n_tasks, swb_ext_result *d_out,
                                    void *stream) {
    if (!sc || (!d_tasks && n_tasks) || (!d_out && n_tasks))
        return set_error(SWB_ERR_INVALID_ARG, "NULL argument");
    if (sc->e_ins <= 0 || sc->e_del <= 0 || sc->o_ins < 0 || sc->o_del < 0 || sc->a < 0 || sc->b < 0 ||
        sc->a > 127 || sc->b > 128)
        return set_error(SWB_ERR_INVALID_ARG, "scoring: need e_ins, e_del > 0, o_* >= 0 and 0 <= a <= 127, 0 <= b <= 128");
    int dev = 0;
    SWB_CUDA(cudaGetDevice(&dev));
    DeviceState *st = nullptr;
    int rc = device_state(dev, &st);   // also for n_tasks == 0: loads the array on this device
    if (rc) return rc;
    if (n_tasks == 0) return SWB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    // Calls from this process's threads share the array; hold it from the
    // status reset until the stream has finished with it.
    std::lock_guard<std::mutex> call_lock(st->call_mu);
    // Every call shares the array: reset the status words (code 0, index ~0).
    SWB_CUDA(cudaMemsetAsync(st->scratch, 0, sizeof(int), s));
    SWB_CUDA(cudaMemsetAsync(st->scratch + sizeof(int), 0xFF, sizeof(int), s));
    ExtArgs a{make_dev_scoring(*sc), d_bases, d_pac, d_tasks, d_out, nullptr, nullptr, nullptr};
    const size_t need = (n_tasks + kStaticT - 1) / kStaticT;
    const size_t grid = std::min<size_t>(need, (size_t)st->sm_count * st->smem_blocks);
    ext_static_smem_kernel<<<(unsigned)grid, kStaticT, kStaticSmemBytes, s>>>(a, n_tasks);
    SWB_CUDA(cudaGetLastError());
    ext_static_global_kernel<<<kStaticSlots / kStaticT, kStaticT, 0, s>>>(a, n_tasks, st->scratch);
    SWB_CUDA(cudaGetLastError());
    int status[2] = {0, 0};
    SWB_CUDA(cudaMemcpyAsync(status, st->scratch, sizeof(status), cudaMemcpyDeviceToHost, s));
    SWB_CUDA(cudaStreamSynchronize(s));
    if (status[0] != 0)
        return set_error(status[0], "task " + std::to_string((unsigned)status[1]) +
                                        ": query longer than 1024 bases needs the int32 path, beyond the static scratch");
    return SWB_OK;
}
