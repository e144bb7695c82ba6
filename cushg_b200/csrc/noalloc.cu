// noalloc.cu — shg_solve_batch_device_noalloc: the batched plain march with its scratch in a
// fixed, statically allocated device array instead of memory allocated per call.
//
// Who needs it: callers that must not allocate device memory while they run.  Examples are
// hosts that hand all free device memory to their own pool allocator at start-up (so a
// cudaMalloc here would fail or break their budget), latency-sensitive loops where an
// allocation can block or synchronise the device at an unpredictable moment, and plugin
// hosts that forbid a library from allocating behind their back.  Such a caller still owns
// and passes the input parameters and the output buffers; this entry point adds nothing
// but kernel launches and copies into memory that exists since the library was loaded.
//
// The scratch (instance descriptors and per-instance power slots) lives in g_noalloc_scratch,
// a file-scope __device__ array of kNoAllocScratchBytes (about 23 KB) that every GPU which loads
// the library holds until the process exits.  Its limit: at most kNoAllocMaxInstances
// instances per call.
//
// In host code the name g_noalloc_scratch is only a host-side stand-in for the device
// symbol, not a device address; the address is obtained once per device with
// cudaGetSymbolAddress while that device is current, on the first call made on it.  That
// first call should therefore come before any stream capture.
//
// All calls share the one array and it keeps the last call's contents.  Each call rewrites
// the descriptors it uses and clears the power slots before its kernels run.  Calls whose
// work overlaps on the GPU (concurrent calls on different streams, or from several host
// threads) race on the array: serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "shg_host.h"
#include "shg_internal.h"
#include "ssfm_variants.h"

namespace shg {

constexpr int kNoAllocMaxInstances = 64;
constexpr size_t kNoAllocDescBytes = sizeof(InstDesc) * kNoAllocMaxInstances;
constexpr size_t kNoAllocScratchBytes = ((kNoAllocDescBytes + 2 * sizeof(double) * kNoAllocMaxInstances + 255) / 256) * 256;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (set up once per device).
static shg_status noalloc_scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(SHG_ERR_UNSUPPORTED, "device ordinal %d too large", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_addr[dev] = ptr;
    }
    *out = g_noalloc_addr[dev];
    return SHG_OK;
}

}  // namespace shg

using namespace shg;

extern "C" shg_status shg_solve_batch_device_noalloc(const shg_params* params, int32_t count,
                                                     void* const* pump_out_dev, void* const* signal_out_dev,
                                                     double* sh_power_out, void* stream_) {
    clear_error();
    if (!params || count < 0) return fail(SHG_ERR_INVALID, "params is NULL or count < 0");
    if (count > kNoAllocMaxInstances)
        return fail(SHG_ERR_INVALID, "count %d exceeds the %d instances the static scratch holds", count,
                    kNoAllocMaxInstances);
    if (count == 0) return SHG_OK;
    for (int i = 0; i < count; ++i) {
        shg_status st = shg_check_params(&params[i]);
        if (st != SHG_OK) return st;
        if (params[i].thermal) return fail(SHG_ERR_UNSUPPORTED, "instance %d: batched runs are plain (thermal == 0)", i);
        if (params[i].precision != params[0].precision)
            return fail(SHG_ERR_INVALID, "instance %d: all instances must share one precision", i);
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    void* base = nullptr;
    shg_status rc = noalloc_scratch_address(&base);
    if (rc != SHG_OK) return rc;
    InstDesc* ddesc = reinterpret_cast<InstDesc*>(base);
    double* dpow = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(base) + kNoAllocDescBytes);

    // descriptors on the stack, grouped by kernel variant, longest march first
    InstDesc descs[kNoAllocMaxInstances];
    const PlainVariant* var[kNoAllocMaxInstances];
    int order[kNoAllocMaxInstances];
    for (int i = 0; i < count; ++i) {
        order[i] = i;
        var[i] = find_plain_variant(params[i].precision, params[i].nx, 0, params[i].march);
        if (var[i]->mp)
            return fail(SHG_ERR_UNSUPPORTED, "instance %d: the multi-pass march (side %d) needs device workspace", i,
                        params[i].nx);
    }
    std::sort(order, order + count, [&](int a, int b) {
        if (var[a] != var[b]) return var[a] < var[b];
        const double ca = (double)params[a].nx * params[a].nx * shg_steps(&params[a]);
        const double cb = (double)params[b].nx * params[b].nx * shg_steps(&params[b]);
        if (ca != cb) return ca > cb;
        return a < b;
    });
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        InstDesc d = make_plain_desc(params[i], params[i].temp, params[i].temp);
        d.slot = i;
        d.pump_out = pump_out_dev ? pump_out_dev[i] : nullptr;
        d.signal_out = signal_out_dev ? signal_out_dev[i] : nullptr;
        d.power_out = dpow + 2 * (size_t)i;
        descs[k] = d;
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(ddesc, descs, sizeof(InstDesc) * (size_t)count, cudaMemcpyHostToDevice, stream)) !=
        cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync descriptors");
    if ((e = cudaMemsetAsync(dpow, 0, 2 * sizeof(double) * (size_t)count, stream)) != cudaSuccess)
        return cuda_fail(e, "cudaMemsetAsync power slots");
    for (int k = 0; k < count;) {
        int j = k;
        while (j < count && var[order[j]] == var[order[k]]) ++j;
        if ((e = var[order[k]]->launch(ddesc + k, j - k, nullptr, stream)) != cudaSuccess)
            return cuda_fail(e, "launch ssfm_plain_kernel");
        k = j;
    }
    if (sh_power_out) {
        double h[2 * kNoAllocMaxInstances];
        if ((e = cudaMemcpyAsync(h, dpow, 2 * sizeof(double) * (size_t)count, cudaMemcpyDeviceToHost, stream)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
            return cuda_fail(e, "batched march");
        for (int i = 0; i < count; ++i) sh_power_out[i] = h[2 * i];
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "batched march");
    return SHG_OK;
}
