// noalloc.cu — shg_solve_batch_device_noalloc: the batched plain march with its scratch in a
// fixed, statically allocated device array instead of memory allocated per call.
//
// Who needs it: callers that must not allocate device memory while they run.  Examples are
// hosts that hand all free device memory to their own pool allocator at start-up (so a
// cudaMalloc here would fail or break their budget), latency-sensitive loops where an
// allocation can block or synchronise the device at an unpredictable moment, and plugin
// hosts that forbid a library from allocating behind their back.  Such a caller still owns
// and passes the input parameters and the output buffers; this entry point adds nothing
// but kernel launches and a copy of the power slots back to the host.
//
// The scratch (instance descriptors and per-instance power slots) lives in g_noalloc_scratch,
// a file-scope __device__ array of kNoAllocScratchBytes (about 23 KB) that every GPU which loads
// the library holds until the process exits.  Its limit: at most kNoAllocMaxInstances
// instances per call.
//
// In host code the name g_noalloc_scratch is only a host-side stand-in for the device
// symbol, not a device address.  The first call made on a device, with that device current,
// sets that device up: it looks the array's address up with cudaGetSymbolAddress and loads
// every kernel this entry point can launch (with CUDA's lazy module loading a kernel's code is
// otherwise loaded at its first launch, and the driver may take device memory for it then).
// So make the first call on each device before the host hands all free device memory to its
// own allocator, and before any stream capture.  Later calls allocate nothing.
//
// The descriptors travel as a kernel parameter (a fixed 24 KB block, copied by the launch),
// so no host staging buffer is involved.  All calls share the one array and it keeps the last
// call's contents: each call rewrites the descriptors it uses and clears the power slots
// before its marches run.  Calls whose work overlaps on the GPU (concurrent calls on
// different streams, or from several host threads) race on the array: serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "shg_host.h"
#include "shg_internal.h"
#include "ssfm_variants.h"

namespace shg {

constexpr int kNoAllocMaxInstances = 64;
constexpr size_t kNoAllocDescBytes = sizeof(InstDesc) * kNoAllocMaxInstances;
constexpr size_t kNoAllocScratchBytes = ((kNoAllocDescBytes + 2 * sizeof(double) * kNoAllocMaxInstances + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The descriptors of one call, passed by value (kernel parameters may take up to 32 KB).
struct NoAllocUpload {
    InstDesc desc[kNoAllocMaxInstances];
    int32_t count;
};
static_assert(sizeof(NoAllocUpload) <= 32000, "descriptor block exceeds the kernel parameter limit");

// Writes the call's descriptors into the scratch and clears its power slots.
__global__ void noalloc_upload_kernel(__grid_constant__ const NoAllocUpload up, InstDesc* ddesc, double* dpow) {
    const int words = (int)(sizeof(InstDesc) / sizeof(uint32_t));
    static_assert(sizeof(InstDesc) % sizeof(uint32_t) == 0, "InstDesc is copied in 32-bit words");
    const uint32_t* src = reinterpret_cast<const uint32_t*>(up.desc);
    uint32_t* dst = reinterpret_cast<uint32_t*>(ddesc);
    for (int i = threadIdx.x; i < up.count * words; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < 2 * up.count; i += blockDim.x) dpow[i] = 0.0;
}

// Once per device: the device address of g_noalloc_scratch, and every kernel this entry point
// launches loaded (a zero-instance launch of each fused plain variant runs its per-device
// attribute set-up, which loads the kernel, and launches nothing).
static PerDevice<void*> g_noalloc_device;

static shg_status noalloc_setup(void** out) {
    const cudaError_t e = g_noalloc_device.get(
        [](int, void*& addr) {
            void* ptr = nullptr;
            cudaError_t r = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (r != cudaSuccess) return r;
            if (!ptr) return cudaErrorInvalidSymbol;
            cudaFuncAttributes fa;
            r = cudaFuncGetAttributes(&fa, noalloc_upload_kernel);
            if (r != cudaSuccess) return r;
            for (int prec : {32, 64}) {
                const PlainVariant* cand[16];
                for (int n = 16; n <= 256; n += 16) {
                    const int k = plain_candidates(prec, n, cand, 16);
                    for (int i = 0; i < k; ++i)
                        if (cand[i]->launch && (r = cand[i]->launch(nullptr, 0, nullptr, nullptr)) != cudaSuccess)
                            return r;
                }
            }
            addr = ptr;
            return cudaSuccess;
        },
        out);
    if (e != cudaSuccess) return cuda_fail(e, "device set-up of the allocation-free march");
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
    shg_status rc = noalloc_setup(&base);
    if (rc != SHG_OK) return rc;
    InstDesc* ddesc = reinterpret_cast<InstDesc*>(base);
    double* dpow = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(base) + kNoAllocDescBytes);

    // kernel variants: the fused march only (the multi-pass march needs workspace); an
    // automatic choice of the multi-pass march falls back to the fused one where it is built
    const PlainVariant* var[kNoAllocMaxInstances];
    int order[kNoAllocMaxInstances], out32[kNoAllocMaxInstances];
    for (int i = 0; i < count; ++i) {
        order[i] = i;
        var[i] = plain_variant_of(params[i], &out32[i]);
        if (var[i] && var[i]->mp && params[i].march == SHG_MARCH_AUTO)
            var[i] = find_plain_variant(params[i].precision, params[i].nx, 0, SHG_MARCH_FUSED);
        if (!var[i] || var[i]->mp)
            return fail(SHG_ERR_UNSUPPORTED, "instance %d: the multi-pass march (side %d) needs device workspace", i,
                        params[i].nx);
    }
    // descriptors grouped by kernel variant, longest march first
    std::sort(order, order + count, [&](int a, int b) {
        if (var[a] != var[b]) return var[a] < var[b];
        const double ca = (double)params[a].nx * params[a].nx * shg_steps(&params[a]);
        const double cb = (double)params[b].nx * params[b].nx * shg_steps(&params[b]);
        if (ca != cb) return ca > cb;
        return a < b;
    });
    NoAllocUpload up;
    std::memset(&up, 0, sizeof(up));
    up.count = count;
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        InstDesc d = make_plain_desc(params[i], params[i].temp, params[i].temp);
        d.slot = i;
        d.out32 = out32[i];
        d.pump_out = pump_out_dev ? pump_out_dev[i] : nullptr;
        d.signal_out = signal_out_dev ? signal_out_dev[i] : nullptr;
        d.power_out = dpow + 2 * (size_t)i;
        up.desc[k] = d;
    }
    cudaError_t e;
    noalloc_upload_kernel<<<1, 256, 0, stream>>>(up, ddesc, dpow);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "launch noalloc_upload_kernel");
    for (int k = 0; k < count;) {
        int j = k;
        while (j < count && var[order[j]] == var[order[k]]) ++j;
        if ((e = var[order[k]]->launch(ddesc + k, j - k, nullptr, stream)) != cudaSuccess)
            return cuda_fail(e, "launch ssfm_plain_kernel");
        k = j;
    }
    if (sh_power_out) {
        // {SH power, pump power} per instance; a NaN or Inf power fails the call as in the
        // allocating batch, naming the instance
        double h[2 * kNoAllocMaxInstances];
        if ((e = cudaMemcpyAsync(h, dpow, 2 * sizeof(double) * (size_t)count, cudaMemcpyDeviceToHost, stream)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
            return cuda_fail(e, "batched march");
        for (int i = 0; i < count; ++i) {
            if (!std::isfinite(h[2 * i]) || !std::isfinite(h[2 * i + 1]))
                return fail(SHG_ERR_NONFINITE, "instance %d: SH / pump power %g / %g", i, h[2 * i], h[2 * i + 1]);
            sh_power_out[i] = h[2 * i];
        }
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "batched march");
    return SHG_OK;
}
