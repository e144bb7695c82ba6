// ssfm_multipass.cu — variants and host sequence of the multi-pass SSFM march
// (ssfm_multipass.cuh): N = 512 (plain and thermal, FP32 and FP64), N = 256 (plain and
// thermal, the side where it can be checked against the fused cluster march) and N = 128
// (thermal).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "shg_host.h"
#include "ssfm_multipass.cuh"
#include "ssfm_variants.h"

namespace shg {

namespace {

// The march of `count` instances of one class: set-up, the first row pass, then per step
// the column pass and the row pass, then the power sums.  The workspace (planes, tables,
// partials, Δk prefix, z_s) is allocated and freed stream-ordered, so the sequence can be
// captured into a CUDA graph.  Instances with fewer steps drop out of later launches.
template <typename T, int N, bool THERM>
cudaError_t mp_march(const InstDesc* dev_descs, const InstDesc* host_descs, int count, cudaStream_t s) {
    using Cfg = MpCfg<T, N>;
    static PerDevice<int> state;  // kernel attributes, once per device
    const cudaError_t attr_err = state.get([](int, int&) {
        cudaError_t e = cudaFuncSetAttribute(mp_row_kernel<T, N, THERM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)Cfg::row_smem_for(THERM));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(mp_col_kernel<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::col_smem);
        return e;
    });
    if (attr_err != cudaSuccess) return attr_err;
    if (count <= 0) return cudaSuccess;
    int max_steps = 0;
    for (int i = 0; i < count; ++i) max_steps = std::max(max_steps, (int)host_descs[i].nsteps);
    MpLayout L = mp_layout<T, N>(nullptr, max_steps, THERM);
    cudaError_t e = dev_alloc((void**)&L.base, L.stride * (size_t)count, s);
    if (e != cudaSuccess) return e;
    const dim3 rgrid(Cfg::RPART, count), cgrid(N / Cfg::CW, 2, count);
    mp_setup_kernel<T, N><<<count, 256, 0, s>>>(dev_descs, L);
    mp_row_kernel<T, N, THERM><<<rgrid, Cfg::row_threads(THERM), Cfg::row_smem_for(THERM), s>>>(dev_descs, L, -1);
    for (int st = 0; st < max_steps; ++st) {
        mp_col_kernel<T, N><<<cgrid, Cfg::CNT, Cfg::col_smem, s>>>(dev_descs, L, st);
        mp_row_kernel<T, N, THERM><<<rgrid, Cfg::row_threads(THERM), Cfg::row_smem_for(THERM), s>>>(dev_descs, L, st);
    }
    mp_power_kernel<T, N><<<count, 32, 0, s>>>(dev_descs, L);
    e = cudaGetLastError();
    const cudaError_t ef = cudaFreeAsync(L.base, s);
    return e != cudaSuccess ? e : ef;
}

#define SHG_MP_VARIANT(T, PREC, N, THERM) \
    {PREC, N, 0, MpCfg<T, N>::row_threads(THERM), 1, THERM ? 1 : 0, MpCfg<T, N>::row_smem_for(THERM), nullptr, &mp_march<T, N, THERM>}

const PlainVariant kTable[] = {
    SHG_MP_VARIANT(float, 32, 512, false),  SHG_MP_VARIANT(double, 64, 512, false),
    SHG_MP_VARIANT(float, 32, 256, false),  SHG_MP_VARIANT(double, 64, 256, false),
    SHG_MP_VARIANT(float, 32, 512, true),   SHG_MP_VARIANT(double, 64, 512, true),
    SHG_MP_VARIANT(float, 32, 256, true),   SHG_MP_VARIANT(double, 64, 256, true),
    SHG_MP_VARIANT(float, 32, 128, true),   SHG_MP_VARIANT(double, 64, 128, true),
};

}  // namespace

VariantTable variants_multipass() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
