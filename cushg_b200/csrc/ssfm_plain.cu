// ssfm_plain.cu — instantiations and launchers of the fused plain SSFM march.
#include <cuda_runtime.h>

#include <mutex>

#include "ssfm_plain.cuh"
#include "ssfm_variants.h"

namespace shg {

template <typename T, int N, int C, int NT, bool THERM, int MINB = 1>
static cudaError_t launch_plain(const InstDesc* descs, int count, cudaStream_t stream) {
    using Cfg = PlainCfg<T, N, C, NT, THERM>;
    auto kern = ssfm_plain_kernel<T, N, C, NT, THERM, MINB>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&]() {
        attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem_bytes);
        if (attr_err == cudaSuccess && C > 8)
            attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    if (attr_err != cudaSuccess) return attr_err;
    if (count <= 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(count * C), 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = Cfg::smem_bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = C > 1 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, descs);
}

#define SHG_PLAIN(T, PREC, N, C, NT) \
    {PREC, N, C, NT, 0, PlainCfg<T, N, C, NT, false>::smem_bytes, &launch_plain<T, N, C, NT, false>}
#define SHG_PLAIN_B(T, PREC, N, C, NT, MINB) \
    {PREC, N, C, NT, 0, PlainCfg<T, N, C, NT, false>::smem_bytes, &launch_plain<T, N, C, NT, false, MINB>}
#define SHG_THERM(T, PREC, N, C, NT) \
    {PREC, N, C, NT, 1, PlainCfg<T, N, C, NT, true>::smem_bytes, &launch_plain<T, N, C, NT, true>}

// Threads per CTA of each variant (tuning knobs, overridable at build time).
#ifndef SHG_NT_F32_SMALL
#define SHG_NT_F32_SMALL 512
#endif
#ifndef SHG_NT_F32_128
#define SHG_NT_F32_128 512
#endif
#ifndef SHG_NT_F32_192
#define SHG_NT_F32_192 384
#endif
#ifndef SHG_NT_F32_256
#define SHG_NT_F32_256 256
#endif
#ifndef SHG_NT_F64
#define SHG_NT_F64 256
#endif
#ifndef SHG_C_F32_128
#define SHG_C_F32_128 2
#endif
#ifndef SHG_C_F32_192
#define SHG_C_F32_192 4
#endif
#ifndef SHG_C_F32_256
#define SHG_C_F32_256 16
#endif
#ifndef SHG_MINB_F32_128
#define SHG_MINB_F32_128 1
#endif
#ifndef SHG_MINB_F32_192
#define SHG_MINB_F32_192 1
#endif
#ifndef SHG_MINB_F32_256
#define SHG_MINB_F32_256 2
#endif
#ifndef SHG_MINB_F32_SMALL
#define SHG_MINB_F32_SMALL 1
#endif

// (precision, grid side) -> cluster size and threads per CTA.  The cluster size keeps
// both planes of one instance in at most ~150 KB of shared memory per CTA.
static const PlainVariant kPlainVariants[] = {
    SHG_PLAIN(float, 32, 32, 1, 128),
    SHG_PLAIN(float, 32, 48, 1, 192),
    SHG_PLAIN_B(float, 32, 64, 1, SHG_NT_F32_SMALL, SHG_MINB_F32_SMALL),
    SHG_PLAIN(float, 32, 96, 1, 192),
    SHG_PLAIN_B(float, 32, 128, SHG_C_F32_128, SHG_NT_F32_128, SHG_MINB_F32_128),
    SHG_PLAIN_B(float, 32, 192, SHG_C_F32_192, SHG_NT_F32_192, SHG_MINB_F32_192),
    SHG_PLAIN_B(float, 32, 256, SHG_C_F32_256, SHG_NT_F32_256, SHG_MINB_F32_256),
    SHG_PLAIN(double, 64, 32, 1, 128),
    SHG_PLAIN(double, 64, 48, 1, 192),
    SHG_PLAIN(double, 64, 64, 1, SHG_NT_F64),
    SHG_PLAIN(double, 64, 96, 2, 192),
    SHG_PLAIN(double, 64, 128, 4, SHG_NT_F64),
    SHG_PLAIN(double, 64, 192, 8, 192),
    SHG_PLAIN(double, 64, 256, 16, SHG_NT_F64),
    // thermal passes (per-voxel n(T), running Δk prefix, Q emission)
    SHG_THERM(float, 32, 32, 1, 128),
    SHG_THERM(float, 32, 64, 1, 256),
    SHG_THERM(float, 32, 128, 2, 256),
    SHG_THERM(float, 32, 256, 8, 256),
    SHG_THERM(double, 64, 32, 1, 128),
    SHG_THERM(double, 64, 64, 1, 256),
    SHG_THERM(double, 64, 128, 4, 256),
    SHG_THERM(double, 64, 256, 16, 256),
};

const PlainVariant* find_plain_variant(int precision, int n, int thermal) {
    for (const auto& v : kPlainVariants)
        if (v.precision == precision && v.n == n && v.thermal == (thermal ? 1 : 0)) return &v;
    return nullptr;
}

}  // namespace shg
