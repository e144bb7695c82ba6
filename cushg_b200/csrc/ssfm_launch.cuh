// ssfm_launch.cuh — launcher of one compiled variant of the fused SSFM march, shared by the
// translation units that instantiate the variants (ssfm_v_*.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "ssfm_plain.cuh"
#include "ssfm_variants.h"

namespace shg {

template <typename T, int N, int C, int NT, bool THERM, int MINB>
cudaError_t launch_plain(const InstDesc* descs, int count, int* queue, cudaStream_t stream) {
    using Cfg = PlainCfg<T, N, C, NT, THERM>;
    auto kern = ssfm_plain_kernel<T, N, C, NT, THERM, MINB>;
    cudaLaunchConfig_t cfg = {};
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
    // once per process: kernel attributes and the clusters that fit on the device at once
    // (the size of a persistent launch); the device is the current one at the first call
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    static int resident = 0;
    std::call_once(once, [&]() {
        attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem_bytes);
        if (attr_err == cudaSuccess && C > 8)
            attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (attr_err != cudaSuccess) return;
        if (C > 1) {
            cfg.gridDim = dim3(C, 1, 1);
            attr_err = cudaOccupancyMaxActiveClusters(&resident, kern, &cfg);
        } else {
            int dev = 0, sms = 0, per_sm = 0;
            attr_err = cudaGetDevice(&dev);
            if (attr_err == cudaSuccess) attr_err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (attr_err == cudaSuccess)
                attr_err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, Cfg::smem_bytes);
            resident = sms * per_sm;
        }
        if (attr_err == cudaSuccess && resident < 1) attr_err = cudaErrorInvalidConfiguration;
    });
    if (attr_err != cudaSuccess) return attr_err;
    if (count <= 0) return cudaSuccess;
    const int clusters = queue ? std::min(count, resident) : count;
    cfg.gridDim = dim3((unsigned)(clusters * C), 1, 1);
    return cudaLaunchKernelEx(&cfg, kern, descs, count, queue);
}

#define SHG_VARIANT(T, PREC, N, C, NT, MINB, THERM)                                                  \
    {PREC, N, C, NT, MINB, THERM ? 1 : 0, PlainCfg<T, N, C, NT, THERM>::smem_bytes,                   \
     &launch_plain<T, N, C, NT, THERM, MINB>, nullptr}

}  // namespace shg
