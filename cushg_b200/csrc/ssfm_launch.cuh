// ssfm_launch.cuh — launcher of one compiled variant of the fused SSFM march, shared by the
// translation units that instantiate the variants (ssfm_v_*.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "per_device.h"

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
    // once per device: kernel attributes and the clusters that fit on the device at once
    // (the size of a persistent launch)
    static PerDevice<int> state;
    int resident = 0;
    const cudaError_t attr_err = state.get(
        [&](int dev, int& res) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem_bytes);
            if (e == cudaSuccess && C > 8) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
            if (C > 1) {
                cudaLaunchConfig_t occ = cfg;
                occ.gridDim = dim3(C, 1, 1);
                e = cudaOccupancyMaxActiveClusters(&res, kern, &occ);
            } else {
                int sms = 0, per_sm = 0;
                e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, Cfg::smem_bytes);
                res = sms * per_sm;
            }
            if (e == cudaSuccess && res < 1) e = cudaErrorInvalidConfiguration;
            return e;
        },
        &resident);
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
