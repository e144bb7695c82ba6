// ssfm_variants.h — registry of the compiled SSFM kernel variants.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "shg_internal.h"

namespace shg {

// One compiled (precision, grid side) variant of the fused plain march.
struct PlainVariant {
    int precision;     // 32 or 64
    int n;             // grid side
    int cluster;       // CTAs per instance
    int threads;       // threads per CTA
    int thermal;       // 1: thermal pass (per-voxel optics, Q emission)
    size_t smem;       // dynamic shared memory per CTA
    cudaError_t (*launch)(const InstDesc* descs, int count, cudaStream_t stream);
};

const PlainVariant* find_plain_variant(int precision, int n, int thermal = 0);

}  // namespace shg
