// ssfm_variants.h — registry of the compiled variants of the fused SSFM march.
//
// A variant fixes the precision, the grid side N, the cluster split C (CTAs per instance),
// the threads per CTA and the CTAs per SM the register budget targets.  Each (precision, N)
// has a default variant and possibly alternatives with another split; shg_autotune times
// them and makes the fastest the one the drivers use.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "shg_internal.h"

namespace shg {

// Launch of `count` instances from `descs`.  queue != nullptr: a persistent launch of at
// most as many clusters as fit on the device, fed by the work queue *queue (an int the
// caller zeroes, stream-ordered, before the launch).  queue == nullptr: one cluster per
// instance.
using PlainLaunch = cudaError_t (*)(const InstDesc* descs, int count, int* queue, cudaStream_t stream);

struct PlainVariant {
    int precision;  // 32 or 64
    int n;          // grid side
    int cluster;    // CTAs per instance
    int threads;    // threads per CTA
    int minb;       // CTAs per SM the register budget targets
    int thermal;    // 1: thermal pass (per-voxel optics, Q emission)
    size_t smem;    // dynamic shared memory per CTA
    PlainLaunch launch;
};

struct VariantTable {
    const PlainVariant* v;
    int count;
};

// per translation unit tables (ssfm_v_*.cu)
VariantTable variants_f32_small();
VariantTable variants_f32_128();
VariantTable variants_f32_192();
VariantTable variants_f32_256();
VariantTable variants_f64_small();
VariantTable variants_f64_large();
VariantTable variants_thermal();

// The variant the drivers use for (precision, n, thermal): the tuned one if shg_autotune
// chose one, else the default (the first compiled).
const PlainVariant* find_plain_variant(int precision, int n, int thermal = 0);
// Every compiled plain variant of (precision, n), default first; returns how many.
int plain_candidates(int precision, int n, const PlainVariant** out, int max);
// Make v the variant find_plain_variant returns for its (precision, n, thermal).
void set_plain_choice(const PlainVariant* v);

}  // namespace shg
