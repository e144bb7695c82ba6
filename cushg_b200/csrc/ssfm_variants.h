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

// Launch of a multi-pass march (ssfm_multipass.cuh): device and host copies of the
// descriptors (the host sequences the per-step launches from the step counts).
using MpLaunch = cudaError_t (*)(const InstDesc* dev_descs, const InstDesc* host_descs, int count,
                                 cudaStream_t stream);

struct PlainVariant {
    int precision;  // 32 or 64
    int n;          // grid side
    int cluster;    // CTAs per instance (0: multi-pass, the planes in global memory)
    int threads;    // threads per CTA (multi-pass: of the row pass)
    int minb;       // CTAs per SM the register budget targets
    int thermal;    // 1: thermal pass (per-voxel optics, Q emission)
    size_t smem;    // dynamic shared memory per CTA (multi-pass: of the row pass)
    PlainLaunch launch;  // fused cluster march, or null
    MpLaunch mp;         // multi-pass march, or null
};

// Run `count` instances through variant v (either kind); queue as for PlainLaunch.
inline cudaError_t run_variant(const PlainVariant* v, const InstDesc* dev_descs, const InstDesc* host_descs, int count,
                               int* queue, cudaStream_t stream) {
    return v->mp ? v->mp(dev_descs, host_descs, count, stream) : v->launch(dev_descs, count, queue, stream);
}

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
VariantTable variants_multipass();

// The variant the drivers use for (precision, n, thermal) under march preference `march`
// (SHG_MARCH_*): automatic = the tuned one if shg_autotune chose one, else the default
// (the first compiled fused variant, else the multi-pass one); fused / multi-pass = the
// default of that kind.  Null if none is built.
const PlainVariant* find_plain_variant(int precision, int n, int thermal = 0, int march = 0);
// Every compiled plain variant of (precision, n), default first; returns how many.
int plain_candidates(int precision, int n, const PlainVariant** out, int max);
// Make v the variant find_plain_variant returns for its (precision, n, thermal).
void set_plain_choice(const PlainVariant* v);
// forget every tuned choice: later runs use the compiled defaults
void clear_plain_choices();

}  // namespace shg
