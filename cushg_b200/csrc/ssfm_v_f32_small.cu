// ssfm_v_f32_small.cu — FP32 variants of the fused march for grid sides 32-96 (one CTA per
// instance).  The first variant of each side is the default.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    SHG_VARIANT(float, 32, 32, 1, 128, 1, false),
    SHG_VARIANT(float, 32, 48, 1, 192, 1, false),
    SHG_VARIANT(float, 32, 64, 1, 512, 1, false),
    SHG_VARIANT(float, 32, 64, 1, 256, 2, false),
    SHG_VARIANT(float, 32, 96, 1, 192, 1, false),
};

VariantTable variants_f32_small() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
