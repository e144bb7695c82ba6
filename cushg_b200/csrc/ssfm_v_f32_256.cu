// ssfm_v_f32_256.cu — FP32 variants of the fused march for 256 x 256 grids.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    SHG_VARIANT(float, 32, 256, 16, 256, 2, false),  // default: 16-CTA clusters, 2 CTAs per SM
    SHG_VARIANT(float, 32, 256, 8, 256, 1, false),
    SHG_VARIANT(float, 32, 256, 16, 512, 1, false),
};

VariantTable variants_f32_256() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
