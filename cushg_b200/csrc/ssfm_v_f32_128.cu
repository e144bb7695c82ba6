// ssfm_v_f32_128.cu — FP32 variants of the fused march for 128 x 128 grids.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    SHG_VARIANT(float, 32, 128, 2, 512, 1, false),  // default
    SHG_VARIANT(float, 32, 128, 2, 256, 1, false),
    SHG_VARIANT(float, 32, 128, 4, 256, 2, false),
};

VariantTable variants_f32_128() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
