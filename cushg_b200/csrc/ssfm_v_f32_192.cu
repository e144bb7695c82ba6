// ssfm_v_f32_192.cu — FP32 variants of the fused march for 192 x 192 grids.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    SHG_VARIANT(float, 32, 192, 4, 384, 1, false),  // default
    SHG_VARIANT(float, 32, 192, 8, 192, 2, false),
};

VariantTable variants_f32_192() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
