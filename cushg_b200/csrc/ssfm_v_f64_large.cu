// ssfm_v_f64_large.cu — FP64 variants of the fused march for grid sides 128-256.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    // the first of each side is its default: the split shg_autotune measured fastest on a
    // device-filling batch of the class (128: 19.5 against 18.3 G pt-steps/s; 192: 14.3
    // against 12.4 G)
    SHG_VARIANT(double, 64, 128, 8, 128, 2, false),
    SHG_VARIANT(double, 64, 128, 4, 256, 1, false),
    SHG_VARIANT(double, 64, 192, 16, 192, 2, false),
    SHG_VARIANT(double, 64, 192, 8, 192, 1, false),
    SHG_VARIANT(double, 64, 256, 16, 256, 1, false),
};

VariantTable variants_f64_large() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
