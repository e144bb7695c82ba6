// ssfm_v_f64_small.cu — FP64 variants of the fused march for grid sides 32-96.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    SHG_VARIANT(double, 64, 32, 1, 128, 1, false),
    SHG_VARIANT(double, 64, 48, 1, 192, 1, false),
    // 64: two-CTA clusters at two per SM measured 27.3 against 26.7 G pt-steps/s
    SHG_VARIANT(double, 64, 64, 2, 256, 2, false),
    SHG_VARIANT(double, 64, 64, 1, 256, 1, false),
    SHG_VARIANT(double, 64, 96, 2, 192, 1, false),
};

VariantTable variants_f64_small() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
