// ssfm_v_f64_large.cu — FP64 variants of the fused march for grid sides 128-256.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    SHG_VARIANT(double, 64, 128, 4, 256, 1, false),  // default
    SHG_VARIANT(double, 64, 128, 8, 128, 2, false),
    SHG_VARIANT(double, 64, 192, 8, 192, 1, false),
    SHG_VARIANT(double, 64, 256, 16, 256, 1, false),
};

VariantTable variants_f64_large() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
