// ssfm_v_thermal.cu — variants of the thermal optical pass (per-voxel n(T), running Δk
// prefix, Q emission), one per precision and grid side.
#include "ssfm_launch.cuh"

namespace shg {

static const PlainVariant kTable[] = {
    SHG_VARIANT(float, 32, 32, 1, 128, 1, true),   SHG_VARIANT(float, 32, 64, 1, 256, 1, true),
    SHG_VARIANT(float, 32, 128, 2, 256, 1, true),  SHG_VARIANT(float, 32, 256, 8, 256, 1, true),
    SHG_VARIANT(double, 64, 32, 1, 128, 1, true),  SHG_VARIANT(double, 64, 64, 1, 256, 1, true),
    SHG_VARIANT(double, 64, 128, 4, 256, 1, true), SHG_VARIANT(double, 64, 256, 16, 256, 1, true),
};

VariantTable variants_thermal() { return {kTable, (int)(sizeof(kTable) / sizeof(kTable[0]))}; }

}  // namespace shg
