// thermal_driver.cu — host driver of thermal runs (the -DTHERMAL outer optical-thermal
// loop of src/headers/Solver.h:321-373).
#include "shg_host.h"

namespace shg {

shg_status thermal_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                                void* temperature_out, shg_stats* stats, cudaStream_t stream) {
    (void)p; (void)signal_in; (void)pump_out; (void)signal_out; (void)temperature_out; (void)stats; (void)stream;
    return fail(SHG_ERR_UNSUPPORTED, "thermal runs are not built yet");
}

}  // namespace shg
