// shg_host.h — host-side helpers shared by the drivers of libshg_b200.
#pragma once

#include <cuda_runtime.h>

#include "../../include/shg.h"
#include "shg_internal.h"

namespace shg {

extern const double kPi, kC, kEps0;

shg_status fail(shg_status st, const char* fmt, ...);
shg_status cuda_fail(cudaError_t e, const char* what);
void clear_error();

double sellmeier(double L, double T);
double delta_k(const shg_params& p, double T);
InstDesc make_plain_desc(const shg_params& p, double Tc, double T_dk);
size_t complex_bytes(const shg_params& p);

// plain runs (plain_driver.cu)
shg_status plain_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                              shg_stats* stats, cudaStream_t stream, void* slices_p = nullptr,
                              void* slices_s = nullptr, const double* poling_dev = nullptr);
shg_status plain_solve_batch(const shg_params* params, int count, void* const* pump_out, void* const* signal_out,
                             double* sh_power_out, cudaStream_t stream);

// thermal runs (thermal_driver.cu)
shg_status thermal_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                                void* temperature_out, shg_stats* stats, cudaStream_t stream,
                                void* slices_p = nullptr, void* slices_s = nullptr);
shg_status heat_sweeps_device(const shg_params& p, void* temperature, const void* q, int64_t sweeps,
                              cudaStream_t stream);

}  // namespace shg
