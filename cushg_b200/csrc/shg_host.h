// shg_host.h — host-side helpers shared by the drivers of libshg_b200.
#pragma once

#include <cuda_runtime.h>

#include <functional>

#include "../../include/shg.h"
#include "shg_internal.h"

namespace shg {

extern const double kPi, kC, kEps0;

shg_status fail(shg_status st, const char* fmt, ...);
shg_status cuda_fail(cudaError_t e, const char* what);
void clear_error();

// Stream-ordered device memory from the library's own pool on the current device, which keeps
// up to kPoolKeepBytes (or SHG_POOL_KEEP_MB megabytes from the environment, read when the
// pool is created) between calls instead of handing it back at every synchronisation (the
// default pool's release threshold is 0, so a repeated call would map its workspace again
// each time).
constexpr unsigned long long kPoolKeepBytes = 2ull << 30;
// Inside a stream capture it falls back to cudaMallocAsync (a graph memory node).
cudaError_t dev_alloc(void** ptr, size_t bytes, cudaStream_t s);

double sellmeier(int crystal, double L, double T);
double delta_k(const shg_params& p, double T);
InstDesc make_plain_desc(const shg_params& p, double Tc, double T_dk);
size_t complex_bytes(const shg_params& p);

// plain runs (plain_driver.cu)
shg_status plain_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                              shg_stats* stats, cudaStream_t stream, void* slices_p = nullptr,
                              void* slices_s = nullptr, const double* poling_dev = nullptr);
// pump_host / signal_host (optional, indexed like params): host arrays the outputs are copied
// to, each group's right after its march on the stream that ran it.
shg_status plain_solve_batch(const shg_params* params, int count, void* const* pump_out, void* const* signal_out,
                             double* sh_power_out, cudaStream_t stream, void* const* pump_host = nullptr,
                             void* const* signal_host = nullptr);

// thermal runs (thermal_driver.cu)
// State of the last optical pass of a thermal run, handed to a ThermalHook before the run
// frees its buffers: the temperature the pass used, its per-voxel optics (working real type),
// its descriptor (host copy and device copy), the Jacobi sweeps of the whole run and the
// centre temperature T(NX/2, NY/2, 0).
struct ThermalState {
    const void* T;
    const void* np;
    const void* ns;
    const void* dk;
    const InstDesc* desc;
    const InstDesc* desc_dev;
    int64_t sweeps;
    double Tc;
};
using ThermalHook = std::function<shg_status(const ThermalState&, cudaStream_t)>;

shg_status thermal_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                                void* temperature_out, shg_stats* stats, cudaStream_t stream,
                                void* slices_p = nullptr, void* slices_s = nullptr,
                                const ThermalHook* hook = nullptr);
shg_status heat_sweeps_device(const shg_params& p, void* temperature, const void* q, int64_t sweeps,
                              cudaStream_t stream);

}  // namespace shg
