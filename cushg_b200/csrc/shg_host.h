// shg_host.h — host-side helpers shared by the drivers of libshg_b200.
#pragma once

#include <cuda_runtime.h>

#include <functional>

#include "../../include/shg.h"
#include "per_device.h"
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
// dn/dT and dΔk/dT in closed form (crystal.cuh)
double sellmeier_dT(int crystal, double L, double T);
double delta_k_dT(const shg_params& p, double T);
InstDesc make_plain_desc(const shg_params& p, double Tc, double T_dk);
// shg_fp32_error_estimate
double fp32_error_estimate(const shg_params& p);
// Precision the march of plain run p computes in: 64 for an FP32 instance whose predicted
// FP32 error exceeds p.fp32_guard (where a fused FP64 march is built for its side; the
// descriptor then gets out32 = 1), else p.precision.
int run_precision(const shg_params& p);
// The compiled variant plain run p marches on (run_precision, p.march); *out32 = 1 when that is
// the FP64 march of an FP32 instance (its descriptor's out32).
struct PlainVariant;
const PlainVariant* plain_variant_of(const shg_params& p, int* out32);
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
// State of one optical pass of a thermal run, handed to a ThermalHook right after the pass is
// enqueued (before the next outer iteration changes the temperature): the temperature the
// pass used, its per-voxel optics (working real type), its descriptor (host copy and device
// copy), the Jacobi sweeps of this outer iteration (from the previous temperature to this
// one), the centre temperature T(NX/2, NY/2, 0), the pass index and whether it is the run's
// last pass (the one whose fields are the outputs).
class HeatDirect;

struct ThermalState {
    const void* T;
    const void* np;
    const void* ns;
    const void* dk;
    const InstDesc* desc;
    const InstDesc* desc_dev;
    int64_t sweeps;
    double Tc;
    int pass;
    bool last;
    int index;  // the instance's position in its batch (0 for a single run)
    // heat_solver DIRECT: the run's solver (its workspace is free between the run's solves,
    // so a hook may solve with it in stream order); NULL for Jacobi runs
    HeatDirect* heat;
};
using ThermalHook = std::function<shg_status(const ThermalState&, cudaStream_t)>;

shg_status thermal_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                                void* temperature_out, shg_stats* stats, cudaStream_t stream,
                                void* slices_p = nullptr, void* slices_s = nullptr,
                                const ThermalHook* hook = nullptr);
// A batch of thermal runs in lockstep (one grid side, precision and nz): every outer iteration
// runs each instance's Jacobi loop, then one optical pass over the instances still iterating,
// then the hook with their states (count of them, in batch order).  Arrays indexed by instance
// (any may be NULL); stats has count entries.  Slices are for single runs only.
using ThermalBatchHook = std::function<shg_status(const ThermalState* states, int count, cudaStream_t)>;
shg_status thermal_solve_batch(const shg_params* ps, int count, const void* const* signal_in, void* const* pump_out,
                               void* const* signal_out, void* const* temperature_out, shg_stats* stats,
                               cudaStream_t stream, void* slices_p = nullptr, void* slices_s = nullptr,
                               const ThermalBatchHook* hook = nullptr);
// shg_heat_steady_device after validation (heat_direct.cu): *residual = max |J(T) - T|
shg_status heat_steady_device(const shg_params& p, void* temperature, const void* q, double* residual,
                              cudaStream_t stream);
shg_status heat_sweeps_device(const shg_params& p, void* temperature, const void* q, int64_t sweeps,
                              cudaStream_t stream);

}  // namespace shg
