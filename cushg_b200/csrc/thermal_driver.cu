// thermal_driver.cu — host driver of thermal runs: the -DTHERMAL outer optical-thermal
// loop of Solver::run (src/headers/Solver.h:321-373).
//
//   T = temp, oven faces = t_peltier, Q = 0                 (Solver.h:319-323)
//   repeat up to max_outer times:
//     Jacobi sweeps until the convergence value, taken on the first sweep of every
//     window of check_every sweeps, falls below tol; a value equal to the previous
//     check counts as converged                              (Solver.h:335-355)
//     (the checked sweep runs alone; the rest of the window runs jacobi_block sweeps
//     per launch through the temporally blocked kernel of jacobi_tb.cu)
//     Δk, n_p, n_s from T; pump, SH and propagators at T(NX/2, NY/2, 0)   (Solver.h:359-362)
//     one optical pass of nz steps that emits Q slice by slice (Solver.h:365, 300)
//     stop after a pass whose Jacobi loop converged at its first sweep (Solver.h:367)
//
// The host reads one scalar per check window; everything else stays on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>

#include "shg_host.h"
#include "ssfm_variants.h"
#include "thermal.h"

namespace shg {

namespace {

// Sweeps per launch: the caller's jacobi_block, else one.  On B200 the one-sweep kernel
// (one voxel per thread, neighbours through L1 / L2) measured faster than the blocked kernel
// at every depth and size tried, from L2-resident grids (128x128x200) to grids 20x the L2
// (512x512x250 FP64): 16.6 vs 28.9 us per sweep at 128x128x200 FP64, 325 vs 357 us at
// 512x512x250 FP64.  The blocked kernel is issue-bound (halo recomputation, one barrier per
// plane), not memory-bound.
int sweep_depth(const shg_params& p) {
    if (p.jacobi_block > 0) return p.jacobi_block;
    return 1;
}

// TMA maps of the two temperature buffers and Q for the blocked sweeps.
template <typename R>
struct SweepMaps {
    CUtensorMap a, b, q;
};

template <typename R>
shg_status make_sweep_maps(const R* Ta, const R* Tb, const R* Q, int n, int nz, SweepMaps<R>* m) {
    shg_status rc;
    if ((rc = make_tb_map<R>(Ta, n, nz, &m->a)) != SHG_OK) return rc;
    if ((rc = make_tb_map<R>(Tb, n, nz, &m->b)) != SHG_OK) return rc;
    return make_tb_map<R>(Q, n, nz, &m->q);
}

// `count` unchecked sweeps, `depth` per launch, ping-ponging cur / nxt (Ta and Tb of the
// maps); on return cur holds the latest temperature.
template <typename R>
cudaError_t run_sweeps(R*& cur, R*& nxt, const R* Ta, const SweepMaps<R>& m, const R* Q, const JacobiCoef<R>& k,
                       int boundary, int depth, int64_t count, unsigned* tb_err, cudaStream_t s) {
    while (count > 0) {
        const int t = (int)std::min<int64_t>(depth, count);
        cudaError_t e;
        if (t >= 2)
            e = launch_jacobi_tb<R>(cur == Ta ? m.a : m.b, m.q, nxt, k, boundary, t, tb_err, s);
        else
            e = launch_jacobi<R>(cur, nxt, Q, k, boundary, false, 0, nullptr, nullptr, s);
        if (e != cudaSuccess) return e;
        std::swap(cur, nxt);
        count -= t;
    }
    return cudaSuccess;
}

template <typename R>
shg_status thermal_run(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                       void* temperature_out, shg_stats* stats, cudaStream_t s, void* slices_p, void* slices_s,
                       const ThermalHook* hook) {
    const PlainVariant* v = find_plain_variant(p.precision, p.nx, 1, p.march);
    if (!v) return fail(SHG_ERR_UNSUPPORTED, "no thermal kernel for grid side %d", p.nx);
    const int n = p.nx, nz = p.nz;
    const size_t nt = (size_t)n * n * nz;
    const size_t arr = sizeof(R) * nt;
    const size_t npart = jacobi_partials(p);
    const size_t bytes = 6 * arr + sizeof(double) * (npart + 4) + sizeof(InstDesc) + 256;
    cudaError_t e;
    char* buf = nullptr;
    if ((e = dev_alloc((void**)&buf, bytes, s)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    R* Ta = reinterpret_cast<R*>(buf);
    R* Tb = Ta + nt;
    R* Q = Tb + nt;
    R* DK = Q + nt;
    R* NP = DK + nt;
    R* NS = NP + nt;
    double* partial = reinterpret_cast<double*>(NS + nt);
    double* resid = partial + npart;   // [0] convergence value, [1] staging-error word
    double* power = resid + 2;         // [2]
    InstDesc* ddesc = reinterpret_cast<InstDesc*>(((uintptr_t)(power + 2) + 255) & ~(uintptr_t)255);
    unsigned* tb_err = reinterpret_cast<unsigned*>(resid + 1);  // set by a blocked sweep whose staging timed out

    shg_status rc = SHG_OK;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    // per-phase timing: the Jacobi loop of an outer iteration runs between ej[0] and ej[1],
    // its optics and optical pass between ej[1] and ej[2]
    cudaEvent_t ej[3] = {nullptr, nullptr, nullptr};
    for (auto& ev : ej) cudaEventCreate(&ev);
    double jacobi_ms = 0.0, optics_ms = 0.0;
    cudaEventRecord(t0, s);
    const JacobiCoef<R> k = make_jacobi_coef<R>(p);
    // Solver.h:332: tol = 5e-4 / TSIZE in the working precision
    const double tol = p.jacobi_tol > 0 ? p.jacobi_tol : (double)(R)(5e-4 / (double)nt);
    const int check_every = p.check_every > 0 ? p.check_every : 5000;
    const int64_t max_sweeps = p.max_sweeps > 0 ? p.max_sweeps : ((int64_t)1 << 40);
    const int max_outer = p.max_outer > 0 ? p.max_outer : 20;
    const int depth = sweep_depth(p);
    int64_t total = 0;
    int outer = 0;
    InstDesc last_d;
    double last_Tc = 0.0;
    double last = 0.0;
    R* cur = Ta;  // holds the latest temperature (the reference's Tinic == Tfinal after its copy)
    R* nxt = Tb;
    SweepMaps<R> maps;
    do {
        if (depth > 1 && (rc = make_sweep_maps<R>(Ta, Tb, Q, n, nz, &maps)) != SHG_OK) break;
        if ((e = cudaMemsetAsync(resid, 0, 2 * sizeof(double), s)) != cudaSuccess) { rc = cuda_fail(e, "memset"); break; }
        if ((e = launch_thermal_init<R>(Ta, Tb, Q, p, s)) != cudaSuccess) { rc = cuda_fail(e, "thermal init"); break; }
        for (int g = 0; g < max_outer && rc == SHG_OK; ++g) {
            double red = 1.0, aux = -1.0;
            int64_t counter = 0;
            cudaEventRecord(ej[0], s);
            if (p.conv_rule == SHG_CONV_FIXED) {
                // exactly max_sweeps sweeps; the last one reports max |Tf - Ti|
                if ((e = run_sweeps<R>(cur, nxt, Ta, maps, Q, k, p.boundary, depth, max_sweeps - 1, tb_err, s)) !=
                        cudaSuccess ||
                    (e = launch_jacobi<R>(cur, nxt, Q, k, p.boundary, true, SHG_CONV_MAXABS, partial, resid, s)) !=
                        cudaSuccess) {
                    rc = cuda_fail(e, "jacobi sweep");
                    break;
                }
                std::swap(cur, nxt);
                double h[2] = {0.0, 0.0};
                if ((e = cudaMemcpyAsync(h, resid, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                    (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                    rc = cuda_fail(e, "jacobi residual");
                    break;
                }
                unsigned staged_err = 0;
                std::memcpy(&staged_err, &h[1], sizeof(staged_err));
                if (staged_err) {
                    rc = fail(SHG_ERR_CUDA, "blocked Jacobi sweep: a staged plane did not arrive");
                    break;
                }
                red = h[0];
                counter = max_sweeps;
                if (!std::isfinite(red)) {
                    rc = fail(SHG_ERR_NONFINITE, "Jacobi residual is %g after %lld sweeps", red, (long long)counter);
                    break;
                }
            }
            while (p.conv_rule != SHG_CONV_FIXED && red >= tol) {
                if (counter >= max_sweeps) {
                    rc = fail(SHG_ERR_NOT_CONVERGED, "Jacobi: %lld sweeps without reaching %g (last %g)",
                              (long long)counter, tol, red);
                    break;
                }
                // the checked sweep of this window
                if ((e = launch_jacobi<R>(cur, nxt, Q, k, p.boundary, true, p.conv_rule, partial, resid, s)) != cudaSuccess) {
                    rc = cuda_fail(e, "jacobi sweep");
                    break;
                }
                std::swap(cur, nxt);
                double h[2] = {0.0, 0.0};
                if ((e = cudaMemcpyAsync(h, resid, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                    (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                    rc = cuda_fail(e, "jacobi residual");
                    break;
                }
                unsigned staged_err = 0;
                std::memcpy(&staged_err, &h[1], sizeof(staged_err));
                if (staged_err) {
                    rc = fail(SHG_ERR_CUDA, "blocked Jacobi sweep: a staged plane did not arrive");
                    break;
                }
                if (counter > 0) aux = red;
                red = p.conv_rule == SHG_CONV_MAXABS ? h[0] : (double)(R)(std::sqrt((R)h[0]) / (R)(double)nt);
                if (!std::isfinite(red)) {
                    rc = fail(SHG_ERR_NONFINITE, "Jacobi residual is %g after %lld sweeps", red, (long long)counter);
                    break;
                }
                if (red == aux) red = 0.5 * tol;
                ++counter;
                if (red < tol) break;
                // the rest of the window, unchecked: `depth` sweeps per launch
                const int64_t left = std::min<int64_t>(check_every - 1, max_sweeps - counter);
                if ((e = run_sweeps<R>(cur, nxt, Ta, maps, Q, k, p.boundary, depth, left, tb_err, s)) != cudaSuccess) {
                    rc = cuda_fail(e, "jacobi sweep");
                    break;
                }
                counter += std::max<int64_t>(left, 0);
            }
            total += counter;
            last = red;
            if (rc != SHG_OK) break;
            cudaEventRecord(ej[1], s);
            // optical pass from the converged temperature
            if ((e = launch_optics<R>(cur, DK, NP, NS, p, s)) != cudaSuccess) { rc = cuda_fail(e, "optics"); break; }
            R tc_h = 0;
            const size_t ic = (size_t)(n / 2) * n + n / 2;  // IDX(NX/2, NY/2, 0)
            if ((e = cudaMemcpyAsync(&tc_h, cur + ic, sizeof(R), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                rc = cuda_fail(e, "read T");
                break;
            }
            const double Tc = (double)tc_h;
            InstDesc d = make_plain_desc(p, Tc, Tc);
            const double dQ = 2.0 * p.deff / kPi, lp = p.lambda_p, ls = 0.5 * lp;
            d.kf_p = 1.0 * kPi * dQ / lp;
            d.kf_s = 0.5 * kPi * dQ / ls;
            d.bf_s = p.beta_s * 0.5 * kEps0 * kC;
            d.q_p = p.alpha_p * 0.5 * kC * kEps0;
            d.q_s = p.alpha_s * 0.5 * kC * kEps0;
            d.q_h = 0.5 * kC * kEps0;
            d.beta_s = p.beta_s;
            d.t_np = NP;
            d.t_ns = NS;
            d.t_dk = DK;
            d.t_q = Q;
            d.pw_s = d.pw_p = 0.5 * kEps0 * kC * d.dx * d.dy;
            d.signal_in = signal_in;
            d.has_signal_in = signal_in ? 1 : 0;
            d.pump_out = pump_out;
            d.signal_out = signal_out;
            d.power_out = power;
            d.slices_p = slices_p;
            d.slices_s = slices_s;
            d.nslices = (slices_p || slices_s) ? nz : 0;
            if ((e = cudaMemcpyAsync(ddesc, &d, sizeof(d), cudaMemcpyHostToDevice, s)) != cudaSuccess) {
                rc = cuda_fail(e, "descriptor");
                break;
            }
            if ((e = run_variant(v, ddesc, &d, 1, nullptr, s)) != cudaSuccess) { rc = cuda_fail(e, "thermal optical pass"); break; }
            last_d = d;
            last_Tc = Tc;
            ++outer;
            cudaEventRecord(ej[2], s);
            if ((e = cudaEventSynchronize(ej[2])) != cudaSuccess) { rc = cuda_fail(e, "thermal optical pass"); break; }
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ej[0], ej[1]);
            cudaEventElapsedTime(&b, ej[1], ej[2]);
            jacobi_ms += a;
            optics_ms += b;
            if (p.conv_rule != SHG_CONV_FIXED && counter == 1 && g != 0) break;  // Solver.h:367
        }
        if (rc != SHG_OK) break;
        if (hook && outer > 0) {
            const ThermalState st = {cur, NP, NS, DK, &last_d, ddesc, total, last_Tc};
            if ((rc = (*hook)(st, s)) != SHG_OK) break;
        }
        if (temperature_out &&
            (e = cudaMemcpyAsync(temperature_out, cur, arr, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) {
            rc = cuda_fail(e, "temperature out");
            break;
        }
        cudaEventRecord(t1, s);
        if (stats) {
            double h[2] = {0, 0};
            if ((e = cudaMemcpyAsync(h, power, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                rc = cuda_fail(e, "thermal run");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            std::memset(stats, 0, sizeof(*stats));
            stats->sh_power = h[0];
            stats->pump_power = h[1];
            stats->jacobi_sweeps = total;
            stats->outer_iterations = outer;
            stats->steps = nz;
            stats->last_residual = last;
            stats->device_ms = ms;
            stats->jacobi_ms = jacobi_ms;
            stats->optics_ms = optics_ms;
            if (!std::isfinite(h[0]) || !std::isfinite(h[1]))
                rc = fail(SHG_ERR_NONFINITE, "SH / pump power %g / %g", h[0], h[1]);
        }
    } while (0);
    cudaFreeAsync(buf, s);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    for (cudaEvent_t ev : ej) cudaEventDestroy(ev);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "thermal run");
    return rc;
}

template <typename R>
shg_status heat_run(const shg_params& p, R* T, const R* Q, int64_t sweeps, cudaStream_t s) {
    const int n = p.nx, nz = p.nz;
    const size_t nt = (size_t)n * n * nz, arr = sizeof(R) * nt;
    // Q null (no heat source, the sweeps read none): one sweep per launch, whose kernels
    // take a null Q as zero
    const int depth = Q ? sweep_depth(p) : 1;
    cudaError_t e;
    char* buf = nullptr;
    if ((e = dev_alloc((void**)&buf, arr + 256, s)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    R* other = reinterpret_cast<R*>(buf);
    unsigned* tb_err = reinterpret_cast<unsigned*>(buf + arr);
    shg_status rc = SHG_OK;
    do {
        SweepMaps<R> maps;
        if (depth > 1 && (rc = make_sweep_maps<R>(T, other, Q, n, nz, &maps)) != SHG_OK) break;
        // both buffers start alike, so the voxels no sweep writes (Dirichlet faces) agree
        if ((e = cudaMemcpyAsync(other, T, arr, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
            (e = cudaMemsetAsync(tb_err, 0, sizeof(unsigned), s)) != cudaSuccess) {
            rc = cuda_fail(e, "heat sweeps set-up");
            break;
        }
        const JacobiCoef<R> k = make_jacobi_coef<R>(p);
        R* cur = T;
        R* nxt = other;
        if ((e = run_sweeps<R>(cur, nxt, T, maps, Q, k, p.boundary, depth, sweeps, tb_err, s)) != cudaSuccess) {
            rc = cuda_fail(e, "jacobi sweep");
            break;
        }
        if (cur != T && (e = cudaMemcpyAsync(T, cur, arr, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) {
            rc = cuda_fail(e, "heat sweeps result");
            break;
        }
        unsigned h = 0;
        if ((e = cudaMemcpyAsync(&h, tb_err, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            rc = cuda_fail(e, "heat sweeps");
            break;
        }
        if (h) rc = fail(SHG_ERR_CUDA, "blocked Jacobi sweep: a staged plane did not arrive");
    } while (0);
    cudaFreeAsync(buf, s);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "heat sweeps");
    return rc;
}

}  // namespace

shg_status heat_sweeps_device(const shg_params& p, void* temperature, const void* q, int64_t sweeps,
                              cudaStream_t stream) {
    if (p.precision == 32)
        return heat_run<float>(p, reinterpret_cast<float*>(temperature), reinterpret_cast<const float*>(q), sweeps, stream);
    return heat_run<double>(p, reinterpret_cast<double*>(temperature), reinterpret_cast<const double*>(q), sweeps, stream);
}

shg_status thermal_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                                void* temperature_out, shg_stats* stats, cudaStream_t stream, void* slices_p,
                                void* slices_s, const ThermalHook* hook) {
    if (p.precision == 32)
        return thermal_run<float>(p, signal_in, pump_out, signal_out, temperature_out, stats, stream, slices_p, slices_s,
                                  hook);
    return thermal_run<double>(p, signal_in, pump_out, signal_out, temperature_out, stats, stream, slices_p, slices_s,
                               hook);
}

}  // namespace shg
