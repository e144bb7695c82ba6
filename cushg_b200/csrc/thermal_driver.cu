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

#include <cmath>
#include <cstring>
#include <utility>

#include "shg_host.h"
#include "ssfm_variants.h"
#include "thermal.h"

namespace shg {

namespace {

template <typename R>
shg_status thermal_run(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                       void* temperature_out, shg_stats* stats, cudaStream_t s, void* slices_p, void* slices_s) {
    const PlainVariant* v = find_plain_variant(p.precision, p.nx, 1);
    if (!v) return fail(SHG_ERR_UNSUPPORTED, "no thermal kernel for grid side %d", p.nx);
    const int n = p.nx, nz = p.nz;
    const size_t nt = (size_t)n * n * nz;
    const size_t arr = sizeof(R) * nt;
    const size_t npart = jacobi_partials(p);
    const size_t bytes = 6 * arr + sizeof(double) * (npart + 4) + sizeof(InstDesc) + 256;
    cudaError_t e;
    char* buf = nullptr;
    if ((e = cudaMallocAsync((void**)&buf, bytes, s)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
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
    cudaEventRecord(t0, s);
    const JacobiCoef<R> k = make_jacobi_coef<R>(p);
    // Solver.h:332: tol = 5e-4 / TSIZE in the working precision
    const double tol = p.jacobi_tol > 0 ? p.jacobi_tol : (double)(R)(5e-4 / (double)nt);
    const int check_every = p.check_every > 0 ? p.check_every : 5000;
    const int64_t max_sweeps = p.max_sweeps > 0 ? p.max_sweeps : ((int64_t)1 << 40);
    const int max_outer = p.max_outer > 0 ? p.max_outer : 20;
    const int depth = p.jacobi_block > 0 ? p.jacobi_block : 4;
    int64_t total = 0;
    int outer = 0;
    double last = 0.0;
    R* cur = Ta;  // holds the latest temperature (the reference's Tinic == Tfinal after its copy)
    R* nxt = Tb;
    CUtensorMap map_a, map_b, map_q;
    do {
        if (depth > 1 && ((rc = make_tb_map<R>(Ta, n, nz, &map_a)) != SHG_OK ||
                          (rc = make_tb_map<R>(Tb, n, nz, &map_b)) != SHG_OK ||
                          (rc = make_tb_map<R>(Q, n, nz, &map_q)) != SHG_OK))
            break;
        if ((e = cudaMemsetAsync(resid, 0, 2 * sizeof(double), s)) != cudaSuccess) { rc = cuda_fail(e, "memset"); break; }
        if ((e = launch_thermal_init<R>(Ta, Tb, Q, p, s)) != cudaSuccess) { rc = cuda_fail(e, "thermal init"); break; }
        for (int g = 0; g < max_outer && rc == SHG_OK; ++g) {
            double red = 1.0, aux = -1.0;
            int64_t counter = 0;
            while (red >= tol) {
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
                if (red == aux) red = 0.5 * tol;
                ++counter;
                if (red < tol) break;
                // the rest of the window, unchecked: `depth` sweeps per launch
                int64_t left = std::min<int64_t>(check_every - 1, max_sweeps - counter);
                while (left > 0) {
                    const int t = (int)std::min<int64_t>(depth, left);
                    if (t >= 2)
                        e = launch_jacobi_tb<R>(cur == Ta ? map_a : map_b, map_q, nxt, k, p.boundary, t, tb_err, s);
                    else
                        e = launch_jacobi<R>(cur, nxt, Q, k, p.boundary, false, p.conv_rule, nullptr, nullptr, s);
                    if (e != cudaSuccess) {
                        rc = cuda_fail(e, "jacobi sweep");
                        break;
                    }
                    std::swap(cur, nxt);
                    counter += t;
                    left -= t;
                }
                if (rc != SHG_OK) break;
            }
            total += counter;
            last = red;
            if (rc != SHG_OK) break;
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
            if ((e = v->launch(ddesc, 1, s)) != cudaSuccess) { rc = cuda_fail(e, "thermal optical pass"); break; }
            ++outer;
            if (counter == 1 && g != 0) break;  // Solver.h:367
        }
        if (rc != SHG_OK) break;
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
        }
    } while (0);
    cudaFreeAsync(buf, s);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "thermal run");
    return rc;
}

}  // namespace

shg_status thermal_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                                void* temperature_out, shg_stats* stats, cudaStream_t stream, void* slices_p,
                                void* slices_s) {
    if (p.precision == 32)
        return thermal_run<float>(p, signal_in, pump_out, signal_out, temperature_out, stats, stream, slices_p, slices_s);
    return thermal_run<double>(p, signal_in, pump_out, signal_out, temperature_out, stats, stream, slices_p, slices_s);
}

}  // namespace shg
