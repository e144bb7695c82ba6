// thermal_grad.cu — shg_thermal_grad: the SH output power of a thermal run and its derivative
// with respect to the oven temperature through the converged temperature field.  No
// counterpart in the reference, which computes no gradients.
//
// The run is the thermal run of shg_solve (Solver.h:321-373).  The oven temperature T_o is
// both the initial temperature and the Dirichlet face value (the reference passes argv[3] as
// both, cuSHG.cu:51-53).  Its derivative is taken in forward mode, since it is one scalar:
//   1. u = dT/dT_o.  Every Jacobi sweep is an affine map of T whose constant part does not
//      depend on T_o once the heat source Q is held fixed, and the initial field moves by 1
//      everywhere.  So u is the homogeneous iteration (T_inf = 0, Q = 0) applied to a field
//      of ones, for the run's total sweep count: the converged field's derivative when the
//      run converged, the exact derivative of its fixed sweep count otherwise.  The
//      temperature is recomputed this way, not stored per sweep.
//   2. The per-voxel tangents u n_p'(T), u n_s'(T), u Δk'(T) (optics_tangent_kernel).
//   3. The tangent-linear march of the last optical pass (ssfm_thermal_jvp.cuh) gives
//      dJ/dT_o.  The feedback of the fields on Q (absorbed power changes with the phase
//      matching) is held fixed: the derivative is first order in the optical-thermal
//      coupling, exact when Q does not depend on T_o.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "shg_host.h"
#include "ssfm_thermal_jvp.cuh"
#include "thermal.h"

namespace shg {

namespace {

template <typename T, int N>
cudaError_t jvp_march(const InstDesc& d, const InstDesc* d_dev, const JvpDesc& jd, cudaStream_t s) {
    using Cfg = MpCfg<T, N>;
    constexpr int row_nt = Cfg::RNT * kJvpPX;
    const size_t row_smem = sizeof(cx<T>) * 4 * (size_t)Cfg::RB * N + sizeof(mult<T>) * N + sizeof(double) * 2 * (row_nt / 32);
    const size_t col_smem = sizeof(cx<T>) * 2 * (size_t)N * Cfg::CW + sizeof(mult<T>) * (2 * (size_t)N + Cfg::CW);
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&] {
        attr_err = cudaFuncSetAttribute(mp_row_jvp_kernel<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem);
        if (attr_err == cudaSuccess)
            attr_err = cudaFuncSetAttribute(mp_col_jvp_kernel<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)col_smem);
    });
    if (attr_err != cudaSuccess) return attr_err;
    MpLayout L = mp_layout<T, N>(nullptr, d.nsteps, true);
    const JvpLayout JL = jvp_layout<T, N>(L);
    cudaError_t e = dev_alloc((void**)&L.base, JL.stride, s);
    if (e != cudaSuccess) return e;
    mp_setup_kernel<T, N><<<1, 256, 0, s>>>(d_dev, L);
    mp_row_jvp_kernel<T, N><<<Cfg::RPART, row_nt, row_smem, s>>>(d_dev, L, JL, jd, -1);
    for (int st = 0; st < d.nsteps; ++st) {
        mp_col_jvp_kernel<T, N><<<dim3(N / Cfg::CW, 2), Cfg::CNT, col_smem, s>>>(d_dev, L, JL, jd, st);
        mp_row_jvp_kernel<T, N><<<Cfg::RPART, row_nt, row_smem, s>>>(d_dev, L, JL, jd, st);
    }
    mp_jvp_sum_kernel<T, N><<<1, 32, 0, s>>>(d_dev, L, jd);
    e = cudaGetLastError();
    const cudaError_t ef = cudaFreeAsync(L.base, s);
    return e != cudaSuccess ? e : ef;
}

// The tangent of a finished thermal run (steps 1-3 above); out[0] the SH power the tangent
// march recomputes, out[1] dJ/dT_o.
template <typename R>
shg_status thermal_tangent(const shg_params& p, const ThermalState& st, double* out, cudaStream_t s) {
    const size_t nt = (size_t)p.nx * p.nx * p.nz, arr = sizeof(R) * nt;
    cudaError_t e;
    char* buf = nullptr;
    if ((e = dev_alloc((void**)&buf, 4 * arr + 256, s)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    R* u = reinterpret_cast<R*>(buf);
    R* ddk = u + nt;
    R* dnp = ddk + nt;
    R* dns = dnp + nt;
    double* dout = reinterpret_cast<double*>(dns + nt);
    shg_status rc = SHG_OK;
    do {
        // 1. u = dT/dT_o: the homogeneous sweeps from a field of ones (no heat source: the
        // sweeps read no Q)
        if ((e = launch_fill<R>(u, nt, (R)1, s)) != cudaSuccess) {
            rc = cuda_fail(e, "tangent set-up");
            break;
        }
        shg_params q = p;
        q.t_inf = 0.0;
        if (st.sweeps > 0 && (rc = heat_sweeps_device(q, u, nullptr, st.sweeps, s)) != SHG_OK) break;
        // 2. per-voxel tangents of the optics
        if ((e = launch_optics_tangent<R>(reinterpret_cast<const R*>(st.T), u, ddk, dnp, dns, p, s)) != cudaSuccess) {
            rc = cuda_fail(e, "optics tangent");
            break;
        }
        R uc_h = 0;
        const size_t ic = (size_t)(p.nx / 2) * p.nx + p.nx / 2;  // IDX(NX/2, NY/2, 0)
        if ((e = cudaMemcpyAsync(&uc_h, u + ic, sizeof(R), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            rc = cuda_fail(e, "read u");
            break;
        }
        // 3. centre-voxel terms (pump, propagators) and the tangent march
        const double uc = (double)uc_h, h = 1e-3, Tc = st.Tc;
        JvpDesc jd;
        std::memset(&jd, 0, sizeof(jd));
        jd.ddk = ddk;
        jd.dnp = dnp;
        jd.dns = dns;
        const InstDesc dp = make_plain_desc(p, Tc + h, Tc + h), dm = make_plain_desc(p, Tc - h, Tc - h);
        const double pert[2][4] = {{dp.amp_re, dp.amp_im, dp.den_re, dp.den_im}, {dm.amp_re, dm.amp_im, dm.den_re, dm.den_im}};
        std::memcpy(jd.pump_pert, pert, sizeof(pert));
        jd.pump_scale = uc / (2 * h);
        jd.adot_p = (dp.a_p - dm.a_p) / (2 * h) * uc;
        jd.adot_s = (dp.a_s - dm.a_s) / (2 * h) * uc;
        jd.out = dout;
        const InstDesc& d = *st.desc;
        if (p.precision == 32)
            e = p.nx == 512 ? jvp_march<float, 512>(d, st.desc_dev, jd, s) : jvp_march<float, 256>(d, st.desc_dev, jd, s);
        else
            e = p.nx == 512 ? jvp_march<double, 512>(d, st.desc_dev, jd, s) : jvp_march<double, 256>(d, st.desc_dev, jd, s);
        if (e != cudaSuccess) { rc = cuda_fail(e, "tangent march"); break; }
        if ((e = cudaMemcpyAsync(out, dout, 2 * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            rc = cuda_fail(e, "tangent result");
            break;
        }
    } while (0);
    cudaFreeAsync(buf, s);
    return rc;
}

}  // namespace

}  // namespace shg

using namespace shg;

extern "C" shg_status shg_thermal_grad(const shg_params* p, shg_thermal_grad_result* out) {
    clear_error();
    shg_status st = shg_check_params(p);
    if (st != SHG_OK) return st;
    if (!out) return fail(SHG_ERR_INVALID, "out is NULL");
    if (!p->thermal) return fail(SHG_ERR_INVALID, "shg_thermal_grad is for thermal runs (thermal == 1)");
    if (p->nx != 256 && p->nx != 512)
        return fail(SHG_ERR_UNSUPPORTED, "the tangent march is built for grid sides 256 and 512 (side %d)", p->nx);
    if (p->waist_y > 0 && p->waist_y != p->waist)
        return fail(SHG_ERR_UNSUPPORTED, "the tangent march is for round beams (waist_y == 0)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    double jv[2] = {0.0, 0.0};
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, s);
    const ThermalHook hook = [&](const ThermalState& ts, cudaStream_t hs) -> shg_status {
        return p->precision == 32 ? thermal_tangent<float>(*p, ts, jv, hs) : thermal_tangent<double>(*p, ts, jv, hs);
    };
    std::memset(out, 0, sizeof(*out));
    shg_status rc = thermal_solve_device(*p, nullptr, nullptr, nullptr, nullptr, &out->stats, s, nullptr, nullptr, &hook);
    cudaEventRecord(t1, s);
    cudaStreamSynchronize(s);
    if (rc == SHG_OK) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        out->sh_power = out->stats.sh_power;
        out->sh_power_tangent_march = jv[0];
        out->d_temp = jv[1];
        out->device_ms = ms;
        if (!std::isfinite(jv[1])) rc = fail(SHG_ERR_NONFINITE, "dJ/dT_oven is %g", jv[1]);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaStreamDestroy(s);
    return rc;
}
