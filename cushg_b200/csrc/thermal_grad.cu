// thermal_grad.cu — shg_thermal_grad: the SH output power of a thermal run and its derivative
// with respect to the oven temperature through the converged temperature field.  No
// counterpart in the reference, which computes no gradients.
//
// The run is the thermal run of shg_solve (Solver.h:321-373).  The oven temperature T_o is
// both the initial temperature and the Dirichlet face value (the reference passes argv[3] as
// both, cuSHG.cu:51-53).  Its derivative is taken in forward mode, since it is one scalar,
// alongside the run, outer iteration by outer iteration:
//   1. u = dT/dT_o.  A Jacobi sweep is affine in (T, Q) with a constant part (T_inf) that does
//      not depend on T_o, and the initial field and the faces move by 1.  So u starts at one
//      everywhere and each outer iteration applies its sweep count of the same sweep with
//      T_inf = 0 and the heat source replaced by q = dQ/dT_o of the previous optical pass
//      (zero before the first).  The temperature is recomputed, not stored per sweep.
//   2. The per-voxel tangents u n_p'(T), u n_s'(T), u Δk'(T) (optics_tangent_kernel, closed
//      form).
//   3. The tangent-linear march of the pass (ssfm_thermal_jvp.cuh): the JVP of every RK4
//      application, the tangent of the running Δk prefix, the propagator term and the
//      centre-voxel pump.  Of the last pass it gives dJ/dT_o.
//   4. Every other pass's tangent march also emits q, the tangent of its heat source
//      (Tfield.h:260-276), which feeds step 1 of the next outer iteration.  So the feedback
//      of the fields on the temperature (absorbed power changes with the phase matching) is
//      carried through every outer iteration: the result is the derivative of the whole
//      computed procedure, for its sweep counts.
//   With heat_solver DIRECT each outer iteration's temperature is the exact solution of the
//   sweep's linear system, so step 1 is that solve applied to u's sources instead of sweeps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "shg_host.h"
#include "ssfm_thermal_jvp.cuh"
#include "thermal.h"

namespace shg {

namespace {

// The tangent-linear march of `count` instances of one class (host and device descriptors,
// device JvpDescs), all in the same launches: grids over the instances.
template <typename T, int N>
cudaError_t jvp_march(const InstDesc* hdescs, const InstDesc* d_dev, const JvpDesc* jds_dev, int count, cudaStream_t s) {
    using Cfg = MpCfg<T, N>;
    constexpr int row_nt = Cfg::RNT * kJvpPX;
    const size_t row_smem = sizeof(cx<T>) * 4 * (size_t)Cfg::RB * N + sizeof(mult<T>) * N + sizeof(double) * 2 * (row_nt / 32);
    const size_t col_smem = sizeof(cx<T>) * 2 * (size_t)N * Cfg::CW + sizeof(mult<T>) * (2 * (size_t)N + Cfg::CW);
    static PerDevice<int> state;  // kernel attributes, once per device
    const cudaError_t attr_err = state.get([&](int, int&) {
        cudaError_t e =
            cudaFuncSetAttribute(mp_row_jvp_kernel<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(mp_col_jvp_kernel<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem);
        return e;
    });
    if (attr_err != cudaSuccess) return attr_err;
    if (count <= 0) return cudaSuccess;
    int max_steps = 0;
    for (int i = 0; i < count; ++i) max_steps = std::max(max_steps, (int)hdescs[i].nsteps);
    MpLayout L = mp_layout<T, N>(nullptr, max_steps, true);
    const JvpLayout JL = jvp_layout<T, N>(L);
    L.stride = JL.stride;  // an instance's region: the march's workspace, then its tangent planes
    cudaError_t e = dev_alloc((void**)&L.base, JL.stride * (size_t)count, s);
    if (e != cudaSuccess) return e;
    mp_setup_kernel<T, N><<<count, 256, 0, s>>>(d_dev, L);
    mp_row_jvp_kernel<T, N><<<dim3(Cfg::RPART, count), row_nt, row_smem, s>>>(d_dev, L, JL, jds_dev, -1);
    for (int st = 0; st < max_steps; ++st) {
        mp_col_jvp_kernel<T, N><<<dim3(N / Cfg::CW, 2, count), Cfg::CNT, col_smem, s>>>(d_dev, L, JL, jds_dev, st);
        mp_row_jvp_kernel<T, N><<<dim3(Cfg::RPART, count), row_nt, row_smem, s>>>(d_dev, L, JL, jds_dev, st);
    }
    mp_jvp_sum_kernel<T, N><<<count, 32, 0, s>>>(d_dev, L, jds_dev);
    e = cudaGetLastError();
    const cudaError_t ef = cudaFreeAsync(L.base, s);
    return e != cudaSuccess ? e : ef;
}

cudaError_t jvp_march_any(int precision, int n, const InstDesc* hdescs, const InstDesc* d_dev, const JvpDesc* jds_dev,
                          int count, cudaStream_t s) {
    if (precision == 32)
        return n == 512 ? jvp_march<float, 512>(hdescs, d_dev, jds_dev, count, s)
                        : jvp_march<float, 256>(hdescs, d_dev, jds_dev, count, s);
    return n == 512 ? jvp_march<double, 512>(hdescs, d_dev, jds_dev, count, s)
                    : jvp_march<double, 256>(hdescs, d_dev, jds_dev, count, s);
}

// The tangent of a thermal run, pass by pass (steps 1-4 above).  Buffers: u = dT/dT_o, the
// tangent heat source q = dQ/dT_o of the latest pass, and the per-voxel optics tangents.
template <typename R>
class ThermalTangent {
  public:
    explicit ThermalTangent(const shg_params& p) : p_(p) {}
    ThermalTangent(const ThermalTangent&) = delete;
    ThermalTangent& operator=(const ThermalTangent&) = delete;
    ~ThermalTangent() {
        if (buf_) cudaFreeAsync(buf_, s_);
    }
    double out[2] = {0.0, 0.0};  // the last pass's SH power (tangent march) and dJ/dT_o

    // Steps 1-2 of one pass and the pass's JvpDesc (step 3's inputs), into *jd.
    shg_status prepare(const ThermalState& st, cudaStream_t s, JvpDesc* jd) {
        const size_t nt = (size_t)p_.nx * p_.nx * p_.nz, arr = sizeof(R) * nt;
        cudaError_t e;
        if (!buf_) {
            s_ = s;
            if ((e = dev_alloc((void**)&buf_, 5 * arr + 1024, s)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
            u_ = reinterpret_cast<R*>(buf_);
            q_ = u_ + nt;
            ddk_ = q_ + nt;
            dnp_ = ddk_ + nt;
            dns_ = dnp_ + nt;
            dout_ = reinterpret_cast<double*>(dns_ + nt);
            jd_dev_ = reinterpret_cast<JvpDesc*>(((uintptr_t)(dout_ + 2) + 255) & ~(uintptr_t)255);
            // T starts at T_o everywhere (faces included): u = 1; no heat source before the
            // first pass: q = 0
            if ((e = launch_fill<R>(u_, nt, (R)1, s)) != cudaSuccess) return cuda_fail(e, "tangent set-up");
        }
        // 1. this outer iteration's sweeps, tangent-linear: T_inf = 0, source q of the
        //    previous pass (none before the first)
        shg_params q = p_;
        q.t_inf = 0.0;
        shg_status rc;
        if (p_.heat_solver == SHG_HEAT_DIRECT) {
            // the direct solve is linear in (Q, faces, T_inf): its tangent is the same solve of
            // the tangent source with faces at 1 (u's initial value there) and T_inf = 0
            if (!st.heat) return fail(SHG_ERR_INVALID, "direct heat tangent without a workspace");
            if ((rc = st.heat->solve<R>(q, u_, st.pass > 0 ? q_ : nullptr, 0.0, s)) != SHG_OK) return rc;
        } else if (st.sweeps > 0 &&
                   (rc = heat_sweeps_device(q, u_, st.pass > 0 ? q_ : nullptr, st.sweeps, s)) != SHG_OK) {
            return rc;
        }
        // 2. per-voxel tangents of the optics
        if ((e = launch_optics_tangent<R>(reinterpret_cast<const R*>(st.T), u_, ddk_, dnp_, dns_, p_, s)) != cudaSuccess)
            return cuda_fail(e, "optics tangent");
        R uc_h = 0;
        const size_t ic = (size_t)(p_.nx / 2) * p_.nx + p_.nx / 2;  // IDX(NX/2, NY/2, 0)
        if ((e = cudaMemcpyAsync(&uc_h, u_ + ic, sizeof(R), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(e, "read u");
        // 3. centre-voxel terms (pump, propagators) of the tangent march, which emits this
        //    pass's q for the next outer iteration (4.)
        const double uc = (double)uc_h, h = 1e-3, Tc = st.Tc;
        std::memset(jd, 0, sizeof(*jd));
        jd->ddk = ddk_;
        jd->dnp = dnp_;
        jd->dns = dns_;
        const InstDesc dp = make_plain_desc(p_, Tc + h, Tc + h), dm = make_plain_desc(p_, Tc - h, Tc - h);
        const double pert[2][4] = {{dp.amp_re, dp.amp_im, dp.den_re, dp.den_im}, {dm.amp_re, dm.amp_im, dm.den_re, dm.den_im}};
        std::memcpy(jd->pump_pert, pert, sizeof(pert));
        jd->pump_scale = uc / (2 * h);
        jd->adot_p = (dp.a_p - dm.a_p) / (2 * h) * uc;
        jd->adot_s = (dp.a_s - dm.a_s) / (2 * h) * uc;
        jd->out = dout_;
        jd->q_dot = st.last ? nullptr : q_;
        return SHG_OK;
    }

    // After the last pass's tangent march: the SH power it recomputed and dJ/dT_o into out.
    shg_status read_out(cudaStream_t s) {
        cudaError_t e;
        if ((e = cudaMemcpyAsync(out, dout_, 2 * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(e, "tangent result");
        return SHG_OK;
    }

    // One pass of a single run: steps 1-3 with a tangent march of its own.
    shg_status pass(const ThermalState& st, cudaStream_t s) {
        JvpDesc jd;
        shg_status rc = prepare(st, s, &jd);
        if (rc != SHG_OK) return rc;
        cudaError_t e;
        if ((e = cudaMemcpyAsync(jd_dev_, &jd, sizeof(jd), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = jvp_march_any(p_.precision, p_.nx, st.desc, st.desc_dev, jd_dev_, 1, s)) != cudaSuccess)
            return cuda_fail(e, "tangent march");
        return st.last ? read_out(s) : SHG_OK;
    }

    const shg_params& params() const { return p_; }

  private:
    shg_params p_;
    cudaStream_t s_ = nullptr;
    char* buf_ = nullptr;
    R *u_ = nullptr, *q_ = nullptr, *ddk_ = nullptr, *dnp_ = nullptr, *dns_ = nullptr;
    double* dout_ = nullptr;
    JvpDesc* jd_dev_ = nullptr;
};

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
    std::memset(out, 0, sizeof(*out));
    shg_status rc;
    {
        ThermalTangent<float> tf(*p);
        ThermalTangent<double> td(*p);
        const ThermalHook hook = [&](const ThermalState& ts, cudaStream_t hs) -> shg_status {
            return p->precision == 32 ? tf.pass(ts, hs) : td.pass(ts, hs);
        };
        rc = thermal_solve_device(*p, nullptr, nullptr, nullptr, nullptr, &out->stats, s, nullptr, nullptr, &hook);
        std::memcpy(jv, p->precision == 32 ? tf.out : td.out, sizeof(jv));
    }
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

namespace shg {
namespace {

// The tangent hook of a thermal batch: steps 1-2 per instance, then ONE tangent march over
// the instances of the pass (their descriptors are contiguous in the batch's pass), then the
// results of the instances whose last pass it was.
template <typename R>
shg_status batch_tangent_pass(std::vector<std::unique_ptr<ThermalTangent<R>>>& tg, const ThermalState* st, int na, JvpDesc* jds_dev,
                              double* d_temp, double* power_tm, cudaStream_t s) {
    std::vector<JvpDesc> jds(na);
    shg_status rc;
    for (int a = 0; a < na; ++a)
        if ((rc = tg[st[a].index]->prepare(st[a], s, &jds[a])) != SHG_OK) return rc;
    cudaError_t e;
    const shg_params& p = tg[st[0].index]->params();
    if ((e = cudaMemcpyAsync(jds_dev, jds.data(), sizeof(JvpDesc) * (size_t)na, cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = jvp_march_any(p.precision, p.nx, st[0].desc, st[0].desc_dev, jds_dev, na, s)) != cudaSuccess)
        return cuda_fail(e, "tangent march");
    for (int a = 0; a < na; ++a)
        if (st[a].last) {
            ThermalTangent<R>& t = *tg[st[a].index];
            if ((rc = t.read_out(s)) != SHG_OK) return rc;
            d_temp[st[a].index] = t.out[1];
            if (power_tm) power_tm[st[a].index] = t.out[0];
        }
    return SHG_OK;
}

template <typename R>
shg_status thermal_batch_grad(const shg_params* ps, int count, void* const* pump_out, void* const* signal_out,
                              void* const* temperature_out, shg_stats* stats, double* d_temp, cudaStream_t s) {
    std::vector<std::unique_ptr<ThermalTangent<R>>> tg;
    for (int i = 0; i < count; ++i) tg.emplace_back(new ThermalTangent<R>(ps[i]));
    JvpDesc* jds_dev = nullptr;
    cudaError_t e = dev_alloc((void**)&jds_dev, sizeof(JvpDesc) * (size_t)count, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    const ThermalBatchHook hook = [&](const ThermalState* st, int na, cudaStream_t hs) {
        return batch_tangent_pass<R>(tg, st, na, jds_dev, d_temp, nullptr, hs);
    };
    shg_status rc = thermal_solve_batch(ps, count, nullptr, pump_out, signal_out, temperature_out, stats, s, nullptr,
                                        nullptr, &hook);
    cudaFreeAsync(jds_dev, s);
    return rc;
}

}  // namespace
}  // namespace shg

extern "C" shg_status shg_thermal_batch(const shg_params* params, int32_t count, void* const* pump_out_dev,
                                        void* const* signal_out_dev, void* const* temperature_out_dev,
                                        shg_stats* stats, double* d_temp_out, void* stream_) {
    clear_error();
    if (!params || count < 0) return fail(SHG_ERR_INVALID, "params is NULL or count < 0");
    if (count == 0) return SHG_OK;
    for (int i = 0; i < count; ++i) {
        shg_status st = shg_check_params(&params[i]);
        if (st != SHG_OK) return fail(st, "instance %d: %s", i, shg_last_error());
        const shg_params& p = params[i];
        if (!p.thermal) return fail(SHG_ERR_INVALID, "instance %d: thermal runs only (thermal == 1)", i);
        if (p.precision != params[0].precision || p.nx != params[0].nx || p.nz != params[0].nz || p.march != params[0].march)
            return fail(SHG_ERR_INVALID, "instance %d: all instances must share precision, grid side, nz and march", i);
        if (d_temp_out) {
            if (p.nx != 256 && p.nx != 512)
                return fail(SHG_ERR_UNSUPPORTED, "the tangent march is built for grid sides 256 and 512 (side %d)", p.nx);
            if (p.waist_y > 0 && p.waist_y != p.waist)
                return fail(SHG_ERR_UNSUPPORTED, "instance %d: the tangent march is for round beams (waist_y == 0)", i);
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    cudaStream_t s = (cudaStream_t)stream_;
    shg_status rc;
    if (d_temp_out)
        rc = params[0].precision == 32
                 ? thermal_batch_grad<float>(params, count, pump_out_dev, signal_out_dev, temperature_out_dev, stats, d_temp_out, s)
                 : thermal_batch_grad<double>(params, count, pump_out_dev, signal_out_dev, temperature_out_dev, stats, d_temp_out, s);
    else
        rc = thermal_solve_batch(params, count, nullptr, pump_out_dev, signal_out_dev, temperature_out_dev, stats, s);
    if (rc == SHG_OK) {
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "thermal batch");
    }
    if (rc == SHG_OK && d_temp_out)
        for (int i = 0; i < count; ++i)
            if (!std::isfinite(d_temp_out[i])) return fail(SHG_ERR_NONFINITE, "instance %d: dJ/dT_oven is %g", i, d_temp_out[i]);
    return rc;
}
