// adjoint.cu — instantiations and host driver of the adjoint march (ssfm_adjoint.cuh):
// shg_grad of include/shg.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "shg_host.h"
#include "ssfm_adjoint.cuh"

namespace shg {

namespace {

struct AdjVariant {
    int precision, n, cluster, threads;
    size_t smem;
    cudaError_t (*launch)(const InstDesc*, const AdjDesc*, cudaStream_t);
};

template <typename T, int N, int C, int NT>
cudaError_t launch_adjoint(const InstDesc* d, const AdjDesc* a, cudaStream_t stream) {
    using Cfg = PlainCfg<T, N, C, NT, false>;
    auto kern = ssfm_adjoint_kernel<T, N, C, NT>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&]() {
        attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem_bytes);
        if (attr_err == cudaSuccess && C > 8)
            attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    if (attr_err != cudaSuccess) return attr_err;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = Cfg::smem_bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = C > 1 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, d, a);
}

#define SHG_ADJ(T, PREC, N, C, NT) {PREC, N, C, NT, PlainCfg<T, N, C, NT, false>::smem_bytes, &launch_adjoint<T, N, C, NT>}

const AdjVariant kAdjVariants[] = {
    SHG_ADJ(float, 32, 32, 1, 128),  SHG_ADJ(float, 32, 64, 1, 256),   SHG_ADJ(float, 32, 128, 2, 256),
    SHG_ADJ(float, 32, 256, 8, 256), SHG_ADJ(double, 64, 32, 1, 128),  SHG_ADJ(double, 64, 64, 1, 256),
    SHG_ADJ(double, 64, 128, 4, 256), SHG_ADJ(double, 64, 256, 16, 256),
};

const AdjVariant* find_adj(int precision, int n) {
    for (const auto& v : kAdjVariants)
        if (v.precision == precision && v.n == n) return &v;
    return nullptr;
}

// pump parameters (Ap0/MX, wX2 MX) of setPump for waist w, focus f and temperature T
void pump_params(const shg_params& p, double w, double f, double T, double* out4) {
    shg_params q = p;
    q.waist = w;
    q.focus = f;
    InstDesc d = make_plain_desc(q, T, T);
    out4[0] = d.amp_re;
    out4[1] = d.amp_im;
    out4[2] = d.den_re;
    out4[3] = d.den_im;
}

}  // namespace

}  // namespace shg

using namespace shg;

extern "C" shg_status shg_grad(const shg_params* p, const double* poling, int32_t checkpoint_every,
                               shg_grad_result* out) {
    shg_status st = shg_check_params(p);
    if (st != SHG_OK) return st;
    if (!out) return fail(SHG_ERR_INVALID, "out is NULL");
    if (p->thermal) return fail(SHG_ERR_UNSUPPORTED, "gradients are for plain runs (thermal == 0)");
    const AdjVariant* v = find_adj(p->precision, p->nx);
    if (!v) return fail(SHG_ERR_UNSUPPORTED, "no adjoint kernel for grid side %d at precision %d", p->nx, p->precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    const int nsteps = shg_steps(p);
    const int K = checkpoint_every > 0 ? std::min(checkpoint_every, nsteps)
                                       : std::max(1, (int)std::lround(std::sqrt((double)nsteps)));
    const int M = (nsteps + K - 1) / K;
    const int C = v->cluster;
    const size_t NN = (size_t)p->nx * p->nx;
    const size_t cb = complex_bytes(*p);

    InstDesc d = make_plain_desc(*p, p->temp, p->temp);
    AdjDesc a;
    std::memset(&a, 0, sizeof(a));
    a.K = K;
    a.M = M;
    // central differences of the closed-form pump
    const double hw = 1e-5 * p->waist, hf = 1e-5 * std::max(std::fabs(p->focus), p->lz), hT = 1e-3;
    pump_params(*p, p->waist + hw, p->focus, p->temp, a.pert[0]);
    pump_params(*p, p->waist - hw, p->focus, p->temp, a.pert[1]);
    pump_params(*p, p->waist, p->focus + hf, p->temp, a.pert[2]);
    pump_params(*p, p->waist, p->focus - hf, p->temp, a.pert[3]);
    pump_params(*p, p->waist, p->focus, p->temp + hT, a.pert[4]);
    pump_params(*p, p->waist, p->focus, p->temp - hT, a.pert[5]);
    a.inv2h[0] = 1.0 / (2 * hw);
    a.inv2h[1] = 1.0 / (2 * hf);
    a.inv2h[2] = 1.0 / (2 * hT);
    std::vector<double> zs(nsteps);
    double z = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        zs[s] = z;
        z += d.dz;  // the forward's accumulation (Solver.h:303)
    }

    // device workspace
    const size_t b_ckpt = (size_t)M * 2 * NN * cb, b_seg = (size_t)K * 2 * NN * cb, b_lam = 2 * NN * cb;
    const size_t b_z = sizeof(double) * nsteps, b_part = sizeof(double) * C * kAdjAcc, b_phi = sizeof(double) * nsteps * C;
    const size_t b_pol = sizeof(double) * nsteps;
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t total = up(b_ckpt) + 3 * up(b_seg) + up(b_lam) + up(b_z) + up(b_part) + up(b_phi) + up(b_pol) +
                         up(sizeof(InstDesc)) + up(sizeof(AdjDesc));
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    char* buf = nullptr;
    shg_status rc = SHG_OK;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    do {
        if ((e = cudaMallocAsync((void**)&buf, total, s)) != cudaSuccess) { rc = cuda_fail(e, "cudaMallocAsync"); break; }
        char* q = buf;
        auto take = [&](size_t b) { char* r = q; q += up(b); return r; };
        a.ckpt = take(b_ckpt);
        a.seg_a2 = take(b_seg);
        a.seg_x = take(b_seg);
        a.seg_y = take(b_seg);
        a.lam = take(b_lam);
        double* dz_ = reinterpret_cast<double*>(take(b_z));
        a.zs = dz_;
        a.part = reinterpret_cast<double*>(take(b_part));
        a.phi = reinterpret_cast<double*>(take(b_phi));
        double* dpol = reinterpret_cast<double*>(take(b_pol));
        InstDesc* dd = reinterpret_cast<InstDesc*>(take(sizeof(InstDesc)));
        AdjDesc* da = reinterpret_cast<AdjDesc*>(take(sizeof(AdjDesc)));
        d.poling = poling ? dpol : nullptr;
        if ((e = cudaMemcpyAsync(dz_, zs.data(), b_z, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (poling && (e = cudaMemcpyAsync(dpol, poling, b_pol, cudaMemcpyHostToDevice, s)) != cudaSuccess) ||
            (e = cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(da, &a, sizeof(a), cudaMemcpyHostToDevice, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync");
            break;
        }
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        if ((e = v->launch(dd, da, s)) != cudaSuccess) { rc = cuda_fail(e, "launch ssfm_adjoint_kernel"); break; }
        cudaEventRecord(t1, s);
        std::vector<double> part((size_t)C * kAdjAcc), phi((size_t)nsteps * C);
        if ((e = cudaMemcpyAsync(part.data(), a.part, b_part, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(phi.data(), a.phi, b_phi, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            rc = cuda_fail(e, "adjoint march");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        double A[kAdjAcc] = {0};
        for (int c = 0; c < C; ++c)
            for (int i = 0; i < kAdjAcc; ++i) A[i] += part[(size_t)c * kAdjAcc + i];
        // temperature derivatives of the scalar constants (central differences in FP64)
        const double lp = p->lambda_p, ls = 0.5 * lp, T = p->temp, h = 1e-3;
        const double np = sellmeier(lp, T), ns = sellmeier(ls, T);
        const double dnp = (sellmeier(lp, T + h) - sellmeier(lp, T - h)) / (2 * h);
        const double dns = (sellmeier(ls, T + h) - sellmeier(ls, T - h)) / (2 * h);
        const double ddk = (delta_k(*p, T + h) - delta_k(*p, T - h)) / (2 * h);
        const double J = d.pw_s * A[kAccJ];
        double dT = 0.0;
        dT += A[kAccKp] * (-dnp / np);                     // κp = π dQ / (n_p λp)
        dT += A[kAccKs] * (-dns / ns);                     // κs = 0.5 π dQ / (n_s λs)
        dT += A[kAccDk] * ddk;                             // Δk(T)
        dT += A[kAccQs] * d.qs * (dns / ns);               // two-photon term ∝ n_s
        dT += d.dz * A[kAccPropP] * d.a_p * (dnp / np);    // propagator phase a = 2π²/k ∝ 1/n
        dT += d.dz * A[kAccPropS] * d.a_s * (dns / ns);
        dT += A[kAccG0T];                                  // initial pump
        dT += J * (dns / ns);                              // power normalisation ∝ n_s
        std::memset(out->reserved, 0, sizeof(out->reserved));
        out->sh_power = J;
        out->d_waist = A[kAccG0w];
        out->d_focus = A[kAccG0f];
        out->d_temp = dT;
        out->device_ms = ms;
        out->checkpoint_every = K;
        out->steps = nsteps;
        if (out->d_poling)
            for (int k = 0; k < nsteps; ++k) {
                double t = 0.0;
                for (int c = 0; c < C; ++c) t += phi[(size_t)k * C + c];
                out->d_poling[k] = t;
            }
    } while (0);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (buf) cudaFreeAsync(buf, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "adjoint");
    return rc;
}
