// adjoint.cu — instantiations and host driver of the adjoint march (ssfm_adjoint.cuh):
// shg_grad and shg_grad_batch of include/shg.h.  A batch is one launch with one cluster per
// instance, each with its own checkpoints, segment buffers and accumulators.
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
    // the full kernel (every phase), and the march-only one (forward and re-march phases)
    cudaError_t (*launch)(const InstDesc*, const AdjDesc*, int count, int phase, int round, cudaStream_t);
    cudaError_t (*launch_march)(const InstDesc*, const AdjDesc*, int count, int phase, int round, cudaStream_t);
};

template <typename T, int N, int C, int NT, bool MARCH_ONLY>
cudaError_t launch_adjoint(const InstDesc* d, const AdjDesc* a, int count, int phase, int round, cudaStream_t stream) {
    using Cfg = PlainCfg<T, N, C, NT, false>;
    auto kern = ssfm_adjoint_kernel<T, N, C, NT, MARCH_ONLY>;
    static PerDevice<int> state;  // kernel attributes, once per device
    const cudaError_t attr_err = state.get([&](int, int&) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem_bytes);
        if (e == cudaSuccess && C > 8) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        return e;
    });
    if (attr_err != cudaSuccess) return attr_err;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(C * count), 1, 1);
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
    return cudaLaunchKernelEx(&cfg, kern, d, a, phase, round);
}

#define SHG_ADJ(T, PREC, N, C, NT)                                                                         \
    {PREC, N, C, NT, PlainCfg<T, N, C, NT, false>::smem_bytes, &launch_adjoint<T, N, C, NT, false>, \
     &launch_adjoint<T, N, C, NT, true>}

const AdjVariant kAdjVariants[] = {
    SHG_ADJ(float, 32, 32, 1, 128),  SHG_ADJ(float, 32, 64, 1, 256),   SHG_ADJ(float, 32, 128, 2, 256),
    SHG_ADJ(float, 32, 256, 16, 256), SHG_ADJ(double, 64, 32, 1, 128),  SHG_ADJ(double, 64, 64, 1, 256),
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

namespace {

// Per-instance host state of a gradient batch.
struct GradJob {
    InstDesc d;
    AdjDesc a;
    int nsteps, K, M;
    size_t off_ckpt, off_seg, off_lam, off_z, off_part, off_phi, off_pol;  // in the instance's workspace
    size_t seg_bytes;  // one segment array: two buffers, or one when a single segment holds the march
    size_t bytes;
};

shg_status grad_batch(const shg_params* ps, int count, const double* const* poling, int32_t checkpoint_every,
                      shg_grad_result* out) {
    for (int i = 0; i < count; ++i) {
        shg_status st = shg_check_params(&ps[i]);
        if (st != SHG_OK) return count > 1 ? fail(st, "instance %d: %s", i, shg_last_error()) : st;
        if (ps[i].thermal) return fail(SHG_ERR_UNSUPPORTED, "gradients are for plain runs (thermal == 0)");
        if (ps[i].waist_y > 0 && ps[i].waist_y != ps[i].waist)
            return fail(SHG_ERR_UNSUPPORTED, "gradients are for round beams (waist_y == 0)");
        if (ps[i].precision != ps[0].precision || ps[i].nx != ps[0].nx)
            return fail(SHG_ERR_INVALID, "instance %d: a gradient batch shares one precision and grid side", i);
    }
    if (!out) return fail(SHG_ERR_INVALID, "out is NULL");
    const shg_params& p0 = ps[0];
    const AdjVariant* v = find_adj(p0.precision, p0.nx);
    if (!v) return fail(SHG_ERR_UNSUPPORTED, "no adjoint kernel for grid side %d at precision %d", p0.nx, p0.precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    const int C = v->cluster;
    const size_t NN = (size_t)p0.nx * p0.nx;
    const size_t cb = complex_bytes(p0);
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    // workspace of one instance with checkpoints every K steps
    auto layout = [&](GradJob& J, int K) {
        J.K = K;
        J.M = (J.nsteps + K - 1) / K;
        J.a.K = J.K;
        J.a.M = J.M;
        size_t o = 0;
        J.off_ckpt = o; o += up((size_t)J.M * 2 * NN * cb);
        // segment m uses buffer m & 1, so a single segment needs no second buffer
        J.seg_bytes = up((size_t)(J.M > 1 ? 2 : 1) * J.K * 2 * NN * cb);
        J.off_seg = o;  o += 3 * J.seg_bytes;
        J.off_lam = o;  o += up(2 * NN * cb);
        J.off_z = o;    o += up(sizeof(double) * J.nsteps);
        J.off_part = o; o += up(sizeof(double) * (J.M + 1) * C * kAdjAcc);
        J.off_phi = o;  o += up(sizeof(double) * (size_t)J.nsteps * C);
        J.off_pol = o;  o += up(sizeof(double) * J.nsteps);
        J.bytes = o;
    };
    std::vector<GradJob> jobs(count);
    for (int i = 0; i < count; ++i) {
        const shg_params& p = ps[i];
        GradJob& J = jobs[i];
        J.nsteps = shg_steps(&p);
        J.d = make_plain_desc(p, p.temp, p.temp);
        std::memset(&J.a, 0, sizeof(J.a));
        // central differences of the closed-form pump
        const double hw = 1e-5 * p.waist, hf = 1e-5 * std::max(std::fabs(p.focus), p.lz), hT = 1e-3;
        pump_params(p, p.waist + hw, p.focus, p.temp, J.a.pert[0]);
        pump_params(p, p.waist - hw, p.focus, p.temp, J.a.pert[1]);
        pump_params(p, p.waist, p.focus + hf, p.temp, J.a.pert[2]);
        pump_params(p, p.waist, p.focus - hf, p.temp, J.a.pert[3]);
        pump_params(p, p.waist, p.focus, p.temp + hT, J.a.pert[4]);
        pump_params(p, p.waist, p.focus, p.temp - hT, J.a.pert[5]);
        J.a.inv2h[0] = 1.0 / (2 * hw);
        J.a.inv2h[1] = 1.0 / (2 * hf);
        J.a.inv2h[2] = 1.0 / (2 * hT);
    }
    // checkpoint_every <= 0: a batch whose clusters cover every SM keeps every step's fields
    // (one segment, no re-march) when they fit in half the free device memory, since such a
    // batch leaves no idle SMs for the re-march to overlap on; a smaller batch, or one too
    // large for that, keeps about sqrt(steps) checkpoints and re-marches on a second stream
    int nsm = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        nsm = 0;
    }
    bool keep_all = false;
    if (checkpoint_every <= 0 && nsm > 0 && (size_t)count * C >= (size_t)nsm) {
        size_t need = 0, fr = 0, tot = 0;
        for (GradJob& J : jobs) {
            layout(J, J.nsteps);
            need += J.bytes;
        }
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) keep_all = need <= fr / 2;
        else cudaGetLastError();
    }
    size_t total = 0;
    for (GradJob& J : jobs) {
        layout(J, checkpoint_every > 0 ? std::min(checkpoint_every, J.nsteps)
                  : keep_all          ? J.nsteps
                                      : std::max(1, (int)std::lround(std::sqrt((double)J.nsteps))));
        total += J.bytes;
    }
    const size_t b_desc = up(sizeof(InstDesc) * (size_t)count), b_adesc = up(sizeof(AdjDesc) * (size_t)count);
    total += b_desc + b_adesc;
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    char* buf = nullptr;
    shg_status rc = SHG_OK;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaStream_t s2 = nullptr;
    std::vector<cudaEvent_t> evs;
    do {
        if ((e = dev_alloc((void**)&buf, total, s)) != cudaSuccess) { rc = cuda_fail(e, "cudaMallocAsync"); break; }
        std::vector<InstDesc> hd(count);
        std::vector<AdjDesc> ha(count);
        char* q = buf + b_desc + b_adesc;
        for (int i = 0; i < count && rc == SHG_OK; ++i) {
            GradJob& J = jobs[i];
            J.a.ckpt = q + J.off_ckpt;
            J.a.seg_a2 = q + J.off_seg;
            J.a.seg_x = q + J.off_seg + J.seg_bytes;
            J.a.seg_y = q + J.off_seg + 2 * J.seg_bytes;
            J.a.lam = q + J.off_lam;
            J.a.zs = reinterpret_cast<const double*>(q + J.off_z);
            J.a.part = reinterpret_cast<double*>(q + J.off_part);
            J.a.phi = reinterpret_cast<double*>(q + J.off_phi);
            J.d.poling = (poling && poling[i]) ? reinterpret_cast<const double*>(q + J.off_pol) : nullptr;
            std::vector<double> zs(J.nsteps);
            double z = 0.0;
            for (int k = 0; k < J.nsteps; ++k) {
                zs[k] = z;
                z += J.d.dz;  // the forward's accumulation (Solver.h:303)
            }
            if ((e = cudaMemcpyAsync(q + J.off_z, zs.data(), sizeof(double) * J.nsteps, cudaMemcpyHostToDevice, s)) !=
                    cudaSuccess ||
                (J.d.poling && (e = cudaMemcpyAsync(q + J.off_pol, poling[i], sizeof(double) * J.nsteps,
                                                    cudaMemcpyHostToDevice, s)) != cudaSuccess))
                rc = cuda_fail(e, "cudaMemcpyAsync");
            hd[i] = J.d;
            ha[i] = J.a;
            q += J.bytes;
        }
        if (rc != SHG_OK) break;
        InstDesc* dd = reinterpret_cast<InstDesc*>(buf);
        AdjDesc* da = reinterpret_cast<AdjDesc*>(buf + b_desc);
        if ((e = cudaMemcpyAsync(dd, hd.data(), sizeof(InstDesc) * count, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(da, ha.data(), sizeof(AdjDesc) * count, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync");
            break;
        }
        // the forward launch, then per round r the adjoint march of segment M-1-r on `s`
        // and, concurrently on `s2`, the re-march of segment M-2-r into the other buffer:
        // a re-march waits for the adjoint march that last read its buffer (round r-1), an
        // adjoint march for the re-march of its segment (round r-1)
        int mmax = 0;
        for (const GradJob& J : jobs) mmax = std::max(mmax, J.M);
        evs.resize(2 * (size_t)mmax + 1);
        for (auto& ev : evs)
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) break;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
        if (e != cudaSuccess) { rc = cuda_fail(e, "adjoint streams"); break; }
        cudaEvent_t* eB = evs.data();
        cudaEvent_t* eR = evs.data() + mmax;
        cudaEvent_t& eF = evs[2 * (size_t)mmax];
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        // A batch whose clusters cover every SM runs its forward and re-march phases on the
        // march-only kernel (two CTAs per SM where its shared memory allows); a smaller one
        // keeps the full kernel, whose one CTA per SM spreads each cluster over twice the SMs
        // (measured: single FP32 256 x 256 x 400 gradient 22.1 ms full, 22.8 ms march-only).
        // The adjoint marches always run the full kernel.
        const bool fills = nsm > 0 && (size_t)count * C >= (size_t)nsm;
        const auto launch_fwd = fills ? v->launch_march : v->launch;
        if ((e = launch_fwd(dd, da, count, kAdjForward, 0, s)) == cudaSuccess &&
            (e = cudaEventRecord(eF, s)) == cudaSuccess)
            e = cudaStreamWaitEvent(s2, eF, 0);
        for (int r = 0; r < mmax && e == cudaSuccess; ++r) {
            if (r + 1 < mmax) {
                if (r >= 1 && (e = cudaStreamWaitEvent(s2, eB[r - 1], 0)) != cudaSuccess) break;
                if ((e = launch_fwd(dd, da, count, kAdjRemarch, r, s2)) != cudaSuccess) break;
                if ((e = cudaEventRecord(eR[r], s2)) != cudaSuccess) break;
            }
            if (r >= 1 && (e = cudaStreamWaitEvent(s, eR[r - 1], 0)) != cudaSuccess) break;
            if ((e = v->launch(dd, da, count, kAdjBackward, r, s)) != cudaSuccess) break;
            if ((e = cudaEventRecord(eB[r], s)) != cudaSuccess) break;
        }
        if (e != cudaSuccess) { rc = cuda_fail(e, "launch ssfm_adjoint_kernel"); break; }
        cudaEventRecord(t1, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) { rc = cuda_fail(e, "adjoint march"); break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        for (int i = 0; i < count && rc == SHG_OK; ++i) {
            const GradJob& J = jobs[i];
            const shg_params& p = ps[i];
            std::vector<double> part((size_t)(J.M + 1) * C * kAdjAcc), phi((size_t)J.nsteps * C);
            if ((e = cudaMemcpy(part.data(), J.a.part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost)) !=
                    cudaSuccess ||
                (e = cudaMemcpy(phi.data(), J.a.phi, sizeof(double) * phi.size(), cudaMemcpyDeviceToHost)) != cudaSuccess) {
                rc = cuda_fail(e, "adjoint results");
                break;
            }
            double A[kAdjAcc] = {0};
            for (int slot = 0; slot <= J.M; ++slot)
                for (int c = 0; c < C; ++c)
                    for (int k = 0; k < kAdjAcc; ++k) A[k] += part[((size_t)slot * C + c) * kAdjAcc + k];
            // temperature derivatives of the scalar constants (closed form, FP64)
            const double lp = p.lambda_p, ls = 0.5 * lp, T = p.temp;
            const int cr = p.crystal;
            const double np = sellmeier(cr, lp, T), ns = sellmeier(cr, ls, T);
            const double dnp = sellmeier_dT(cr, lp, T), dns = sellmeier_dT(cr, ls, T);
            const double ddk = delta_k_dT(p, T);
            const InstDesc& d = J.d;
            const double Jp = d.pw_s * A[kAccJ];
            double dT = 0.0;
            dT += A[kAccKp] * (-dnp / np);                     // κp = π dQ / (n_p λp)
            dT += A[kAccKs] * (-dns / ns);                     // κs = 0.5 π dQ / (n_s λs)
            dT += A[kAccDk] * ddk;                             // Δk(T)
            dT += A[kAccQs] * d.qs * (dns / ns);               // two-photon term ∝ n_s
            dT += d.dz * A[kAccPropP] * d.a_p * (dnp / np);    // propagator phase a = 2π²/k ∝ 1/n
            dT += d.dz * A[kAccPropS] * d.a_s * (dns / ns);
            dT += A[kAccG0T];                                  // initial pump
            dT += Jp * (dns / ns);                             // power normalisation ∝ n_s
            shg_grad_result& r = out[i];
            std::memset(r.reserved, 0, sizeof(r.reserved));
            r.sh_power = Jp;
            r.d_waist = A[kAccG0w];
            r.d_focus = A[kAccG0f];
            r.d_temp = dT;
            r.device_ms = ms;
            r.checkpoint_every = J.K;
            r.steps = J.nsteps;
            if (r.d_poling)
                for (int k = 0; k < J.nsteps; ++k) {
                    double t = 0.0;
                    for (int c = 0; c < C; ++c) t += phi[(size_t)k * C + c];
                    r.d_poling[k] = t;
                }
        }
    } while (0);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (buf) cudaFreeAsync(buf, s);
    cudaStreamSynchronize(s);
    if (s2) {
        cudaStreamSynchronize(s2);
        cudaStreamDestroy(s2);
    }
    for (cudaEvent_t ev : evs)
        if (ev) cudaEventDestroy(ev);
    cudaStreamDestroy(s);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "adjoint");
    return rc;
}

}  // namespace

extern "C" shg_status shg_grad(const shg_params* p, const double* poling, int32_t checkpoint_every,
                               shg_grad_result* out) {
    clear_error();
    if (!p) return fail(SHG_ERR_INVALID, "params is NULL");
    return grad_batch(p, 1, &poling, checkpoint_every, out);
}

extern "C" shg_status shg_grad_batch(const shg_params* params, int32_t count, const double* const* poling,
                                     int32_t checkpoint_every, shg_grad_result* out) {
    clear_error();
    if (!params || count <= 0) return fail(SHG_ERR_INVALID, "params is NULL or count <= 0");
    return grad_batch(params, count, poling, checkpoint_every, out);
}
