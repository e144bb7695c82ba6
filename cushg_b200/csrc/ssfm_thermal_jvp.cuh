// ssfm_thermal_jvp.cuh — tangent-linear (forward-mode) march of the thermal optical pass:
// the derivative of the SH output power with respect to the oven temperature, carried step by
// step beside the fields.  No counterpart in the reference, which computes no gradients.
//
// The oven temperature T_o moves the converged temperature field by u = dT/dT_o at every
// voxel (computed by the caller), and the optical pass sees T only through
//   * the per-voxel n_p(T), n_s(T) and Δk(T) of the RK4 stages (Solver.h:33-55), with the
//     running Δk prefix DKint (PhaseMatching.h:27-44), and the two-photon term ∝ n_s;
//   * n(T_c) at the centre voxel (NX/2, NY/2, 0): the initial pump (Efields.h:84-119) and
//     the diffraction propagators (Efields.h:122-141);
//   * the power weights n_s(T) of the output slice.
// The tangent fields (Ṗ, Ṡ) go through the same four-step transforms as the fields (the
// transforms do not depend on T), the propagator product gains the term i θ̇ D X, and the
// RK4 applications are replaced by their Jacobian-vector products.  The planes live in
// global memory as in the multi-pass march (ssfm_multipass.cuh); every step is a row launch
// and a column launch over the four planes P, S, Ṗ, Ṡ.
#pragma once

#include "ssfm_multipass.cuh"

namespace shg {

// Tangent inputs of one instance.
struct JvpDesc {
    const void* ddk;         // u dΔk/dT per voxel (working real type, index z*n*n + y*n + x)
    const void* dnp;         // u dn_p/dT
    const void* dns;         // u dn_s/dT
    double pump_pert[2][4];  // (amp_re, amp_im, den_re, den_im) of setPump at T_c + h, T_c - h
    double pump_scale;       // u(T_c voxel) / (2 h)
    double adot_p, adot_s;   // d a / dT_o of the propagator coefficients a = 2π²/k (pump, SH)
    double* out;             // device [2]: SH power, its derivative
    void* q_dot;             // or null: the tangent of the heat source Q this pass emits
                             // (Tfield.h:260-276), slice by slice like the forward march
};

// dA/dz (dadz) and its derivative along (ṗ, ṡ) and the coefficient tangents (ċP, ċS, q̇s).
template <typename T>
__device__ __forceinline__ void dadz_jvp(cx<T> p, cx<T> s, cx<T> pd, cx<T> sd, cx<T> cP, cx<T> cS, cx<T> cPd,
                                         cx<T> cSd, T hap, T has, T qs, T qsd, cx<T>& dp, cx<T>& ds, cx<T>& dpd,
                                         cx<T>& dsd) {
    dadz<T>(p, s, cP, cS, hap, has, qs, dp, ds);
    // dP = cP s conj(p) - hap p
    const cx<T> sp = mulc<T>(s, p);
    const cx<T> t1 = mul<T>(cPd, sp);
    const cx<T> t2 = mul<T>(cP, add<T>(mulc<T>(sd, p), mulc<T>(s, pd)));
    dpd = mk<T>(t1.x + t2.x - hap * pd.x, t1.y + t2.y - hap * pd.y);
    // dS = cS p^2 - (has + qs |s|^2) s
    const cx<T> pp = mk<T>(p.x * p.x - p.y * p.y, (T)2 * p.x * p.y);
    const cx<T> u1 = mul<T>(cSd, pp);
    const cx<T> ppd = scale<T>(mul<T>(p, pd), (T)2);
    const cx<T> u2 = mul<T>(cS, ppd);
    const T a2 = s.x * s.x + s.y * s.y, a2d = (T)2 * (s.x * sd.x + s.y * sd.y);
    const T g = has + qs * a2, gd = qsd * a2 + qs * a2d;
    dsd = mk<T>(u1.x + u2.x - g * sd.x - gd * s.x, u1.y + u2.y - g * sd.y - gd * s.y);
}

// One application of the reference's RK4 scheme (rk4_point) with its tangent: cf / cfd the
// stage coefficients and their tangents, qsd the tangent of the two-photon coefficient.
template <typename T>
__device__ __forceinline__ void rk4_jvp(cx<T>& P, cx<T>& S, cx<T>& Pd, cx<T>& Sd, const cx<T>* cf, const cx<T>* cfd,
                                        T hap, T has, T qs, T qsd, T dz6) {
    using V = cx<T>;
    const V p = P, s = S, pd = Pd, sd = Sd;
    V kp, ks, kpd, ksd, ap, as, apd, asd;
    dadz_jvp<T>(p, s, pd, sd, cf[0], cf[3], cfd[0], cfd[3], hap, has, qs, qsd, kp, ks, kpd, ksd);
    ap = kp; as = ks; apd = kpd; asd = ksd;
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
        const T w = j < 2 ? (T)0.5 : (T)1;  // stage inputs A + 0.5 k1, A + 0.5 k2, A + k3
        const V up = mk<T>(p.x + w * kp.x, p.y + w * kp.y), us = mk<T>(s.x + w * ks.x, s.y + w * ks.y);
        const V upd = mk<T>(pd.x + w * kpd.x, pd.y + w * kpd.y), usd = mk<T>(sd.x + w * ksd.x, sd.y + w * ksd.y);
        const int c = j < 2 ? 1 : 2;
        dadz_jvp<T>(up, us, upd, usd, cf[c], cf[3 + c], cfd[c], cfd[3 + c], hap, has, qs, qsd, kp, ks, kpd, ksd);
        const T m = j < 2 ? (T)2 : (T)1;  // weights 1, 2, 2, 1
        ap = mk<T>(ap.x + m * kp.x, ap.y + m * kp.y);
        as = mk<T>(as.x + m * ks.x, as.y + m * ks.y);
        apd = mk<T>(apd.x + m * kpd.x, apd.y + m * kpd.y);
        asd = mk<T>(asd.x + m * ksd.x, asd.y + m * ksd.y);
    }
    P = mk<T>(p.x + ap.x * dz6, p.y + ap.y * dz6);
    S = mk<T>(s.x + as.x * dz6, s.y + as.y * dz6);
    Pd = mk<T>(pd.x + apd.x * dz6, pd.y + apd.y * dz6);
    Sd = mk<T>(sd.x + asd.x * dz6, sd.y + asd.y * dz6);
}

// Thermal stage coefficients (thermal_coef) and their tangents from the voxel's tangents
// of DKint, n_p and n_s.
template <typename T>
__device__ __forceinline__ void thermal_coef_jvp(const InstDesc& d, double dki, double dkid, int sl, double np,
                                                 double ns, double npd, double nsd, cx<T>* cf, cx<T>* cfd) {
    const double sr = (double)sl, b = sr + 1.0;
    if constexpr (sizeof(T) == 4) {
        // FP32 run: cf exactly as thermal_coef computes it (FP64 phase and reduction, FP32
        // sine, cosine and κ/n), so the tangent march's forward part repeats the forward
        // march; the tangents in FP32
        const double q = dki / b, qd = dkid / b, two_pi = 6.283185307179586476925,
                     inv_two_pi = 0.159154943091895335769;
        const float kp = (float)d.kf_p / (float)np, ks = (float)d.kf_s / (float)ns;
        const float kpd = -kp * (float)npd / (float)np, ksd = -ks * (float)nsd / (float)ns;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double inc = j == 0 ? 0.0 : (j == 1 ? 0.25 : 0.5);
            const double zj = d.dz * inc + sr * d.dz;
            const double phi = q * zj;
            const float r = (float)fma(-two_pi, rint(phi * inv_two_pi), phi);
            const float phid = (float)(qd * zj);
            float sn, cs;
            sincosf(r, &sn, &cs);
            cf[j] = mk<T>(kp * sn, kp * cs);
            cf[3 + j] = mk<T>(-ks * sn, ks * cs);
            cfd[j] = mk<T>(kpd * sn + kp * cs * phid, kpd * cs - kp * sn * phid);
            cfd[3 + j] = mk<T>(-ksd * sn - ks * cs * phid, ksd * cs - ks * sn * phid);
        }
        return;
    }
    const double kp = d.kf_p / np, ks = d.kf_s / ns;
    const double kpd = -kp * npd / np, ksd = -ks * nsd / ns;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const double inc = j == 0 ? 0.0 : (j == 1 ? 0.25 : 0.5);
        const double w = (d.dz * inc + sr * d.dz) / b;
        const double phi = dki * w, phid = dkid * w;
        double sn, cs;
        sincos(phi, &sn, &cs);
        // cP = κp (sin φ, cos φ), cS = κs (-sin φ, cos φ)
        cf[j] = mk<T>((T)(kp * sn), (T)(kp * cs));
        cf[3 + j] = mk<T>((T)(-ks * sn), (T)(ks * cs));
        cfd[j] = mk<T>((T)(kpd * sn + kp * cs * phid), (T)(kpd * cs - kp * sn * phid));
        cfd[3 + j] = mk<T>((T)(-ksd * sn - ks * cs * phid), (T)(ksd * cs - ks * sn * phid));
    }
}

// Offsets of the tangent planes and the tangent Δk prefix in a multi-pass workspace laid
// out by mp_layout plus jvp_extra_bytes.
struct JvpLayout {
    size_t off_pd, off_sd, off_dkd, stride;
};

template <typename T, int N>
__host__ __device__ inline JvpLayout jvp_layout(const MpLayout& L) {
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t plane = sizeof(cx<T>) * (size_t)N * N;
    JvpLayout J;
    J.off_pd = L.stride;
    J.off_sd = J.off_pd + up(plane);
    J.off_dkd = J.off_sd + up(plane);
    J.stride = J.off_dkd + up(sizeof(double) * (size_t)N * N);
    return J;
}

// Threads per (row, n1) job in the tangent row pass's pointwise work, as in the thermal row
// pass (two: the tangent RK4 needs more registers than a 512-thread block allows).
constexpr int kJvpPX = 2;

// Row pass of the tangent march (grid (N / RB, instances); the workspace of instance i at
// L.base + i * L.stride, L.stride covering the tangent planes of JL): as mp_row_kernel's thermal
// pass over the four planes P, S, Ṗ, Ṡ, with the JVP of the RK4 applications; the pass with
// s + 1 = out_after sums this CTA's SH power and its derivative into the partials
// (part[2 r], part[2 r + 1]).
template <typename T, int N>
__global__ void __launch_bounds__(MpCfg<T, N>::RNT * kJvpPX)
    mp_row_jvp_kernel(const InstDesc* __restrict__ descs, MpLayout L, JvpLayout JL, const JvpDesc* __restrict__ jds,
                      int s) {
    using Cfg = MpCfg<T, N>;
    constexpr int R2 = Cfg::R2, RB = Cfg::RB, SW = Cfg::SW;
    constexpr int JOBS = Cfg::RNT, PX = kJvpPX, NT = JOBS * PX;
    using V = cx<T>;
    using W = mult<T>;
    using R = T;
    const InstDesc d = descs[blockIdx.y];
    if (s >= d.nsteps) return;
    const JvpDesc jd = jds[blockIdx.y];
    const int mode = s < 0 ? 0 : (s + 1 < d.nsteps ? 1 : 2);
    char* wbase = L.base + (size_t)blockIdx.y * L.stride;
    V* g[4] = {reinterpret_cast<V*>(wbase), reinterpret_cast<V*>(wbase + L.off_s), reinterpret_cast<V*>(wbase + JL.off_pd),
               reinterpret_cast<V*>(wbase + JL.off_sd)};
    const W* gtab = reinterpret_cast<const W*>(wbase + L.off_tab);
    double* dkint = reinterpret_cast<double*>(wbase + L.off_dk);
    double* dkind = reinterpret_cast<double*>(wbase + JL.off_dkd);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* F4[4];
    F4[0] = reinterpret_cast<V*>(smem_raw);
#pragma unroll
    for (int f = 1; f < 4; ++f) F4[f] = F4[f - 1] + RB * N;
    W* tw = reinterpret_cast<W*>(F4[3] + RB * N);
    double* red = reinterpret_cast<double*>(tw + N);
    const int tid = threadIdx.x, y0 = blockIdx.x * RB;
    auto cj = [](V a) { return mk<T>(a.x, -a.y); };
    if (s + 2 < d.nsteps) {
        // step s reads slices s and s + 1 of the optics and their tangents; warm this CTA's
        // rows of slice s + 2 in L2 for the next row pass
        const size_t off = (size_t)(s + 2) * N * N + (size_t)y0 * N, rb = sizeof(R) * RB * N;
        const void* arrs[6] = {d.t_np, d.t_ns, d.t_dk, jd.dnp, jd.dns, jd.ddk};
#pragma unroll
        for (int a = 0; a < 6; ++a) l2_prefetch(reinterpret_cast<const R*>(arrs[a]) + off, rb, tid, NT);
    }
    for (int j = tid; j < N; j += NT) tw[j] = gtab[j];
    if (mode == 0) {
        // setPump at T_c and its tangent (central difference of the closed form times u_c)
        for (int e = tid; e < RB * N; e += NT) {
            const int lr = e / N, x = e % N, y = y0 + lr;
            const double2 pv = pump_value(d, x, y, d.amp_re, d.amp_im, d.den_re, d.den_im);
            const double2 pp = pump_value(d, x, y, jd.pump_pert[0][0], jd.pump_pert[0][1], jd.pump_pert[0][2], jd.pump_pert[0][3]);
            const double2 pm = pump_value(d, x, y, jd.pump_pert[1][0], jd.pump_pert[1][1], jd.pump_pert[1][2], jd.pump_pert[1][3]);
            const int o = sidx<N, R2, SW>(lr, x);
            F4[0][o] = mk<T>((T)pv.x, (T)pv.y);
            F4[1][o] = mk<T>((T)0, (T)0);
            F4[2][o] = mk<T>((T)((pp.x - pm.x) * jd.pump_scale), (T)((pp.y - pm.y) * jd.pump_scale));
            F4[3][o] = mk<T>((T)0, (T)0);
        }
    } else {
        for (int e = tid; e < RB * N; e += NT) {
            const int lr = e / N, x = e % N;
            const size_t gi = (size_t)(y0 + lr) * N + x;
#pragma unroll
            for (int f = 0; f < 4; ++f) F4[f][sidx<N, R2, SW>(lr, x)] = g[f][gi];
        }
    }
    __syncthreads();
    auto n1_pass = [&](bool inv) {
        for (int j = tid; j < RB * R2; j += NT) {
            const int k2 = j % R2, lr = j / R2;
#pragma unroll 1
            for (int f = 0; f < 4; ++f) {
                V* F = F4[f];
                V u[16];
#pragma unroll
                for (int n = 0; n < 16; ++n) {
                    u[n] = F[sidx<N, R2, SW>(lr, n + 16 * k2)];
                    if (inv) u[n] = cj(u[n]);
                }
                Dft<16, -1, T>::run(u);
#pragma unroll
                for (int n = 0; n < 16; ++n) F[sidx<N, R2, SW>(lr, n + 16 * k2)] = inv ? cj(u[n]) : u[n];
            }
        }
    };
    // the R2 stages of planes [f0, f1) of job (lr, n1)
    auto r2_pass = [&](int n1, int lr, bool inv, int f0, int f1) {
#pragma unroll 1
        for (int f = f0; f < f1; ++f) {
            V v[R2];
#pragma unroll
            for (int k = 0; k < R2; ++k) v[k] = F4[f][sidx<N, R2, SW>(lr, n1 + 16 * k)];
            r2_stage<T, R2>(v, tw, n1, inv);
#pragma unroll
            for (int k = 0; k < R2; ++k) F4[f][sidx<N, R2, SW>(lr, n1 + 16 * k)] = v[k];
        }
    };
    if (mode != 0) {
        n1_pass(true);
        __syncthreads();
    }
    const R* tnp = reinterpret_cast<const R*>(d.t_np);
    const R* tns = reinterpret_cast<const R*>(d.t_ns);
    const R* tdk = reinterpret_cast<const R*>(d.t_dk);
    const R* dnp = reinterpret_cast<const R*>(jd.dnp);
    const R* dns = reinterpret_cast<const R*>(jd.dns);
    const R* ddk = reinterpret_cast<const R*>(jd.ddk);
    const T hap = (T)d.hap, has = (T)d.has, dz6 = (T)(d.dz / 6.0);
    const size_t nn = (size_t)N * N;
    double acc_j = 0.0, acc_jd = 0.0;
    {
        // one (row, n1) job per JOBS threads: its R2 stages on the first, its points shared
        const int job = tid % JOBS, part = tid / JOBS;
        const int n1 = job & 15, lr = job >> 4;
        // the four planes' R2 stages split over the job's PX threads
        const int f0 = part * 4 / PX, f1 = (part + 1) * 4 / PX;
        if (mode != 0) r2_pass(n1, lr, true, f0, f1);
        __syncthreads();
        const int h0 = mode == 0 ? 1 : 0, h1 = mode == 2 ? 1 : 2;
        // the per-voxel optics and their tangents of both half steps and the running prefixes
        // of point k, read before any arithmetic so that the loads are in flight together
        // (the march never writes the optics); the next point's are read before this one's
        // arithmetic starts
        struct Pre {
            R np[2], ns[2], dnp[2], dns[2], dk, ddk;
            double dki, dkid;
        };
        auto fetch = [&](int k) {
            Pre f;
            const size_t gi = (size_t)(y0 + lr) * N + n1 + 16 * k;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                f.np[h] = f.ns[h] = f.dnp[h] = f.dns[h] = 0;
                if (h < h0 || h >= h1) continue;
                const size_t gz = (size_t)(s + h) * nn + gi;
                f.np[h] = __ldg(tnp + gz);
                f.ns[h] = __ldg(tns + gz);
                f.dnp[h] = __ldg(dnp + gz);
                f.dns[h] = __ldg(dns + gz);
            }
            f.dk = h1 == 2 ? __ldg(tdk + (size_t)(s + 1) * nn + gi) : (R)0;
            f.ddk = h1 == 2 ? __ldg(ddk + (size_t)(s + 1) * nn + gi) : (R)0;
            f.dki = mode == 0 ? 0.0 : dkint[gi];
            f.dkid = mode == 0 ? 0.0 : dkind[gi];
            return f;
        };
        Pre nxt;
        if (part < R2) nxt = fetch(part);
#pragma unroll 1
        for (int k = part; k < R2; k += PX) {
            const int x = n1 + 16 * k;
            const int o = sidx<N, R2, SW>(lr, x);
            const size_t gi = (size_t)(y0 + lr) * N + x;
            const Pre cur = nxt;
            if (k + PX < R2) nxt = fetch(k + PX);
            V p = F4[0][o], q = F4[1][o], pd = F4[2][o], qd = F4[3][o];
            const R pdk = cur.dk, pddk = cur.ddk;
            double dki = cur.dki, dkid = cur.dkid;
#pragma unroll 1
            for (int h = h0; h < h1; ++h) {
                const int sl = s + h;
                const size_t gz = (size_t)sl * nn + gi;
                if (h == 1) {
                    dki += (double)pdk;
                    dkid += (double)pddk;
                    dkint[gi] = dki;
                    dkind[gi] = dkid;
                }
                // this half step's values (selects, so that the rolled loop indexes no array)
                const double np = (double)(h ? cur.np[1] : cur.np[0]), ns = (double)(h ? cur.ns[1] : cur.ns[0]);
                const double npd = (double)(h ? cur.dnp[1] : cur.dnp[0]), nsd = (double)(h ? cur.dns[1] : cur.dns[0]);
                V cf[6], cfd[6];
                thermal_coef_jvp<T>(d, dki, dkid, sl, np, ns, npd, nsd, cf, cfd);
                rk4_jvp<T>(p, q, pd, qd, cf, cfd, hap, has, (T)(0.5 * (d.bf_s * ns)), (T)(0.5 * (d.bf_s * nsd)), dz6);
                if (h == 0 && jd.q_dot) {
                    // tangent of kernelSetQ for slice s after its step:
                    // Q = q_p n_p |P|^2 + q_s n_s |S|^2 + βs (q_h n_s |S|^2)^2
                    const double ap2 = (double)p.x * p.x + (double)p.y * p.y;
                    const double as2 = (double)q.x * q.x + (double)q.y * q.y;
                    const double ap2d = 2.0 * ((double)p.x * pd.x + (double)p.y * pd.y);
                    const double as2d = 2.0 * ((double)q.x * qd.x + (double)q.y * qd.y);
                    const double is = d.q_h * ns * as2, isd = d.q_h * (nsd * as2 + ns * as2d);
                    reinterpret_cast<R*>(jd.q_dot)[gz] =
                        (R)(d.q_p * (npd * ap2 + np * ap2d) + d.q_s * (nsd * as2 + ns * as2d) + 2.0 * d.beta_s * is * isd);
                }
                if (h == 0 && s + 1 == d.out_after) {
                    // J = pw sum n_s |S|^2 over the output slice, and its tangent
                    const size_t go = (size_t)(s + 1) * nn + gi;
                    const double ws = (double)tns[go], wsd = (double)dns[go];
                    const double a2 = (double)q.x * q.x + (double)q.y * q.y;
                    acc_j += ws * a2;
                    acc_jd += wsd * a2 + ws * 2.0 * ((double)q.x * qd.x + (double)q.y * qd.y);
                }
            }
            if (mode != 2) {
                F4[0][o] = p;
                F4[1][o] = q;
                F4[2][o] = pd;
                F4[3][o] = qd;
            }
        }
        __syncthreads();
        if (mode != 2) r2_pass(n1, lr, false, f0, f1);
    }
    __syncthreads();
    if (s + 1 == d.out_after) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc_j += __shfl_down_sync(0xffffffffu, acc_j, o);
            acc_jd += __shfl_down_sync(0xffffffffu, acc_jd, o);
        }
        if ((tid & 31) == 0) {
            red[2 * (tid >> 5)] = acc_j;
            red[2 * (tid >> 5) + 1] = acc_jd;
        }
        __syncthreads();
        if (tid == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < NT / 32; ++w) {
                a += red[2 * w];
                b += red[2 * w + 1];
            }
            double* part = reinterpret_cast<double*>(wbase + L.off_part);
            part[2 * blockIdx.x] = a;
            part[2 * blockIdx.x + 1] = b;
        }
    }
    if (mode != 2) {
        n1_pass(false);
        __syncthreads();
        for (int e = tid; e < RB * N; e += NT) {
            const int lr = e / N, x = e % N;
            const size_t gi = (size_t)(y0 + lr) * N + x;
#pragma unroll
            for (int f = 0; f < 4; ++f) g[f][gi] = F4[f][sidx<N, R2, SW>(lr, x)];
        }
    }
}

// Column pass of the tangent march: the diffraction of one field (blockIdx.y) and of its
// tangent over CW columns.  Ẏ = D Ẋ + i θ̇ D X with θ̇ = -dz ȧ (dfx² sx² + dfy² sy²), ȧ
// the derivative of the propagator coefficient of that field.  Grid (N / CW, 2, instances).
template <typename T, int N>
__global__ void __launch_bounds__(MpCfg<T, N>::CNT)
    mp_col_jvp_kernel(const InstDesc* __restrict__ descs, MpLayout L, JvpLayout JL, const JvpDesc* __restrict__ jds,
                      int s) {
    using Cfg = MpCfg<T, N>;
    constexpr int R2 = Cfg::R2, CW = Cfg::CW, NT = Cfg::CNT;
    using V = cx<T>;
    using W = mult<T>;
    const InstDesc d = descs[blockIdx.z];
    if (s >= d.nsteps) return;
    const double adot = blockIdx.y ? jds[blockIdx.z].adot_s : jds[blockIdx.z].adot_p;
    const int f = blockIdx.y;
    char* wbase = L.base + (size_t)blockIdx.z * L.stride;
    V* F = reinterpret_cast<V*>(wbase + (f ? L.off_s : 0));
    V* Fd = reinterpret_cast<V*>(wbase + (f ? JL.off_sd : JL.off_pd));
    const W* gtab = reinterpret_cast<const W*>(wbase + L.off_tab);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);  // (y, c) at y * CW + c
    V* tiled = tile + N * CW;
    W* tw = reinterpret_cast<W*>(tiled + N * CW);
    W* py = tw + N;
    W* px = py + N;
    const int tid = threadIdx.x, x0 = blockIdx.x * CW;
    auto cj = [](V a) { return mk<T>(a.x, -a.y); };
    for (int j = tid; j < N; j += NT) {
        tw[j] = gtab[j];
        py[j] = gtab[(f ? 4 : 3) * N + j];
    }
    if (tid < CW) px[tid] = gtab[(f ? 2 : 1) * N + x0 + tid];
    for (int e = tid; e < N * CW; e += NT) {
        const int y = e / CW, c = e % CW;
        tile[e] = F[(size_t)y * N + x0 + c];
        tiled[e] = Fd[(size_t)y * N + x0 + c];
    }
    __syncthreads();
    auto col_stage = [&](V* tl, bool inv) {
        const int c = tid % CW, n1 = tid / CW;
        V v[R2];
#pragma unroll
        for (int k = 0; k < R2; ++k) v[k] = tl[(n1 + 16 * k) * CW + c];
        r2_stage<T, R2>(v, tw, n1, inv);
#pragma unroll
        for (int k = 0; k < R2; ++k) tl[(n1 + 16 * k) * CW + c] = v[k];
    };
    col_stage(tile, false);
    col_stage(tiled, false);
    __syncthreads();
    for (int j = tid; j < R2 * CW; j += NT) {
        const int c = j % CW, k2 = j / CW;
        const int x = x0 + c;
        const int fx = (x >> 4) + R2 * (x & 15);
        const double sx = (double)(fx < N / 2 ? fx : fx - N);
        V u[16], ud[16];
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            u[n] = tile[(n + 16 * k2) * CW + c];
            ud[n] = tiled[(n + 16 * k2) * CW + c];
        }
        Dft<16, -1, T>::run(u);
        Dft<16, -1, T>::run(ud);
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1) {
            const int fy = k2 + R2 * k1;
            const double sy = (double)(fy < N / 2 ? fy : fy - N);
            const T thd = (T)(-d.dz * adot * (d.dfx * d.dfx * (sx * sx) + d.dfy * d.dfy * (sy * sy)));
            const V y = mulw(mulw(u[k1], py[fy]), px[c]);
            const V yd = mulw(mulw(ud[k1], py[fy]), px[c]);
            u[k1] = y;
            ud[k1] = mk<T>(yd.x - thd * y.y, yd.y + thd * y.x);
        }
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            u[n] = cj(u[n]);
            ud[n] = cj(ud[n]);
        }
        Dft<16, -1, T>::run(u);
        Dft<16, -1, T>::run(ud);
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            tile[(n + 16 * k2) * CW + c] = cj(u[n]);
            tiled[(n + 16 * k2) * CW + c] = cj(ud[n]);
        }
    }
    __syncthreads();
    col_stage(tile, true);
    col_stage(tiled, true);
    __syncthreads();
    for (int e = tid; e < N * CW; e += NT) {
        const int y = e / CW, c = e % CW;
        F[(size_t)y * N + x0 + c] = tile[e];
        Fd[(size_t)y * N + x0 + c] = tiled[e];
    }
}

// SH power and its derivative from the row-pass partials (fixed order), times pw_s; one
// block per instance.
template <typename T, int N>
__global__ void mp_jvp_sum_kernel(const InstDesc* __restrict__ descs, MpLayout L, const JvpDesc* __restrict__ jds) {
    if (threadIdx.x != 0) return;
    const int i = blockIdx.x;
    const double* part = reinterpret_cast<const double*>(L.base + (size_t)i * L.stride + L.off_part);
    double a = 0.0, b = 0.0;
    for (int r = 0; r < MpCfg<T, N>::RPART; ++r) {
        a += part[2 * r];
        b += part[2 * r + 1];
    }
    jds[i].out[0] = a * descs[i].pw_s;
    jds[i].out[1] = b * descs[i].pw_s;
}

}  // namespace shg
