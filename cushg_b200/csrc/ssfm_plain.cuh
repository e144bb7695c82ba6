// ssfm_plain.cuh — the fused, persistent SSFM march of a plain (non-thermal) run.
//
// One thread-block cluster of C CTAs owns one instance for its whole z-march.  The
// pump and SH planes never leave on-chip memory between steps: CTA c holds the global
// rows y ≡ c (mod C) of both fields in shared memory, and every SSFM step
//
//     RK4(z) -> FFT2 -> × propagator -> IFFT2 -> RK4(z)        (Solver.h:267-273)
//
// runs as seven shared-memory passes with no HBM traffic and no kernel launch:
//
//   RA  rows, DFT over n2 (R2 points) + twiddle, fused with the RK4 half-steps
//   RB  rows, DFT over n1 (16 points)
//   CA  columns, DFT over n2 + twiddle           (rows of this CTA only)
//   CB  columns, DFT over n1, propagator, IDFT   (reads / writes the cluster's DSMEM)
//   CA' columns, conj twiddle + IDFT over n2
//   RB' rows, IDFT over n1
//   RA' rows, conj twiddle + IDFT, RK4(z_s), RK4(z_{s+1}), then RA of the next step
//
// The transverse transform is a four-step FFT with N = 16 * R2: x = n1 + 16 n2 and
// frequency k = k2 + R2 k1 stored at position k1 + 16 k2 (digit-reversed); the
// propagator is applied in that order and the inverse undoes it, so no reordering
// pass exists.  Rows are XOR-swizzled so every pass is free of bank conflicts.
//
// Reference counterparts: Solver::solverRK4 / dAdz / linealCombination / kernelRK4
// (src/headers/Solver.h:33-113,189-264), Solver::diffraction with cuFFT,
// kernelComplexProduct and cuFFTscale (Solver.h:17-30,153-186, Efields.h:15-29),
// the propagators and their fftshift (Efields.h:32-81,122-141), setPump
// (Efields.h:84-119) and the z-loop of Solver::CWES (Solver.h:276-308).
#pragma once

#include <cooperative_groups.h>


#include "dft.cuh"
#include "shg_internal.h"

namespace shg {

namespace cg = cooperative_groups;

template <typename T, int N, int C, int NT, bool THERM = false>
struct PlainCfg {
    static constexpr int R1 = 16;
    static constexpr int R2 = N / 16;
    static constexpr int RL = N / C;           // rows per CTA
    static constexpr int SW = sizeof(T) == 4 ? 16 : 8;  // complex slots per 128 B
    static constexpr int JA = RL * 16;         // RA jobs: (row, n1)
    static constexpr int JB = RL * R2;         // RB jobs: (row, k2)
    static constexpr int JCA = N * (16 / C);   // CA jobs: (column, n1 of this CTA)
    static constexpr int JCB = N * R2 / C;     // CB jobs: (column, k2)
    static constexpr int PLANE = RL * N;       // complex elements per field per CTA
    static_assert(N % 16 == 0 && 16 % C == 0 && RL * C == N, "bad grid / cluster split");
    // dynamic shared memory: P, S planes, twiddles + 4 propagator vectors (multiplier
    // tables), 2x6 coefficients, reduction scratch
    // (thermal: plus the running Δk prefix of this CTA's points, FP64)
    // (plain FP32: plus the packed RK4 stage constants, 2 steps x 3 phases of Rk4Pack)
    static constexpr size_t smem_bytes = sizeof(cx<T>) * (2 * (size_t)PLANE + 12) + sizeof(mult<T>) * 5 * (size_t)N +
                                         sizeof(double) * (2 * (NT / 32) + 4) +
                                         (THERM ? sizeof(double) * (size_t)PLANE
                                                : (sizeof(T) == 4 ? 6 * sizeof(float2) * 6 : 0));
};

// physical offset of logical position p of local row lr
template <int N, int R2, int SW>
__device__ __forceinline__ int sidx(int lr, int p) {
    return lr * N + (p ^ (((p >> 4) + lr * R2) & (SW - 1)));
}

// dA/dz of the coupled equations at one point (Solver.h:57-80):
//   dP = cP * S * conj(P) - 0.5 αp P,   cP = i κp e^{-iφ}
//   dS = cS * P^2 - 0.5 (αs + βs 0.5 c ε0 n_s |S|^2) S,   cS = i κs e^{+iφ}
template <typename T>
__device__ __forceinline__ void dadz(cx<T> p, cx<T> s, cx<T> cP, cx<T> cS, T hap, T has, T qs, cx<T>& dp,
                                     cx<T>& ds) {
    cx<T> sp = mulc<T>(s, p);
    cx<T> tp = mul<T>(cP, sp);
    dp = mk<T>(tp.x - hap * p.x, tp.y - hap * p.y);
    cx<T> pp = mk<T>(p.x * p.x - p.y * p.y, (T)2 * p.x * p.y);
    cx<T> ts = mul<T>(cS, pp);
    T g = has + qs * (s.x * s.x + s.y * s.y);
    ds = mk<T>(ts.x - g * s.x, ts.y - g * s.y);
}

// One application of the reference's RK4 scheme (Solver.h:231-259): stage inputs
// A + 0.5 k1, A + 0.5 k2, A + k3 (no dz factor), stage phases at z, z + dz/4 (twice)
// and z + dz/2; A += (k1 + 2 k2 + 2 k3 + k4) dz / 6.  cf[0..2] = cP of the three
// phases, cf[3..5] = cS.
template <typename T>
__device__ __forceinline__ void rk4_point(cx<T>& P, cx<T>& S, const cx<T>* cf, T hap, T has, T qs, T dz6) {
    cx<T> p = P, s = S, kp, ks, ap, as;
    dadz<T>(p, s, cf[0], cf[3], hap, has, qs, kp, ks);
    ap = kp; as = ks;
    dadz<T>(mk<T>(p.x + (T)0.5 * kp.x, p.y + (T)0.5 * kp.y), mk<T>(s.x + (T)0.5 * ks.x, s.y + (T)0.5 * ks.y), cf[1],
            cf[4], hap, has, qs, kp, ks);
    ap = mk<T>(ap.x + (T)2 * kp.x, ap.y + (T)2 * kp.y);
    as = mk<T>(as.x + (T)2 * ks.x, as.y + (T)2 * ks.y);
    dadz<T>(mk<T>(p.x + (T)0.5 * kp.x, p.y + (T)0.5 * kp.y), mk<T>(s.x + (T)0.5 * ks.x, s.y + (T)0.5 * ks.y), cf[1],
            cf[4], hap, has, qs, kp, ks);
    ap = mk<T>(ap.x + (T)2 * kp.x, ap.y + (T)2 * kp.y);
    as = mk<T>(as.x + (T)2 * ks.x, as.y + (T)2 * ks.y);
    dadz<T>(add<T>(p, kp), add<T>(s, ks), cf[2], cf[5], hap, has, qs, kp, ks);
    ap = add<T>(ap, kp);
    as = add<T>(as, ks);
    P = mk<T>(p.x + ap.x * dz6, p.y + ap.y * dz6);
    S = mk<T>(s.x + as.x * dz6, s.y + as.y * dz6);
}

// Two points of the FP32 RK4 at once in packed two-lane arithmetic (sm_100 f32x2): the real
// parts of the two points share one register pair, the imaginary parts another, and each
// packed instruction does the work of two scalar ones.  The per-phase stage constants are
// held with each value in both lanes (Rk4Pack, written by stage_pack).  The operations and
// their order are those of dadz / rk4_point; only where the compiler would choose to fuse
// a multiply into an add is fixed here.
struct Cx2 {
    float2 r, i;
};
struct Rk4Pack {
    float2 cpr, cpi, ncpi, csr, csi, ncsi;  // cP, cS and the negated imaginary parts
};

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

__device__ __forceinline__ void dadz_pair(const Cx2& p, const Cx2& s, const Rk4Pack& k, float2 nhap, float2 nhas,
                                          float2 nqs, Cx2& dp, Cx2& ds) {
    const float2 npi = __fmul2_rn(bc2(-1.f), p.i);
    // sp = s conj(p)
    const float2 spr = __ffma2_rn(s.i, p.i, __fmul2_rn(s.r, p.r));
    const float2 spi = __ffma2_rn(s.r, npi, __fmul2_rn(s.i, p.r));
    // dP = cP sp - 0.5 αp P
    const float2 tpr = __ffma2_rn(k.ncpi, spi, __fmul2_rn(k.cpr, spr));
    const float2 tpi = __ffma2_rn(k.cpi, spr, __fmul2_rn(k.cpr, spi));
    dp.r = __ffma2_rn(nhap, p.r, tpr);
    dp.i = __ffma2_rn(nhap, p.i, tpi);
    // pp = P^2
    const float2 ppr = __ffma2_rn(p.i, npi, __fmul2_rn(p.r, p.r));
    const float2 ppi = __fmul2_rn(__fadd2_rn(p.r, p.r), p.i);
    // dS = cS pp - (0.5 αs + qs |S|^2) S
    const float2 tsr = __ffma2_rn(k.ncsi, ppi, __fmul2_rn(k.csr, ppr));
    const float2 tsi = __ffma2_rn(k.csi, ppr, __fmul2_rn(k.csr, ppi));
    const float2 ng = __ffma2_rn(nqs, __ffma2_rn(s.i, s.i, __fmul2_rn(s.r, s.r)), nhas);
    ds.r = __ffma2_rn(ng, s.r, tsr);
    ds.i = __ffma2_rn(ng, s.i, tsi);
}

// rk4_point for two points; k[0..2]: the stage phases z, z + dz/4, z + dz/2
__device__ __forceinline__ void rk4_pair(Cx2& P, Cx2& S, const Rk4Pack* k, float2 nhap, float2 nhas, float2 nqs,
                                         float2 dz6) {
    const float2 half = bc2(0.5f), two = bc2(2.f);
    const Cx2 p = P, s = S;
    Cx2 kp, ks, ap, as, xp, xs;
    dadz_pair(p, s, k[0], nhap, nhas, nqs, kp, ks);
    ap = kp;
    as = ks;
#pragma unroll
    for (int st = 0; st < 2; ++st) {
        xp.r = __ffma2_rn(half, kp.r, p.r);
        xp.i = __ffma2_rn(half, kp.i, p.i);
        xs.r = __ffma2_rn(half, ks.r, s.r);
        xs.i = __ffma2_rn(half, ks.i, s.i);
        dadz_pair(xp, xs, k[1], nhap, nhas, nqs, kp, ks);
        ap.r = __ffma2_rn(two, kp.r, ap.r);
        ap.i = __ffma2_rn(two, kp.i, ap.i);
        as.r = __ffma2_rn(two, ks.r, as.r);
        as.i = __ffma2_rn(two, ks.i, as.i);
    }
    xp.r = __fadd2_rn(p.r, kp.r);
    xp.i = __fadd2_rn(p.i, kp.i);
    xs.r = __fadd2_rn(s.r, ks.r);
    xs.i = __fadd2_rn(s.i, ks.i);
    dadz_pair(xp, xs, k[2], nhap, nhas, nqs, kp, ks);
    ap.r = __fadd2_rn(ap.r, kp.r);
    ap.i = __fadd2_rn(ap.i, kp.i);
    as.r = __fadd2_rn(as.r, ks.r);
    as.i = __fadd2_rn(as.i, ks.i);
    P.r = __ffma2_rn(ap.r, dz6, p.r);
    P.i = __ffma2_rn(ap.i, dz6, p.i);
    S.r = __ffma2_rn(as.r, dz6, s.r);
    S.i = __ffma2_rn(as.i, dz6, s.i);
}

// the packed constants of phase j from the scalar ones (cf[j] = cP, cf[3 + j] = cS)
__device__ __forceinline__ void stage_pack(const float2* cf, int j, Rk4Pack* kp) {
    const float2 cp = cf[j], cs = cf[3 + j];
    kp[j] = Rk4Pack{bc2(cp.x), bc2(cp.y), bc2(-cp.y), bc2(cs.x), bc2(cs.y), bc2(-cs.y)};
}

// stage coefficients of the plain dAdz of step s at position z: phases (z + dz*{0, 1/4,
// 1/2}) Δk (Solver.h:68-74 with increment 0.5*{0, 0.5, 1}) plus the step's poling phase,
// computed in FP64
template <typename T>
__device__ __forceinline__ void stage_coef(const InstDesc& d, int s, double z, int j, cx<T>* cf) {
    const double inc = j == 0 ? 0.0 : (j == 1 ? 0.25 : 0.5);
    const double phi = (z + d.dz * inc) * d.dk + (d.poling ? d.poling[s] : 0.0);
    double sn, cs;
    sincos(phi, &sn, &cs);
    // i κ e^{-iφ} = κ (sin φ, cos φ);  i κ e^{+iφ} = κ (-sin φ, cos φ)
    cf[j] = mk<T>((T)(d.kap_p * sn), (T)(d.kap_p * cs));
    cf[3 + j] = mk<T>((T)(-d.kap_s * sn), (T)(d.kap_s * cs));
}

// Multiplier tables of one instance: twiddles tw[k*16 + n1] = W_N^{n1 k}; the x factors of
// the pump / SH propagators by physical column position (frequency perm(j) = (j>>4) +
// R2*(j&15)); the y factors by frequency with the 1/(NX*NY) of the inverse FFT folded in.
// Propagator phase θ = -dz (a (dfx^2 sx^2 + dfy^2 sy^2) + b sx) (Efields.h:122-141) with the
// fftshift of Efields.h:32-81 expressed through signed frequency indices.
template <typename T, int N>
__device__ __forceinline__ void init_tables(const InstDesc& d, mult<T>* tw, mult<T>* pxp, mult<T>* pxs, mult<T>* pyp,
                                            mult<T>* pys, int tid, int nt) {
    constexpr int R2 = N / 16;
    for (int j = tid; j < N; j += nt) {
        double sn, cs;
        sincospi(-2.0 * (double)((j & 15) * (j >> 4)) / (double)N, &sn, &cs);
        tw[j] = make_mult<T>(cs, sn);
        const int fx = (j >> 4) + R2 * (j & 15);
        const double sx = (double)(fx < N / 2 ? fx : fx - N);
        const double thxp = -d.dz * (d.a_p * (d.dfx * d.dfx * (sx * sx)) + d.b_p * sx);
        const double thxs = -d.dz * (d.a_s * (d.dfx * d.dfx * (sx * sx)) + d.b_s * sx);
        sincos(thxp, &sn, &cs);
        pxp[j] = make_mult<T>(cs, sn);
        sincos(thxs, &sn, &cs);
        pxs[j] = make_mult<T>(cs, sn);
        const double sy = (double)(j < N / 2 ? j : j - N);
        const double inv = 1.0 / ((double)N * (double)N);
        const double thyp = -d.dz * (d.a_p * (d.dfy * d.dfy * (sy * sy)));
        const double thys = -d.dz * (d.a_s * (d.dfy * d.dfy * (sy * sy)));
        sincos(thyp, &sn, &cs);
        pyp[j] = make_mult<T>(cs * inv, sn * inv);
        sincos(thys, &sn, &cs);
        pys[j] = make_mult<T>(cs * inv, sn * inv);
    }
}

// Focused Gaussian pump at grid point (x, y), setPump (Efields.h:84-119):
// (Ap0 / MX) exp(-(((x - uX) dx)^2 + ((y - uY) dy)^2) / (wX2 MX)), in FP64; with d.elliptic
// the separable variant amp * exp(-ax^2 / (wX2 MX) - ay^2 / (wY2 MY)) (Efields.h:113-115).
__device__ __forceinline__ double2 pump_value(const InstDesc& d, int x, int y, double amp_re, double amp_im,
                                              double den_re, double den_im) {
    const double ax = ((double)x - d.ux) * d.dx, ay = ((double)y - d.uy) * d.dy;
    if (d.elliptic) {
        const double dx2 = den_re * den_re + den_im * den_im;
        const double dy2 = d.deny_re * d.deny_re + d.deny_im * d.deny_im;
        const double are = -(ax * ax) * den_re / dx2 - (ay * ay) * d.deny_re / dy2;
        const double aim = (ax * ax) * den_im / dx2 + (ay * ay) * d.deny_im / dy2;
        const double ex = exp(are);
        double sn, cs;
        sincos(aim, &sn, &cs);
        const double er = ex * cs, ei = ex * sn;
        return make_double2(amp_re * er - amp_im * ei, amp_re * ei + amp_im * er);
    }
    const double num = -(ax * ax) - (ay * ay);
    const double dd = den_re * den_re + den_im * den_im;
    const double are = (num * den_re) / dd, aim = (-num * den_im) / dd;
    const double ex = exp(are);
    double sn, cs;
    sincos(aim, &sn, &cs);
    const double er = ex * cs, ei = ex * sn;
    return make_double2(amp_re * er - amp_im * ei, amp_re * ei + amp_im * er);
}

// Caller buffers of an instance (signal_in, outputs, slices) hold complex values of the
// working type, or FP32 complex when an FP64 march runs an FP32 instance (d.out32): the
// march reads and rounds at the buffer, nothing else changes.
template <typename T>
__device__ __forceinline__ void put_field(const InstDesc& d, void* base, size_t i, cx<T> v) {
    if constexpr (sizeof(T) == 8) {
        if (d.out32) {
            reinterpret_cast<float2*>(base)[i] = make_float2((float)v.x, (float)v.y);
            return;
        }
    }
    reinterpret_cast<cx<T>*>(base)[i] = v;
}
template <typename T>
__device__ __forceinline__ cx<T> get_field(const InstDesc& d, const void* base, size_t i) {
    if constexpr (sizeof(T) == 8) {
        if (d.out32) {
            const float2 v = reinterpret_cast<const float2*>(base)[i];
            return mk<T>((T)v.x, (T)v.y);
        }
    }
    return reinterpret_cast<const cx<T>*>(base)[i];
}

// Thermal stage coefficients at one voxel (Solver.h:33-55): κ = kf / n(λ, T(x,y,s)) and the
// phase DKint (dz inc + s dz) / (s + 1), DKint the running sum of Δk over slices 0..s
// (PhaseMatching.h:27-44), in FP64.
template <typename T>
__device__ __forceinline__ void thermal_coef(const InstDesc& d, double dki, int sl, double np, double ns, cx<T>* cf) {
    const double sr = (double)sl, b = sr + 1.0;
    if constexpr (sizeof(T) == 4) {
        // FP32 run: the phases (up to hundreds of radians) and their reduction to [-π, π] in
        // FP64, then sine, cosine and κ/n in FP32, accurate to the float rounding the
        // coefficients get anyway; one FP64 division instead of five and no FP64 sincos
        const double q = dki / b, two_pi = 6.283185307179586476925, inv_two_pi = 0.159154943091895335769;
        const float kp = (float)d.kf_p / (float)np, ks = (float)d.kf_s / (float)ns;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double inc = j == 0 ? 0.0 : (j == 1 ? 0.25 : 0.5);
            const double phi = q * (d.dz * inc + sr * d.dz);
            const float r = (float)fma(-two_pi, rint(phi * inv_two_pi), phi);
            float sn, cs;
            sincosf(r, &sn, &cs);
            cf[j] = mk<T>(kp * sn, kp * cs);
            cf[3 + j] = mk<T>(-ks * sn, ks * cs);
        }
    } else {
        const double kp = d.kf_p / np, ks = d.kf_s / ns;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double inc = j == 0 ? 0.0 : (j == 1 ? 0.25 : 0.5);
            const double phi = dki * (d.dz * inc + sr * d.dz) / b;
            double sn, cs;
            sincos(phi, &sn, &cs);
            cf[j] = mk<T>((T)(kp * sn), (T)(kp * cs));
            cf[3 + j] = mk<T>((T)(-ks * sn), (T)(ks * cs));
        }
    }
}

// The per-voxel values a thermal boundary_point reads from global memory, fetched apart from
// its arithmetic so that a caller can issue the next point's loads before this point's work:
// n_p and n_s of the slices of both half steps, Δk of slice s + 1 (when the second half step
// runs), and the point's running Δk prefix through slice s.
template <typename R>
struct ThermPre {
    R np[2], ns[2], dk;
    double dki;
};

template <typename T, bool THERM>
__device__ __forceinline__ ThermPre<T> thermal_pre(const InstDesc& d, int mode, int s, size_t g, size_t nn,
                                                   const double* dki) {
    ThermPre<T> t;
    t.np[0] = t.np[1] = t.ns[0] = t.ns[1] = t.dk = (T)0;
    t.dki = 0.0;
    if constexpr (THERM) {
        const T* tnp = reinterpret_cast<const T*>(d.t_np);
        const T* tns = reinterpret_cast<const T*>(d.t_ns);
        const T* tdk = reinterpret_cast<const T*>(d.t_dk);
        const int h0 = mode == 0 ? 1 : 0, h1 = mode == 2 ? 1 : 2;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h < h0 || h >= h1) continue;
            const size_t gz = (size_t)(s + h) * nn + g;
            t.np[h] = __ldg(tnp + gz);
            t.ns[h] = __ldg(tns + gz);
        }
        if (h1 == 2) t.dk = __ldg(tdk + (size_t)(s + 1) * nn + g);
        if (mode != 0) t.dki = *dki;
    }
    return t;
}

// The pointwise work of a row pass at grid point g (index y*n + x in the plane): the RK4
// applications around a step boundary, h = 0 the second half of step s and h = 1 the first
// half of step s+1 (Solver.h:267-273); mode 0 (s = -1, the first pass) runs h = 1 only, mode
// 2 (the last step) h = 0 only.  With them: the heat source of slice s (thermal), the
// per-slice record of the fields before step s+1 and the outputs after step out_after with
// their power sums.  Thermal: pre holds the point's optics and running Δk prefix
// (thermal_pre), and dki receives the prefix through slice s + 1.
template <typename T, bool THERM>
__device__ __forceinline__ void boundary_point(const InstDesc& d, int mode, int s, size_t g, size_t nn, cx<T>& p,
                                               cx<T>& q, const cx<T>* cf_prev, const cx<T>* cf_next, T hap, T has,
                                               T qs, T dz6, double* dki, double& acc_s, double& acc_p,
                                               const ThermPre<T>& pre) {
    using V = cx<T>;
    using R = T;  // real type of the thermal 3D arrays
    const R* tnp = reinterpret_cast<const R*>(d.t_np);
    const R* tns = reinterpret_cast<const R*>(d.t_ns);
    R* tq = reinterpret_cast<R*>(d.t_q);
    const int h0 = mode == 0 ? 1 : 0, h1 = mode == 2 ? 1 : 2;
    double dk_run = pre.dki;  // thermal: the running Δk prefix through this half step's slice
#pragma unroll 1
    for (int h = h0; h < h1; ++h) {
        const int sl = s + h;  // slice of this half step
        if constexpr (THERM) {
            const size_t gz = (size_t)sl * nn + g;
            if (h == 1) {
                dk_run += (double)pre.dk;
                *dki = dk_run;
            }
            // this half step's optics (selects, so that the rolled loop indexes no array)
            const double np = (double)(h ? pre.np[1] : pre.np[0]), ns = (double)(h ? pre.ns[1] : pre.ns[0]);
            V cf[6];
            thermal_coef<T>(d, dk_run, sl, np, ns, cf);
            rk4_point<T>(p, q, cf, hap, has, (T)(0.5 * (d.bf_s * ns)), dz6);
            if (h == 0 && tq) {
                // kernelSetQ (Tfield.h:260-276) for slice s, after its step
                const R ap2 = p.x * p.x + p.y * p.y, as2 = q.x * q.x + q.y * q.y;
                const R is = (R)d.q_h * (R)ns * as2;
                tq[gz] = (R)d.q_p * (R)np * ap2 + (R)d.q_s * (R)ns * as2 + (R)d.beta_s * (is * is);
            }
        } else {
            (void)dki;
            (void)pre;
            rk4_point<T>(p, q, h ? cf_next : cf_prev, hap, has, qs, dz6);
        }
        if (h == 0 && s + 1 < d.nslices) {
            // per-slice record: the fields before step s+1 (Solver.h:289-295)
            const size_t gs = (size_t)(s + 1) * nn + g;
            if (d.slices_p) put_field<T>(d, d.slices_p, gs, p);
            if (d.slices_s) put_field<T>(d, d.slices_s, gs, q);
        }
        if (h == 0 && s + 1 == d.out_after) {
            if (d.pump_out) put_field<T>(d, d.pump_out, g, p);
            if (d.signal_out) put_field<T>(d, d.signal_out, g, q);
            double ws = 1.0, wp = 1.0;
            if constexpr (THERM) {
                ws = (double)tns[(size_t)(s + 1) * nn + g];
                wp = (double)tnp[(size_t)(s + 1) * nn + g];
            }
            acc_s += ws * ((double)q.x * (double)q.x + (double)q.y * (double)q.y);
            acc_p += wp * ((double)p.x * (double)p.x + (double)p.y * (double)p.y);
        }
    }
}

// Persistent march: each cluster takes instances from the device work queue *queue (an
// atomic counter the host zeroes before the launch, instances in the descriptor order the
// host chose: longest march first) until the queue is empty.  queue == nullptr: one
// instance per cluster, instance = cluster index.
template <typename T, int N, int C, int NT, bool THERM, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB)
    ssfm_plain_kernel(const InstDesc* __restrict__ descs, int count, int* __restrict__ queue) {
    using Cfg = PlainCfg<T, N, C, NT, THERM>;
    constexpr int R2 = Cfg::R2, SW = Cfg::SW;
    constexpr int JA = Cfg::JA, JB = Cfg::JB, JCA = Cfg::JCA, JCB = Cfg::JCB;
    constexpr int CPR = 16 / C;  // column sub-rows per n1 of this CTA
    using V = cx<T>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* Ps = reinterpret_cast<V*>(smem_raw);
    V* Ss = Ps + Cfg::PLANE;
    using W = mult<T>;
    V* coef = Ss + Cfg::PLANE;   // [2][6] RK4 stage coefficients
    W* tw = reinterpret_cast<W*>(coef + 12);  // tw[k*16 + n1] = W_N^{n1 k}, forward sign
    W* pxp = tw + N;             // pump propagator, x factor, by physical column position
    W* pxs = pxp + N;            // SH   propagator, x factor
    W* pyp = pxs + N;            // pump propagator, y factor by frequency, × 1/N^2
    W* pys = pyp + N;            // SH   propagator, y factor
    double* red = reinterpret_cast<double*>(pys + N);  // [2*(NT/32)] + [4]
    double* dkint = red + 2 * (NT / 32) + 4;           // thermal: [RL*N] running Δk prefix
    // plain FP32: packed RK4 stage constants [2][3], in the place of the thermal prefix
    Rk4Pack* kpk = reinterpret_cast<Rk4Pack*>(dkint);
    constexpr bool PACK = !THERM && sizeof(T) == 4;

    const int tid = threadIdx.x;
    const int crank = (C > 1) ? (int)cg::this_cluster().block_rank() : 0;

    auto cluster_sync = [&]() {
        if constexpr (C > 1) cg::this_cluster().sync();
        else __syncthreads();
    };

    // next instance of this cluster: rank 0 takes it from the queue and the others read it
    // from rank 0's shared memory; the second barrier keeps rank 0 (and its shared memory)
    // alive until every CTA has read it
    __shared__ int s_next;
    auto take = [&]() -> int {
        if (crank == 0 && tid == 0) s_next = atomicAdd(queue, 1);
        cluster_sync();
        int v = s_next;
        if constexpr (C > 1) v = *cg::this_cluster().map_shared_rank(&s_next, 0);
        cluster_sync();
        return v;
    };
    int inst = queue ? take() : (int)(blockIdx.x / C);
#pragma unroll 1
    while (inst < count) {
        const InstDesc d = descs[inst];
        const int nsteps = d.nsteps;

        // ---- tables -----------------------------------------------------------------
        init_tables<T, N>(d, tw, pxp, pxs, pyp, pys, tid, NT);
        if (!THERM && tid < 3) {
            stage_coef<T>(d, 0, 0.0, tid, coef);
            if constexpr (PACK) stage_pack(coef, tid, kpk);
        }

        // ---- initial fields: setPump (Efields.h:84-119), SH = 0 or given ---------------
        for (int e = tid; e < Cfg::PLANE; e += NT) {
            const int lr = e / N, x = e % N;
            const int y = crank + C * lr;
            const double2 pv = pump_value(d, x, y, d.amp_re, d.amp_im, d.den_re, d.den_im);
            Ps[sidx<N, R2, SW>(lr, x)] = mk<T>((T)pv.x, (T)pv.y);
            Ss[sidx<N, R2, SW>(lr, x)] = d.has_signal_in ? get_field<T>(d, d.signal_in, (size_t)y * N + x)
                                                         : mk<T>((T)0, (T)0);
            if (d.slices_p) put_field<T>(d, d.slices_p, (size_t)y * N + x, Ps[sidx<N, R2, SW>(lr, x)]);
            if (d.slices_s) put_field<T>(d, d.slices_s, (size_t)y * N + x, Ss[sidx<N, R2, SW>(lr, x)]);
        }
        __syncthreads();

        const T hap = (T)d.hap, has = (T)d.has, qs = (T)d.qs, dz6 = (T)(d.dz / 6.0);

        // nsteps >= 1 (the host rejects nz < 2)
        //
        // Code size matters more than instruction count here: the step loop cycles through
        // every pass, so each pass keeps a single copy of its transform (the inverse is computed
        // as conj(DFT(conj(x))) with the forward body) and the two fields go through it in a
        // rolled loop.  Forward R2 stage: DFT then twiddle W_N^{n1 k}; inverse: conj twiddle then
        // IDFT, i.e. conj(DFT(conj(x) W)).
        auto cj = [](V a) { return mk<T>(a.x, -a.y); };

        // ---- RA: rows, R2-point stage of (row lr, n1) and the pointwise RK4 half-steps -----
        // mode 0: first (natural order in: RK4(z_0), forward), 1: middle (inverse, RK4(z_s),
        // RK4(z_{s+1}), forward), 2: last (inverse, RK4(z_s), outputs)

        // s: index of the step that ends in this pass (-1 in the first pass)
        auto pass_ra = [&](int mode, int s, const V* cf_prev, const V* cf_next, double& acc_s, double& acc_p) {
            for (int j = tid; j < JA; j += NT) {
                const int n1 = j & 15, lr = j >> 4;
#pragma unroll 1
                for (int ph = 0; ph < 5; ++ph) {
                    if (ph == 2) {
                        // pointwise: the two RK4 applications around the step boundary (the second
                        // half of step s, then the first half of step s+1)
                        if constexpr (PACK) {
                            if (mode == 1 && s + 1 >= d.nslices) {
                                // a middle step that records nothing: two points at a time in
                                // packed arithmetic
                                const Rk4Pack* kprev = kpk + 3 * (s & 1);
                                const Rk4Pack* knext = kpk + 3 * ((s + 1) & 1);
                                const float2 nhap = bc2(-hap), nhas = bc2(-has), nqs = bc2(-qs), dzz = bc2(dz6);
#pragma unroll 1
                                for (int k = 0; k + 1 < R2; k += 2) {
                                    const int o0 = sidx<N, R2, SW>(lr, n1 + 16 * k);
                                    const int o1 = sidx<N, R2, SW>(lr, n1 + 16 * k + 16);
                                    const V p0 = Ps[o0], q0 = Ss[o0], p1 = Ps[o1], q1 = Ss[o1];
                                    Cx2 P{make_float2(p0.x, p1.x), make_float2(p0.y, p1.y)};
                                    Cx2 S{make_float2(q0.x, q1.x), make_float2(q0.y, q1.y)};
                                    rk4_pair(P, S, kprev, nhap, nhas, nqs, dzz);
                                    rk4_pair(P, S, knext, nhap, nhas, nqs, dzz);
                                    Ps[o0] = make_float2(P.r.x, P.i.x);
                                    Ps[o1] = make_float2(P.r.y, P.i.y);
                                    Ss[o0] = make_float2(S.r.x, S.i.x);
                                    Ss[o1] = make_float2(S.r.y, S.i.y);
                                }
                                if constexpr (R2 & 1) {
                                    const int o = sidx<N, R2, SW>(lr, n1 + 16 * (R2 - 1));
                                    V p = Ps[o], q = Ss[o];
                                    rk4_point<T>(p, q, cf_prev, hap, has, qs, dz6);
                                    rk4_point<T>(p, q, cf_next, hap, has, qs, dz6);
                                    Ps[o] = p;
                                    Ss[o] = q;
                                }
                                continue;
                            }
                        }
                        // otherwise point by point, two interleaved for instruction-level
                        // parallelism
#pragma unroll 2
                        for (int k = 0; k < R2; ++k) {
                            const int x = n1 + 16 * k;
                            const int o = sidx<N, R2, SW>(lr, x);
                            const size_t g = (size_t)(crank + C * lr) * N + x;
                            V p = Ps[o], q = Ss[o];
                            double* dkp = THERM ? &dkint[lr * N + x] : nullptr;
                            const ThermPre<T> pre = thermal_pre<T, THERM>(d, mode, s, g, (size_t)N * N, dkp);
                            boundary_point<T, THERM>(d, mode, s, g, (size_t)N * N, p, q, cf_prev, cf_next, hap, has,
                                                     qs, dz6, dkp, acc_s, acc_p, pre);
                            if (mode != 2) {
                                Ps[o] = p;
                                Ss[o] = q;
                            }
                        }
                        continue;
                    }
                    const bool inv = ph < 2;
                    if ((inv && mode == 0) || (!inv && mode == 2)) continue;
                    V* F = (ph == 1 || ph == 3) ? Ss : Ps;
                    V v[R2];
#pragma unroll
                    for (int k = 0; k < R2; ++k) v[k] = F[sidx<N, R2, SW>(lr, n1 + 16 * k)];
                    if (inv) {
                        v[0] = cj(v[0]);
#pragma unroll
                        for (int k = 1; k < R2; ++k) v[k] = mulw(cj(v[k]), tw[k * 16 + n1]);
                    }
                    Dft<R2, -1, T>::run(v);
                    if (inv) {
#pragma unroll
                        for (int k = 0; k < R2; ++k) v[k] = cj(v[k]);
                    } else {
#pragma unroll
                        for (int k = 1; k < R2; ++k) v[k] = mulw(v[k], tw[k * 16 + n1]);
                    }
#pragma unroll
                    for (int k = 0; k < R2; ++k) F[sidx<N, R2, SW>(lr, n1 + 16 * k)] = v[k];
                }
            }
        };

        // ---- RB: rows, 16-point DFT over n1 (in place, digit-reversed output) ----------
        auto pass_rb = [&](bool inv) {
            for (int j = tid; j < JB; j += NT) {
                const int k2 = j % R2, lr = j / R2;
#pragma unroll 1
                for (int f = 0; f < 2; ++f) {
                    V* F = f ? Ss : Ps;
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

        // ---- CA: columns, R2-point stage over n2 on this CTA's rows ----------------------
        auto pass_ca = [&](bool inv) {
            for (int j = tid; j < JCA; j += NT) {
                const int x = j % N, n1l = j / N;
                const int n1 = crank + C * n1l;
#pragma unroll 1
                for (int f = 0; f < 2; ++f) {
                    V* F = f ? Ss : Ps;
                    V v[R2];
#pragma unroll
                    for (int k = 0; k < R2; ++k) v[k] = F[sidx<N, R2, SW>(n1l + CPR * k, x)];
                    if (inv) {
                        v[0] = cj(v[0]);
#pragma unroll
                        for (int k = 1; k < R2; ++k) v[k] = mulw(cj(v[k]), tw[k * 16 + n1]);
                    }
                    Dft<R2, -1, T>::run(v);
                    if (inv) {
#pragma unroll
                        for (int k = 0; k < R2; ++k) v[k] = cj(v[k]);
                    } else {
#pragma unroll
                        for (int k = 1; k < R2; ++k) v[k] = mulw(v[k], tw[k * 16 + n1]);
                    }
#pragma unroll
                    for (int k = 0; k < R2; ++k) F[sidx<N, R2, SW>(n1l + CPR * k, x)] = v[k];
                }
            }
        };

        // ---- CB: columns, DFT over n1 across the cluster, propagator, IDFT ----------------
        auto pass_cb = [&]() {
            V* rP[C];
            V* rS[C];
#pragma unroll
            for (int r = 0; r < C; ++r) {
                if constexpr (C > 1) {
                    rP[r] = cg::this_cluster().map_shared_rank(Ps, r);
                    rS[r] = cg::this_cluster().map_shared_rank(Ss, r);
                } else {
                    rP[r] = Ps;
                    rS[r] = Ss;
                }
            }
            for (int j = tid; j < JCB; j += NT) {
                const int xl = j % (N / C), k2 = j / (N / C);
                const int x = crank * (N / C) + xl;
#pragma unroll 1
                for (int f = 0; f < 2; ++f) {
                    V* const* R = f ? rS : rP;
                    const W px = f ? pxs[x] : pxp[x];
                    const W* py = f ? pys : pyp;
                    V u[16];
#pragma unroll
                    for (int n = 0; n < 16; ++n) u[n] = R[n % C][sidx<N, R2, SW>(n / C + CPR * k2, x)];
#pragma unroll 1
                    for (int it = 0; it < 2; ++it) {
                        if (it) {
#pragma unroll
                            for (int n = 0; n < 16; ++n) u[n] = cj(u[n]);
                        }
                        Dft<16, -1, T>::run(u);
                        if (!it) {
#pragma unroll
                            for (int k1 = 0; k1 < 16; ++k1) u[k1] = mulw(mulw(u[k1], py[k2 + R2 * k1]), px);
                        } else {
#pragma unroll
                            for (int n = 0; n < 16; ++n) u[n] = cj(u[n]);
                        }
                    }
#pragma unroll
                    for (int n = 0; n < 16; ++n) R[n % C][sidx<N, R2, SW>(n / C + CPR * k2, x)] = u[n];
                }
            }
        };

        // Between the two row passes a CTA-wide barrier is needed only where a warp's RA jobs
        // and RB jobs touch different rows.  With R2 == 16 both passes give job j the row j / 16
        // and every thread the same jobs, so each warp owns its rows for RB, RA and RB' / RA'
        // alike, and a warp barrier orders them.
        auto row_sync = [&]() {
            if constexpr (R2 == 16) __syncwarp();
            else __syncthreads();
        };

        double acc_s = 0.0, acc_p = 0.0;
        pass_ra(0, -1, coef, coef, acc_s, acc_p);
        row_sync();

        double z = 0.0;
        for (int s = 0; s < nsteps; ++s) {
            V* cf_cur = coef + 6 * (s & 1);
            V* cf_nxt = coef + 6 * ((s + 1) & 1);
            pass_rb(false);
            __syncthreads();
            pass_ca(false);
            cluster_sync();
            if (!THERM && tid < 3 && s + 1 < nsteps) {
                stage_coef<T>(d, s + 1, z + d.dz, tid, cf_nxt);
                if constexpr (PACK) stage_pack(cf_nxt, tid, kpk + 3 * ((s + 1) & 1));
            }
            pass_cb();
            cluster_sync();
            pass_ca(true);
            __syncthreads();
            pass_rb(true);
            row_sync();
            pass_ra(s + 1 < nsteps ? 1 : 2, s, cf_cur, cf_nxt, acc_s, acc_p);
            row_sync();
            z += d.dz;
        }

        // ---- SH and pump power: deterministic block + cluster reduction --------------------
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc_s += __shfl_down_sync(0xffffffffu, acc_s, o);
            acc_p += __shfl_down_sync(0xffffffffu, acc_p, o);
        }
        const int warp = tid >> 5, lane = tid & 31;
        if (lane == 0) {
            red[2 * warp] = acc_s;
            red[2 * warp + 1] = acc_p;
        }
        __syncthreads();
        double* part = red + 2 * (NT / 32);
        if (tid == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < NT / 32; ++w) { a += red[2 * w]; b += red[2 * w + 1]; }
            part[0] = a;
            part[1] = b;
        }
        cluster_sync();
        if (crank == 0 && tid == 0 && d.power_out) {
            double a = 0.0, b = 0.0;
            for (int r = 0; r < C; ++r) {
                const double* pr = part;
                if constexpr (C > 1) pr = cg::this_cluster().map_shared_rank(part, r);
                a += pr[0];
                b += pr[1];
            }
            d.power_out[0] = a * d.pw_s;
            d.power_out[1] = b * d.pw_p;
        }
        cluster_sync();
        if (!queue) break;
        inst = take();
    }  // instances
}

}  // namespace shg
