// ssfm_adjoint.cuh — hand-written adjoint of the plain SSFM march: gradients of the SH output
// power J = pw_s sum |S|^2 with respect to the beam waist, the focal position, the oven
// temperature and a per-step poling-phase vector.  No counterpart in the reference, which
// has no gradients; the forward model is the reference's scheme (Solver.h:189-308).
//
// Forward step s:  x_s --N_s--> a1 --L--> a2_s --N_s--> x_{s+1}   (N_s: the RK4 application
// at z_s, L: diffraction).  Backward, with adjoints g = dJ/dRe + i dJ/dIm of the fields:
//     mu2 = N_s^T(a2_s) lambda_{s+1},   mu1 = L^H mu2,   lambda_s = N_s^T(x_s) mu1
// where N_s^T is the vector-Jacobian product of the RK4 scheme (stage values recomputed from
// the input point) and L^H the diffraction with the conjugate propagator.
//
// One cluster owns an instance for the whole computation (a launch holds one cluster per
// instance of a batch), with the same shared-memory layout and transform passes as the
// forward march (ssfm_plain.cuh):
//   1. forward march, keeping x_{mK} (checkpoints every K steps) in global memory;
//   2. for each segment m from the last: re-march from x_{mK}, keeping x_s, a2_s and the
//      propagated spectra of each step of the segment (the last segment's come from step 1
//      directly); then march the adjoint back through the segment; the adjoint fields are
//      parked in global memory between segments.
// Each phase is a launch (kAdjForward, kAdjRemarch, kAdjBackward, one round of segments
// per launch), the segment buffers are double-buffered by segment parity, so the host can
// run the re-march of segment m-1 on other SMs while the adjoint march of segment m runs.
// Parameter sensitivities are accumulated on the way: the stage coefficients' dependence
// on κ, Δk, the two-photon term and the poling phase (RK4 adjoint), the propagator phases'
// dependence on n(T) (adjoint diffraction, with the stored spectra), and the initial pump's
// dependence on waist, focus and T (central differences of the closed-form Gaussian).
#pragma once

#include "ssfm_plain.cuh"

namespace shg {

// accumulators (per CTA) of the adjoint
enum {
    kAccKp = 0,     // sum Re(conj(g_dP) t)          = κp dJ/dκp
    kAccKs = 1,     // sum Re(conj(g_dS) u)          = κs dJ/dκs
    kAccDk = 2,     // sum phase sensitivity (z + dz inc)   = dJ/dΔk
    kAccQs = 3,     // sum Re(conj(g_dS) (-|S|^2 S)) = dJ/dqs
    kAccPropP = 4,  // sum over steps, frequencies of Re(conj(Λ) i Y) q   (pump)
    kAccPropS = 5,  //                                                 (SH)
    kAccG0w = 6,    // Re <λ0_P, dP0/dwaist>
    kAccG0f = 7,    // Re <λ0_P, dP0/dfocus>
    kAccG0T = 8,    // Re <λ0_P, dP0/dT>
    kAccJ = 9,      // sum |S_out|^2
    kAdjAcc = 10
};

// launch phases of ssfm_adjoint_kernel
enum { kAdjForward = 0, kAdjRemarch = 1, kAdjBackward = 2 };

struct AdjDesc {
    int32_t K;          // checkpoint interval (steps)
    int32_t M;          // number of checkpoints (x_{mK}, m = 0..M-1)
    void* ckpt;         // M x 2 x n*n complex (pump, SH) before step mK, natural layout
    void* seg_a2;       // 2 x K x 2 x n*n: fields after the diffraction of each step of a segment
    void* seg_x;        // 2 x K x 2 x n*n: fields before each step of a segment
    void* seg_y;        // 2 x K x 2 x n*n: propagated spectra of each step (CB order: fy*n + column)
                        // (two buffers each, the one of segment m at parity m & 1)
    void* lam;          // 2 x n*n: adjoint fields between segments
    const double* zs;   // nsteps: z at the start of each step (the forward's accumulation)
    double* part;       // [M + 1][C][kAdjAcc] per-CTA accumulators: slot 0 the forward launch,
                        // slot 1 + m the adjoint march of segment m
    double* phi;        // [nsteps][C] per-CTA dJ/dφ_s
    double pert[6][4];  // pump (amp_re, amp_im, den_re, den_im) at waist±hw, focus±hf, T±hT
    double inv2h[3];    // 1 / (2 h) of those differences
};

// Vector-Jacobian product of dA/dz at (p, s) (see dadz): adds to (gp, gs) the adjoints of
// the inputs given the adjoints (gdp, gds) of (dp, ds), and to sens[] the parameter terms in
// the working precision: sens[0] κp, [1] κs, [2] Σ inc·e_φ, [3] qs, [4] Σ e_φ, where e_φ is
// the mismatch-phase term and inc the stage's offset in units of dz (0, 1/4, 1/2), so that
// the Δk term of a step at z is z·sens[4] + dz·sens[2] and its poling term sens[4].
template <typename T>
__device__ __forceinline__ void dadz_vjp(cx<T> p, cx<T> s, cx<T> cP, cx<T> cS, T hap, T has, T qs, cx<T> gdp,
                                         cx<T> gds, cx<T>& gp, cx<T>& gs, T inc, T* sens) {
    const cx<T> t = mul<T>(cP, mulc<T>(s, p));                   // cP s conj(p)
    const cx<T> pp = mk<T>(p.x * p.x - p.y * p.y, (T)2 * p.x * p.y);
    const cx<T> u = mul<T>(cS, pp);                               // cS p^2
    const T a2 = s.x * s.x + s.y * s.y;
    // g_p: -hap g_dP + cP s conj(g_dP) + conj(2 cS p) g_dS
    const cx<T> a = mulc<T>(mul<T>(cP, s), gdp);
    const cx<T> b = mulc<T>(gds, mul<T>(cS, p));
    gp = mk<T>(gp.x - hap * gdp.x + a.x + (T)2 * b.x, gp.y - hap * gdp.y + a.y + (T)2 * b.y);
    // g_s: conj(cP) p g_dP + (-has - 2 qs |s|^2) g_dS - qs s^2 conj(g_dS)
    const cx<T> c = mul<T>(mulc<T>(p, cP), gdp);
    const cx<T> ss = mk<T>(s.x * s.x - s.y * s.y, (T)2 * s.x * s.y);
    const cx<T> e = mulc<T>(ss, gds);
    const T h = -has - (T)2 * qs * a2;
    gs = mk<T>(gs.x + c.x + h * gds.x - qs * e.x, gs.y + c.y + h * gds.y - qs * e.y);
    const T eph = (gdp.x * t.y - gdp.y * t.x) - (gds.x * u.y - gds.y * u.x);
    sens[0] += gdp.x * t.x + gdp.y * t.y;
    sens[1] += gds.x * u.x + gds.y * u.y;
    sens[2] += eph * inc;
    sens[3] += -a2 * (gds.x * s.x + gds.y * s.y);
    sens[4] += eph;
}

// Vector-Jacobian product of one RK4 application (rk4_point) at input (p, s) with stage
// coefficients cf (phases at z, z + dz/4, z + dz/2): (gp, gs) holds the adjoint of the
// output on entry and of the input on return; sens[] as for dadz_vjp.
template <typename T>
__device__ __forceinline__ void rk4_vjp(cx<T> p, cx<T> s, const cx<T>* cf, T hap, T has, T qs, T dz6, cx<T>& gp,
                                        cx<T>& gs, T* sens) {
    using V = cx<T>;
    V k1p, k1s, k2p, k2s, k3p, k3s, k4p, k4s;
    dadz<T>(p, s, cf[0], cf[3], hap, has, qs, k1p, k1s);
    const V u2p = mk<T>(p.x + (T)0.5 * k1p.x, p.y + (T)0.5 * k1p.y), u2s = mk<T>(s.x + (T)0.5 * k1s.x, s.y + (T)0.5 * k1s.y);
    dadz<T>(u2p, u2s, cf[1], cf[4], hap, has, qs, k2p, k2s);
    const V u3p = mk<T>(p.x + (T)0.5 * k2p.x, p.y + (T)0.5 * k2p.y), u3s = mk<T>(s.x + (T)0.5 * k2s.x, s.y + (T)0.5 * k2s.y);
    dadz<T>(u3p, u3s, cf[1], cf[4], hap, has, qs, k3p, k3s);
    const V u4p = add<T>(p, k3p), u4s = add<T>(s, k3s);
    (void)k4p;
    (void)k4s;
    const V gop = gp, gos = gs;
    V g3p = scale<T>(gop, (T)2 * dz6), g3s = scale<T>(gos, (T)2 * dz6);
    V g2p = g3p, g2s = g3s;
    V g1p = scale<T>(gop, dz6), g1s = scale<T>(gos, dz6);
    V hp = mk<T>(0, 0), hs = mk<T>(0, 0);
    dadz_vjp<T>(u4p, u4s, cf[2], cf[5], hap, has, qs, g1p, g1s, hp, hs, (T)0.5, sens);  // g_k4 = dz6 g
    gp = add<T>(gop, hp);
    gs = add<T>(gos, hs);
    g3p = add<T>(g3p, hp);
    g3s = add<T>(g3s, hs);
    hp = mk<T>(0, 0);
    hs = mk<T>(0, 0);
    dadz_vjp<T>(u3p, u3s, cf[1], cf[4], hap, has, qs, g3p, g3s, hp, hs, (T)0.25, sens);
    gp = add<T>(gp, hp);
    gs = add<T>(gs, hs);
    g2p = add<T>(g2p, scale<T>(hp, (T)0.5));
    g2s = add<T>(g2s, scale<T>(hs, (T)0.5));
    hp = mk<T>(0, 0);
    hs = mk<T>(0, 0);
    dadz_vjp<T>(u2p, u2s, cf[1], cf[4], hap, has, qs, g2p, g2s, hp, hs, (T)0.25, sens);
    gp = add<T>(gp, hp);
    gs = add<T>(gs, hs);
    g1p = add<T>(g1p, scale<T>(hp, (T)0.5));
    g1s = add<T>(g1s, scale<T>(hs, (T)0.5));
    hp = mk<T>(0, 0);
    hs = mk<T>(0, 0);
    dadz_vjp<T>(p, s, cf[0], cf[3], hap, has, qs, g1p, g1s, hp, hs, (T)0, sens);
    gp = add<T>(gp, hp);
    gs = add<T>(gs, hs);
}

// dadz_vjp for two points at once in packed FP32 (see rk4_pair): the same terms, lane 0 the
// first point and lane 1 the second; the five sensitivities are accumulated per lane.
// Constant pairs: nhap = -hap, nhas = -has, nqs = -qs, n2qs = -2 qs, inc in both lanes.
__device__ __forceinline__ void dadz_vjp_pair(const Cx2& p, const Cx2& s, const Rk4Pack& K, float2 nhap, float2 nhas,
                                              float2 nqs, float2 n2qs, const Cx2& gdp, const Cx2& gds, Cx2& gp,
                                              Cx2& gs, float2 inc, float2* sens) {
    const float2 m1 = bc2(-1.f), two = bc2(2.f);
    const float2 npi = __fmul2_rn(m1, p.i), nsi = __fmul2_rn(m1, s.i);
    const float2 ngdpi = __fmul2_rn(m1, gdp.i), ngdsr = __fmul2_rn(m1, gds.r), ngdsi = __fmul2_rn(m1, gds.i);
    // t = cP s conj(p)
    const float2 spr = __ffma2_rn(s.i, p.i, __fmul2_rn(s.r, p.r));
    const float2 spi = __ffma2_rn(s.r, npi, __fmul2_rn(s.i, p.r));
    const float2 tr = __ffma2_rn(K.ncpi, spi, __fmul2_rn(K.cpr, spr));
    const float2 ti = __ffma2_rn(K.cpi, spr, __fmul2_rn(K.cpr, spi));
    // u = cS p^2
    const float2 ppr = __ffma2_rn(p.i, npi, __fmul2_rn(p.r, p.r));
    const float2 ppi = __fmul2_rn(__fadd2_rn(p.r, p.r), p.i);
    const float2 ur = __ffma2_rn(K.ncsi, ppi, __fmul2_rn(K.csr, ppr));
    const float2 ui = __ffma2_rn(K.csi, ppr, __fmul2_rn(K.csr, ppi));
    const float2 a2 = __ffma2_rn(s.i, s.i, __fmul2_rn(s.r, s.r));
    // g_p += -hap g_dP + (cP s) conj(g_dP) + 2 g_dS conj(cS p)
    const float2 cps_r = __ffma2_rn(K.ncpi, s.i, __fmul2_rn(K.cpr, s.r));
    const float2 cps_i = __ffma2_rn(K.cpi, s.r, __fmul2_rn(K.cpr, s.i));
    const float2 ar = __ffma2_rn(cps_i, gdp.i, __fmul2_rn(cps_r, gdp.r));
    const float2 ai = __ffma2_rn(cps_r, ngdpi, __fmul2_rn(cps_i, gdp.r));
    const float2 csp_r = __ffma2_rn(K.ncsi, p.i, __fmul2_rn(K.csr, p.r));
    const float2 csp_i = __ffma2_rn(K.csi, p.r, __fmul2_rn(K.csr, p.i));
    const float2 br = __ffma2_rn(gds.i, csp_i, __fmul2_rn(gds.r, csp_r));
    const float2 bi = __ffma2_rn(ngdsr, csp_i, __fmul2_rn(gds.i, csp_r));
    gp.r = __ffma2_rn(two, br, __fadd2_rn(__ffma2_rn(nhap, gdp.r, gp.r), ar));
    gp.i = __ffma2_rn(two, bi, __fadd2_rn(__ffma2_rn(nhap, gdp.i, gp.i), ai));
    // g_s += (p conj(cP)) g_dP + (-has - 2 qs |s|^2) g_dS - qs s^2 conj(g_dS)
    const float2 pcc_r = __ffma2_rn(p.i, K.cpi, __fmul2_rn(p.r, K.cpr));
    const float2 pcc_i = __ffma2_rn(p.r, K.ncpi, __fmul2_rn(p.i, K.cpr));
    const float2 cr = __ffma2_rn(pcc_i, ngdpi, __fmul2_rn(pcc_r, gdp.r));
    const float2 ci = __ffma2_rn(pcc_i, gdp.r, __fmul2_rn(pcc_r, gdp.i));
    const float2 ssr = __ffma2_rn(s.i, nsi, __fmul2_rn(s.r, s.r));
    const float2 ssi = __fmul2_rn(__fadd2_rn(s.r, s.r), s.i);
    const float2 er = __ffma2_rn(ssi, gds.i, __fmul2_rn(ssr, gds.r));
    const float2 ei = __ffma2_rn(ssr, ngdsi, __fmul2_rn(ssi, gds.r));
    const float2 h = __ffma2_rn(n2qs, a2, nhas);
    gs.r = __ffma2_rn(nqs, er, __ffma2_rn(h, gds.r, __fadd2_rn(gs.r, cr)));
    gs.i = __ffma2_rn(nqs, ei, __ffma2_rn(h, gds.i, __fadd2_rn(gs.i, ci)));
    // sensitivities
    const float2 e1 = __ffma2_rn(ngdpi, tr, __fmul2_rn(gdp.r, ti));
    const float2 e2 = __ffma2_rn(ngdsi, ur, __fmul2_rn(gds.r, ui));
    const float2 eph = __ffma2_rn(m1, e2, e1);
    sens[0] = __fadd2_rn(sens[0], __ffma2_rn(gdp.i, ti, __fmul2_rn(gdp.r, tr)));
    sens[1] = __fadd2_rn(sens[1], __ffma2_rn(gds.i, ui, __fmul2_rn(gds.r, ur)));
    sens[2] = __ffma2_rn(eph, inc, sens[2]);
    sens[3] = __ffma2_rn(__fmul2_rn(m1, a2), __ffma2_rn(gds.i, s.i, __fmul2_rn(gds.r, s.r)), sens[3]);
    sens[4] = __fadd2_rn(sens[4], eph);
}

// rk4_vjp for two points at once in packed FP32; k[0..2] the stage phases (see rk4_pair)
__device__ __forceinline__ void rk4_vjp_pair(const Cx2& p, const Cx2& s, const Rk4Pack* k, float2 nhap, float2 nhas,
                                             float2 nqs, float2 n2qs, float2 dz6, Cx2& gp, Cx2& gs, float2* sens) {
    const float2 half = bc2(0.5f), z0 = bc2(0.f);
    auto axpy = [](float2 a, const Cx2& x, const Cx2& y) {  // a x + y
        return Cx2{__ffma2_rn(a, x.r, y.r), __ffma2_rn(a, x.i, y.i)};
    };
    auto sum = [](const Cx2& x, const Cx2& y) { return Cx2{__fadd2_rn(x.r, y.r), __fadd2_rn(x.i, y.i)}; };
    auto scl = [](const Cx2& x, float2 a) { return Cx2{__fmul2_rn(x.r, a), __fmul2_rn(x.i, a)}; };
    Cx2 k1p, k1s, k2p, k2s, k3p, k3s;
    dadz_pair(p, s, k[0], nhap, nhas, nqs, k1p, k1s);
    const Cx2 u2p = axpy(half, k1p, p), u2s = axpy(half, k1s, s);
    dadz_pair(u2p, u2s, k[1], nhap, nhas, nqs, k2p, k2s);
    const Cx2 u3p = axpy(half, k2p, p), u3s = axpy(half, k2s, s);
    dadz_pair(u3p, u3s, k[1], nhap, nhas, nqs, k3p, k3s);
    const Cx2 u4p = sum(p, k3p), u4s = sum(s, k3s);
    const Cx2 gop = gp, gos = gs;
    const float2 dz3 = __fadd2_rn(dz6, dz6);
    Cx2 g3p = scl(gop, dz3), g3s = scl(gos, dz3);
    Cx2 g2p = g3p, g2s = g3s;
    Cx2 g1p = scl(gop, dz6), g1s = scl(gos, dz6);
    Cx2 hp{z0, z0}, hs{z0, z0};
    dadz_vjp_pair(u4p, u4s, k[2], nhap, nhas, nqs, n2qs, g1p, g1s, hp, hs, bc2(0.5f), sens);  // g_k4 = dz6 g
    gp = sum(gop, hp);
    gs = sum(gos, hs);
    g3p = sum(g3p, hp);
    g3s = sum(g3s, hs);
    hp = Cx2{z0, z0};
    hs = Cx2{z0, z0};
    dadz_vjp_pair(u3p, u3s, k[1], nhap, nhas, nqs, n2qs, g3p, g3s, hp, hs, bc2(0.25f), sens);
    gp = sum(gp, hp);
    gs = sum(gs, hs);
    g2p = axpy(half, hp, g2p);
    g2s = axpy(half, hs, g2s);
    hp = Cx2{z0, z0};
    hs = Cx2{z0, z0};
    dadz_vjp_pair(u2p, u2s, k[1], nhap, nhas, nqs, n2qs, g2p, g2s, hp, hs, bc2(0.25f), sens);
    gp = sum(gp, hp);
    gs = sum(gs, hs);
    g1p = axpy(half, hp, g1p);
    g1s = axpy(half, hs, g1s);
    hp = Cx2{z0, z0};
    hs = Cx2{z0, z0};
    dadz_vjp_pair(p, s, k[0], nhap, nhas, nqs, n2qs, g1p, g1s, hp, hs, z0, sens);
    gp = sum(gp, hp);
    gs = sum(gs, hs);
}

// (a0, a1), (b0, b1) of two complex values as one packed pair and back
__device__ __forceinline__ Cx2 pack2(float2 a, float2 b) { return Cx2{make_float2(a.x, b.x), make_float2(a.y, b.y)}; }
__device__ __forceinline__ float2 lane0(const Cx2& v) { return make_float2(v.r.x, v.i.x); }
__device__ __forceinline__ float2 lane1(const Cx2& v) { return make_float2(v.r.y, v.i.y); }

// MARCH_ONLY: an instantiation with the forward and re-march phases only.  Without the
// adjoint march's code it needs half the registers, so two CTAs fit on an SM where the full
// kernel fits one; the march it runs is the same code as the full kernel's.
template <typename T, int N, int C, int NT, bool MARCH_ONLY = false>
__global__ void __launch_bounds__(NT, MARCH_ONLY ? 2 : 1) ssfm_adjoint_kernel(const InstDesc* __restrict__ descs,
                                                                              const AdjDesc* __restrict__ adescs,
                                                                              int phase, int round) {
    using Cfg = PlainCfg<T, N, C, NT, false>;
    constexpr int R2 = Cfg::R2, SW = Cfg::SW;
    constexpr int JA = Cfg::JA, JB = Cfg::JB, JCA = Cfg::JCA, JCB = Cfg::JCB;
    constexpr int CPR = 16 / C;
    constexpr size_t NN = (size_t)N * N;
    using V = cx<T>;
    using W = mult<T>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* Ps = reinterpret_cast<V*>(smem_raw);
    V* Ss = Ps + Cfg::PLANE;
    V* coef = Ss + Cfg::PLANE;  // [2][6], by step parity
    W* tw = reinterpret_cast<W*>(coef + 12);
    W* pxp = tw + N;
    W* pxs = pxp + N;
    W* pyp = pxs + N;
    W* pys = pyp + N;
    double* red = reinterpret_cast<double*>(pys + N);  // [2*(NT/32)] + [4]
    // FP32: the packed RK4 stage constants [2][3] by step parity (after the reduction area)
    Rk4Pack* kpk = reinterpret_cast<Rk4Pack*>(red + 2 * (NT / 32) + 4);
    constexpr bool PACK = sizeof(T) == 4;
    constexpr int KP = PACK ? (R2 & ~1) : 0;  // points of a job that go in packed pairs

    const int tid = threadIdx.x;
    const int crank = (C > 1) ? (int)cg::this_cluster().block_rank() : 0;
    const int inst = blockIdx.x / C;  // one cluster per instance
    const InstDesc d = descs[inst];
    const AdjDesc& a = adescs[inst];
    const int nsteps = d.nsteps;
    const int K = a.K;
    const T hap = (T)d.hap, has = (T)d.has, qs = (T)d.qs, dz6 = (T)(d.dz / 6.0);
    // segment of this launch: round r runs the adjoint march of segment M-1-r and the
    // re-march of segment M-2-r (the forward launch covers segment M-1); instances with
    // fewer segments have nothing to do in the late rounds
    const int m = phase == kAdjForward ? a.M - 1 : (phase == kAdjBackward ? a.M - 1 - round : a.M - 2 - round);
    if (m < 0) return;
    const size_t seg_stride = (size_t)K * 2 * NN;
    const size_t seg_off = (size_t)(m & 1) * seg_stride;
    V* ckpt = reinterpret_cast<V*>(a.ckpt);
    V* seg_a2 = reinterpret_cast<V*>(a.seg_a2) + seg_off;
    V* seg_y = reinterpret_cast<V*>(a.seg_y) + seg_off;
    V* lam = reinterpret_cast<V*>(a.lam);

    auto cluster_sync = [&]() {
        if constexpr (C > 1) cg::this_cluster().sync();
        else __syncthreads();
    };
    auto cj = [](V v) { return mk<T>(v.x, -v.y); };

    init_tables<T, N>(d, tw, pxp, pxs, pyp, pys, tid, NT);

    // accumulators (kAcc*), kept as scalars so that nothing is indexed at run time
    double acc_kp = 0.0, acc_ks = 0.0, acc_dk = 0.0, acc_qs = 0.0, acc_pp = 0.0, acc_ps = 0.0;
    double acc_g0w = 0.0, acc_g0f = 0.0, acc_g0T = 0.0, acc_j = 0.0;
    V* seg_x = reinterpret_cast<V*>(a.seg_x) + seg_off;

    // L2 prefetch of what adjoint step s of the segment from sb reads from global memory:
    // x_s, the stored spectra of step s and (s > sb) a2_{s-1}, each two planes in one
    // contiguous block. Each CTA of the cluster fetches its 1/C share of each block in 4 KB
    // bulk prefetches (16-byte aligned: a share is a multiple of 256 bytes), so the loads of
    // the point loop and of the column pass find it in L2 one step later.
    auto prefetch_step = [&](int s, int sb) {
        constexpr size_t kPair = 2 * (size_t)N * N * sizeof(V), kShare = kPair / C, kChunk = 4096;
        constexpr int kChunks = (int)((kShare + kChunk - 1) / kChunk);
        static_assert(kShare % 16 == 0, "bulk prefetch needs 16-byte multiples");
        for (int i = tid; i < 3 * kChunks; i += NT) {
            const int arr = i / kChunks, ch = i % kChunks;
            const int slot = arr == 2 ? s - 1 - sb : s - sb;
            if (slot < 0 || slot >= K) continue;
            const V* blk = arr == 0 ? seg_x : (arr == 1 ? seg_y : seg_a2);
            const char* src = reinterpret_cast<const char*>(blk) + (size_t)slot * kPair + (size_t)crank * kShare +
                              (size_t)ch * kChunk;
            const size_t rem = kShare - (size_t)ch * kChunk;
            const unsigned bytes = (unsigned)(rem < kChunk ? rem : kChunk);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
        }
    };

    // ---- plane transfers between shared memory and global (natural layout) ------------
    auto load_planes = [&](const V* gp, const V* gs) {
        for (int e = tid; e < Cfg::PLANE; e += NT) {
            const int lr = e / N, x = e % N;
            const size_t g = (size_t)(crank + C * lr) * N + x;
            Ps[sidx<N, R2, SW>(lr, x)] = gp[g];
            Ss[sidx<N, R2, SW>(lr, x)] = gs[g];
        }
    };
    auto store_planes = [&](V* gp, V* gs) {
        for (int e = tid; e < Cfg::PLANE; e += NT) {
            const int lr = e / N, x = e % N;
            const size_t g = (size_t)(crank + C * lr) * N + x;
            gp[g] = Ps[sidx<N, R2, SW>(lr, x)];
            gs[g] = Ss[sidx<N, R2, SW>(lr, x)];
        }
    };

    // ---- transform passes (as in the forward march) -----------------------------------
    // R2-point row stage of job (lr, n1): forward = DFT then twiddle; inverse =
    // conj(DFT(conj(x) W)).
    auto row_a = [&](V* F, int lr, int n1, bool inv) {
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
    };
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
    // CB: forward (store the propagated spectrum of step slot `ys` when ys >= 0) or
    // adjoint (conjugate propagator; accumulate the n(T) sensitivity with the stored spectrum)
    auto pass_cb = [&](bool adjoint, int ys) {
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
        const T dfy2 = (T)(d.dfy * d.dfy);
        for (int j = tid; j < JCB; j += NT) {
            const int xl = j % (N / C), k2 = j / (N / C);
            const int x = crank * (N / C) + xl;
            const int fx = (x >> 4) + R2 * (x & 15);
            const double sx = (double)(fx < N / 2 ? fx : fx - N);
            const T fxq = (T)(d.dfx * d.dfx * (sx * sx));  // dfx^2 sx^2 of this column
#pragma unroll 1
            for (int f = 0; f < 2; ++f) {
                V* const* R = f ? rS : rP;
                const W px = f ? pxs[x] : pxp[x];
                const W* py = f ? pys : pyp;
                V* ybuf = (ys >= 0) ? seg_y + ((size_t)ys * 2 + f) * NN : nullptr;
                T wsum = 0;  // this job's propagator-phase sensitivity (adjoint)
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
                        for (int k1 = 0; k1 < 16; ++k1) {
                            const int fy = k2 + R2 * k1;
                            const size_t yo = (size_t)fy * N + x;
                            if (!adjoint) {
                                u[k1] = mulw(mulw(u[k1], py[fy]), px);
                                if (ybuf) __stcs(&ybuf[yo], u[k1]);  // read by a later launch: evict first
                            } else {
                                // dJ/dθ_f = Re(conj(Λ) i Y): Λ = this spectrum / N^2, Y = stored D X,
                                // stored as D X / N^2 -> Re(conj(u) i Ystored)
                                const V yv = __ldcs(&ybuf[yo]);  // read once: evict first
                                const T c = u[k1].y * yv.x - u[k1].x * yv.y;
                                const T sy = (T)(fy < N / 2 ? fy : fy - N);
                                wsum += c * (fxq + dfy2 * (sy * sy));
                                // conjugate propagator: conj(py) conj(px), via conj(conj(u) py px)
                                u[k1] = cj(mulw(mulw(cj(u[k1]), py[fy]), px));
                            }
                        }
                    } else {
#pragma unroll
                        for (int n = 0; n < 16; ++n) u[n] = cj(u[n]);
                    }
                }
                if (adjoint) {
                    if (f) acc_ps += (double)wsum;
                    else acc_pp += (double)wsum;
                }
#pragma unroll
                for (int n = 0; n < 16; ++n) R[n % C][sidx<N, R2, SW>(n / C + CPR * k2, x)] = u[n];
            }
        }
    };

    auto coefs = [&](int s) {  // stage coefficients of step s into its parity slot
        if (tid < 3) {
            stage_coef<T>(d, s, a.zs[s], tid, coef + 6 * (s & 1));
            if constexpr (PACK) stage_pack(coef + 6 * (s & 1), tid, kpk + 3 * (s & 1));
        }
    };
    // the per-instance constants in both lanes (FP32)
    const float2 nhap2 = bc2(-(float)hap), nhas2 = bc2(-(float)has), nqs2 = bc2(-(float)qs);
    const float2 n2qs2 = bc2(-2.f * (float)qs), dz62 = bc2((float)dz6);

    // ---- forward march over steps [sb, se) from the fields in shared memory ------------
    // ckpt_mode: keep x_{mK} as checkpoints.  Steps s >= seg_from keep x_s, a2_s and their
    // propagated spectra in the segment buffers (slot s - seg_from).  seed: the march runs to
    // the end and turns the SH output into the adjoint seed lambda = (0, 2 pw_s S)
    // (accumulating J); otherwise it stops after a2_{se-1}.
    auto march = [&](int sb, int se, bool ckpt_mode, int seg_from, bool seed) {
        coefs(sb);
        if (ckpt_mode && sb % K == 0) store_planes(ckpt + (size_t)(sb / K) * 2 * NN, ckpt + ((size_t)(sb / K) * 2 + 1) * NN);
        if (sb >= seg_from)
            store_planes(seg_x + (size_t)(sb - seg_from) * 2 * NN, seg_x + ((size_t)(sb - seg_from) * 2 + 1) * NN);
        __syncthreads();
        // first half of step sb, forward row stage
        for (int j = tid; j < JA; j += NT) {
            const int n1 = j & 15, lr = j >> 4;
            if constexpr (PACK) {
#pragma unroll 1
                for (int k = 0; k < KP; k += 2) {
                    const int o0 = sidx<N, R2, SW>(lr, n1 + 16 * k), o1 = sidx<N, R2, SW>(lr, n1 + 16 * k + 16);
                    Cx2 P = pack2(Ps[o0], Ps[o1]), S = pack2(Ss[o0], Ss[o1]);
                    rk4_pair(P, S, kpk + 3 * (sb & 1), nhap2, nhas2, nqs2, dz62);
                    Ps[o0] = lane0(P);
                    Ps[o1] = lane1(P);
                    Ss[o0] = lane0(S);
                    Ss[o1] = lane1(S);
                }
            }
#pragma unroll 1
            for (int k = KP; k < R2; ++k) {
                const int o = sidx<N, R2, SW>(lr, n1 + 16 * k);
                V p = Ps[o], q = Ss[o];
                rk4_point<T>(p, q, coef + 6 * (sb & 1), hap, has, qs, dz6);
                Ps[o] = p;
                Ss[o] = q;
            }
#pragma unroll 1
            for (int f = 0; f < 2; ++f) row_a(f ? Ss : Ps, lr, n1, false);
        }
        __syncthreads();
        for (int s = sb; s < se; ++s) {
            const bool keep = s >= seg_from;
            pass_rb(false);
            __syncthreads();
            pass_ca(false);
            cluster_sync();
            if (s + 1 < nsteps) coefs(s + 1);
            pass_cb(false, keep ? s - seg_from : -1);
            cluster_sync();
            pass_ca(true);
            __syncthreads();
            pass_rb(true);
            __syncthreads();
            const bool last = (s + 1 == se);
            for (int j = tid; j < JA; j += NT) {
                const int n1 = j & 15, lr = j >> 4;
#pragma unroll 1
                for (int f = 0; f < 2; ++f) row_a(f ? Ss : Ps, lr, n1, true);
                if constexpr (PACK) {
                    // the loop below for points k and k + 1 at once
#pragma unroll 1
                    for (int k = 0; k < KP; k += 2) {
                        const int x = n1 + 16 * k;
                        const int o0 = sidx<N, R2, SW>(lr, x), o1 = sidx<N, R2, SW>(lr, x + 16);
                        const size_t g0 = (size_t)(crank + C * lr) * N + x, g1 = g0 + 16;
                        const V p0 = Ps[o0], q0 = Ss[o0], p1 = Ps[o1], q1 = Ss[o1];
                        if (keep) {
                            const size_t b = (size_t)(s - seg_from) * 2 * NN;
                            __stcs(&seg_a2[b + g0], p0);
                            __stcs(&seg_a2[b + g1], p1);
                            __stcs(&seg_a2[b + NN + g0], q0);
                            __stcs(&seg_a2[b + NN + g1], q1);
                        }
                        if (last && !seed) continue;
                        Cx2 P = pack2(p0, p1), S = pack2(q0, q1);
                        rk4_pair(P, S, kpk + 3 * (s & 1), nhap2, nhas2, nqs2, dz62);  // x_{s+1}
                        if (s + 1 == nsteps) {
                            const V e0 = lane0(S), e1 = lane1(S);
                            acc_j += (double)e0.x * e0.x + (double)e0.y * e0.y;
                            acc_j += (double)e1.x * e1.x + (double)e1.y * e1.y;
                            Ps[o0] = mk<T>(0, 0);
                            Ps[o1] = mk<T>(0, 0);
                            Ss[o0] = mk<T>((T)(2.0 * d.pw_s * e0.x), (T)(2.0 * d.pw_s * e0.y));
                            Ss[o1] = mk<T>((T)(2.0 * d.pw_s * e1.x), (T)(2.0 * d.pw_s * e1.y));
                            continue;
                        }
                        if (ckpt_mode && (s + 1) % K == 0) {
                            const size_t b = (size_t)((s + 1) / K) * 2 * NN;
                            __stcs(&ckpt[b + g0], lane0(P));
                            __stcs(&ckpt[b + g1], lane1(P));
                            __stcs(&ckpt[b + NN + g0], lane0(S));
                            __stcs(&ckpt[b + NN + g1], lane1(S));
                        }
                        if (s + 1 >= seg_from) {
                            const size_t b = (size_t)(s + 1 - seg_from) * 2 * NN;
                            __stcs(&seg_x[b + g0], lane0(P));
                            __stcs(&seg_x[b + g1], lane1(P));
                            __stcs(&seg_x[b + NN + g0], lane0(S));
                            __stcs(&seg_x[b + NN + g1], lane1(S));
                        }
                        rk4_pair(P, S, kpk + 3 * ((s + 1) & 1), nhap2, nhas2, nqs2, dz62);
                        Ps[o0] = lane0(P);
                        Ps[o1] = lane1(P);
                        Ss[o0] = lane0(S);
                        Ss[o1] = lane1(S);
                    }
                }
#pragma unroll 1
                for (int k = KP; k < R2; ++k) {
                    const int x = n1 + 16 * k;
                    const int o = sidx<N, R2, SW>(lr, x);
                    const size_t g = (size_t)(crank + C * lr) * N + x;
                    V p = Ps[o], q = Ss[o];
                    if (keep) {
                        __stcs(&seg_a2[((size_t)(s - seg_from) * 2) * NN + g], p);
                        __stcs(&seg_a2[((size_t)(s - seg_from) * 2 + 1) * NN + g], q);
                    }
                    if (last && !seed) continue;
                    rk4_point<T>(p, q, coef + 6 * (s & 1), hap, has, qs, dz6);  // x_{s+1}
                    if (s + 1 == nsteps) {
                        // adjoint seed: J = pw_s sum |S|^2 -> g_S = 2 pw_s S, g_P = 0
                        acc_j += (double)q.x * q.x + (double)q.y * q.y;
                        Ps[o] = mk<T>(0, 0);
                        Ss[o] = mk<T>((T)(2.0 * d.pw_s * q.x), (T)(2.0 * d.pw_s * q.y));
                        continue;
                    }
                    if (ckpt_mode && (s + 1) % K == 0) {
                        __stcs(&ckpt[((size_t)((s + 1) / K) * 2) * NN + g], p);
                        __stcs(&ckpt[((size_t)((s + 1) / K) * 2 + 1) * NN + g], q);
                    }
                    if (s + 1 >= seg_from) {
                        __stcs(&seg_x[((size_t)(s + 1 - seg_from) * 2) * NN + g], p);
                        __stcs(&seg_x[((size_t)(s + 1 - seg_from) * 2 + 1) * NN + g], q);
                    }
                    rk4_point<T>(p, q, coef + 6 * ((s + 1) & 1), hap, has, qs, dz6);
                    Ps[o] = p;
                    Ss[o] = q;
                }
                if (!last) {
#pragma unroll 1
                    for (int f = 0; f < 2; ++f) row_a(f ? Ss : Ps, lr, n1, false);
                }
            }
            __syncthreads();
        }
    };

    // ---- per-step poling sensitivity: block sum of each thread's part of Φ_s -------------
    double* wred = red;  // [NT/32]
    auto flush_phi = [&](int s, double v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) wred[tid >> 5] = v;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < NT / 32; ++w) t += wred[w];
            a.phi[(size_t)s * C + crank] = t;
        }
        __syncthreads();
    };
    // a job's working-precision partials of step s into the FP64 accumulators; returns the
    // poling term
    auto add_sens = [&](const T* sn, int s) -> double {
        acc_kp += (double)sn[0];
        acc_ks += (double)sn[1];
        acc_dk += a.zs[s] * (double)sn[4] + d.dz * (double)sn[2];
        acc_qs += (double)sn[3];
        return (double)sn[4];
    };

    // ---- adjoint march back over [sb, se) from lambda_se in shared memory ---------------
    auto backward = [&](int sb, int se) {
        prefetch_step(se - 1, sb);
        coefs(se - 1);
        __syncthreads();
        double phi_cur = 0.0;  // this thread's part of Φ_s for the step being finished
        // mu2_{se-1} = N^T(a2_{se-1}) lambda_se, then the forward row stage
        for (int j = tid; j < JA; j += NT) {
            const int n1 = j & 15, lr = j >> 4;
            T sn[5] = {0, 0, 0, 0, 0};
            if constexpr (PACK) {
                float2 sp[5] = {bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f)};
#pragma unroll 1
                for (int k = 0; k < KP; k += 2) {
                    const int x = n1 + 16 * k;
                    const int o0 = sidx<N, R2, SW>(lr, x), o1 = sidx<N, R2, SW>(lr, x + 16);
                    const size_t g0 = (size_t)(crank + C * lr) * N + x, g1 = g0 + 16;
                    const size_t sl = (size_t)(se - 1 - sb) * 2;
                    Cx2 gp = pack2(Ps[o0], Ps[o1]), gs = pack2(Ss[o0], Ss[o1]);
                    rk4_vjp_pair(pack2(__ldcs(&seg_a2[sl * NN + g0]), __ldcs(&seg_a2[sl * NN + g1])),
                                 pack2(__ldcs(&seg_a2[(sl + 1) * NN + g0]), __ldcs(&seg_a2[(sl + 1) * NN + g1])),
                                 kpk + 3 * ((se - 1) & 1), nhap2, nhas2, nqs2, n2qs2, dz62, gp, gs, sp);
                    Ps[o0] = lane0(gp);
                    Ps[o1] = lane1(gp);
                    Ss[o0] = lane0(gs);
                    Ss[o1] = lane1(gs);
                }
#pragma unroll
                for (int i = 0; i < 5; ++i) sn[i] = sp[i].x + sp[i].y;
            }
#pragma unroll 1
            for (int k = KP; k < R2; ++k) {
                const int x = n1 + 16 * k;
                const int o = sidx<N, R2, SW>(lr, x);
                const size_t g = (size_t)(crank + C * lr) * N + x;
                const size_t sl = (size_t)(se - 1 - sb) * 2;
                V gp = Ps[o], gs = Ss[o];
                rk4_vjp<T>(__ldcs(&seg_a2[sl * NN + g]), __ldcs(&seg_a2[(sl + 1) * NN + g]), coef + 6 * ((se - 1) & 1), hap, has, qs, dz6,
                           gp, gs, sn);
                Ps[o] = gp;
                Ss[o] = gs;
            }
            phi_cur += add_sens(sn, se - 1);
#pragma unroll 1
            for (int f = 0; f < 2; ++f) row_a(f ? Ss : Ps, lr, n1, false);
        }
        __syncthreads();
        for (int s = se - 1; s >= sb; --s) {
            if (s > sb) prefetch_step(s - 1, sb);
            pass_rb(false);
            __syncthreads();
            pass_ca(false);
            cluster_sync();
            if (s > sb) coefs(s - 1);
            pass_cb(true, s - sb);
            cluster_sync();
            pass_ca(true);
            __syncthreads();
            pass_rb(true);
            __syncthreads();
            double phi_prev = 0.0;  // this thread's part of Φ_{s-1} (from a2_{s-1})
            for (int j = tid; j < JA; j += NT) {
                const int n1 = j & 15, lr = j >> 4;
                T sn[5] = {0, 0, 0, 0, 0}, sn2[5] = {0, 0, 0, 0, 0};  // step s, step s-1
#pragma unroll 1
                for (int f = 0; f < 2; ++f) row_a(f ? Ss : Ps, lr, n1, true);
                if constexpr (PACK) {
                    // the loop below for points k and k + 1 at once
                    float2 sp[5] = {bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f)};
                    float2 sp2[5] = {bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f)};
#pragma unroll 1
                    for (int k = 0; k < KP; k += 2) {
                        const int x = n1 + 16 * k;
                        const int o0 = sidx<N, R2, SW>(lr, x), o1 = sidx<N, R2, SW>(lr, x + 16);
                        const size_t g0 = (size_t)(crank + C * lr) * N + x, g1 = g0 + 16;
                        Cx2 gp = pack2(Ps[o0], Ps[o1]), gs = pack2(Ss[o0], Ss[o1]);
                        const size_t sx_ = (size_t)(s - sb) * 2;
                        const Cx2 xp = pack2(__ldcs(&seg_x[sx_ * NN + g0]), __ldcs(&seg_x[sx_ * NN + g1]));
                        const Cx2 xs = pack2(__ldcs(&seg_x[(sx_ + 1) * NN + g0]), __ldcs(&seg_x[(sx_ + 1) * NN + g1]));
                        rk4_vjp_pair(xp, xs, kpk + 3 * (s & 1), nhap2, nhas2, nqs2, n2qs2, dz62, gp, gs, sp);
                        if (s > sb) {
                            const size_t sl = (size_t)(s - 1 - sb) * 2;
                            const Cx2 bp = pack2(__ldcs(&seg_a2[sl * NN + g0]), __ldcs(&seg_a2[sl * NN + g1]));
                            const Cx2 bs = pack2(__ldcs(&seg_a2[(sl + 1) * NN + g0]), __ldcs(&seg_a2[(sl + 1) * NN + g1]));
                            rk4_vjp_pair(bp, bs, kpk + 3 * ((s - 1) & 1), nhap2, nhas2, nqs2, n2qs2, dz62, gp, gs, sp2);
                        }
                        Ps[o0] = lane0(gp);
                        Ps[o1] = lane1(gp);
                        Ss[o0] = lane0(gs);
                        Ss[o1] = lane1(gs);
                    }
#pragma unroll
                    for (int i = 0; i < 5; ++i) {
                        sn[i] = sp[i].x + sp[i].y;
                        sn2[i] = sp2[i].x + sp2[i].y;
                    }
                }
#pragma unroll 1
                for (int k = KP; k < R2; ++k) {
                    const int x = n1 + 16 * k;
                    const int o = sidx<N, R2, SW>(lr, x);
                    const size_t g = (size_t)(crank + C * lr) * N + x;
                    V gp = Ps[o], gs = Ss[o];
                    // x_s and (inside the segment) a2_{s-1} from the segment buffers
                    const size_t sx_ = (size_t)(s - sb) * 2;
                    const V xp = __ldcs(&seg_x[sx_ * NN + g]), xs = __ldcs(&seg_x[(sx_ + 1) * NN + g]);
                    V bp = mk<T>(0, 0), bs = mk<T>(0, 0);
                    if (s > sb) {
                        const size_t sl = (size_t)(s - 1 - sb) * 2;
                        bp = __ldcs(&seg_a2[sl * NN + g]);
                        bs = __ldcs(&seg_a2[(sl + 1) * NN + g]);
                    }
                    rk4_vjp<T>(xp, xs, coef + 6 * (s & 1), hap, has, qs, dz6, gp, gs, sn);
                    if (s > sb) {
                        // step s-1's second application: mu2_{s-1} = N^T(a2_{s-1}) lambda_s
                        rk4_vjp<T>(bp, bs, coef + 6 * ((s - 1) & 1), hap, has, qs, dz6, gp, gs, sn2);
                    }
                    Ps[o] = gp;
                    Ss[o] = gs;
                }
                phi_cur += add_sens(sn, s);
                if (s > sb) phi_prev += add_sens(sn2, s - 1);
                if (s > sb) {
#pragma unroll 1
                    for (int f = 0; f < 2; ++f) row_a(f ? Ss : Ps, lr, n1, false);
                }
            }
            __syncthreads();
            flush_phi(s, phi_cur);
            phi_cur = phi_prev;
        }
    };

    // ============================ the computation ======================================
    // One call site each for march and backward (keeps them inlined, with the accumulators
    // in registers).
    const int last_sb = (a.M - 1) * K;
    const int sb = m * K, se = min(sb + K, nsteps);
    if (phase != kAdjBackward) {
        if (phase == kAdjForward) {
            // x_0: the pump of setPump, SH = 0
            for (int e = tid; e < Cfg::PLANE; e += NT) {
                const int lr = e / N, x = e % N;
                const double2 pv = pump_value(d, x, crank + C * lr, d.amp_re, d.amp_im, d.den_re, d.den_im);
                Ps[sidx<N, R2, SW>(lr, x)] = mk<T>((T)pv.x, (T)pv.y);
                Ss[sidx<N, R2, SW>(lr, x)] = mk<T>((T)0, (T)0);
            }
        } else {
            load_planes(ckpt + (size_t)m * 2 * NN, ckpt + ((size_t)m * 2 + 1) * NN);
        }
        __syncthreads();
        // the full march (keeping checkpoints and the last segment, ending in the adjoint
        // seed), or the re-march of segment m
        const bool fwd = phase == kAdjForward;
        march(fwd ? 0 : sb, se, fwd, fwd ? last_sb : sb, fwd);
        if (!fwd) return;
        store_planes(lam, lam + NN);
    } else if constexpr (!MARCH_ONLY) {
        load_planes(lam, lam + NN);
        __syncthreads();
        backward(sb, se);
        __syncthreads();
        if (m > 0) {
            store_planes(lam, lam + NN);
        } else {
            // dJ/dθ of the initial pump: Re <λ0_P, dP0/dθ>, dP0/dθ by central differences of
            // the closed form (waist, focus, T)
            for (int e = tid; e < Cfg::PLANE; e += NT) {
                const int lr = e / N, x = e % N, y = crank + C * lr;
                const V l0 = Ps[sidx<N, R2, SW>(lr, x)];
#pragma unroll 1
                for (int q = 0; q < 3; ++q) {
                    const double2 pp =
                        pump_value(d, x, y, a.pert[2 * q][0], a.pert[2 * q][1], a.pert[2 * q][2], a.pert[2 * q][3]);
                    const double2 pm = pump_value(d, x, y, a.pert[2 * q + 1][0], a.pert[2 * q + 1][1],
                                                  a.pert[2 * q + 1][2], a.pert[2 * q + 1][3]);
                    const double dre = (pp.x - pm.x) * a.inv2h[q], dim = (pp.y - pm.y) * a.inv2h[q];
                    const double v = (double)l0.x * dre + (double)l0.y * dim;
                    if (q == 0) acc_g0w += v;
                    else if (q == 1) acc_g0f += v;
                    else acc_g0T += v;
                }
            }
        }
    }
    // per-CTA accumulators, block-reduced in a fixed order
    const double av[kAdjAcc] = {acc_kp, acc_ks, acc_dk, acc_qs, acc_pp, acc_ps, acc_g0w, acc_g0f, acc_g0T, acc_j};
#pragma unroll
    for (int i = 0; i < kAdjAcc; ++i) {
        double v = av[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) wred[tid >> 5] = v;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < NT / 32; ++w) t += wred[w];
            const size_t slot = phase == kAdjForward ? 0 : 1 + (size_t)m;
            a.part[(slot * C + crank) * kAdjAcc + i] = t;
        }
        __syncthreads();
    }
    cluster_sync();
}

}  // namespace shg
