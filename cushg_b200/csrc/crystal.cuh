// crystal.cuh — extraordinary refractive index n(λ, T) and the grating's thermal expansion of
// the supported crystals, in FP64, for host and device code alike (λ in µm, T in °C).
//
//   SHG_CRYSTAL_MGO_SPPLT  MgO:sPPLT, Bruner et al. (src/headers/Crystal.h:54-70) with the
//                          grating expansion of src/headers/PhaseMatching.h:53,75
//   SHG_CRYSTAL_MGO_PPLN   5 mol% MgO:PPLN, the temperature-dependent Sellmeier equation of
//                          Gayer et al., Appl. Phys. B 91, 343 (2008), extraordinary index.
//                          The reference's README names this crystal but its Crystal.h carries
//                          only sPPLT.
#pragma once

#include <math.h>

#include "../../include/shg.h"

namespace shg {

// n^2 = A + (B + b)/(L^2 - (C + c)^2) + E/(L^2 - F^2) + G/(L^2 - H^2) + D L^2,
// b = 3.483933e-8 (T + 273.15)^2, c = 1.607839e-8 (T + 273.15)^2.
__host__ __device__ inline double n_spplt(double L, double T) {
    const double A = 4.502483, B = 0.007294, C = 0.185087, D = -0.02357;
    const double E = 0.073423, F = 0.199595, G = 0.001, H = 7.99724;
    const double TK = T + 273.15;
    const double b = 3.483933e-8 * (TK * TK);
    const double c = 1.607839e-8 * (TK * TK);
    const double L2 = L * L;
    return sqrt(A + (B + b) / (L2 - (C + c) * (C + c)) + E / (L2 - F * F) + G / (L2 - H * H) + D * L2);
}

// n^2 = a1 + b1 f + (a2 + b2 f)/(L^2 - (a3 + b3 f)^2) + (a4 + b4 f)/(L^2 - a5^2) - a6 L^2,
// f = (T - 24.5)(T + 570.82).
__host__ __device__ inline double n_ppln(double L, double T) {
    const double a1 = 5.756, a2 = 0.0983, a3 = 0.2020, a4 = 189.32, a5 = 12.52, a6 = 1.32e-2;
    const double b1 = 2.860e-6, b2 = 4.700e-8, b3 = 6.113e-8, b4 = 1.516e-4;
    const double f = (T - 24.5) * (T + 570.82);
    const double L2 = L * L;
    const double p = a3 + b3 * f;
    return sqrt(a1 + b1 * f + (a2 + b2 * f) / (L2 - p * p) + (a4 + b4 * f) / (L2 - a5 * a5) - a6 * L2);
}

__host__ __device__ inline double crystal_n(int crystal, double L, double T) {
    return crystal == SHG_CRYSTAL_MGO_PPLN ? n_ppln(L, T) : n_spplt(L, T);
}

// dn/dT of n_spplt, differentiated in closed form: d(n^2)/dT = b'/(L^2 - (C + c)^2)
// + 2 (B + b)(C + c) c' / (L^2 - (C + c)^2)^2 with b' = 2 * 3.483933e-8 TK, c' = 2 * 1.607839e-8 TK,
// and dn/dT = d(n^2)/dT / (2 n).
__host__ __device__ inline double dn_spplt(double L, double T) {
    const double B = 0.007294, C = 0.185087;
    const double TK = T + 273.15;
    const double b = 3.483933e-8 * (TK * TK), db = 2 * 3.483933e-8 * TK;
    const double c = 1.607839e-8 * (TK * TK), dc = 2 * 1.607839e-8 * TK;
    const double g = L * L - (C + c) * (C + c);
    const double dn2 = db / g + (B + b) * 2 * (C + c) * dc / (g * g);
    return dn2 / (2 * n_spplt(L, T));
}

// dn/dT of n_ppln: d(n^2)/df = b1 + b2/(L^2 - p^2) + 2 (a2 + b2 f) p b3/(L^2 - p^2)^2
// + b4/(L^2 - a5^2), df/dT = 2 T + 570.82 - 24.5.
__host__ __device__ inline double dn_ppln(double L, double T) {
    const double a2 = 0.0983, a3 = 0.2020, a5 = 12.52;
    const double b1 = 2.860e-6, b2 = 4.700e-8, b3 = 6.113e-8, b4 = 1.516e-4;
    const double f = (T - 24.5) * (T + 570.82), df = 2 * T + 570.82 - 24.5;
    const double L2 = L * L;
    const double p = a3 + b3 * f;
    const double g = L2 - p * p;
    const double dn2 = b1 + b2 / g + 2 * (a2 + b2 * f) * p * b3 / (g * g) + b4 / (L2 - a5 * a5);
    return dn2 * df / (2 * n_ppln(L, T));
}

__host__ __device__ inline double crystal_dn_dT(int crystal, double L, double T) {
    return crystal == SHG_CRYSTAL_MGO_PPLN ? dn_ppln(L, T) : dn_spplt(L, T);
}

// Grating period at T: Λ (1 + α (T - 25) + β (T - 25)^2).  sPPLT: α = 2.2e-6, β = -5.9e-9
// (PhaseMatching.h:53,75).  LN: α = 1.54e-5, β = 5.3e-9, the expansion of lithium niobate
// along the poling period's axis that goes with the Gayer equation.
__host__ __device__ inline void crystal_expansion(int crystal, double* a, double* b) {
    if (crystal == SHG_CRYSTAL_MGO_PPLN) {
        *a = 1.54e-5;
        *b = 5.3e-9;
    } else {
        *a = 2.2e-6;
        *b = -5.9e-9;
    }
}

// Δk = 2π (2 n(λp)/λp - n(λs)/λs + 1/Λ(T)), λs = λp / 2 (PhaseMatching.h:47-85).
__host__ __device__ inline double crystal_delta_k(int crystal, double lp, double period, double T) {
    const double ls = 0.5 * lp, pi = 3.14159265358979323846;
    double a, b;
    crystal_expansion(crystal, &a, &b);
    const double d = T - 25.;
    return 2 * pi * (2 * crystal_n(crystal, lp, T) / lp - crystal_n(crystal, ls, T) / ls + 1 / (period * (1. + a * d + b * (d * d))));
}

// dΔk/dT of crystal_delta_k in closed form: 2π (2 n'(λp)/λp - n'(λs)/λs
// - (α + 2 β d) / (Λ (1 + α d + β d^2)^2)), d = T - 25.
__host__ __device__ inline double crystal_ddk_dT(int crystal, double lp, double period, double T) {
    const double ls = 0.5 * lp, pi = 3.14159265358979323846;
    double a, b;
    crystal_expansion(crystal, &a, &b);
    const double d = T - 25.;
    const double e = 1. + a * d + b * (d * d);
    return 2 * pi * (2 * crystal_dn_dT(crystal, lp, T) / lp - crystal_dn_dT(crystal, ls, T) / ls -
                     (a + 2 * b * d) / (period * (e * e)));
}

}  // namespace shg
