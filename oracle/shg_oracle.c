/*
 * shg_oracle.c — CPU oracle for the cuSHG focused-beam SHG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path in
 * libshg_b200 is compared against, and the timed CPU baseline of bench.py.  The
 * product never links, loads or calls it.
 *
 * It restates, in plain C with OpenMP, the algorithm of alfredos84/cuSHG
 * (src/headers/Solver.h, Efields.h, PhaseMatching.h, Tfield.h, Crystal.h,
 * Operators.h).  The reference itself is CUDA-only and needs a GPU; this
 * restatement is pinned against fixtures produced by running the reference's
 * own FP64 build on a B200 (tests/golden/, made by oracle/make_golden.py).
 *
 * Build: make -C oracle   (liboracle.so next to this file)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/shg.h"

static int shgo_threads = 1;

/* Sellmeier equation of MgO:sPPLT (Bruner et al.), src/headers/Crystal.h:54-70:
 * n^2 = A + (B+b(T))/(L^2-(C+c(T))^2) + E/(L^2-F^2) + G/(L^2-H^2) + D L^2,
 * b(T) = 3.483933e-8 (T+273.15)^2, c(T) = 1.607839e-8 (T+273.15)^2, L in µm.
 * With single != 0 the coefficients, b, c, B+b and C+c are rounded to float and
 * the rest is evaluated in double, which is what the float build of the
 * reference does (its pow() calls promote to double). */
static double shgo_sellmeier_any(double L, double T, int single) {
    double A = 4.502483, B = 0.007294, C = 0.185087, D = -0.02357;
    double E = 0.073423, F = 0.199595, G = 0.001, H = 7.99724;
    const double TK = T + 273.15;
    double b = 3.483933e-8 * (TK * TK);
    double c = 1.607839e-8 * (TK * TK);
    double Bb, Cc;
    if (single) {
        A = (float)A; B = (float)B; C = (float)C; D = (float)D;
        E = (float)E; F = (float)F; G = (float)G; H = (float)H;
        b = (float)b; c = (float)c;
        Bb = (float)((float)B + (float)b);
        Cc = (float)((float)C + (float)c);
    } else {
        Bb = B + b;
        Cc = C + c;
    }
    const double L2 = L * L;
    return sqrt(A + Bb / (L2 - Cc * Cc) + E / (L2 - F * F) + G / (L2 - H * H) + D * L2);
}

/* 5 mol% MgO:PPLN, extraordinary index (Gayer et al., Appl. Phys. B 91, 343 (2008)):
 * n^2 = a1 + b1 f + (a2 + b2 f)/(L^2 - (a3 + b3 f)^2) + (a4 + b4 f)/(L^2 - a5^2) - a6 L^2,
 * f = (T - 24.5)(T + 570.82).  The reference has no code for this crystal, so both
 * precisions evaluate it in double. */
static double shgo_ppln(double L, double T) {
    const double a1 = 5.756, a2 = 0.0983, a3 = 0.2020, a4 = 189.32, a5 = 12.52, a6 = 1.32e-2;
    const double b1 = 2.860e-6, b2 = 4.700e-8, b3 = 6.113e-8, b4 = 1.516e-4;
    const double f = (T - 24.5) * (T + 570.82);
    const double L2 = L * L, p = a3 + b3 * f;
    return sqrt(a1 + b1 * f + (a2 + b2 * f) / (L2 - p * p) + (a4 + b4 * f) / (L2 - a5 * a5) - a6 * L2);
}

double shgo_sellmeier_d(double L, double T) { return shgo_sellmeier_any(L, T, 0); }
/* n(L, T) of crystal SHG_CRYSTAL_* in double */
double shgo_crystal_n(int crystal, double L, double T) {
    return crystal == SHG_CRYSTAL_MGO_PPLN ? shgo_ppln(L, T) : shgo_sellmeier_any(L, T, 0);
}
static double shgo_crystal_n_s(int crystal, double L, double T) {
    return crystal == SHG_CRYSTAL_MGO_PPLN ? shgo_ppln(L, T) : shgo_sellmeier_any(L, T, 1);
}

/* ---- double instantiation ---- */
#define R double
#define SFX(name) name##_f64
#define SELLMEIER shgo_crystal_n
#define COS cos
#define SIN sin
#define EXP exp
#define SQRT sqrt
#define TAN tan
#include "shg_oracle_impl.h"
#undef R
#undef SFX
#undef COS
#undef SIN
#undef EXP
#undef SQRT
#undef TAN
#undef SELLMEIER

/* ---- float instantiation (the reference's own precision, src/cuSHG.cu:7-8) ---- */
#define R float
#define SFX(name) name##_f32
#define SELLMEIER shgo_crystal_n_s
#define COS cosf
#define SIN sinf
#define EXP expf
#define SQRT sqrtf
#define TAN tanf
#include "shg_oracle_impl.h"
#undef R
#undef SFX
#undef COS
#undef SIN
#undef EXP
#undef SQRT
#undef TAN
#undef SELLMEIER

/* ------------------------------------------------------------------------- */
/* Exported entry points (ctypes).                                            */

void shgo_set_threads(int n) { shgo_threads = n > 0 ? n : 1; }

int shgo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Whole run, like shg_solve: precision selects the buffer element type.  poling (plain
 * runs only, may be NULL): a phase in rad added to the mismatch phase of every RK4 stage of
 * step s, one value per step. */
int shgo_solve_poling(const shg_params* p, const void* signal_in, const double* poling, void* pump_out, void* signal_out,
                      void* T_out, shg_stats* st) {
    if (!p || p->nx != p->ny || p->nx < 4 || (p->nx & 1) || p->nz < 2 || p->nx > 1024) return SHG_ERR_INVALID;
    if (p->precision == 32) {
        return p->thermal ? solve_thermal_f32(p, (const float*)signal_in, (float*)pump_out, (float*)signal_out, (float*)T_out, st)
                          : solve_plain_f32(p, (const float*)signal_in, poling, (float*)pump_out, (float*)signal_out, st);
    }
    return p->thermal ? solve_thermal_f64(p, (const double*)signal_in, (double*)pump_out, (double*)signal_out, (double*)T_out, st)
                      : solve_plain_f64(p, (const double*)signal_in, poling, (double*)pump_out, (double*)signal_out, st);
}

int shgo_solve(const shg_params* p, const void* signal_in, void* pump_out, void* signal_out, void* T_out, shg_stats* st) {
    return shgo_solve_poling(p, signal_in, NULL, pump_out, signal_out, T_out, st);
}

/* Plain march of `steps` SSFM steps from the given fields (in place), FP64.
 * Used for size-bounded checks and the bounded CPU baseline sample. */
int shgo_march_plain_f64(const shg_params* p, int steps, double* pump, double* signal) {
    cfg_f64 c;
    make_cfg_f64(p, &c);
    optics_f64 o;
    optics_init_f64(&o, &c, c.temp);
    cwes_plain_f64(&c, &o, steps, NULL, (cpx_f64*)pump, (cpx_f64*)signal);
    optics_free_f64(&o);
    return SHG_OK;
}

int shgo_march_plain_f32(const shg_params* p, int steps, float* pump, float* signal) {
    cfg_f32 c;
    make_cfg_f32(p, &c);
    optics_f32 o;
    optics_init_f32(&o, &c, c.temp);
    cwes_plain_f32(&c, &o, steps, NULL, (cpx_f32*)pump, (cpx_f32*)signal);
    optics_free_f32(&o);
    return SHG_OK;
}

/* Batch of independent plain instances, one instance per OpenMP thread
 * (the CPU baseline of the batched sweep).  steps[i] < 0 marches nz-1 steps.
 * Returns SHG_OK; sh_power[i] receives each SH power. */
int shgo_batch_plain(const shg_params* ps, int count, const int* steps, double* sh_power, int nthreads) {
    int saved = shgo_threads;
    shgo_threads = 1;
    int status = SHG_OK;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int i = 0; i < count; ++i) {
        const shg_params* p = &ps[i];
        int st = steps ? steps[i] : -1;
        if (st < 0) st = p->nz - 1;
        size_t n = (size_t)p->nx * p->ny;
        if (p->precision == 32) {
            cfg_f32 c; make_cfg_f32(p, &c);
            cpx_f32* P = (cpx_f32*)malloc(sizeof(cpx_f32) * n);
            cpx_f32* S = (cpx_f32*)calloc(n, sizeof(cpx_f32));
            optics_f32 o; optics_init_f32(&o, &c, c.temp);
            set_pump_f32(&c, c.temp, P);
            cwes_plain_f32(&c, &o, st, NULL, P, S);
            if (sh_power) sh_power[i] = power_of_f32(&c, S, NULL, sellmeier_f32(&c, c.ls, c.temp));
            optics_free_f32(&o); free(P); free(S);
        } else {
            cfg_f64 c; make_cfg_f64(p, &c);
            cpx_f64* P = (cpx_f64*)malloc(sizeof(cpx_f64) * n);
            cpx_f64* S = (cpx_f64*)calloc(n, sizeof(cpx_f64));
            optics_f64 o; optics_init_f64(&o, &c, c.temp);
            set_pump_f64(&c, c.temp, P);
            cwes_plain_f64(&c, &o, st, NULL, P, S);
            if (sh_power) sh_power[i] = power_of_f64(&c, S, NULL, sellmeier_f64(&c, c.ls, c.temp));
            optics_free_f64(&o); free(P); free(S);
        }
    }
    shgo_threads = saved;
    return status;
}

/* ---- pieces, for unit tests (FP64) ---- */

double shgo_delta_k(const shg_params* p, double T) {
    cfg_f64 c; make_cfg_f64(p, &c);
    return delta_k_f64(&c, T);
}

void shgo_set_pump(const shg_params* p, double Tc, double* pump) {
    cfg_f64 c; make_cfg_f64(p, &c);
    set_pump_f64(&c, Tc, (cpx_f64*)pump);
}

void shgo_propagators(const shg_params* p, double Tc, double* prop_p, double* prop_s) {
    cfg_f64 c; make_cfg_f64(p, &c);
    set_propagators_f64(&c, Tc, (cpx_f64*)prop_p, (cpx_f64*)prop_s);
}

/* Unnormalised 2D FFT of an n x n plane in place (inverse != 0: e^{+i}). */
void shgo_fft2(int n, double* a, int inverse) {
    fftplan_f64 pl; fft_plan_init_f64(&pl, n);
    fft2_f64(&pl, (cpx_f64*)a, n, inverse);
    fft_plan_free_f64(&pl);
}

/* One Jacobi sweep (boundary per p->boundary) from Ti into Tf. */
void shgo_jacobi_sweep(const shg_params* p, const double* Ti, double* Tf, const double* Q) {
    cfg_f64 c; make_cfg_f64(p, &c);
    if (p->boundary == SHG_BOUNDARY_OVEN_SURROUNDED) jacobi_oven_f64(&c, Ti, Tf, Q);
    else jacobi_top_open_f64(&c, Ti, Tf, Q);
}

void shgo_jacobi_sweep_f32(const shg_params* p, const float* Ti, float* Tf, const float* Q) {
    cfg_f32 c; make_cfg_f32(p, &c);
    if (p->boundary == SHG_BOUNDARY_OVEN_SURROUNDED) jacobi_oven_f32(&c, Ti, Tf, Q);
    else jacobi_top_open_f32(&c, Ti, Tf, Q);
}

/* kernelSetQ for slice s. */
void shgo_set_q(const shg_params* p, const double* T, const double* P, const double* S, int s, double* Q) {
    cfg_f64 c; make_cfg_f64(p, &c);
    set_q_f64(&c, T, (const cpx_f64*)P, (const cpx_f64*)S, s, Q);
}

double shgo_sh_power(const shg_params* p, const double* S, double temp) {
    cfg_f64 c; make_cfg_f64(p, &c);
    return power_of_f64(&c, (const cpx_f64*)S, NULL, sellmeier_f64(&c, c.ls, temp));
}
