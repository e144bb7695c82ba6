/*
 * shg_oracle_impl.h — body of the CPU oracle, compiled twice by shg_oracle.c:
 * once with R = double (suffix _f64) and once with R = float (suffix _f32).
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for libshg_b200 and the timed
 * CPU baseline.  Nothing in the product links it.
 *
 * Every function restates one piece of alfredos84/cuSHG (paths relative to the
 * reference project) in plain C.  The formulas are kept term-for-term the same
 * because parity requires the same arithmetic; the code structure is our own.
 */

#define CPX SFX(cpx)
typedef struct { R re, im; } CPX;

static inline CPX SFX(cmk)(R re, R im) { CPX c; c.re = re; c.im = im; return c; }
static inline CPX SFX(cadd)(CPX a, CPX b) { return SFX(cmk)(a.re + b.re, a.im + b.im); }
static inline CPX SFX(csub)(CPX a, CPX b) { return SFX(cmk)(a.re - b.re, a.im - b.im); }
static inline CPX SFX(cmul)(CPX a, CPX b) {
    /* Operators.h:139-145 */
    return SFX(cmk)(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline CPX SFX(cscale)(CPX a, R s) { return SFX(cmk)(a.re * s, a.im * s); }
static inline CPX SFX(conj_)(CPX a) { return SFX(cmk)(a.re, -a.im); }
static inline R SFX(abs2)(CPX a) { return a.re * a.re + a.im * a.im; } /* Operators.h:184-190 */
/* real / complex: Operators.h:159-167 */
static inline CPX SFX(rdivc)(R a, CPX b) {
    R den = b.re * b.re + b.im * b.im;
    return SFX(cmk)((a * b.re) / den, (-a * b.im) / den);
}
/* e^{i a}: Operators.h:146-151 */
static inline CPX SFX(cexpi)(R a) { return SFX(cmk)(COS(a), SIN(a)); }
/* principal square root: sqrt((|z| + re) / 2) + i sign(im) sqrt((|z| - re) / 2) */
static inline CPX SFX(csqrt)(CPX a) {
    R m = SQRT(a.re * a.re + a.im * a.im);
    R r = SQRT((m + a.re) / (R)2), i = SQRT((m - a.re) / (R)2);
    return SFX(cmk)(r, a.im < 0 ? -i : i);
}
/* e^{a.re + i a.im}: Operators.h:155-161 */
static inline CPX SFX(cexpc)(CPX a) {
    R e = EXP(a.re);
    return SFX(cmk)(e * COS(a.im), e * SIN(a.im));
}

/* ------------------------------------------------------------------------- */
/* Physical constants, Crystal.h:19-21 (µm, ps, W, V).                        */
static const R SFX(K_PI) = (R)3.14159265358979323846;
static const R SFX(K_C) = (R)(299792458 * 1E6 / 1E12);
static const R SFX(K_EPS0) = (R)(8.8541878128E-12 * 1E12 / 1E6);

typedef struct {
    int nx, ny, nz;
    R lx, ly, lz, dx, dy, dz;
    R lp, ls;
    R deff, dQ, Lambda, alpha_p, alpha_s, beta_s, rho_p, rho_s;
    R kappa, hconv;
    R power, waist, focus, temp, t_inf, t_peltier;
    R waist_y; /* <= 0 or == waist: round beam */
    int crystal; /* SHG_CRYSTAL_* */
} SFX(cfg);

/* Extraordinary index of the run's crystal (sPPLT: Crystal.h:54-70), rounded to real_t like
 * the reference's n(L, T). */
static R SFX(sellmeier)(const SFX(cfg)* c, R L, R T) {
    return (R)SELLMEIER(c->crystal, (double)L, (double)T);
}

/* Grid steps dx = LX/(NX-1) etc., Crystal.h:34-36; dQ = 2 deff/π, Crystal.h:41. */
static void SFX(make_cfg)(const shg_params* p, SFX(cfg)* c) {
    c->nx = p->nx; c->ny = p->ny; c->nz = p->nz;
    c->lx = (R)p->lx; c->ly = (R)p->ly; c->lz = (R)p->lz;
    c->dx = c->lx / (R)(c->nx - 1);
    c->dy = c->ly / (R)(c->ny - 1);
    c->dz = c->lz / (R)(c->nz - 1);
    c->lp = (R)p->lambda_p;
    c->ls = (R)0.5 * c->lp;
    c->deff = (R)p->deff;
    c->dQ = (R)2.0 * c->deff / SFX(K_PI);
    c->Lambda = (R)p->period;
    c->alpha_p = (R)p->alpha_p; c->alpha_s = (R)p->alpha_s; c->beta_s = (R)p->beta_s;
    c->rho_p = (R)p->rho_p; c->rho_s = (R)p->rho_s;
    c->kappa = (R)p->kappa; c->hconv = (R)p->h_conv;
    c->power = (R)p->power; c->waist = (R)p->waist; c->focus = (R)p->focus;
    c->waist_y = (R)p->waist_y;
    c->temp = (R)p->temp; c->t_inf = (R)p->t_inf; c->t_peltier = (R)p->t_peltier;
    c->crystal = p->crystal;
}

/* ------------------------------------------------------------------------- */
/* FFT: our own mixed-radix (4, 2, 3) decimation-in-time transform, standing  */
/* in for cufftExecC2C / Z2Z (Solver.h:159-183).  Unnormalised, forward       */
/* kernel e^{-2πi jk/n}, inverse e^{+2πi jk/n}, like cuFFT.  Twiddles are     */
/* computed in long double and rounded once.                                   */

typedef struct { int n; CPX* fw; CPX* bw; } SFX(fftplan);

static void SFX(fft_plan_init)(SFX(fftplan)* pl, int n) {
    pl->n = n;
    pl->fw = (CPX*)malloc(sizeof(CPX) * (size_t)n);
    pl->bw = (CPX*)malloc(sizeof(CPX) * (size_t)n);
    for (int t = 0; t < n; ++t) {
        long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)n;
        long double cs = cosl(a), sn = sinl(a);
        pl->fw[t] = SFX(cmk)((R)cs, (R)(-sn));
        pl->bw[t] = SFX(cmk)((R)cs, (R)sn);
    }
}
static void SFX(fft_plan_free)(SFX(fftplan)* pl) { free(pl->fw); free(pl->bw); }

/* out[k] = sum_j in[j*is] W_n^{jk}; tw = table of W_N^t, twstep = N/n. */
static void SFX(fft_rec)(int n, const CPX* in, int is, CPX* out, const CPX* tw, int N, int twstep, int inverse) {
    if (n == 1) { out[0] = in[0]; return; }
    int r = (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : n;
    int m = n / r;
    for (int q = 0; q < r; ++q)
        SFX(fft_rec)(m, in + (size_t)q * is, is * r, out + (size_t)q * m, tw, N, twstep * r, inverse);
    CPX y[64];
    for (int k = 0; k < m; ++k) {
        for (int q = 0; q < r; ++q) {
            CPX v = out[(size_t)q * m + k];
            if (q && k) v = SFX(cmul)(v, tw[((size_t)q * k * twstep) % (size_t)N]);
            y[q] = v;
        }
        if (r == 2) {
            out[k] = SFX(cadd)(y[0], y[1]);
            out[k + m] = SFX(csub)(y[0], y[1]);
        } else if (r == 4) {
            CPX a0 = SFX(cadd)(y[0], y[2]), a1 = SFX(csub)(y[0], y[2]);
            CPX b0 = SFX(cadd)(y[1], y[3]), b1 = SFX(csub)(y[1], y[3]);
            /* W_4 = -i (forward), +i (inverse) */
            CPX jb1 = inverse ? SFX(cmk)(-b1.im, b1.re) : SFX(cmk)(b1.im, -b1.re);
            out[k] = SFX(cadd)(a0, b0);
            out[k + m] = SFX(cadd)(a1, jb1);
            out[k + 2 * m] = SFX(csub)(a0, b0);
            out[k + 3 * m] = SFX(csub)(a1, jb1);
        } else {
            /* generic radix (3 or a prime leftover): direct DFT over q */
            for (int s = 0; s < r; ++s) {
                CPX acc = y[0];
                for (int q = 1; q < r; ++q) {
                    size_t e = ((size_t)q * s * (size_t)m * twstep) % (size_t)N;
                    acc = SFX(cadd)(acc, SFX(cmul)(y[q], tw[e]));
                }
                out[k + (size_t)s * m] = acc;
            }
        }
    }
}

/* In-place 1D transform of n points with element stride `stride`. */
static void SFX(fft1)(const SFX(fftplan)* pl, CPX* x, int stride, CPX* tmp_in, CPX* tmp_out, int inverse) {
    int n = pl->n;
    for (int j = 0; j < n; ++j) tmp_in[j] = x[(size_t)j * stride];
    SFX(fft_rec)(n, tmp_in, 1, tmp_out, inverse ? pl->bw : pl->fw, n, 1, inverse);
    for (int j = 0; j < n; ++j) x[(size_t)j * stride] = tmp_out[j];
}

/* 2D transform of an ny x nx row-major plane (nx == ny, as cufftPlan2d(NX,NY)). */
static void SFX(fft2)(const SFX(fftplan)* pl, CPX* a, int n, int inverse) {
#pragma omp parallel for schedule(static) if (shgo_threads > 1) num_threads(shgo_threads)
    for (int y = 0; y < n; ++y) {
        CPX ti[1024], to[1024];
        SFX(fft1)(pl, a + (size_t)y * n, 1, ti, to, inverse);
    }
#pragma omp parallel for schedule(static) if (shgo_threads > 1) num_threads(shgo_threads)
    for (int x = 0; x < n; ++x) {
        CPX ti[1024], to[1024];
        SFX(fft1)(pl, a + x, n, ti, to, inverse);
    }
}

/* ------------------------------------------------------------------------- */
/* Initial fields and propagators.                                            */

/* Focused Gaussian pump at z = 0, setPump (Efields.h:84-119): index centre
 * uX = NX/2 (not (NX-1)/2), n at the temperature of voxel (NX/2, NY/2, 0). */
static void SFX(set_pump)(const SFX(cfg)* c, R Tc, CPX* pump) {
    const R PI = SFX(K_PI);
    R np = SFX(sellmeier)(c, c->lp, Tc);
    R uX = (R)0.5 * (R)c->nx, uY = (R)0.5 * (R)c->ny;
    R wX2 = c->waist * c->waist;
    R zRX = PI * np * wX2 / c->lp;
    R Ap0 = SQRT((R)4 * c->power / (SFX(K_EPS0) * SFX(K_C) * PI * np * wX2));
    R etaX = c->focus / zRX;
    CPX MX = SFX(cmk)((R)1, -etaX);
    CPX amp = SFX(rdivc)(Ap0, MX);
    CPX den = SFX(cscale)(MX, wX2);
    if (c->waist_y > 0 && c->waist_y != c->waist) {
        /* the elliptical variant (Efields.h:113-115, commented out in the reference):
         * (A / (sqrt(MX) sqrt(MY))) exp(-ax^2 / (wX2 MX) - ay^2 / (wY2 MY)), A normalised with
         * waist * waist_y so that the beam carries the pump power */
        R wY2 = c->waist_y * c->waist_y;
        R etaY = c->focus / (PI * np * wY2 / c->lp);
        R A = SQRT((R)4 * c->power / (SFX(K_EPS0) * SFX(K_C) * PI * np * c->waist * c->waist_y));
        CPX MY = SFX(cmk)((R)1, -etaY);
        CPX ampe = SFX(rdivc)(A, SFX(cmul)(SFX(csqrt)(MX), SFX(csqrt)(MY)));
        CPX deny = SFX(cscale)(MY, wY2);
        for (int y = 0; y < c->ny; ++y)
            for (int x = 0; x < c->nx; ++x) {
                R ax = ((R)x - uX) * c->dx, ay = ((R)y - uY) * c->dy;
                CPX arg = SFX(cadd)(SFX(rdivc)(-(ax * ax), den), SFX(rdivc)(-(ay * ay), deny));
                pump[(size_t)y * c->nx + x] = SFX(cmul)(ampe, SFX(cexpc)(arg));
            }
        return;
    }
    for (int y = 0; y < c->ny; ++y)
        for (int x = 0; x < c->nx; ++x) {
            R ax = ((R)x - uX) * c->dx, ay = ((R)y - uY) * c->dy;
            R num = -(ax * ax) - (ay * ay);
            CPX arg = SFX(rdivc)(num, den);
            pump[(size_t)y * c->nx + x] = SFX(cmul)(amp, SFX(cexpc)(arg));
        }
}

/* Diffraction propagators beamPropagator (Efields.h:122-141) followed by the
 * 2D fftshift of fftShift2D (Efields.h:32-81; for even N the V-then-H half
 * swaps equal out[y][x] = in[(y+N/2)%N][(x+N/2)%N]). */
static void SFX(set_propagators)(const SFX(cfg)* c, R Tc, CPX* prop_p, CPX* prop_s) {
    const R PI = SFX(K_PI);
    int nx = c->nx, ny = c->ny;
    R kp = (R)2 * PI * SFX(sellmeier)(c, c->lp, Tc) / c->lp;
    R ks = (R)2 * PI * SFX(sellmeier)(c, c->ls, Tc) / c->ls;
    R dfX = (R)1 / c->dx / (R)nx, dfY = (R)1 / c->dy / (R)ny;
    R uX = (R)0.5 * (R)nx, uY = (R)0.5 * (R)ny;
    R tp = TAN(c->rho_p), ts = TAN(c->rho_s);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            /* unshifted centred value at (xc, yc) lands at the shifted slot (x, y) */
            int xc = (x + nx / 2) % nx, yc = (y + ny / 2) % ny;
            R fx = (R)xc - uX, fy = (R)yc - uY;
            R rad = dfX * dfX * (fx * fx) + dfY * dfY * (fy * fy);
            R thp = -c->dz * ((R)2 * (PI * PI) / kp * rad + (R)2 * PI * dfX * tp * fx);
            R ths = -c->dz * ((R)2 * (PI * PI) / ks * rad + (R)2 * PI * dfX * ts * fx);
            prop_p[(size_t)y * nx + x] = SFX(cexpi)(thp);
            prop_s[(size_t)y * nx + x] = SFX(cexpi)(ths);
        }
}

/* Phase mismatch at one temperature, kernelSetInicialDKConstant /
 * kernelSetInicialDKThermal (PhaseMatching.h:47-85), with the grating's
 * thermal expansion: sPPLT α = 2.2e-6, β = -5.9e-9 (PhaseMatching.h:53,75);
 * MgO:PPLN α = 1.54e-5, β = 5.3e-9 (lithium niobate). */
static R SFX(delta_k)(const SFX(cfg)* c, R T) {
    const R PI = SFX(K_PI);
    const int ln = c->crystal == SHG_CRYSTAL_MGO_PPLN;
    const R a = ln ? (R)1.54e-5 : (R)2.2e-6, b = ln ? (R)5.3e-9 : (R)-5.9e-9;
    R d = T - (R)25.;
    return (R)2 * PI * ((R)2 * SFX(sellmeier)(c, c->lp, T) / c->lp - SFX(sellmeier)(c, c->ls, T) / c->ls +
                        (R)1 / (c->Lambda * ((R)1. + a * d + b * (d * d))));
}

/* ------------------------------------------------------------------------- */
/* Nonlinear step: the reference's RK4 scheme (Solver.h:189-264) with dAdz    */
/* (Solver.h:33-80).  Stages: k1 = f(A, 0); k2 = f(A + 0.5 k1, dz/4);          */
/* k3 = f(A + 0.5 k2, dz/4); k4 = f(A + k3, dz/2); A += dz/6 (k1+2k2+2k3+k4). */
/* The stage increments carry no dz factor, as in linealCombination calls     */
/* (Solver.h:239-250).                                                         */

typedef struct {
    /* per-point optical constants */
    R kap_p, kap_s;   /* π dQ/(n_p λp), 0.5 π dQ/(n_s λs) */
    R ab_s;           /* beta_s * 0.5 * c * eps0 * n_s */
} SFX(pointc);

static inline SFX(pointc) SFX(point_consts)(const SFX(cfg)* c, R np, R ns, int thermal) {
    SFX(pointc) k;
    const R PI = SFX(K_PI);
    k.kap_p = (R)1 * PI * c->dQ / (np * c->lp);
    k.kap_s = (R)0.5 * PI * c->dQ / (ns * c->ls);
    /* the plain dAdz multiplies C*EPS0 (Solver.h:74), the thermal one EPS0*C (Solver.h:50) */
    k.ab_s = thermal ? c->beta_s * (R)0.5 * SFX(K_EPS0) * SFX(K_C) * ns
                     : c->beta_s * (R)0.5 * SFX(K_C) * SFX(K_EPS0) * ns;
    return k;
}

/* dA/dz at one point for a mismatch phase phi (dP uses e^{-i phi}, dS e^{+i phi}). */
static inline void SFX(dadz)(const SFX(cfg)* c, const SFX(pointc)* k, R phi, CPX P, CPX S, CPX* dP, CPX* dS) {
    CPX em = SFX(cexpi)(-phi), ep = SFX(cexpi)(phi);
    CPX t = SFX(cmul)(SFX(cmul)(SFX(cmk)((R)0, k->kap_p), S), SFX(conj_)(P));
    t = SFX(cmul)(t, em);
    *dP = SFX(csub)(t, SFX(cscale)(P, (R)0.5 * c->alpha_p));
    CPX u = SFX(cmul)(SFX(cmul)(SFX(cmk)((R)0, k->kap_s), P), P);
    u = SFX(cmul)(u, ep);
    R g = (R)0.5 * (c->alpha_s + k->ab_s * SFX(abs2)(S));
    *dS = SFX(csub)(u, SFX(cscale)(S, g));
}

/* One RK4 application at one point.  phi0/phi1/phi2: mismatch phases of the
 * stages with z-offset 0, dz/4 and dz/2. */
static inline void SFX(rk4_point)(const SFX(cfg)* c, const SFX(pointc)* k, R phi0, R phi1, R phi2, CPX* P, CPX* S) {
    CPX k1p, k1s, k2p, k2s, k3p, k3s, k4p, k4s;
    CPX p = *P, s = *S;
    SFX(dadz)(c, k, phi0, p, s, &k1p, &k1s);
    SFX(dadz)(c, k, phi1, SFX(cadd)(p, SFX(cscale)(k1p, (R)0.5)), SFX(cadd)(s, SFX(cscale)(k1s, (R)0.5)), &k2p, &k2s);
    SFX(dadz)(c, k, phi1, SFX(cadd)(p, SFX(cscale)(k2p, (R)0.5)), SFX(cadd)(s, SFX(cscale)(k2s, (R)0.5)), &k3p, &k3s);
    SFX(dadz)(c, k, phi2, SFX(cadd)(p, SFX(cscale)(k3p, (R)1.0)), SFX(cadd)(s, SFX(cscale)(k3s, (R)1.0)), &k4p, &k4s);
    /* kernelRK4, Solver.h:83-97: A + (k1 + 2k2 + 2k3 + k4) * dz / 6 */
    CPX sp = SFX(cadd)(SFX(cadd)(SFX(cadd)(k1p, SFX(cscale)(k2p, (R)2)), SFX(cscale)(k3p, (R)2)), k4p);
    CPX ss = SFX(cadd)(SFX(cadd)(SFX(cadd)(k1s, SFX(cscale)(k2s, (R)2)), SFX(cscale)(k3s, (R)2)), k4s);
    sp = SFX(cscale)(sp, c->dz);
    ss = SFX(cscale)(ss, c->dz);
    *P = SFX(cadd)(p, SFX(cmk)(sp.re / (R)6, sp.im / (R)6));
    *S = SFX(cadd)(s, SFX(cmk)(ss.re / (R)6, ss.im / (R)6));
}

/* solverRK4 of a plain run (uniform T, Δk; Solver.h:231-259): the stage phase
 * is (z + dz*inc) * Δk with inc in {0, 0.25, 0.5}, plus the step's poling phase (a
 * per-slice phase of the QPM grating; zero in the reference, which has a uniform grating). */
static void SFX(rk4_plain)(const SFX(cfg)* c, const SFX(pointc)* k, R dk, R z, R poling, CPX* P, CPX* S) {
    int n = c->nx * c->ny;
    R phi0 = (z + c->dz * (R)0.0) * dk + poling;
    R phi1 = (z + c->dz * (R)0.25) * dk + poling;
    R phi2 = (z + c->dz * (R)0.5) * dk + poling;
#pragma omp parallel for schedule(static) if (shgo_threads > 1) num_threads(shgo_threads)
    for (int i = 0; i < n; ++i) SFX(rk4_point)(c, k, phi0, phi1, phi2, &P[i], &S[i]);
}

/* solverRK4 of a thermal run (Solver.h:198-229): per-voxel n(λ, T(x,y,s)) and
 * phase DKint * (dz*inc + s*dz)/(s+1), DKint = sum_{z<=s} Δk (PhaseMatching.h:27-44). */
static void SFX(rk4_thermal)(const SFX(cfg)* c, const R* T, const R* dkint, int s, CPX* P, CPX* S) {
    int n = c->nx * c->ny;
    R sr = (R)s;
    R a0 = c->dz * (R)0.0 + sr * c->dz;
    R a1 = c->dz * (R)0.25 + sr * c->dz;
    R a2 = c->dz * (R)0.5 + sr * c->dz;
    R b = sr + (R)1.0;
    const R* Ts = T + (size_t)s * n;
#pragma omp parallel for schedule(static) if (shgo_threads > 1) num_threads(shgo_threads)
    for (int i = 0; i < n; ++i) {
        SFX(pointc) k = SFX(point_consts)(c, SFX(sellmeier)(c, c->lp, Ts[i]), SFX(sellmeier)(c, c->ls, Ts[i]), 1);
        SFX(rk4_point)(c, &k, dkint[i] * a0 / b, dkint[i] * a1 / b, dkint[i] * a2 / b, &P[i], &S[i]);
    }
}

/* diffraction (Solver.h:153-186): A <- IFFT2(prop * FFT2(A)) / (NX*NY). */
static void SFX(diffraction)(const SFX(cfg)* c, const SFX(fftplan)* pl, const CPX* prop, CPX* A) {
    int n = c->nx * c->ny;
    R size = (R)(c->nx * c->ny);
    SFX(fft2)(pl, A, c->nx, 0);
    for (int i = 0; i < n; ++i) A[i] = SFX(cmul)(prop[i], A[i]);
    SFX(fft2)(pl, A, c->nx, 1);
    for (int i = 0; i < n; ++i) A[i] = SFX(cmk)(A[i].re / size, A[i].im / size);
}

/* SH / pump power: sum 0.5 eps0 c n |A|^2 dx dy, summed in double. */
static double SFX(power_of)(const SFX(cfg)* c, const CPX* A, const R* nmap, R nconst) {
    int n = c->nx * c->ny;
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
        double nn = nmap ? (double)nmap[i] : (double)nconst;
        acc += 0.5 * (double)SFX(K_EPS0) * (double)SFX(K_C) * nn * ((double)A[i].re * A[i].re + (double)A[i].im * A[i].im);
    }
    return acc * (double)c->dx * (double)c->dy;
}

/* ------------------------------------------------------------------------- */
/* Heat equation (Tfield.h).                                                   */

#define TIDX(x, y, z) (((size_t)(z) * (size_t)(ny) + (size_t)(y)) * (size_t)(nx) + (size_t)(x))

/* One Jacobi sweep of kernelHeatEquationTopOpen (Tfield.h:93-201): writes Tf
 * at every voxel except the y = 0 face, which stays at the oven temperature. */
static void SFX(jacobi_top_open)(const SFX(cfg)* c, const R* Ti, R* Tf, const R* Q) {
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const R dx = c->dx, dy = c->dy, dz = c->dz, K = c->kappa, Tinf = c->t_inf;
    const R Bix = c->hconv * dx / K, Biy = c->hconv * dy / K, Biz = c->hconv * dz / K;
    const R ax = dx * dx / ((R)2 * dy * dy), ay = dy * dy / ((R)2 * dx * dx), az = dz * dz / ((R)2 * dx * dx);
    const R bx = dx * dx / ((R)2 * dz * dz), by = dy * dy / ((R)2 * dz * dz), bz = dz * dz / ((R)2 * dy * dy);
    const R av = dz / ((R)2 * dx), bv = dx / ((R)2 * dz), cv = dx * dz / ((R)4 * dy * dy);
    const R V = (R)1 / (av + bv + (R)2 * cv + (R)0.5 * (Bix + Biz));
    const R ah = dz / ((R)2 * dy), bh = dy / ((R)2 * dz), ch = dy * dz / ((R)4 * dx * dx);
    const R H = (R)1 / (ah + bh + (R)2 * ch + (R)0.5 * (Biy + Biz));
    const R ad = dx / ((R)2 * dy), bd = dy / ((R)2 * dx), cd = dx * dy / ((R)4 * dz * dz);
    const R D = (R)1 / (ad + bd + (R)2 * cd + (R)0.5 * (Bix + Biy));
    const R AV = dy * dz / dx, BV = dx * dz / dy, CV = dx * dy / dz, BiD = Bix * dy + Biy * dz + Biz * dx;
    const R GV = (R)1 / (AV + BV + CV + BiD);
    const R L2 = (R)1 / ((R)2 / (dx * dx) + (R)2 / (dy * dy) + (R)2 / (dz * dz));
#pragma omp parallel for schedule(static) if (shgo_threads > 1) num_threads(shgo_threads)
    for (int z = 0; z < nz; ++z) {
        const int zi = (z > 0 && z < nz - 1);
        for (int y = 1; y < ny; ++y) {
            const int yi = (y < ny - 1);
            for (int x = 0; x < nx; ++x) {
                const int xi = (x > 0 && x < nx - 1);
                R v;
                if (xi && yi && zi) {            /* inner points */
                    v = L2 * ((Ti[TIDX(x + 1, y, z)] + Ti[TIDX(x - 1, y, z)]) / (dx * dx) +
                              (Ti[TIDX(x, y + 1, z)] + Ti[TIDX(x, y - 1, z)]) / (dy * dy) +
                              (Ti[TIDX(x, y, z + 1)] + Ti[TIDX(x, y, z - 1)]) / (dz * dz) + Q[TIDX(x, y, z)] / K);
                } else if (!xi && yi && zi) {    /* faces x = 0 / x = Lx */
                    int xn = (x == 0) ? 1 : x - 1;
                    v = (Ti[TIDX(xn, y, z)] + ax * (Ti[TIDX(x, y + 1, z)] + Ti[TIDX(x, y - 1, z)]) +
                         bx * (Ti[TIDX(x, y, z + 1)] + Ti[TIDX(x, y, z - 1)]) + Bix * Tinf) /
                        ((R)1 + (R)2 * ax + (R)2 * bx + Bix);
                } else if (xi && !yi && zi) {    /* face y = Ly */
                    v = (Ti[TIDX(x, y - 1, z)] + ay * (Ti[TIDX(x + 1, y, z)] + Ti[TIDX(x - 1, y, z)]) +
                         by * (Ti[TIDX(x, y, z + 1)] + Ti[TIDX(x, y, z - 1)]) + Biy * Tinf) /
                        ((R)1 + (R)2 * ay + (R)2 * by + Biy);
                } else if (xi && yi && !zi) {    /* faces z = 0 / z = Lcr */
                    int zn = (z == 0) ? 1 : z - 1;
                    v = (Ti[TIDX(x, y, zn)] + az * (Ti[TIDX(x + 1, y, z)] + Ti[TIDX(x - 1, y, z)]) +
                         bz * (Ti[TIDX(x, y + 1, z)] + Ti[TIDX(x, y - 1, z)]) + Biz * Tinf) /
                        ((R)1 + (R)2 * az + (R)2 * bz + Biz);
                } else if (!xi && yi && !zi) {   /* vertical edges (x, z on the boundary) */
                    int xn = (x == 0) ? 1 : x - 1, zn = (z == 0) ? 1 : z - 1;
                    v = (av * Ti[TIDX(xn, y, z)] + bv * Ti[TIDX(x, y, zn)] +
                         cv * (Ti[TIDX(x, y + 1, z)] + Ti[TIDX(x, y - 1, z)]) + (R)0.5 * Tinf * (Bix + Biz)) * V;
                } else if (xi && !yi && !zi) {   /* horizontal edges (y = Ly, z on the boundary) */
                    int zn = (z == 0) ? 1 : z - 1;
                    v = (ah * Ti[TIDX(x, y - 1, z)] + bh * Ti[TIDX(x, y, zn)] +
                         ch * (Ti[TIDX(x - 1, y, z)] + Ti[TIDX(x + 1, y, z)]) + (R)0.5 * Tinf * (Biy + Biz)) * H;
                } else if (!xi && !yi && zi) {   /* depth edges (x on the boundary, y = Ly) */
                    int xn = (x == 0) ? 1 : x - 1;
                    v = (ad * Ti[TIDX(x, y - 1, z)] + bd * Ti[TIDX(xn, y, z)] +
                         cd * (Ti[TIDX(x, y, z + 1)] + Ti[TIDX(x, y, z - 1)]) + (R)0.5 * Tinf * (Bix + Biy)) * D;
                } else {                         /* vertices (x, z on the boundary, y = Ly) */
                    int xn = (x == 0) ? 1 : x - 1, zn = (z == 0) ? 1 : z - 1;
                    v = (AV * Ti[TIDX(xn, y, z)] + BV * Ti[TIDX(x, y - 1, z)] + CV * Ti[TIDX(x, y, zn)] + Tinf * BiD) * GV;
                }
                Tf[TIDX(x, y, z)] = v;
            }
        }
    }
}

/* One Jacobi sweep of kernelHeatEquationOvenSurrounded (Tfield.h:205-240):
 * inner points plus Robin z faces; every other voxel keeps its value. */
static void SFX(jacobi_oven)(const SFX(cfg)* c, const R* Ti, R* Tf, const R* Q) {
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const R dx = c->dx, dy = c->dy, dz = c->dz, K = c->kappa, Tinf = c->t_inf;
    const R Biz = c->hconv * dz / K;
    const R az = dz * dz / ((R)2 * dx * dx), bz = dz * dz / ((R)2 * dy * dy);
    const R L2 = (R)1 / ((R)2 / (dx * dx) + (R)2 / (dy * dy) + (R)2 / (dz * dz));
#pragma omp parallel for schedule(static) if (shgo_threads > 1) num_threads(shgo_threads)
    for (int z = 0; z < nz; ++z)
        for (int y = 1; y < ny - 1; ++y)
            for (int x = 1; x < nx - 1; ++x) {
                if (z > 0 && z < nz - 1) {
                    Tf[TIDX(x, y, z)] = L2 * ((Ti[TIDX(x + 1, y, z)] + Ti[TIDX(x - 1, y, z)]) / (dx * dx) +
                                              (Ti[TIDX(x, y + 1, z)] + Ti[TIDX(x, y - 1, z)]) / (dy * dy) +
                                              (Ti[TIDX(x, y, z + 1)] + Ti[TIDX(x, y, z - 1)]) / (dz * dz) + Q[TIDX(x, y, z)] / K);
                } else {
                    int zn = (z == 0) ? 1 : z - 1;
                    Tf[TIDX(x, y, z)] = (Ti[TIDX(x, y, zn)] + az * (Ti[TIDX(x + 1, y, z)] + Ti[TIDX(x - 1, y, z)]) +
                                         bz * (Ti[TIDX(x, y + 1, z)] + Ti[TIDX(x, y - 1, z)]) + Biz * Tinf) /
                                        ((R)1 + (R)2 * az + (R)2 * bz + Biz);
                }
            }
}

/* Convergence value of checkConvergence (Tfield.h:13-25, 366-376):
 * sqrt(sum (Tf-Ti)^2)/TSIZE (rule 0) or max |Tf-Ti| (rule 1). */
static double SFX(conv_value)(const SFX(cfg)* c, const R* Tf, const R* Ti, int rule) {
    size_t n = (size_t)c->nx * c->ny * c->nz;
    double acc = 0.0;
    if (rule == SHG_CONV_MAXABS) {
        for (size_t i = 0; i < n; ++i) { double d = fabs((double)Tf[i] - (double)Ti[i]); if (d > acc) acc = d; }
        return acc;
    }
    for (size_t i = 0; i < n; ++i) { R d = (R)(Tf[i] - Ti[i]); R d2 = d * d; acc += (double)d2; }
    return (double)(R)(sqrt(acc) / (double)n);
}

/* kernelSetQ (Tfield.h:260-276): Q(x,y,s) = αp Ip + αs Is + βs Is^2. */
static void SFX(set_q)(const SFX(cfg)* c, const R* T, const CPX* P, const CPX* S, int s, R* Q) {
    const int n = c->nx * c->ny;
    const R* Ts = T + (size_t)s * n;
    R* Qs = Q + (size_t)s * n;
    const R C0 = SFX(K_C), E0 = SFX(K_EPS0);
    for (int i = 0; i < n; ++i) {
        R np = SFX(sellmeier)(c, c->lp, Ts[i]), ns = SFX(sellmeier)(c, c->ls, Ts[i]);
        R Is = (R)0.5 * C0 * E0 * ns * SFX(abs2)(S[i]);
        Qs[i] = c->alpha_p * (R)0.5 * C0 * E0 * np * SFX(abs2)(P[i]) + c->alpha_s * (R)0.5 * C0 * E0 * ns * SFX(abs2)(S[i]) +
                c->beta_s * (Is * Is);
    }
}

/* ------------------------------------------------------------------------- */
/* Optical pass: CWES (Solver.h:276-308).  Marches `steps` SSFM steps          */
/* RK4 - diffraction - RK4 (Solver.h:267-273); `record` receives the fields    */
/* before step nz-1, as Solver.h:283-286 saves them.                           */

typedef struct {
    const SFX(cfg)* c;
    SFX(fftplan) pl;
    CPX *prop_p, *prop_s;
} SFX(optics);

static void SFX(optics_init)(SFX(optics)* o, const SFX(cfg)* c, R Tc) {
    size_t n = (size_t)c->nx * c->ny;
    o->c = c;
    SFX(fft_plan_init)(&o->pl, c->nx);
    o->prop_p = (CPX*)malloc(sizeof(CPX) * n);
    o->prop_s = (CPX*)malloc(sizeof(CPX) * n);
    SFX(set_propagators)(c, Tc, o->prop_p, o->prop_s);
}
static void SFX(optics_free)(SFX(optics)* o) { SFX(fft_plan_free)(&o->pl); free(o->prop_p); free(o->prop_s); }

/* One SSFM step of a plain run at position z. */
static void SFX(ssfm_plain)(const SFX(optics)* o, const SFX(pointc)* k, R dk, R z, R poling, CPX* P, CPX* S) {
    SFX(rk4_plain)(o->c, k, dk, z, poling, P, S);
    SFX(diffraction)(o->c, &o->pl, o->prop_p, P);
    SFX(diffraction)(o->c, &o->pl, o->prop_s, S);
    SFX(rk4_plain)(o->c, k, dk, z, poling, P, S);
}

/* Plain CWES: nsteps steps from z = 0, z accumulated as z += dz (Solver.h:303). */
static void SFX(cwes_plain)(const SFX(cfg)* c, const SFX(optics)* o, int nsteps, const double* poling, CPX* P, CPX* S) {
    SFX(pointc) k = SFX(point_consts)(c, SFX(sellmeier)(c, c->lp, c->temp), SFX(sellmeier)(c, c->ls, c->temp), 0);
    R dk = SFX(delta_k)(c, c->temp);
    R z = (R)0.0;
    for (int s = 0; s < nsteps; ++s) {
        SFX(ssfm_plain)(o, &k, dk, z, poling ? (R)poling[s] : (R)0, P, S);
        z += c->dz;
    }
}

/* ------------------------------------------------------------------------- */
/* Public entry points of this precision.                                      */

static void SFX(init_signal)(CPX* S, const R* signal_in, size_t n) {
    for (size_t i = 0; i < n; ++i)
        S[i] = signal_in ? SFX(cmk)(signal_in[2 * i], signal_in[2 * i + 1]) : SFX(cmk)((R)0, (R)0);
}

/* Plain run, Solver.h:376-383. */
static int SFX(solve_plain)(const shg_params* p, const R* signal_in, const double* poling, R* pump_out, R* signal_out,
                            shg_stats* st) {
    SFX(cfg) c;
    SFX(make_cfg)(p, &c);
    size_t n = (size_t)c.nx * c.ny;
    CPX* P = (CPX*)malloc(sizeof(CPX) * n);
    CPX* S = (CPX*)malloc(sizeof(CPX) * n);
    if (!P || !S) { free(P); free(S); return SHG_ERR_NOMEM; }
    SFX(optics) o;
    SFX(optics_init)(&o, &c, c.temp);
    SFX(set_pump)(&c, c.temp, P);
    SFX(init_signal)(S, signal_in, n);
    int steps = c.nz - 1;
    SFX(cwes_plain)(&c, &o, steps, poling, P, S);
    if (pump_out) memcpy(pump_out, P, sizeof(CPX) * n);
    if (signal_out) memcpy(signal_out, S, sizeof(CPX) * n);
    if (st) {
        memset(st, 0, sizeof(*st));
        st->sh_power = SFX(power_of)(&c, S, NULL, SFX(sellmeier)(&c, c.ls, c.temp));
        st->pump_power = SFX(power_of)(&c, P, NULL, SFX(sellmeier)(&c, c.lp, c.temp));
        st->steps = steps;
        st->outer_iterations = 1;
    }
    SFX(optics_free)(&o);
    free(P); free(S);
    return SHG_OK;
}

/* Thermal run, Solver.h:319-373. */
static int SFX(solve_thermal)(const shg_params* p, const R* signal_in, R* pump_out, R* signal_out, R* T_out, shg_stats* st) {
    SFX(cfg) c;
    SFX(make_cfg)(p, &c);
    const int nx = c.nx, ny = c.ny, nz = c.nz;
    size_t n = (size_t)nx * ny, nt = n * (size_t)nz;
    R* Ti = (R*)malloc(sizeof(R) * nt);
    R* Tf = (R*)malloc(sizeof(R) * nt);
    R* Q = (R*)calloc(nt, sizeof(R));
    R* DK = (R*)malloc(sizeof(R) * nt);
    R* dkint = (R*)malloc(sizeof(R) * n);
    CPX* P = (CPX*)malloc(sizeof(CPX) * n);
    CPX* S = (CPX*)malloc(sizeof(CPX) * n);
    CPX* Pout = (CPX*)malloc(sizeof(CPX) * n);
    CPX* Sout = (CPX*)malloc(sizeof(CPX) * n);
    if (!Ti || !Tf || !Q || !DK || !dkint || !P || !S || !Pout || !Sout) {
        free(Ti); free(Tf); free(Q); free(DK); free(dkint); free(P); free(S); free(Pout); free(Sout);
        return SHG_ERR_NOMEM;
    }
    /* setTemperature (Tfield.h:300-314) then the boundary temperatures */
    for (size_t i = 0; i < nt; ++i) Ti[i] = Tf[i] = c.temp;
    if (p->boundary == SHG_BOUNDARY_OVEN_SURROUNDED) {
        /* kernelSetOvenSurrounded (Tfield.h:64-90) */
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x)
                    if (y == 0 || y == ny - 1 || x == 0 || x == nx - 1) Ti[TIDX(x, y, z)] = Tf[TIDX(x, y, z)] = c.t_peltier;
    } else {
        /* kernelSetBottomOvensTemperature (Tfield.h:46-61) */
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x) Ti[TIDX(x, 0, z)] = Tf[TIDX(x, 0, z)] = c.t_peltier;
    }
    double tol = p->jacobi_tol > 0 ? p->jacobi_tol : (double)(R)(5e-4 / (double)nt);
    int check_every = p->check_every > 0 ? p->check_every : 5000;
    int64_t max_sweeps = p->max_sweeps > 0 ? p->max_sweeps : ((int64_t)1 << 40);
    int max_outer = p->max_outer > 0 ? p->max_outer : 20;
    int64_t total_sweeps = 0;
    int outer = 0, status = SHG_OK;
    double last = 0.0;
    SFX(fftplan) pl;
    SFX(fft_plan_init)(&pl, nx);
    CPX* prop_p = (CPX*)malloc(sizeof(CPX) * n);
    CPX* prop_s = (CPX*)malloc(sizeof(CPX) * n);
    R* nsmap = (R*)malloc(sizeof(R) * n);
    R* npmap = (R*)malloc(sizeof(R) * n);
    for (int g = 0; g < max_outer; ++g) {
        /* Jacobi loop, Solver.h:335-355 */
        double red = 1.0, aux = -1.0;
        int64_t counter = 0;
        if (p->conv_rule == SHG_CONV_FIXED) {
            /* the library's fixed rule (no counterpart in the reference): exactly max_sweeps
               sweeps per outer iteration and exactly max_outer outer iterations */
            for (; counter < p->max_sweeps; ++counter) {
                if (p->boundary == SHG_BOUNDARY_OVEN_SURROUNDED) SFX(jacobi_oven)(&c, Ti, Tf, Q);
                else SFX(jacobi_top_open)(&c, Ti, Tf, Q);
                memcpy(Ti, Tf, sizeof(R) * nt);
            }
            red = 0.0;
        }
        while (red >= tol) {
            if (counter >= max_sweeps) { status = SHG_ERR_NOT_CONVERGED; break; }
            if (p->boundary == SHG_BOUNDARY_OVEN_SURROUNDED) SFX(jacobi_oven)(&c, Ti, Tf, Q);
            else SFX(jacobi_top_open)(&c, Ti, Tf, Q);
            if (counter % check_every == 0) {
                if (counter > 0) aux = red;
                red = SFX(conv_value)(&c, Tf, Ti, p->conv_rule);
                if (red == aux) red = 0.5 * tol;
            }
            memcpy(Ti, Tf, sizeof(R) * nt);
            ++counter;
        }
        last = red;
        total_sweeps += counter;
        if (status != SHG_OK) break;
        /* setDKFromTemperature, setInputPump, setNoisyField, setPropagators (Solver.h:359-362) */
        for (size_t i = 0; i < nt; ++i) DK[i] = SFX(delta_k)(&c, Tf[i]);
        R Tc = Tf[TIDX(nx / 2, ny / 2, 0)];
        SFX(set_pump)(&c, Tc, P);
        SFX(init_signal)(S, signal_in, n);
        SFX(set_propagators)(&c, Tc, prop_p, prop_s);
        /* CWES with Q updates (Solver.h:276-308, 300) */
        for (size_t i = 0; i < n; ++i) dkint[i] = (R)0.0;
        for (int s = 0; s < nz; ++s) {
            if (s == nz - 1) { memcpy(Pout, P, sizeof(CPX) * n); memcpy(Sout, S, sizeof(CPX) * n); }
            /* running prefix: the same additions in the same order as kernelIntegrateDK */
            for (size_t i = 0; i < n; ++i) dkint[i] += DK[(size_t)s * n + i];
            SFX(rk4_thermal)(&c, Tf, dkint, s, P, S);
            SFX(diffraction)(&c, &pl, prop_p, P);
            SFX(diffraction)(&c, &pl, prop_s, S);
            SFX(rk4_thermal)(&c, Tf, dkint, s, P, S);
            SFX(set_q)(&c, Tf, P, S, s, Q);
        }
        ++outer;
        if (p->conv_rule != SHG_CONV_FIXED && counter == 1 && g != 0) break; /* Solver.h:367 */
    }
    if (pump_out) memcpy(pump_out, Pout, sizeof(CPX) * n);
    if (signal_out) memcpy(signal_out, Sout, sizeof(CPX) * n);
    if (T_out) memcpy(T_out, Tf, sizeof(R) * nt);
    if (st) {
        memset(st, 0, sizeof(*st));
        const R* Tl = Tf + (size_t)(nz - 1) * n;
        for (size_t i = 0; i < n; ++i) { nsmap[i] = SFX(sellmeier)(&c, c.ls, Tl[i]); npmap[i] = SFX(sellmeier)(&c, c.lp, Tl[i]); }
        st->sh_power = SFX(power_of)(&c, Sout, nsmap, 0);
        st->pump_power = SFX(power_of)(&c, Pout, npmap, 0);
        st->jacobi_sweeps = total_sweeps;
        st->outer_iterations = outer;
        st->steps = nz;
        st->last_residual = last;
    }
    SFX(fft_plan_free)(&pl);
    free(prop_p); free(prop_s); free(nsmap); free(npmap);
    free(Ti); free(Tf); free(Q); free(DK); free(dkint); free(P); free(S); free(Pout); free(Sout);
    return status;
}

#undef TIDX
#undef CPX
