// shg_api.cu — host side of libshg_b200: the C ABI of include/shg.h.
//
// This is the C++ counterpart of the reference's Solver::run (src/headers/Solver.h:311-390)
// and of the argv / compile-time configuration of src/cuSHG.cu:11-58: it validates a
// runtime shg_params, derives every per-instance constant in FP64 with the reference's
// formulas, and drives the fused kernels.  Errors are returned as shg_status codes; the
// message of the last failure on the calling thread is kept for shg_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/shg.h"
#include "crystal.cuh"
#include "shg_host.h"
#include "shg_internal.h"
#include "ssfm_variants.h"

namespace shg {

static thread_local std::string g_last_error;

shg_status fail(shg_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

shg_status cuda_fail(cudaError_t e, const char* what) {
    const shg_status st = e == cudaErrorMemoryAllocation ? SHG_ERR_NOMEM : SHG_ERR_CUDA;
    return fail(st, "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
}

void clear_error() { g_last_error.clear(); }

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

cudaError_t dev_alloc(void** ptr, size_t bytes, cudaStream_t s) {
    std::mutex& mu = g_pool_mu;
    cudaMemPool_t* pools = g_pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(s, &cap)) != cudaSuccess) return e;
    // inside a stream capture the allocation becomes a graph memory node
    if (dev < 0 || dev >= 64 || cap != cudaStreamCaptureStatusNone) return cudaMallocAsync(ptr, bytes, s);
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if ((e = cudaMemPoolCreate(&pools[dev], &props)) != cudaSuccess) {
                pools[dev] = nullptr;
                return e;
            }
            unsigned long long keep = kPoolKeepBytes;
            if (const char* env = std::getenv("SHG_POOL_KEEP_MB")) {
                char* end = nullptr;
                const unsigned long long mb = std::strtoull(env, &end, 10);
                if (end != env) keep = mb << 20;
            }
            cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = pools[dev];
    }
    return cudaMallocFromPoolAsync(ptr, bytes, pool, s);
}

// Physical constants, src/headers/Crystal.h:19-21 (µm, ps, W, V).
const double kPi = 3.14159265358979323846;
const double kC = 299792458 * 1E6 / 1E12;
const double kEps0 = 8.8541878128E-12 * 1E12 / 1E6;

// Extraordinary index of the chosen crystal (crystal.cuh; sPPLT: src/headers/Crystal.h:54-70).
double sellmeier(int crystal, double L, double T) { return crystal_n(crystal, L, T); }

// Δk at temperature T with the grating's thermal expansion (PhaseMatching.h:47-85).
double delta_k(const shg_params& p, double T) { return crystal_delta_k(p.crystal, p.lambda_p, p.period, T); }
double sellmeier_dT(int crystal, double L, double T) { return crystal_dn_dT(crystal, L, T); }
double delta_k_dT(const shg_params& p, double T) { return crystal_ddk_dT(p.crystal, p.lambda_p, p.period, T); }

// Constants of one plain optical pass at uniform temperature Tc (the reference reads
// T at voxel (NX/2, NY/2, 0) for the pump and propagators, Efields.h:88,124).
InstDesc make_plain_desc(const shg_params& p, double Tc, double T_dk) {
    InstDesc d;
    std::memset(&d, 0, sizeof(d));
    const double dx = p.lx / (p.nx - 1), dy = p.ly / (p.ny - 1), dz = p.lz / (p.nz - 1);
    const double lp = p.lambda_p, ls = 0.5 * lp;
    const double dQ = 2.0 * p.deff / kPi;
    const double np = sellmeier(p.crystal, lp, Tc), ns = sellmeier(p.crystal, ls, Tc);
    d.n = p.nx;
    d.nsteps = shg_steps(&p);
    d.out_after = p.thermal ? d.nsteps - 1 : d.nsteps;
    d.dz = dz;
    d.dk = delta_k(p, T_dk);
    d.kap_p = 1 * kPi * dQ / (np * lp);
    d.kap_s = 0.5 * kPi * dQ / (ns * ls);
    d.hap = 0.5 * p.alpha_p;
    d.has = 0.5 * p.alpha_s;
    d.qs = 0.5 * (p.beta_s * 0.5 * kC * kEps0 * ns);
    // setPump, Efields.h:92-110
    const double wX2 = p.waist * p.waist;
    const double zRX = kPi * np * wX2 / lp;
    const double Ap0 = std::sqrt(4 * p.power / (kEps0 * kC * kPi * np * wX2));
    const double etaX = p.focus / zRX;
    const double mre = 1.0, mim = -etaX;  // MX = 1 - i etaX
    const double den = mre * mre + mim * mim;
    d.amp_re = (Ap0 * mre) / den;
    d.amp_im = (-Ap0 * mim) / den;
    d.den_re = wX2 * mre;
    d.den_im = wX2 * mim;
    if (p.waist_y > 0 && p.waist_y != p.waist) {
        // elliptical beam (the commented-out variant of setPump, Efields.h:113-115):
        // (Ap0 / (sqrt(MX) sqrt(MY))) exp(-ax^2 / (wX2 MX) - ay^2 / (wY2 MY)), Ap0 normalised
        // with wX wY
        const double wY2 = p.waist_y * p.waist_y;
        const double zRY = kPi * np * wY2 / lp;
        const double etaY = p.focus / zRY;
        const double A = std::sqrt(4 * p.power / (kEps0 * kC * kPi * np * p.waist * p.waist_y));
        const std::complex<double> m = std::sqrt(std::complex<double>(1.0, -etaX)) *
                                       std::sqrt(std::complex<double>(1.0, -etaY));
        const std::complex<double> a = A / m;
        d.elliptic = 1;
        d.amp_re = a.real();
        d.amp_im = a.imag();
        d.deny_re = wY2;
        d.deny_im = wY2 * -etaY;
    }
    d.ux = 0.5 * p.nx;
    d.uy = 0.5 * p.ny;
    d.dx = dx;
    d.dy = dy;
    // beamPropagator, Efields.h:124-137
    const double kp = 2 * kPi * np / lp, ks = 2 * kPi * ns / ls;
    d.dfx = 1 / dx / p.nx;
    d.dfy = 1 / dy / p.ny;
    d.a_p = 2 * (kPi * kPi) / kp;
    d.a_s = 2 * (kPi * kPi) / ks;
    d.b_p = 2 * kPi * d.dfx * std::tan(p.rho_p);
    d.b_s = 2 * kPi * d.dfx * std::tan(p.rho_s);
    d.pw_s = 0.5 * kEps0 * kC * ns * dx * dy;
    d.pw_p = 0.5 * kEps0 * kC * np * dx * dy;
    return d;
}

size_t complex_bytes(const shg_params& p) { return p.precision == 32 ? 8 : 16; }

}  // namespace shg

using namespace shg;

namespace shg {

// Relative L2 error of the FP32 SH output field per (peak-to-final ratio × sqrt(steps)): the
// median ratio measured between the FP32 and FP64 marches of the 256-instance parameter
// sweep (grid sides 64-256, nz 100-400), where the measured field errors follow
// c * sqrt(steps) with a correlation of 0.96 in log scale.
constexpr double kFp32StepError = 1.3e-7;

double fp32_error_estimate(const shg_params& p) {
    const double lp = p.lambda_p;
    const double np = sellmeier(p.crystal, lp, p.temp);
    const double wy = p.waist_y > 0 ? p.waist_y : p.waist;
    const double zrx = kPi * np * p.waist * p.waist / lp, zry = kPi * np * wy * wy / lp;
    const double dk = delta_k(p, p.temp);
    // trapezoid rule with at least 16 points per period of e^{i Δk z}; the phase factor by
    // rotation, recomputed every 64 points; round beams need no complex square root
    const int m = (int)std::min(65536.0, std::max(512.0, std::ceil(16.0 * std::fabs(dk) * p.lz / (2 * kPi))));
    const double h = p.lz / m;
    const bool round = wy == p.waist;
    auto envelope = [&](double z) {
        const double ax = (z - p.focus) / zrx;
        if (round) return std::complex<double>(1.0, -ax) / (1.0 + ax * ax);
        const double ay = (z - p.focus) / zry;
        return 1.0 / std::sqrt(std::complex<double>(1.0, ax) * std::complex<double>(1.0, ay));
    };
    const std::complex<double> rot = std::polar(1.0, dk * h);
    std::complex<double> ph = 1.0, H = 0.0, prev = envelope(0.0);
    double peak = 0.0;
    for (int i = 1; i <= m; ++i) {
        ph = (i & 63) ? ph * rot : std::polar(1.0, dk * h * i);
        const std::complex<double> cur = ph * envelope(h * i);
        H += 0.5 * h * (prev + cur);
        peak = std::max(peak, std::abs(H));
        prev = cur;
    }
    const double c = peak / std::max(std::abs(H), 1e-300 * peak + 1e-300);
    return kFp32StepError * c * std::sqrt((double)std::max(1, shg_steps(&p)));
}

int run_precision(const shg_params& p) {
    if (p.precision != 32 || p.thermal || !(p.fp32_guard > 0)) return p.precision;
    if (!find_plain_variant(64, p.nx, 0, SHG_MARCH_FUSED)) return p.precision;
    return fp32_error_estimate(p) > p.fp32_guard ? 64 : 32;
}

const PlainVariant* plain_variant_of(const shg_params& p, int* out32) {
    const int rp = run_precision(p);
    *out32 = rp != p.precision ? 1 : 0;
    return *out32 ? find_plain_variant(rp, p.nx, 0, SHG_MARCH_FUSED) : find_plain_variant(p.precision, p.nx, 0, p.march);
}

}  // namespace shg

extern "C" {

void shg_default_params(shg_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->nx = p->ny = 128;
    p->nz = 100;
    p->precision = 32;
    p->lx = 2000.0;
    p->ly = 1000.0;
    p->lz = 30000.0;
    p->lambda_p = 1.064;
    p->deff = 11.00e-6;
    p->period = 7.97;
    p->alpha_p = 0.17e-6;
    p->alpha_s = 1.57e-6;
    p->beta_s = 5e-5;
    p->rho_p = p->rho_s = 0.0;
    p->kappa = 8.4e-6;
    p->h_conv = 10e-12;
    p->power = 30.0;
    p->waist = 29.0;
    p->focus = 0.5 * 30000.0;
    p->temp = 55.66;
    p->t_inf = 25.0;
    p->t_peltier = 55.66;
    p->thermal = 0;
    p->boundary = SHG_BOUNDARY_TOP_OPEN;
    p->max_outer = 20;
    p->check_every = 5000;
    p->conv_rule = SHG_CONV_REFERENCE;
    p->crystal = SHG_CRYSTAL_MGO_SPPLT;
    p->jacobi_tol = 0.0;
    p->max_sweeps = 0;
    p->jacobi_block = 0;
    p->march = SHG_MARCH_AUTO;
    p->heat_solver = SHG_HEAT_JACOBI;
    p->waist_y = 0.0;
    p->fp32_guard = 0.0;
}

static bool finite_all(const shg_params* p) {
    const double v[] = {p->lx, p->ly, p->lz, p->lambda_p, p->deff, p->period, p->alpha_p, p->alpha_s, p->beta_s,
                        p->rho_p, p->rho_s, p->kappa, p->h_conv, p->power, p->waist, p->focus, p->temp, p->t_inf,
                        p->t_peltier, p->jacobi_tol, p->waist_y, p->fp32_guard};
    for (double x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

static shg_status check_params_impl(const shg_params* p, bool need_kernel) {
    clear_error();
    if (!p) return fail(SHG_ERR_INVALID, "params is NULL");
    if (!finite_all(p)) return fail(SHG_ERR_INVALID, "a parameter is NaN or infinite");
    if (p->precision != 32 && p->precision != 64) return fail(SHG_ERR_INVALID, "precision must be 32 or 64");
    if (p->nx != p->ny) return fail(SHG_ERR_INVALID, "nx (%d) must equal ny (%d)", p->nx, p->ny);
    if (p->nx < 2 || (p->nx & 1)) return fail(SHG_ERR_INVALID, "grid side %d must be even and >= 2", p->nx);
    if (p->nz < 2) return fail(SHG_ERR_INVALID, "nz must be >= 2 (dz = lz/(nz-1))");
    if (!(p->lx > 0 && p->ly > 0 && p->lz > 0)) return fail(SHG_ERR_INVALID, "lx, ly, lz must be > 0");
    if (!(p->lambda_p > 0.3 && p->lambda_p < 6.0)) return fail(SHG_ERR_INVALID, "lambda_p out of range");
    if (!(p->waist > 0) || p->power < 0 || !(p->period > 0)) return fail(SHG_ERR_INVALID, "waist/power/period");
    if (p->waist_y < 0) return fail(SHG_ERR_INVALID, "waist_y must be >= 0 (0: round beam)");
    if (p->fp32_guard < 0) return fail(SHG_ERR_INVALID, "fp32_guard must be >= 0 (0: off)");
    if (p->alpha_p < 0 || p->alpha_s < 0 || p->beta_s < 0) return fail(SHG_ERR_INVALID, "negative absorption");
    if (p->crystal != SHG_CRYSTAL_MGO_SPPLT && p->crystal != SHG_CRYSTAL_MGO_PPLN)
        return fail(SHG_ERR_UNSUPPORTED, "unknown crystal %d", p->crystal);
    if (p->thermal) {
        if (!(p->kappa > 0) || p->h_conv < 0) return fail(SHG_ERR_INVALID, "kappa must be > 0, h_conv >= 0");
        if (p->boundary != SHG_BOUNDARY_TOP_OPEN && p->boundary != SHG_BOUNDARY_OVEN_SURROUNDED)
            return fail(SHG_ERR_INVALID, "unknown boundary %d", p->boundary);
        if (p->conv_rule != SHG_CONV_REFERENCE && p->conv_rule != SHG_CONV_MAXABS && p->conv_rule != SHG_CONV_FIXED)
            return fail(SHG_ERR_INVALID, "unknown conv_rule %d", p->conv_rule);
        if (p->conv_rule == SHG_CONV_FIXED && (p->max_sweeps <= 0 || p->max_outer <= 0))
            return fail(SHG_ERR_INVALID, "conv_rule FIXED needs max_sweeps > 0 and max_outer > 0");
        if (p->nz < 3 || p->nx < 3) return fail(SHG_ERR_INVALID, "thermal grid needs nx, nz >= 3");
        if (p->jacobi_block < 0 || p->jacobi_block > 4)
            return fail(SHG_ERR_INVALID, "jacobi_block %d must be in 0..4", p->jacobi_block);
        if (p->heat_solver != SHG_HEAT_JACOBI && p->heat_solver != SHG_HEAT_DIRECT)
            return fail(SHG_ERR_INVALID, "unknown heat_solver %d", p->heat_solver);
    }
    if (p->march < SHG_MARCH_AUTO || p->march > SHG_MARCH_MULTIPASS)
        return fail(SHG_ERR_INVALID, "unknown march %d", p->march);
    if (need_kernel && !find_plain_variant(p->precision, p->nx, p->thermal, p->march))
        return fail(SHG_ERR_UNSUPPORTED, "no %s%s kernel built for grid side %d at precision %d",
                    p->march == SHG_MARCH_FUSED ? "fused " : p->march == SHG_MARCH_MULTIPASS ? "multi-pass " : "",
                    p->thermal ? "thermal" : "plain", p->nx, p->precision);
    return SHG_OK;
}

shg_status shg_check_params(const shg_params* p) { return check_params_impl(p, true); }

int32_t shg_steps(const shg_params* p) {
    if (!p) return 0;
    return p->thermal ? p->nz : p->nz - 1;
}


double shg_fp32_error_estimate(const shg_params* p) {
    if (!p || !(p->waist > 0) || !(p->lz > 0) || !(p->lambda_p > 0) || p->nz < 2) return -1.0;
    return fp32_error_estimate(*p);
}

const char* shg_last_error(void) { return g_last_error.c_str(); }

const char* shg_status_string(int32_t s) {
    switch (s) {
        case SHG_OK: return "ok";
        case SHG_ERR_INVALID: return "invalid argument";
        case SHG_ERR_UNSUPPORTED: return "unsupported configuration";
        case SHG_ERR_CUDA: return "CUDA error";
        case SHG_ERR_NOMEM: return "out of memory";
        case SHG_ERR_NOT_CONVERGED: return "Jacobi did not converge";
        case SHG_ERR_NO_DEVICE: return "no CUDA device";
        case SHG_ERR_NONFINITE: return "non-finite result";
        default: return "unknown status";
    }
}

const char* shg_version(void) { return "libshg_b200 0.1 (sm_100a)"; }

shg_status shg_solve_device(const shg_params* p, const void* signal_in_dev, void* pump_out_dev, void* signal_out_dev,
                            void* temperature_out_dev, shg_stats* stats, void* stream_) {
    shg_status st = shg_check_params(p);
    if (st != SHG_OK) return st;
    cudaStream_t stream = (cudaStream_t)stream_;
    if (p->thermal) return thermal_solve_device(*p, signal_in_dev, pump_out_dev, signal_out_dev, temperature_out_dev, stats, stream);
    return plain_solve_device(*p, signal_in_dev, pump_out_dev, signal_out_dev, stats, stream);
}

// Host-buffer solve shared by shg_solve (last slice) and shg_solve_slices (every slice).
static shg_status solve_host(const shg_params* p, const void* signal_in, void* pump_out, void* signal_out,
                             void* temperature_out, shg_stats* stats, bool slices) {
    shg_status st = shg_check_params(p);
    if (st != SHG_OK) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    const size_t plane = (size_t)p->nx * p->ny * complex_bytes(*p);
    const size_t outb = slices ? plane * (size_t)p->nz : plane;
    const size_t tbytes = (size_t)p->nx * p->ny * p->nz * (p->precision == 32 ? 4 : 8);
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    void *din = nullptr, *dp = nullptr, *ds = nullptr, *dT = nullptr;
    shg_status rc = SHG_OK;
    do {
        if (signal_in && (e = dev_alloc((void**)&din, plane, s)) != cudaSuccess) { rc = cuda_fail(e, "cudaMallocAsync"); break; }
        if (pump_out && (e = dev_alloc((void**)&dp, outb, s)) != cudaSuccess) { rc = cuda_fail(e, "cudaMallocAsync"); break; }
        if (signal_out && (e = dev_alloc((void**)&ds, outb, s)) != cudaSuccess) { rc = cuda_fail(e, "cudaMallocAsync"); break; }
        if (temperature_out && p->thermal && (e = dev_alloc((void**)&dT, tbytes, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMallocAsync");
            break;
        }
        if (din && (e = cudaMemcpyAsync(din, signal_in, plane, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync H2D");
            break;
        }
        if (slices) {
            rc = p->thermal ? thermal_solve_device(*p, din, nullptr, nullptr, dT, stats, s, dp, ds)
                            : plain_solve_device(*p, din, nullptr, nullptr, stats, s, dp, ds);
        } else {
            rc = shg_solve_device(p, din, dp, ds, dT, stats, s);
        }
        if (rc != SHG_OK) break;
        if (dp && (e = cudaMemcpyAsync(pump_out, dp, outb, cudaMemcpyDeviceToHost, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync D2H");
            break;
        }
        if (ds && (e = cudaMemcpyAsync(signal_out, ds, outb, cudaMemcpyDeviceToHost, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync D2H");
            break;
        }
        if (dT && (e = cudaMemcpyAsync(temperature_out, dT, tbytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync D2H");
            break;
        }
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) { rc = cuda_fail(e, "cudaStreamSynchronize"); break; }
    } while (0);
    if (din) cudaFreeAsync(din, s);
    if (dp) cudaFreeAsync(dp, s);
    if (ds) cudaFreeAsync(ds, s);
    if (dT) cudaFreeAsync(dT, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}

shg_status shg_solve(const shg_params* p, const void* signal_in, void* pump_out, void* signal_out,
                     void* temperature_out, shg_stats* stats) {
    return solve_host(p, signal_in, pump_out, signal_out, temperature_out, stats, false);
}

shg_status shg_solve_slices(const shg_params* p, const void* signal_in, void* pump_slices, void* signal_slices,
                            void* temperature_out, shg_stats* stats) {
    return solve_host(p, signal_in, pump_slices, signal_slices, temperature_out, stats, true);
}

shg_status shg_sh_power(const shg_params* p, const double* poling, double* sh_power) {
    shg_status st = shg_check_params(p);
    if (st != SHG_OK) return st;
    if (!sh_power) return fail(SHG_ERR_INVALID, "sh_power is NULL");
    if (p->thermal) return fail(SHG_ERR_UNSUPPORTED, "shg_sh_power is for plain runs");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    const int nsteps = shg_steps(p);
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    double* dpol = nullptr;
    shg_status rc = SHG_OK;
    do {
        if (poling) {
            if ((e = dev_alloc((void**)&dpol, sizeof(double) * nsteps, s)) != cudaSuccess ||
                (e = cudaMemcpyAsync(dpol, poling, sizeof(double) * nsteps, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
                rc = cuda_fail(e, "poling upload");
                break;
            }
        }
        shg_stats stats;
        rc = plain_solve_device(*p, nullptr, nullptr, nullptr, &stats, s, nullptr, nullptr, dpol);
        if (rc == SHG_OK) *sh_power = stats.sh_power;
    } while (0);
    if (dpol) cudaFreeAsync(dpol, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}

shg_status shg_heat_sweeps_device(const shg_params* p, void* temperature_dev, const void* q_dev, int64_t sweeps,
                                  void* stream) {
    clear_error();
    if (!p) return fail(SHG_ERR_INVALID, "params is NULL");
    shg_params q = *p;
    q.thermal = 1;
    shg_status st = check_params_impl(&q, false);  // the heat solve needs no optical kernel
    if (st != SHG_OK) return st;
    if (!temperature_dev || !q_dev) return fail(SHG_ERR_INVALID, "temperature or Q is NULL");
    // the sweep reads voxel pairs (float2 / double2): both arrays aligned to two reals
    const uintptr_t al = 2 * (p->precision == 32 ? 4 : 8) - 1;
    if (((uintptr_t)temperature_dev & al) || ((uintptr_t)q_dev & al))
        return fail(SHG_ERR_INVALID, "temperature and Q must be aligned to %d bytes", (int)al + 1);
    if (sweeps < 0) return fail(SHG_ERR_INVALID, "sweeps must be >= 0");
    if (sweeps == 0) return SHG_OK;
    return heat_sweeps_device(q, temperature_dev, q_dev, sweeps, (cudaStream_t)stream);
}

shg_status shg_heat_steady_device(const shg_params* p, void* temperature_dev, const void* q_dev, double* residual_out,
                                  void* stream) {
    clear_error();
    if (!p) return fail(SHG_ERR_INVALID, "params is NULL");
    shg_params q = *p;
    q.thermal = 1;
    shg_status st = check_params_impl(&q, false);  // the heat solve needs no optical kernel
    if (st != SHG_OK) return st;
    if (!temperature_dev) return fail(SHG_ERR_INVALID, "temperature is NULL");
    const uintptr_t al = (p->precision == 32 ? 4 : 8) - 1;
    if (((uintptr_t)temperature_dev & al) || ((uintptr_t)q_dev & al))
        return fail(SHG_ERR_INVALID, "temperature and Q must be aligned to %d bytes", (int)al + 1);
    return heat_steady_device(q, temperature_dev, q_dev, residual_out, (cudaStream_t)stream);
}

shg_status shg_reserve_device_memory(int64_t bytes) {
    clear_error();
    if (bytes < 0) return fail(SHG_ERR_INVALID, "bytes must be >= 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (bytes == 0) return SHG_OK;
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    void* p = nullptr;
    shg_status rc = SHG_OK;
    if ((e = dev_alloc(&p, (size_t)bytes, s)) != cudaSuccess) {
        rc = cuda_fail(e, "reserve");
    } else {
        // keep at least the reserved bytes in the pool from now on
        int dev = 0;
        cudaGetDevice(&dev);
        {
            std::lock_guard<std::mutex> lk(g_pool_mu);
            if (dev >= 0 && dev < 64 && g_pools[dev]) {
                unsigned long long keep = 0;
                cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
                if (keep < (unsigned long long)bytes) {
                    keep = (unsigned long long)bytes;
                    cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
                }
            }
        }
        cudaFreeAsync(p, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) rc = cuda_fail(e, "reserve");
    }
    cudaStreamDestroy(s);
    return rc;
}

shg_status shg_solve_batch(const shg_params* params, int32_t count, void* const* pump_out, void* const* signal_out,
                           double* sh_power_out) {
    clear_error();
    if (!params || count < 0) return fail(SHG_ERR_INVALID, "params is NULL or count < 0");
    for (int i = 0; i < count; ++i) {
        shg_status st = shg_check_params(&params[i]);
        if (st != SHG_OK) return fail(st, "instance %d: %s", i, g_last_error.c_str());
        if (params[i].thermal) return fail(SHG_ERR_UNSUPPORTED, "instance %d: batched runs are plain (thermal == 0)", i);
        if (params[i].precision != params[0].precision)
            return fail(SHG_ERR_INVALID, "instance %d: all instances must share one precision", i);
    }
    if (count == 0) return SHG_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    // Page-locked host outputs are written by the march itself through their device mapping,
    // as each instance finishes, so the transfer spreads over the whole launch; pageable ones
    // go through a device buffer and one copy per class as soon as that class's march ends.
    auto mapped = [](void* h) -> void* {
        if (!h) return nullptr;
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
    };
    std::vector<void*> mp(count, nullptr), ms(count, nullptr);
    std::vector<size_t> off(2 * (size_t)count + 1, 0);
    for (int i = 0; i < count; ++i) {
        const size_t plane = (size_t)params[i].nx * params[i].ny * complex_bytes(params[i]);
        if (pump_out) mp[i] = mapped(pump_out[i]);
        if (signal_out) ms[i] = mapped(signal_out[i]);
        off[2 * i + 1] = off[2 * i] + ((pump_out && pump_out[i] && !mp[i]) ? plane : 0);
        off[2 * i + 2] = off[2 * i + 1] + ((signal_out && signal_out[i] && !ms[i]) ? plane : 0);
    }
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    char* buf = nullptr;
    shg_status rc = SHG_OK;
    do {
        if (off.back() && (e = dev_alloc((void**)&buf, off.back(), s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMallocAsync");
            break;
        }
        std::vector<void*> dp(mp), ds(ms), hp(count, nullptr), hs(count, nullptr);
        for (int i = 0; i < count; ++i) {
            if (off[2 * i + 1] > off[2 * i]) {
                dp[i] = buf + off[2 * i];
                hp[i] = pump_out[i];
            }
            if (off[2 * i + 2] > off[2 * i + 1]) {
                ds[i] = buf + off[2 * i + 1];
                hs[i] = signal_out[i];
            }
        }
        // staged outputs: each grid-size class's are copied as soon as its march ends,
        // overlapping the others
        if ((rc = plain_solve_batch(params, count, dp.data(), ds.data(), sh_power_out, s, hp.data(), hs.data())) !=
            SHG_OK)
            break;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) rc = cuda_fail(e, "cudaStreamSynchronize");
    } while (0);
    if (buf) cudaFreeAsync(buf, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}

shg_status shg_solve_batch_device(const shg_params* params, int32_t count, void* const* pump_out_dev,
                                  void* const* signal_out_dev, double* sh_power_out, void* stream_) {
    clear_error();
    if (!params || count < 0) return fail(SHG_ERR_INVALID, "params is NULL or count < 0");
    for (int i = 0; i < count; ++i) {
        shg_status st = shg_check_params(&params[i]);
        if (st != SHG_OK) return fail(st, "instance %d: %s", i, g_last_error.c_str());
        if (params[i].thermal) return fail(SHG_ERR_UNSUPPORTED, "instance %d: batched runs are plain (thermal == 0)", i);
        if (params[i].precision != params[0].precision)
            return fail(SHG_ERR_INVALID, "instance %d: all instances must share one precision", i);
    }
    return plain_solve_batch(params, count, pump_out_dev, signal_out_dev, sh_power_out, (cudaStream_t)stream_);
}

}  // extern "C"
