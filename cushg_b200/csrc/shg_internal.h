// shg_internal.h — structures shared by the host driver and the kernels of
// libshg_b200 (not part of the public C ABI).
#pragma once

#include <stdint.h>

namespace shg {

// Per-instance constants of one plain optical pass.  The host fills them in FP64
// from shg_params with the reference's formulas (src/headers/Solver.h:57-80,
// Efields.h:84-141, PhaseMatching.h:68-85, Crystal.h:34-41); the kernels round to
// the working precision only where a value enters field arithmetic.
struct InstDesc {
    int32_t n;             // grid side (nx == ny)
    int32_t nsteps;        // SSFM steps to march
    int32_t has_signal_in; // 1: SH starts from signal_in, 0: from zero
    int32_t slot;          // output slot (batch index)
    double dz;             // LZ/(NZ-1)
    double dk;             // phase mismatch Δk at the (uniform) temperature
    double kap_p, kap_s;   // π dQ/(n_p λp), 0.5 π dQ/(n_s λs)
    double hap, has, qs;   // 0.5 αp, 0.5 αs, 0.5 βs 0.5 c ε0 n_s
    // pump at z = 0: P = amp * exp(-(ax^2 + ay^2) / den), ax = (x - ux) dx
    double amp_re, amp_im, den_re, den_im;
    double ux, uy, dx, dy;
    int32_t elliptic;      // 1: elliptical pump, P = amp * exp(-ax^2 / den - ay^2 / deny)
    int32_t out32;         // FP64 march of an FP32 instance: signal_in, the outputs and the
                           // slices are FP32 complex (the march rounds what it writes)
    double deny_re, deny_im;
    // propagator phase θ = -dz (a (dfx^2 sx^2 + dfy^2 sy^2) + b sx) per field,
    // sx, sy the signed FFT frequency indices
    double a_p, b_p, a_s, b_s, dfx, dfy;
    double pw_s, pw_p;     // power = pw * sum w |A|^2: plain w = 1, pw = 0.5 eps0 c n dx dy;
                           // thermal w = n(λ, T) of the output slice, pw = 0.5 eps0 c dx dy
    const void* signal_in; // device, n*n complex (natural layout) or null
    void* pump_out;        // device, n*n complex or null
    void* signal_out;      // device, n*n complex or null
    double* power_out;     // device, [2] = {SH power, pump power} or null
    const double* poling;  // device, per-step poling phase [rad] added to the mismatch phase, or null
    int32_t out_after;     // the outputs are the fields after this many steps
    int32_t nslices;       // number of planes in slices_p / slices_s (nz), 0 if none
    void* slices_p;        // device, nslices*n*n complex: the fields before each step s
    void* slices_s;        //   (the reference's save_only_last = false dump), or null
    // thermal pass only (Solver.h:33-55, Tfield.h:260-276); null / zero in plain runs.
    // 3D arrays of the working real type, index z*n*n + y*n + x.
    const void* t_np;      // n(λp, T) per voxel
    const void* t_ns;      // n(λs, T) per voxel
    const void* t_dk;      // Δk(T) per voxel
    void* t_q;             // heat source Q, written slice by slice
    double kf_p, kf_s;     // 1.0 π dQ / λp, 0.5 π dQ / λs (κ = kf / n)
    double bf_s;           // βs 0.5 ε0 c (the two-photon term is bf_s n_s |S|^2)
    double q_p, q_s, q_h;  // αp 0.5 c ε0, αs 0.5 c ε0, 0.5 c ε0: Q = q_p n_p |P|^2 + q_s n_s |S|^2 + βs (q_h n_s |S|^2)^2
    double beta_s;         // βs
};

}  // namespace shg
