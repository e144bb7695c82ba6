/*
 * shg.h — C ABI of the B200-native focused-beam SHG solver (libshg_b200.so).
 *
 * This is the drop-in boundary for the split-step Fourier (SSFM) march of the
 * coupled pump / second-harmonic (SH) fields and the 3D Jacobi heat solve of
 * alfredos84/cuSHG.  The reference exposes that path as one C++ method with its
 * parameters split between compile-time constants and arguments:
 *
 *   Solver::run(Power, waist, focalpoint, Temp, T_inf, Tpeltier,
 *               save_only_last, save_temperature)      src/headers/Solver.h:149,311
 *   NX, NY, NZ                                          src/cuSHG.cu:11-13
 *   crystal / beam constants                            src/headers/Crystal.h:19-52
 *   -DTHERMAL                                           src/headers/Solver.h:32,321
 *   outputs Pump_out_{r,i}.dat, Signal_out_{r,i}.dat    src/headers/Solver.h:283-286
 *   temperature tensor Tfinal_<z>.dat                   src/headers/Solver.h:372-373
 *
 * Here every one of those is a runtime field of shg_params, the fields come back
 * in caller-owned buffers as interleaved complex (re, im) in the reference's
 * row-major layout (x fastest: index y*nx + x, src/headers/Common.h:88-90), and
 * errors come back as a status code instead of exit(1) (src/headers/Common.h:10-20).
 *
 * Element types: precision 64 -> double (re, im pairs, like cufftDoubleComplex),
 * precision 32 -> float (like cufftComplex).  Real 3D arrays (temperature) use
 * the same scalar type, index z*nx*ny + y*nx + x.
 *
 * Units follow the reference: lengths in µm, time in ps, power in W,
 * temperatures in °C.
 */
#ifndef CUSHG_B200_SHG_H
#define CUSHG_B200_SHG_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SHG_API __attribute__((visibility("default")))
#else
#define SHG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum shg_status {
    SHG_OK = 0,
    SHG_ERR_INVALID = 1,       /* a parameter is out of range, NaN, or a pointer is NULL */
    SHG_ERR_UNSUPPORTED = 2,   /* grid size / precision combination not built */
    SHG_ERR_CUDA = 3,          /* a CUDA runtime call failed; see shg_last_error() */
    SHG_ERR_NOMEM = 4,         /* device or host allocation failed */
    SHG_ERR_NOT_CONVERGED = 5, /* Jacobi hit max_sweeps before its tolerance */
    SHG_ERR_NO_DEVICE = 6,     /* no CUDA device is visible */
    SHG_ERR_NONFINITE = 7      /* the run produced NaN or Inf (SH power or Jacobi residual):
                                  parameters outside the range the discretisation resolves */
} shg_status;

/* Heat-equation boundary models (src/headers/Tfield.h). */
enum {
    SHG_BOUNDARY_TOP_OPEN = 0,        /* kernelHeatEquationTopOpen, Tfield.h:93-201:
                                         y=0 face Dirichlet at t_peltier, Robin elsewhere */
    SHG_BOUNDARY_OVEN_SURROUNDED = 1  /* kernelHeatEquationOvenSurrounded, Tfield.h:205-240:
                                         4 lateral faces at t_peltier, Robin on z faces */
};

/* Jacobi stopping rules. */
enum {
    SHG_CONV_REFERENCE = 0, /* sqrt(sum (Tf-Ti)^2)/TSIZE < tol, checked every check_every
                               sweeps, stagnation exit (Solver.h:332-351) */
    SHG_CONV_MAXABS = 1,    /* max |Tf-Ti| < tol, checked every check_every sweeps */
    SHG_CONV_FIXED = 2      /* exactly max_sweeps sweeps per outer iteration and exactly
                               max_outer iterations, no convergence test (a fixed cost per
                               optical-thermal update); last_residual = max |Tf-Ti| of the
                               last sweep */
};

/* Crystals (Sellmeier equations). */
enum {
    SHG_CRYSTAL_MGO_SPPLT = 0, /* Bruner et al., src/headers/Crystal.h:54-70 */
    SHG_CRYSTAL_MGO_PPLN = 1   /* 5 mol% MgO:PPLN, Gayer et al. 2008; named in the reference's
                                  README.md:52, absent from its Crystal.h */
};

typedef struct shg_params {
    /* grid: src/cuSHG.cu:11-13 (NX, NY, NZ).  nx == ny, even. */
    int32_t nx, ny, nz;
    int32_t precision;      /* 64 (double) or 32 (float): src/cuSHG.cu:7-8 */
    /* window and crystal [µm]: Crystal.h:31-33 (LX, LY, LZ); dx = lx/(nx-1) */
    double lx, ly, lz;
    double lambda_p;        /* pump wavelength [µm], SH at lambda_p/2: Crystal.h:27-28 */
    double deff;            /* effective nonlinearity [µm/V]: Crystal.h:40 */
    double period;          /* QPM grating period Λ [µm]: Crystal.h:42 */
    double alpha_p;         /* pump linear absorption [1/µm]: Crystal.h:43 */
    double alpha_s;         /* SH linear absorption [1/µm]: Crystal.h:44 */
    double beta_s;          /* SH two-photon absorption [µm/W]: Crystal.h:45 */
    double rho_p, rho_s;    /* walk-off angles [rad]: Crystal.h:46-47 */
    double kappa;           /* thermal conductivity [W/(µm K)]: Crystal.h:51 */
    double h_conv;          /* heat transfer coefficient [W/(µm² K)]: Crystal.h:52 */
    /* Solver::run arguments: Solver.h:311 and cuSHG.cu:46-53 */
    double power;           /* pump power [W] */
    double waist;           /* beam waist radius [µm] */
    double focus;           /* focal position from the input face [µm] */
    double temp;            /* initial / phase-matching temperature [°C] */
    double t_inf;           /* environment temperature [°C] (25 in cuSHG.cu:52) */
    double t_peltier;       /* oven temperature [°C] */
    int32_t thermal;        /* 0: plain run; 1: -DTHERMAL outer optical-thermal loop */
    int32_t boundary;       /* SHG_BOUNDARY_* */
    int32_t max_outer;      /* outer iterations, 20 in Solver.h:325 */
    int32_t check_every;    /* Jacobi check period, 5000 in Solver.h:342 */
    int32_t conv_rule;      /* SHG_CONV_* */
    int32_t crystal;        /* SHG_CRYSTAL_* */
    double jacobi_tol;      /* <= 0 selects the reference tolerance 5e-4/TSIZE (Solver.h:332) */
    int64_t max_sweeps;     /* Jacobi sweep cap per outer iteration (<= 0: 2^40) */
    /* Sweeps fused per launch between convergence checks (temporal blocking): 0 = automatic
     * (one sweep per launch, the fastest on B200 at every grid size measured), 1 = one
     * sweep per launch, 2..4 = that many through the TMA-staged blocked kernel.  Every setting gives the same
     * temperatures bit for bit; the checked sweep of each window always runs alone. */
    int32_t jacobi_block;
    /* Which SSFM march to run (SHG_MARCH_*): automatic picks, for plain runs, the fused
     * cluster march where one is built for the grid side (planes in shared memory, sides
     * <= 256) and the multi-pass march otherwise (planes in global memory, side 512); for
     * thermal runs, the multi-pass march where one is built (sides 128, 256, 512), since a
     * single instance's optical pass then spreads over the GPU, and the fused march
     * otherwise. */
    int32_t march;
    /* How each outer iteration of a thermal run solves the heat equation (SHG_HEAT_*):
     * Jacobi sweeps as the reference runs them (default), or the sweeps' fixed point computed
     * directly.  No counterpart in the reference. */
    int32_t heat_solver;
    /* Beam waist radius in y [µm].  <= 0 (default): a round beam of radius `waist`, setPump
     * as the reference runs it (Efields.h:94, waistY = waistX).  Otherwise the elliptical beam
     * of the reference's commented-out variant (Efields.h:113-115), with its own Rayleigh
     * length and focusing term in y, and Ap0 normalised with waist * waist_y so that the beam
     * carries `power` (the commented code keeps waist^2, which would not). */
    double waist_y;
    /* FP32 plain runs only (precision 32, thermal 0, fused grid sides up to 256): the largest
     * predicted relative error of the FP32 SH output field this instance accepts.  The FP32
     * march rounds both fields at every step; when the crystal is far from phase matching the
     * SH grows and cancels along the crystal, so the output is a small remainder of a larger
     * field and its relative error grows with that ratio.  shg_fp32_error_estimate predicts
     * it before the march.  An instance whose prediction exceeds fp32_guard runs the FP64
     * march instead, with its outputs rounded to FP32 (same buffers, same layout).
     * 0 (default): every FP32 instance runs in FP32.  No counterpart in the reference. */
    double fp32_guard;
} shg_params;

/* Heat solvers of a thermal run. */
enum {
    SHG_HEAT_JACOBI = 0, /* Jacobi sweeps under conv_rule (Solver.h:335-355); bit-identical to the
                            reference */
    SHG_HEAT_DIRECT = 1  /* the temperature the sweeps converge to, solved directly for every
                            outer iteration (shg_heat_steady_device), in FP64.  jacobi_block,
                            check_every and max_sweeps are ignored; jacobi_sweeps reports 0;
                            last_residual is the conv_rule value (max |ΔT| for MAXABS and
                            FIXED) of one FP64 Jacobi sweep applied to the solution.  The outer
                            loop stops after max_outer iterations, or (conv_rule REFERENCE or
                            MAXABS) after the first iteration g > 0 whose solution moved by less
                            than the Jacobi tolerance, by the rule's own measure. */
};

enum {
    SHG_MARCH_AUTO = 0,     /* plain runs: fused where built (the autotuner's choice if it ran), else
                               multi-pass; thermal runs: multi-pass where built, else fused */
    SHG_MARCH_FUSED = 1,     /* one thread-block cluster per instance, fields in shared memory */
    SHG_MARCH_MULTIPASS = 2  /* fields in global memory, a row and a column launch per step */
};

/* Per-call report. */
typedef struct shg_stats {
    double sh_power;          /* SH output power [W]: sum 0.5*eps0*c*n_s*|S|^2*dx*dy */
    double pump_power;        /* pump output power [W], same normalisation */
    int64_t jacobi_sweeps;    /* total Jacobi sweeps over all outer iterations */
    int32_t outer_iterations; /* outer optical-thermal iterations run */
    int32_t steps;            /* SSFM steps marched per optical pass */
    double last_residual;     /* last Jacobi convergence value */
    double device_ms;         /* device time of the call (CUDA events) */
    double jacobi_ms;         /* thermal runs: device time of the Jacobi sweeps and checks */
    double optics_ms;         /* thermal runs: device time of the per-voxel optics and optical
                                 passes (plain runs: 0; device_ms is the march) */
} shg_stats;

/* Fill *p with the reference's compile-time defaults (cuSHG.cu:11-13, Crystal.h:19-52,
 * cuSHG.cu:46-53 with argv = 30 W, 29 µm, 55.66 °C from cuSHG.sh:43-45). */
SHG_API void shg_default_params(shg_params* p);

/* Validate a parameter set; SHG_OK or SHG_ERR_INVALID / SHG_ERR_UNSUPPORTED. */
SHG_API shg_status shg_check_params(const shg_params* p);

/* Number of SSFM steps a plain optical pass marches for these parameters: the
 * reference records the fields before its last step (Solver.h:283-286), so a
 * plain pass marches nz-1 steps and a thermal pass nz (its last step feeds Q). */
SHG_API int32_t shg_steps(const shg_params* p);

/* Predicted relative L2 error of the SH output field of the FP32 march against the FP64
 * march, for a plain run of these parameters: K * c * sqrt(steps), where c is the ratio of
 * the peak to the final magnitude of the undepleted Gaussian-beam SH amplitude
 *   H(z) = integral_0^z e^{i Δk z'} / sqrt((1 + i (z' - f)/z_Rx) (1 + i (z' - f)/z_Ry)) dz'
 * (the phase-mismatch cancellation along the crystal) and K the per-step rounding of the
 * FP32 march, fitted on the 256-instance parameter sweep (grid sides 64-256).  The SH power's
 * relative error is typically below it.  Host-only arithmetic; no counterpart in the
 * reference. */
SHG_API double shg_fp32_error_estimate(const shg_params* p);

/*
 * Solve one instance.  Replaces Solver::run (Solver.h:311-390) with
 * save_only_last = true.  Host buffers, synchronous.
 *   signal_in   nx*ny complex or NULL.  NULL starts the SH at zero; the reference
 *               starts from clock-seeded N(0,1e-20) noise (Efields.h:144-168).
 *   pump_out, signal_out   nx*ny complex each (Pump_out / Signal_out), may be NULL.
 *   temperature_out        nx*ny*nz reals (Tfinal), thermal runs only, may be NULL.
 *   stats                  may be NULL.
 */
SHG_API shg_status shg_solve(const shg_params* p, const void* signal_in, void* pump_out,
                     void* signal_out, void* temperature_out, shg_stats* stats);

/*
 * Solve one instance and keep the fields of every slice: the save_only_last = false mode of
 * Solver::run, which writes Pump_<s> / Signal_<s> before each step s (Solver.h:289-295).
 * pump_slices, signal_slices: host buffers of nz planes of nx*ny complex each (plane s holds
 * the fields before step s; plane nz-1 equals shg_solve's outputs), may be NULL.
 */
SHG_API shg_status shg_solve_slices(const shg_params* p, const void* signal_in, void* pump_slices,
                                    void* signal_slices, void* temperature_out, shg_stats* stats);

/* The same with device buffers on a caller stream (a cudaStream_t, NULL = legacy
 * default stream).  Plain runs are asynchronous; thermal runs synchronise at each
 * Jacobi convergence check.  stats, if given, is filled after a synchronise. */
SHG_API shg_status shg_solve_device(const shg_params* p, const void* signal_in_dev,
                            void* pump_out_dev, void* signal_out_dev,
                            void* temperature_out_dev, shg_stats* stats, void* stream);

/*
 * Batched plain runs: `count` independent instances, each with its own parameter
 * set (grid size, nz, crystal, beam), in one persistent launch per grid-size class
 * fed by a device work queue.  Replaces the one-process-per-point sweep of
 * src/cuSHG.sh:58-94.  All instances must share `precision` and have thermal == 0.
 * pump_out[i] / signal_out[i]: device buffers (nx_i*ny_i complex) or NULL entries.
 * sh_power_out: host array of `count` doubles or NULL.
 */
SHG_API shg_status shg_solve_batch_device(const shg_params* params, int32_t count,
                                  void* const* pump_out_dev, void* const* signal_out_dev,
                                  double* sh_power_out, void* stream);

/*
 * shg_solve_batch_device with host buffers: pump_out[i] / signal_out[i] are host arrays of
 * nx_i*ny_i complex (or NULL entries), sh_power_out a host array of `count` doubles or NULL.
 * Synchronous.  The sweep of src/cuSHG.sh:58-94 as one call.  Page-locked buffers
 * (cudaHostAlloc / cudaMallocHost / cudaHostRegister) are written by the march directly as
 * each instance finishes; pageable ones are staged on the device and copied per grid-size
 * class.
 */
SHG_API shg_status shg_solve_batch(const shg_params* params, int32_t count, void* const* pump_out,
                                   void* const* signal_out, double* sh_power_out);

/*
 * Batch plans: the batched march of shg_solve_batch_device captured once into a CUDA graph,
 * with its descriptors, work-queue counters and power slots allocated at creation, then
 * replayed by shg_batch_plan_launch with one graph launch (no host work per replay).  For
 * sweeps run repeatedly over the same parameter sets and output buffers (optimisation
 * loops, repeated measurements).  No counterpart in the reference, whose sweep is one
 * process per point (src/cuSHG.sh:58-94).
 *   shg_batch_plan_create   validates like shg_solve_batch_device, uploads the descriptors
 *                           and captures the launches (current device); synchronous.
 *   shg_batch_plan_launch   replays the graph on `stream`; launches of one plan that overlap
 *                           on the GPU race on its work queues and power slots.
 *   shg_batch_plan_powers   copies the SH powers of the last finished replay to the host
 *                           array sh_power_out[count] (stream-ordered, then synchronises).
 *   shg_batch_plan_destroy  synchronises the device and frees the plan.
 */
typedef struct shg_batch_plan shg_batch_plan;
SHG_API shg_status shg_batch_plan_create(const shg_params* params, int32_t count, void* const* pump_out_dev,
                                         void* const* signal_out_dev, shg_batch_plan** plan);
SHG_API shg_status shg_batch_plan_launch(shg_batch_plan* plan, void* stream);
SHG_API shg_status shg_batch_plan_powers(shg_batch_plan* plan, double* sh_power_out, void* stream);
SHG_API void shg_batch_plan_destroy(shg_batch_plan* plan);

/* Result of shg_autotune. */
typedef struct shg_tune_result {
    int32_t precision, n;       /* the grid-size class tuned */
    int32_t cluster, threads;   /* the chosen split: CTAs per instance, threads per CTA */
    int32_t candidates;         /* compiled variants timed */
    int32_t reserved;
    double pt_steps_per_s;      /* the chosen variant's rate on the tuning batch */
    double default_pt_steps_per_s; /* the default variant's rate on the same batch */
} shg_tune_result;

/*
 * Autotuner of the fused march's schedule for one (precision, grid side) class: times every
 * compiled variant of the class (cluster split and threads per CTA of the row / column FFT
 * passes) on a synthetic batch that fills the device several times over, and makes the
 * fastest the variant every later plain run and batch of that class uses in this process
 * (results are the same to the last bit of the fields; SH powers may differ in the last
 * bits, the cluster reduction order being the split's).  Synchronous; call it before any
 * stream capture.  No counterpart in the reference (compile-time launch shapes,
 * src/cuSHG.cu:22-23).
 */
SHG_API shg_status shg_autotune(int32_t precision, int32_t n, shg_tune_result* out);

/*
 * Autotuner for a given mixed batch (shg_solve_batch_device arguments, all march ==
 * SHG_MARCH_AUTO): the classes of a batch run side by side and share the SMs, so the split
 * that is fastest for a class alone can slow the batch.  Starting from the compiled
 * defaults, each class (largest total work first) tries its other compiled variants with the
 * rest fixed, and keeps one that makes the whole batch at least 1 % faster on this device.
 * The choices hold for every later plain run and batch in this process, as for
 * shg_autotune.  out[0 .. *n_out-1]: one entry per class, largest work first, with
 * pt_steps_per_s the batch's rate with the chosen schedule and default_pt_steps_per_s its
 * rate with the defaults.  Synchronous (runs the batch 4 times per trial); call it before
 * any stream capture.  No counterpart in the reference.
 */
SHG_API shg_status shg_autotune_batch(const shg_params* params, int32_t count, shg_tune_result* out,
                                      int32_t max_out, int32_t* n_out);

/* Grow the library's device memory pool on the current device to hold `bytes`, and keep at
 * least that much from now on (raises the keep threshold of SHG_POOL_KEEP_MB).  Later calls
 * draw their workspace from it without mapping new memory: a 512 x 512 x 1000 thermal run
 * takes about 11 GB, and growing the pool to that is most of a first run's extra time.
 * Synchronous.  No counterpart in the reference. */
SHG_API shg_status shg_reserve_device_memory(int64_t bytes);

/* Forget the choices of shg_autotune / shg_autotune_batch: later runs use the compiled
 * default schedules.  No counterpart in the reference. */
SHG_API void shg_autotune_reset(void);

/* Choose a class's compiled variant by its split (the cluster and threads fields of a
 * shg_tune_result), without timing: e.g. to reuse a schedule that shg_autotune_batch found in
 * an earlier process.  SHG_ERR_UNSUPPORTED if no such variant is compiled.  No counterpart in
 * the reference. */
SHG_API shg_status shg_set_schedule(int32_t precision, int32_t n, int32_t cluster, int32_t threads);

/*
 * The batched plain march of shg_solve_batch_device without any device allocation.  This
 * entry point has no counterpart in the reference.  It is for callers that cannot allocate
 * device memory while they run (hosts that give all free memory to their own allocator,
 * latency-bound loops where an allocation may block or synchronise, plugin hosts that forbid
 * it): its scratch (instance descriptors, power slots) is a fixed ~23 KB __device__ array of
 * the library, held by every GPU that loads it until exit.  Limit: count <= 64 instances
 * (larger counts return SHG_ERR_INVALID), grid sides of the fused march (up to 256).  The
 * first call on a device sets that device up: it looks the array's address up and loads the
 * kernels it launches, for which the CUDA driver may take device memory.  Make that first
 * call before the host hands all free memory to its own allocator, and before any stream
 * capture; later calls allocate nothing.  Calls share the array: calls that overlap on the
 * GPU (other streams, other threads) race and must be serialised.
 * Arguments as shg_solve_batch_device; sh_power_out (host, may be NULL) synchronises, and a
 * NaN or Inf SH or pump power then returns SHG_ERR_NONFINITE naming the instance.
 */
SHG_API shg_status shg_solve_batch_device_noalloc(const shg_params* params, int32_t count,
                                                  void* const* pump_out_dev, void* const* signal_out_dev,
                                                  double* sh_power_out, void* stream);

/*
 * `sweeps` Jacobi sweeps of the heat equation on caller device buffers, without
 * convergence checks: the Tfield::upDate loop of the thermal run (Tfield.h:350-364,
 * Solver.h:339-355; kernelHeatEquationTopOpen / OvenSurrounded, Tfield.h:93-240).
 *   temperature_dev  nx*ny*nz reals: the starting temperature on entry, the result on
 *                    return; voxels the model holds fixed (Dirichlet faces) keep their value.
 *   q_dev            nx*ny*nz reals: the heat source Q.
 * Uses the grid, precision, kappa, h_conv, t_inf, boundary and jacobi_block of *p (p->thermal
 * is ignored).  Both buffers aligned to two reals (8 bytes in FP32, 16 in FP64; any cudaMalloc
 * pointer is), else SHG_ERR_INVALID.  Stream-ordered on `stream`; synchronises once at the end.
 */
SHG_API shg_status shg_heat_sweeps_device(const shg_params* p, void* temperature_dev, const void* q_dev,
                                          int64_t sweeps, void* stream);

/*
 * The temperature that shg_heat_sweeps_device's sweeps converge to, computed directly: the
 * fixed point T = J(T) of one Jacobi sweep J for the heat source Q.  No counterpart in the
 * reference, whose Jacobi loop (Solver.h:339-355) approaches it one sweep at a time.
 * With the faces' coefficients of Tfield.h:93-240 scaled to a common form the sweep's linear
 * system is the sum of three one-dimensional operators (Robin, or next to a Dirichlet face,
 * at each end); the solve diagonalises the x and y operators (FP64 transforms cached per
 * device and operator) and solves a tridiagonal system along z for every (x, y) mode.
 *   temperature_dev  nx*ny*nz reals: the Dirichlet voxels hold their values on entry and keep
 *                    them; every other voxel receives the solution (rounded to the precision).
 *   q_dev            nx*ny*nz reals: the heat source Q, or NULL for none.
 *   residual_out     optional: max |J(T) - T| of one FP64 Jacobi sweep applied to the FP64
 *                    solution (the sweep's own measure of how far T is from its fixed point).
 * Uses the grid, precision, kappa, h_conv, t_inf and boundary of *p.  Works in FP64 with two
 * workspace buffers of nx*ny*nz doubles from the stream's pool.  Stream-ordered on `stream`;
 * synchronises once at the end.
 */
SHG_API shg_status shg_heat_steady_device(const shg_params* p, void* temperature_dev, const void* q_dev,
                                          double* residual_out, void* stream);

/*
 * The one-dimensional operator of the direct heat solve for one grid direction, and its
 * eigendecomposition (host only; no device needed).  m unknowns at spacing d; each end is
 * next to a Dirichlet voxel (robin = 0) or a Robin face with Biot number bi (robin = 1).  In the
 * scaled form each row reads (2u_i - u_{i-1} - u_{i+1}) / d^2, and a Robin end row
 * (2(1 + bi) u_0 - 2 u_1) / d^2.  On return lambda_out[k] (m) are its eigenvalues,
 * forward_out (m x m, row-major, row k) maps values to mode amplitudes and inverse_out
 * (m x m, row-major, row i) maps them back: M = inverse * diag(lambda) * forward and
 * forward * inverse = I.
 */
SHG_API shg_status shg_heat_operator_modes(int32_t m, double d, int32_t lo_robin, int32_t hi_robin, double bi,
                                           double* lambda_out, double* forward_out, double* inverse_out);

/*
 * A batch of thermal runs: the -DTHERMAL outer loop of Solver::run (Solver.h:321-373) for each
 * parameter set, which the reference's sweep script runs as one process per point
 * (cuSHG.sh:58-94), marched in lockstep on `stream`.  Every outer iteration runs each
 * instance's Jacobi loop (its own stopping rule and counts), then the optical passes of all
 * instances still iterating as one launch sequence of the thermal march (grids over the
 * instances), so the optical passes of small batches fill the GPU.  An instance stops after
 * its own last pass.  Each instance's fields, temperature, powers and counts equal its
 * shg_solve_device run bit for bit.  All instances share precision, grid side, nz and march;
 * thermal == 1.
 *   pump_out_dev, signal_out_dev, temperature_out_dev  arrays of count device buffers, or NULL
 *                  (an array, or any entry of one); fields nx*ny complex, temperature nx*ny*nz.
 *   stats          count entries, or NULL; device_ms is the whole batch's time, optics_ms the
 *                  time of the batched optical passes the instance took part in.
 *   d_temp_out     count doubles (host), or NULL.  With it, each instance's dJ/dT_oven as
 *                  shg_thermal_grad computes it (grid sides 256 and 512, round beams), with the
 *                  tangent marches of every outer iteration batched the same way.
 * Synchronises `stream` before returning.  No counterpart in the reference.
 */
SHG_API shg_status shg_thermal_batch(const shg_params* params, int32_t count, void* const* pump_out_dev,
                                     void* const* signal_out_dev, void* const* temperature_out_dev,
                                     shg_stats* stats, double* d_temp_out, void* stream);

/*
 * Diagnostics: the bounded wait of the TMA-staged Jacobi sweeps (jacobi_block >= 2).  Runs two
 * blocked sweeps of a 64 x 64 x 32 grid with every wait for a staged plane limited to wait_us
 * microseconds and, with withhold_plane in 0..31, that plane's staging never issued, so its
 * wait runs out: the kernel then stops, waits (bounded) for the loads it did issue, and
 * reports through a status word.  Returns SHG_ERR_CUDA when a wait ran out, SHG_OK when every
 * plane arrived (withhold_plane = -1).  The device stays usable either way.  No counterpart
 * in the reference.
 */
SHG_API shg_status shg_selftest_bounded_wait(int32_t precision, double wait_us, int32_t withhold_plane);

/* Gradients of the SH output power (plain runs), from shg_grad. */
typedef struct shg_grad_result {
    double sh_power;          /* J = SH output power [W] */
    double d_waist;           /* dJ/dwaist [W/µm] */
    double d_focus;           /* dJ/dfocus [W/µm] */
    double d_temp;            /* dJ/dtemp [W/K]: the oven temperature of a plain run (n, Δk, pump, propagators) */
    double* d_poling;         /* caller array of shg_steps(p) values dJ/dφ_s [W/rad], or NULL */
    double device_ms;         /* device time of the forward + adjoint march */
    int32_t checkpoint_every; /* checkpoint interval used (steps) */
    int32_t steps;            /* steps marched */
    double reserved[4];
} shg_grad_result;

/*
 * Gradient of the SH output power of a plain run by the adjoint of the SSFM march.  No
 * counterpart in the reference (which computes no power and no gradients); the forward
 * model is the reference's scheme.  poling: NULL or shg_steps(p) phases [rad], a per-step
 * phase of the QPM grating added to the mismatch phase of that step's RK4 stages (zero for
 * the reference's uniform grating).  checkpoint_every: fields are kept every that many steps
 * and re-marched in between (<= 0: about sqrt(steps); >= steps: every step is kept and
 * nothing is re-marched).  Host buffers, synchronous.
 */
SHG_API shg_status shg_grad(const shg_params* p, const double* poling, int32_t checkpoint_every,
                            shg_grad_result* out);

/*
 * Gradients of `count` plain runs in one launch (one thread-block cluster per instance), for
 * sweeps and optimisers that need many gradients at once.  All instances share precision and
 * grid side (nz and every other parameter may differ).  poling: NULL, or an array of `count`
 * pointers each NULL or to shg_steps(&params[i]) phases.  out[i] as for shg_grad (its
 * d_poling, if set, receives instance i's vector); device_ms is the whole launch.
 * checkpoint_every <= 0 keeps every step's fields (no re-march) when the batch's clusters
 * cover every SM and its workspace fits in half the free device memory, else about
 * sqrt(steps); out[i].checkpoint_every says which.  No counterpart in the reference.
 */
SHG_API shg_status shg_grad_batch(const shg_params* params, int32_t count, const double* const* poling,
                                  int32_t checkpoint_every, shg_grad_result* out);

/* Result of shg_thermal_grad. */
typedef struct shg_thermal_grad_result {
    double sh_power;               /* SH output power of the thermal run [W] */
    double d_temp;                 /* dJ/dT_oven [W/K] through the converged temperature field */
    double sh_power_tangent_march; /* J as the tangent march recomputes it (a consistency check) */
    double device_ms;              /* device time of the run and its tangent */
    shg_stats stats;               /* the thermal run's report */
    double reserved[4];
} shg_thermal_grad_result;

/*
 * A thermal run (thermal == 1, as shg_solve) and the derivative of its SH output power with
 * respect to the oven temperature, i.e. temp and t_peltier moved together (the reference
 * passes argv[3] as both, src/cuSHG.cu:51-53).  Forward mode: the temperature field's
 * derivative is the homogeneous Jacobi iteration from a field of ones over the run's total
 * sweep count (recomputed, not stored), then a tangent-linear march of the last optical pass
 * through the per-voxel n_p, n_s, Δk and the centre-voxel pump and propagators.  The heat
 * source Q is held fixed in the derivative: first order in the optical-thermal coupling, exact
 * when Q does not depend on the oven temperature.  Grid sides 256 and 512, round beams.
 * Synchronous.  No counterpart in the reference.
 */
SHG_API shg_status shg_thermal_grad(const shg_params* p, shg_thermal_grad_result* out);

/* SH output power of a plain run with an optional per-step poling phase (as shg_grad),
 * forward only.  Host, synchronous. */
SHG_API shg_status shg_sh_power(const shg_params* p, const double* poling, double* sh_power);

/* Message of the last failing call on this thread ("" if none). */
SHG_API const char* shg_last_error(void);
SHG_API const char* shg_status_string(int32_t status);

/* Library version string. */
SHG_API const char* shg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CUSHG_B200_SHG_H */
