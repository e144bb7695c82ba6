// thermal.h — launchers of the heat-solve and temperature-optics kernels (thermal.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/shg.h"

namespace shg {

// Coefficients of one Jacobi sweep of kernelHeatEquationTopOpen / OvenSurrounded
// (src/headers/Tfield.h:99-106, 211-215), computed in FP64 and rounded to R; divisions
// of the reference become multiplications by these reciprocals.
template <typename R>
struct JacobiCoef {
    int n, nz;
    R L2, idx2, idy2, idz2, iK, Tinf;
    R Bix, Biy, Biz;
    R ax, ay, az, bx, by, bz, fx, fy, fz;
    R av, bv, cv, V, tv;
    R ah, bh, ch, H, th;
    R ad, bd, cd, D, td;
    R AV, BV, CV, BiD, GV;
};

template <typename R> JacobiCoef<R> make_jacobi_coef(const shg_params& p);
template <typename R> cudaError_t launch_thermal_init(R* Ta, R* Tb, R* Q, const shg_params& p, cudaStream_t s);
template <typename R> cudaError_t launch_optics(const R* T, R* dk, R* np, R* ns, const shg_params& p, cudaStream_t s);
// u * (dΔk/dT, dn_p/dT, dn_s/dT) at every voxel (u = dT/dT_oven)
template <typename R>
cudaError_t launch_optics_tangent(const R* T, const R* u, R* ddk, R* dnp, R* dns, const shg_params& p, cudaStream_t s);
template <typename R> cudaError_t launch_fill(R* a, size_t total, R v, cudaStream_t s);
// one sweep Ti -> Tf; with resid, also the convergence value of that sweep into *out
template <typename R>
cudaError_t launch_jacobi(const R* Ti, R* Tf, const R* Q, const JacobiCoef<R>& k, int boundary, bool resid, int rule,
                          double* partial, double* out, cudaStream_t s);
size_t jacobi_partials(const shg_params& p);

// Temporally blocked sweeps (jacobi_tb.cu): `depth` (2..4) sweeps Ti -> Tf in one launch,
// with Ti and Q read through 3D TMA maps made by make_tb_map.  *err is set to 1 if a
// staged plane never arrived.
int jacobi_tb_chunk(int tiles, int nz, int depth, int sms);
template <typename R> shg_status make_tb_map(const R* base, int n, int nz, CUtensorMap* map);
// Bound of each wait for a staged plane (2 s by default: a plane that takes longer is an
// error), and a plane never staged (the self-test of that bound; -1: none).
struct TbWait {
    uint64_t limit_ns = 2000000000ull;
    int withhold = -1;
};
template <typename R>
cudaError_t launch_jacobi_tb(const CUtensorMap& tmT, const CUtensorMap& tmQ, R* Tf, const JacobiCoef<R>& k,
                             int boundary, int depth, unsigned* err, cudaStream_t s, TbWait w = TbWait());

// The fixed point of the Jacobi sweeps for a heat source, solved directly (heat_direct.cu).
// One object holds the FP64 workspace of one grid size; its solves run in stream order, so
// the instances of a batch and their tangents share it.
class HeatDirect {
  public:
    HeatDirect() = default;
    HeatDirect(const HeatDirect&) = delete;
    HeatDirect& operator=(const HeatDirect&) = delete;
    ~HeatDirect();
    // T (n*n*nz): Dirichlet voxels keep their values, the others receive the fixed point for
    // heat source Q (NULL: none) and environment temperature t_inf; p gives the grid,
    // boundary, kappa and h_conv.
    template <typename R>
    shg_status solve(const shg_params& p, R* T, const R* Q, double t_inf, cudaStream_t s);
    // Of the latest solve (synchronises s): the FP64 Jacobi-sweep residual of the solution and
    // the change from the temperature T held before, each as the `rule` measures it
    // (SHG_CONV_REFERENCE: sqrt(sum d^2) / voxels; otherwise max |d|).
    shg_status result(int rule, double* residual, double* change, cudaStream_t s);
    // Frees the workspace on s (which must outlive the call).
    void release(cudaStream_t s);

  private:
    double* ws_ = nullptr;  // two compact FP64 volumes, then the four reduction slots
    size_t cap_ = 0;        // doubles per volume
    size_t nt_ = 0;         // voxels of the latest solve
};

}  // namespace shg
