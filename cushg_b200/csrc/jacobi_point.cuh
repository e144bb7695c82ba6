// jacobi_point.cuh — the value of one voxel after one Jacobi sweep of the heat equation,
// shared by the one-sweep kernel (thermal.cu) and the temporally blocked kernel
// (jacobi_tb.cu) so that both evaluate the same expressions in the same order and give the
// same bits.
//
// Reference: kernelHeatEquationTopOpen, src/headers/Tfield.h:93-201 (inner points, Robin
// faces, edges and vertices; the y = 0 face is Dirichlet at the oven temperature) and
// kernelHeatEquationOvenSurrounded, Tfield.h:205-240 (four lateral faces at the oven
// temperature, Robin z faces).  The reference's divisions are multiplications by the
// reciprocals in JacobiCoef (computed once in FP64).
#pragma once

#include "../../include/shg.h"
#include "thermal.h"

namespace shg {

// The inner-point update (Tfield.h:113-115) from the six neighbours and Q; jacobi_point's inner
// branch, and the fast path of kernels that know a voxel is inner.
template <typename R>
__device__ __forceinline__ R jacobi_inner(R xp, R xm, R yp, R ym, R zp, R zm, R q, const JacobiCoef<R>& k) {
    return k.L2 * ((xp + xm) * k.idx2 + (yp + ym) * k.idy2 + (zp + zm) * k.idz2 + q * k.iK);
}

// get(dx, dy, dz) returns the current temperature of voxel (x+dx, y+dy, z+dz); only
// neighbours inside the grid are asked for.  q is Q at (x, y, z).  Returns false (and
// leaves *v alone) for voxels the reference never writes.
template <typename R, int BOUND, typename Get>
__device__ __forceinline__ bool jacobi_point(int x, int y, int z, const JacobiCoef<R>& k, R q, Get&& get, R* v) {
    const int n = k.n, nz = k.nz;
    const bool xi = x > 0 && x < n - 1, yi = y > 0 && y < n - 1, zi = z > 0 && z < nz - 1;
    if (BOUND == SHG_BOUNDARY_TOP_OPEN) {
        if (y == 0) return false;  // Dirichlet face at the oven temperature
        if (xi && yi && zi) {      // inner points (Tfield.h:113-115)
            *v = jacobi_inner<R>(get(1, 0, 0), get(-1, 0, 0), get(0, 1, 0), get(0, -1, 0), get(0, 0, 1), get(0, 0, -1), q, k);
        } else if (!xi && yi && zi) {  // faces x = 0 / x = Lx (Tfield.h:119-125)
            const int xn = x == 0 ? 1 : -1;
            *v = (get(xn, 0, 0) + k.ax * (get(0, 1, 0) + get(0, -1, 0)) + k.bx * (get(0, 0, 1) + get(0, 0, -1)) +
                  k.Bix * k.Tinf) * k.fx;
        } else if (xi && !yi && zi) {  // face y = Ly (Tfield.h:127-129)
            *v = (get(0, -1, 0) + k.ay * (get(1, 0, 0) + get(-1, 0, 0)) + k.by * (get(0, 0, 1) + get(0, 0, -1)) +
                  k.Biy * k.Tinf) * k.fy;
        } else if (xi && yi && !zi) {  // faces z = 0 / z = Lcr (Tfield.h:131-137)
            const int zn = z == 0 ? 1 : -1;
            *v = (get(0, 0, zn) + k.az * (get(1, 0, 0) + get(-1, 0, 0)) + k.bz * (get(0, 1, 0) + get(0, -1, 0)) +
                  k.Biz * k.Tinf) * k.fz;
        } else if (!xi && yi && !zi) {  // vertical edges (Tfield.h:143-157)
            const int xn = x == 0 ? 1 : -1, zn = z == 0 ? 1 : -1;
            *v = (k.av * get(xn, 0, 0) + k.bv * get(0, 0, zn) + k.cv * (get(0, 1, 0) + get(0, -1, 0)) + k.tv) * k.V;
        } else if (xi && !yi && !zi) {  // horizontal edges (Tfield.h:161-167)
            const int zn = z == 0 ? 1 : -1;
            *v = (k.ah * get(0, -1, 0) + k.bh * get(0, 0, zn) + k.ch * (get(-1, 0, 0) + get(1, 0, 0)) + k.th) * k.H;
        } else if (!xi && !yi && zi) {  // depth edges (Tfield.h:171-177)
            const int xn = x == 0 ? 1 : -1;
            *v = (k.ad * get(0, -1, 0) + k.bd * get(xn, 0, 0) + k.cd * (get(0, 0, 1) + get(0, 0, -1)) + k.td) * k.D;
        } else {  // vertices (Tfield.h:181-196)
            const int xn = x == 0 ? 1 : -1, zn = z == 0 ? 1 : -1;
            *v = (k.AV * get(xn, 0, 0) + k.BV * get(0, -1, 0) + k.CV * get(0, 0, zn) + k.Tinf * k.BiD) * k.GV;
        }
        return true;
    } else {
        if (!(xi && yi)) return false;  // lateral faces held at the oven temperature
        if (zi) {
            *v = jacobi_inner<R>(get(1, 0, 0), get(-1, 0, 0), get(0, 1, 0), get(0, -1, 0), get(0, 0, 1), get(0, 0, -1), q, k);
        } else {  // z faces (Tfield.h:229-236)
            const int zn = z == 0 ? 1 : -1;
            *v = (get(0, 0, zn) + k.az * (get(1, 0, 0) + get(-1, 0, 0)) + k.bz * (get(0, 1, 0) + get(0, -1, 0)) +
                  k.Biz * k.Tinf) * k.fz;
        }
        return true;
    }
}

}  // namespace shg
