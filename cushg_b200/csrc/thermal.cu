// thermal.cu — kernels of the 3D heat solve and the temperature-dependent optics.
//
// Reference counterparts (src/headers/Tfield.h, PhaseMatching.h):
//   kernelSetTemperature / kernelSetBottomOvensTemperature / kernelSetOvenSurrounded
//       -> thermal_init_kernel
//   kernelHeatEquationTopOpen / kernelHeatEquationOvenSurrounded (one Jacobi sweep)
//       -> jacobi_zb2_kernel (unchecked sweeps) and jacobi_kernel (the checked sweep of each
//          window); Ti -> Tf, the reference's Tf -> Ti device copy after every sweep becomes
//          a ping-pong of two buffers
//   kernelDifSquareVectors + thrust::reduce (checkConvergence)
//       -> the RESID form of jacobi_kernel (per-block partials) + reduce_partials_kernel
//   kernelSetInicialDKThermal and the per-voxel n(λ, T) of dAdz / kernelSetQ
//       -> optics_kernel (Δk, n_p, n_s per voxel, once per optical pass)
#include <cuda_runtime.h>

#include <cstdint>

#include "crystal.cuh"
#include "jacobi_point.cuh"
#include "shg_host.h"
#include "thermal.h"

namespace shg {

template <typename R>
__global__ void thermal_init_kernel(R* Ta, R* Tb, R* Q, int n, int nz, R temp, R tpelt, int boundary) {
    const size_t total = (size_t)n * n * nz;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % n), y = (int)((i / n) % n);
        bool face;
        if (boundary == SHG_BOUNDARY_OVEN_SURROUNDED) face = (y == 0 || y == n - 1 || x == 0 || x == n - 1);
        else face = (y == 0);
        const R v = face ? tpelt : temp;
        Ta[i] = v;
        Tb[i] = v;
        Q[i] = (R)0;
    }
}

// Δk (PhaseMatching.h:47-65), n(λp, T) and n(λs, T) at every voxel, in FP64 (crystal.cuh).
template <typename R>
__global__ void optics_kernel(const R* __restrict__ T, R* __restrict__ dk, R* __restrict__ np, R* __restrict__ ns,
                              size_t total, double lp, double period, int crystal) {
    const double ls = 0.5 * lp;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const double t = (double)T[i];
        dk[i] = (R)crystal_delta_k(crystal, lp, period, t);
        np[i] = (R)crystal_n(crystal, lp, t);
        ns[i] = (R)crystal_n(crystal, ls, t);
    }
}

// Derivatives of the per-voxel optics with respect to the oven temperature: u = dT/dT_oven at
// every voxel times dn/dT and dΔk/dT, both in closed form (crystal.cuh), in FP64.
template <typename R>
__global__ void optics_tangent_kernel(const R* __restrict__ T, const R* __restrict__ u, R* __restrict__ ddk,
                                      R* __restrict__ dnp, R* __restrict__ dns, size_t total, double lp,
                                      double period, int crystal) {
    const double ls = 0.5 * lp;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const double t = (double)T[i], w = (double)u[i];
        ddk[i] = (R)(crystal_ddk_dT(crystal, lp, period, t) * w);
        dnp[i] = (R)(crystal_dn_dT(crystal, lp, t) * w);
        dns[i] = (R)(crystal_dn_dT(crystal, ls, t) * w);
    }
}

template <typename R>
__global__ void fill_kernel(R* __restrict__ a, size_t total, R v) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) a[i] = v;
}

// One Jacobi sweep Ti -> Tf.  Thread block (32, 8) over (x, y), one z plane per grid z.
// Voxels the reference never writes (the Dirichlet faces) are left untouched, which with
// two buffers initialised alike keeps them at the oven temperature in both.
// RESID: each block also writes its partial of sum (Tf - Ti)^2 (rule 0) or max |Tf - Ti|.
template <typename R, int BOUND, bool RESID>
__global__ void __launch_bounds__(256) jacobi_kernel(const R* __restrict__ Ti, R* __restrict__ Tf, const R* __restrict__ Q,
                                                     JacobiCoef<R> k, int rule, double* __restrict__ partial) {
    const int n = k.n;
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    double dres = 0.0;
    if (x < n && y < n) {
        const size_t sy = (size_t)n, sz = (size_t)n * n;
        const size_t i = (size_t)z * sz + (size_t)y * sy + x;
        auto get = [&](int dx, int dy, int dz) -> R { return Ti[i + (ptrdiff_t)dz * sz + (ptrdiff_t)dy * sy + dx]; };
        R v;
        if (jacobi_point<R, BOUND>(x, y, z, k, Q[i], get, &v)) {
            Tf[i] = v;
            if (RESID) {
                const double dd = (double)(R)(v - Ti[i]);
                dres = rule == SHG_CONV_MAXABS ? fabs(dd) : dd * dd;
            }
        }
    }
    if (RESID) {
        const bool mx = rule == SHG_CONV_MAXABS;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double other = __shfl_down_sync(0xffffffffu, dres, o);
            dres = mx ? fmax(dres, other) : dres + other;
        }
        __shared__ double wsum[8];
        const int w = threadIdx.y;
        if (threadIdx.x == 0) wsum[w] = dres;
        __syncthreads();
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            double a = 0.0;
            for (int q = 0; q < 8; ++q) a = mx ? fmax(a, wsum[q]) : a + wsum[q];
            partial[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = a;
        }
    }
}

// Unchecked Jacobi sweeps Ti -> Tf, z-blocked: a thread walks a column of ZB planes,
// keeping T at z-1, z and z+1 in registers as it goes up, so each voxel costs one new load of
// the centre column and its lateral neighbours, and the boundary classification and index
// arithmetic are paid once per column step.
//
// One voxel per thread with every neighbour loaded was bound by instruction issue in FP32 (91
// thread instructions per voxel, DRAM at 34 % of peak at 256x256x400).  Measured per sweep:
//   FP32 512x512x250: 249 us (one voxel) -> 203 (z-blocked) -> 166 (z-blocked, pairs), 4.7 TB/s
//   FP64 512x512x250: 318 us (one voxel) -> 282 (z-blocked, pairs), 5.6 TB/s
//   FP64 128x128x200 (L2-resident): 16.6 -> 14.5 us
// Planes per z-block: 16.  Per sweep at 512x512x250, z-blocks of 4 / 8 / 16 planes measured
// 145 / 142 / 141 us (FP32) and 286 / 280 / 276 us (FP64); at 128x128x200 FP64 all three take
// 14.4 us (the 79 MB sweep streams at HBM speed either way).
constexpr int kJacobiZB = 16;

// The z-blocked sweep with two x-adjacent voxels per thread: the centre column, its y
// neighbours and Q are read as float2 / double2 (rows are 8- / 16-byte aligned since n is
// even), the x neighbours outside the pair as scalars.  Each voxel is still jacobi_point of
// the same operands.  Thread block (32, 8) covers 64 x 8 voxels; grid (n/64, n/8, nz/ZB).
template <typename R> struct pair_t;
template <> struct pair_t<float> { using type = float2; };
template <> struct pair_t<double> { using type = double2; };

template <typename R, int BOUND>
__global__ void __launch_bounds__(256, 5) jacobi_zb2_kernel(const R* __restrict__ Ti, R* __restrict__ Tf,
                                                         const R* __restrict__ Q, JacobiCoef<R> k) {
    using R2 = typename pair_t<R>::type;
    const int n = k.n, nz = k.nz;
    const int x = 2 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= n || y >= n) return;
    const int z0 = blockIdx.z * kJacobiZB, z1 = min(nz, z0 + kJacobiZB);
    const size_t sy = (size_t)n, sz = (size_t)n * n;
    size_t i = (size_t)z0 * sz + (size_t)y * sy + x;
    auto ld2 = [&](size_t j) { return *reinterpret_cast<const R2*>(Ti + j); };
    R2 zero2;
    zero2.x = zero2.y = (R)0;
    R2 below = z0 > 0 ? ld2(i - sz) : zero2;
    R2 cur = ld2(i);
    // both voxels of the pair are inner in x and y (a pair starts at an even x)
    const bool inner_xy = x >= 2 && x + 3 < n && y >= 1 && y + 1 < n;
#pragma unroll 2
    for (int z = z0; z < z1; ++z, i += sz) {
        const R2 above = z + 1 < nz ? ld2(i + sz) : zero2;
        const R2 ym = y > 0 ? ld2(i - sy) : zero2, yp = y + 1 < n ? ld2(i + sy) : zero2;
        const R xm = x > 0 ? Ti[i - 1] : (R)0, xp = x + 2 < n ? Ti[i + 2] : (R)0;
        const R2 q = Q ? *reinterpret_cast<const R2*>(Q + i) : zero2;  // Q null: no heat source
        auto get0 = [&](int dx, int dy, int dz) -> R {
            if (dz) return dz > 0 ? above.x : below.x;
            if (dy) return dy > 0 ? yp.x : ym.x;
            return dx > 0 ? cur.y : xm;
        };
        auto get1 = [&](int dx, int dy, int dz) -> R {
            if (dz) return dz > 0 ? above.y : below.y;
            if (dy) return dy > 0 ? yp.y : ym.y;
            return dx > 0 ? xp : cur.x;
        };
        R v0, v1;
        bool w0 = true, w1 = true;
        if (inner_xy && z >= 1 && z + 1 < nz) {
            // inner voxels: jacobi_point's inner branch without the classification
            v0 = jacobi_inner<R>(cur.y, xm, yp.x, ym.x, above.x, below.x, q.x, k);
            v1 = jacobi_inner<R>(xp, cur.x, yp.y, ym.y, above.y, below.y, q.y, k);
        } else {
            w0 = jacobi_point<R, BOUND>(x, y, z, k, q.x, get0, &v0);
            w1 = jacobi_point<R, BOUND>(x + 1, y, z, k, q.y, get1, &v1);
        }
        if (w0 && w1) {
            R2 o;
            o.x = v0;
            o.y = v1;
            *reinterpret_cast<R2*>(Tf + i) = o;
        } else {
            if (w0) Tf[i] = v0;
            if (w1) Tf[i + 1] = v1;
        }
        below = cur;
        cur = above;
    }
}

// FP32: the same sweep with four x-adjacent voxels per thread (float4 loads of the centre
// column, its y neighbours and Q; the x neighbours outside the quad as scalars), half the
// loads and index arithmetic per voxel of the pairs.  Launched when n is a multiple of 4 and
// the three arrays are 16-byte aligned (launch_jacobi checks both), so the quads tile every
// row and every float4 access is aligned; otherwise the pairs run.  Each voxel is
// jacobi_point / jacobi_inner of the same operands as in every other sweep kernel.  Thread
// block (32, 8) covers 128 x 8 voxels; grid (n/128, n/8, nz/ZB).
template <int BOUND>
__global__ void __launch_bounds__(256) jacobi_zb4_kernel(const float* __restrict__ Ti, float* __restrict__ Tf,
                                                         const float* __restrict__ Q, JacobiCoef<float> k) {
    using R = float;
    const int n = k.n, nz = k.nz;
    const int x = 4 * (blockIdx.x * 32 + threadIdx.x);
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= n || y >= n) return;
    const int z0 = blockIdx.z * kJacobiZB, z1 = min(nz, z0 + kJacobiZB);
    const size_t sy = (size_t)n, sz = (size_t)n * n;
    size_t i = (size_t)z0 * sz + (size_t)y * sy + x;
    auto ld4 = [&](size_t j) { return *reinterpret_cast<const float4*>(Ti + j); };
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    auto arr = [](float4 v, R* a) { a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w; };
    R below[4], cur[4];
    arr(z0 > 0 ? ld4(i - sz) : zero4, below);
    arr(ld4(i), cur);
    // all four voxels of the quad are inner in x and y (a quad starts at a multiple of 4)
    const bool inner_xy = x >= 4 && x + 4 < n && y >= 1 && y + 1 < n;
#pragma unroll 1
    for (int z = z0; z < z1; ++z, i += sz) {
        R above[4], ym[4], yp[4], q[4], v[4];
        arr(z + 1 < nz ? ld4(i + sz) : zero4, above);
        arr(y > 0 ? ld4(i - sy) : zero4, ym);
        arr(y + 1 < n ? ld4(i + sy) : zero4, yp);
        arr(Q ? *reinterpret_cast<const float4*>(Q + i) : zero4, q);  // Q null: no heat source
        const R xm = x > 0 ? Ti[i - 1] : (R)0, xp = x + 4 < n ? Ti[i + 4] : (R)0;
        bool w[4] = {true, true, true, true};
        if (inner_xy && z >= 1 && z + 1 < nz) {
            // inner voxels: jacobi_point's inner branch without the classification
#pragma unroll
            for (int j = 0; j < 4; ++j)
                v[j] = jacobi_inner<R>(j < 3 ? cur[j + 1] : xp, j > 0 ? cur[j - 1] : xm, yp[j], ym[j], above[j],
                                       below[j], q[j], k);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                auto get = [&](int dx, int dy, int dz) -> R {
                    if (dz) return dz > 0 ? above[j] : below[j];
                    if (dy) return dy > 0 ? yp[j] : ym[j];
                    return dx > 0 ? (j < 3 ? cur[j + 1] : xp) : (j > 0 ? cur[j - 1] : xm);
                };
                w[j] = jacobi_point<R, BOUND>(x + j, y, z, k, q[j], get, &v[j]);
            }
        }
        if (w[0] && w[1] && w[2] && w[3]) {
            *reinterpret_cast<float4*>(Tf + i) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (w[j]) Tf[i + j] = v[j];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            below[j] = cur[j];
            cur[j] = above[j];
        }
    }
}

// Deterministic second stage: one block sums (or maxes) the partials in a fixed order.
__global__ void reduce_partials_kernel(const double* __restrict__ partial, size_t count, int rule, double* out) {
    __shared__ double s[256];
    const bool mx = rule == SHG_CONV_MAXABS;
    double a = 0.0;
    for (size_t i = threadIdx.x; i < count; i += blockDim.x) a = mx ? fmax(a, partial[i]) : a + partial[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] = mx ? fmax(s[threadIdx.x], s[threadIdx.x + o]) : s[threadIdx.x] + s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

template <typename R>
JacobiCoef<R> make_jacobi_coef(const shg_params& p) {
    JacobiCoef<R> k;
    const double dx = p.lx / (p.nx - 1), dy = p.ly / (p.ny - 1), dz = p.lz / (p.nz - 1);
    const double K = p.kappa, h = p.h_conv, Tinf = p.t_inf;
    const double Bix = h * dx / K, Biy = h * dy / K, Biz = h * dz / K;
    const double ax = dx * dx / (2 * dy * dy), ay = dy * dy / (2 * dx * dx), az = dz * dz / (2 * dx * dx);
    const double bx = dx * dx / (2 * dz * dz), by = dy * dy / (2 * dz * dz), bz = dz * dz / (2 * dy * dy);
    const double av = dz / (2 * dx), bv = dx / (2 * dz), cv = dx * dz / (4 * dy * dy);
    const double ah = dz / (2 * dy), bh = dy / (2 * dz), ch = dy * dz / (4 * dx * dx);
    const double ad = dx / (2 * dy), bd = dy / (2 * dx), cd = dx * dy / (4 * dz * dz);
    const double AV = dy * dz / dx, BV = dx * dz / dy, CV = dx * dy / dz, BiD = Bix * dy + Biy * dz + Biz * dx;
    k.n = p.nx;
    k.nz = p.nz;
    k.L2 = (R)(1 / (2 / (dx * dx) + 2 / (dy * dy) + 2 / (dz * dz)));
    k.idx2 = (R)(1 / (dx * dx));
    k.idy2 = (R)(1 / (dy * dy));
    k.idz2 = (R)(1 / (dz * dz));
    k.iK = (R)(1 / K);
    k.Tinf = (R)Tinf;
    k.Bix = (R)Bix; k.Biy = (R)Biy; k.Biz = (R)Biz;
    k.ax = (R)ax; k.ay = (R)ay; k.az = (R)az; k.bx = (R)bx; k.by = (R)by; k.bz = (R)bz;
    k.fx = (R)(1 / (1 + 2 * ax + 2 * bx + Bix));
    k.fy = (R)(1 / (1 + 2 * ay + 2 * by + Biy));
    k.fz = (R)(1 / (1 + 2 * az + 2 * bz + Biz));
    k.av = (R)av; k.bv = (R)bv; k.cv = (R)cv;
    k.V = (R)(1 / (av + bv + 2 * cv + 0.5 * (Bix + Biz)));
    k.tv = (R)(0.5 * Tinf * (Bix + Biz));
    k.ah = (R)ah; k.bh = (R)bh; k.ch = (R)ch;
    k.H = (R)(1 / (ah + bh + 2 * ch + 0.5 * (Biy + Biz)));
    k.th = (R)(0.5 * Tinf * (Biy + Biz));
    k.ad = (R)ad; k.bd = (R)bd; k.cd = (R)cd;
    k.D = (R)(1 / (ad + bd + 2 * cd + 0.5 * (Bix + Biy)));
    k.td = (R)(0.5 * Tinf * (Bix + Biy));
    k.AV = (R)AV; k.BV = (R)BV; k.CV = (R)CV; k.BiD = (R)BiD;
    k.GV = (R)(1 / (AV + BV + CV + BiD));
    return k;
}

template <typename R>
cudaError_t launch_thermal_init(R* Ta, R* Tb, R* Q, const shg_params& p, cudaStream_t s) {
    const size_t total = (size_t)p.nx * p.nx * p.nz;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    thermal_init_kernel<R><<<blocks, 256, 0, s>>>(Ta, Tb, Q, p.nx, p.nz, (R)p.temp, (R)p.t_peltier, p.boundary);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_optics(const R* T, R* dk, R* np, R* ns, const shg_params& p, cudaStream_t s) {
    const size_t total = (size_t)p.nx * p.nx * p.nz;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    optics_kernel<R><<<blocks, 256, 0, s>>>(T, dk, np, ns, total, p.lambda_p, p.period, p.crystal);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_optics_tangent(const R* T, const R* u, R* ddk, R* dnp, R* dns, const shg_params& p, cudaStream_t s) {
    const size_t total = (size_t)p.nx * p.nx * p.nz;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    optics_tangent_kernel<R><<<blocks, 256, 0, s>>>(T, u, ddk, dnp, dns, total, p.lambda_p, p.period, p.crystal);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_fill(R* a, size_t total, R v, cudaStream_t s) {
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    fill_kernel<R><<<blocks, 256, 0, s>>>(a, total, v);
    return cudaGetLastError();
}

size_t jacobi_partials(const shg_params& p) {
    return (size_t)((p.nx + 31) / 32) * ((p.nx + 7) / 8) * p.nz;
}

template <typename R>
cudaError_t launch_jacobi(const R* Ti, R* Tf, const R* Q, const JacobiCoef<R>& k, int boundary, bool resid, int rule,
                          double* partial, double* out, cudaStream_t s) {
    dim3 block(32, 8, 1);
    dim3 grid((k.n + 31) / 32, (k.n + 7) / 8, k.nz);
    if (!resid) {
        if constexpr (sizeof(R) == 4) {
            auto al16 = [](const void* a) { return ((uintptr_t)a & 15) == 0; };
            if ((k.n & 3) == 0 && al16(Ti) && al16(Tf) && al16(Q)) {
                // quads tile every row when n is a multiple of 4, and every row starts
                // 16-byte aligned when the arrays do
                const dim3 qgrid((k.n + 127) / 128, grid.y, (k.nz + kJacobiZB - 1) / kJacobiZB);
                if (boundary == SHG_BOUNDARY_OVEN_SURROUNDED)
                    jacobi_zb4_kernel<SHG_BOUNDARY_OVEN_SURROUNDED><<<qgrid, block, 0, s>>>(Ti, Tf, Q, k);
                else
                    jacobi_zb4_kernel<SHG_BOUNDARY_TOP_OPEN><<<qgrid, block, 0, s>>>(Ti, Tf, Q, k);
                return cudaGetLastError();
            }
        }
        // n is even (shg_check_params), so the voxel pairs tile every row
        const dim3 zgrid((k.n + 63) / 64, grid.y, (k.nz + kJacobiZB - 1) / kJacobiZB);
        if (boundary == SHG_BOUNDARY_OVEN_SURROUNDED)
            jacobi_zb2_kernel<R, SHG_BOUNDARY_OVEN_SURROUNDED><<<zgrid, block, 0, s>>>(Ti, Tf, Q, k);
        else
            jacobi_zb2_kernel<R, SHG_BOUNDARY_TOP_OPEN><<<zgrid, block, 0, s>>>(Ti, Tf, Q, k);
        return cudaGetLastError();
    }
    if (boundary == SHG_BOUNDARY_OVEN_SURROUNDED) {
        if (resid) jacobi_kernel<R, SHG_BOUNDARY_OVEN_SURROUNDED, true><<<grid, block, 0, s>>>(Ti, Tf, Q, k, rule, partial);
        else jacobi_kernel<R, SHG_BOUNDARY_OVEN_SURROUNDED, false><<<grid, block, 0, s>>>(Ti, Tf, Q, k, rule, partial);
    } else {
        if (resid) jacobi_kernel<R, SHG_BOUNDARY_TOP_OPEN, true><<<grid, block, 0, s>>>(Ti, Tf, Q, k, rule, partial);
        else jacobi_kernel<R, SHG_BOUNDARY_TOP_OPEN, false><<<grid, block, 0, s>>>(Ti, Tf, Q, k, rule, partial);
    }
    if (resid) reduce_partials_kernel<<<1, 256, 0, s>>>(partial, (size_t)grid.x * grid.y * grid.z, rule, out);
    return cudaGetLastError();
}

template JacobiCoef<float> make_jacobi_coef<float>(const shg_params&);
template JacobiCoef<double> make_jacobi_coef<double>(const shg_params&);
template cudaError_t launch_thermal_init<float>(float*, float*, float*, const shg_params&, cudaStream_t);
template cudaError_t launch_thermal_init<double>(double*, double*, double*, const shg_params&, cudaStream_t);
template cudaError_t launch_optics<float>(const float*, float*, float*, float*, const shg_params&, cudaStream_t);
template cudaError_t launch_optics<double>(const double*, double*, double*, double*, const shg_params&, cudaStream_t);
template cudaError_t launch_optics_tangent<float>(const float*, const float*, float*, float*, float*, const shg_params&,
                                                  cudaStream_t);
template cudaError_t launch_optics_tangent<double>(const double*, const double*, double*, double*, double*,
                                                   const shg_params&, cudaStream_t);
template cudaError_t launch_fill<float>(float*, size_t, float, cudaStream_t);
template cudaError_t launch_fill<double>(double*, size_t, double, cudaStream_t);
template cudaError_t launch_jacobi<float>(const float*, float*, const float*, const JacobiCoef<float>&, int, bool, int,
                                          double*, double*, cudaStream_t);
template cudaError_t launch_jacobi<double>(const double*, double*, const double*, const JacobiCoef<double>&, int, bool,
                                           int, double*, double*, cudaStream_t);

}  // namespace shg
