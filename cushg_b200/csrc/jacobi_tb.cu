// jacobi_tb.cu — several Jacobi sweeps of the heat equation per launch (temporal blocking),
// with the temperature and heat-source planes staged into shared memory by TMA.
//
// The reference runs one sweep per kernel launch, copies Tf back to Ti and round-trips to
// the host after every sweep (src/headers/Solver.h:335-355, Tfield.h:350-364).  Between two
// convergence checks the sweeps are pure data movement over the 3D grid, so here TL of them
// (2..4) are fused into one pass over HBM:
//
//   * A CTA owns a 32 x 32 staged tile of the (x, y) plane.  Its output is the inner
//     TX x TY part; the rest is halo, recomputed by the neighbouring tiles.  The CTA streams
//     along z through a chunk of planes.
//   * Each iteration stages one plane of T and one of Q.  Thread 0 issues a 3D TMA load
//     (cp.async.bulk.tensor) two planes ahead, completing on an mbarrier.  Loads outside
//     the grid are zero-filled and never read by a grid voxel.
//   * Thread (u, v) keeps its own column in registers: the last three planes of every
//     level 0..TL-1, and Q of the last TL+1 planes.  So the z neighbours come from
//     registers.  The x / y neighbours come from the previous iteration's plane of the level
//     below, published in shared memory (two planes per level).  That needs one barrier per
//     iteration.
//   * Level l of iteration j is sweep l applied to plane j - l.  Level TL is written to HBM.
//
// Every voxel value is computed by jacobi_point (jacobi_point.cuh) from the same operands as
// in the one-sweep kernel.  TL fused sweeps therefore give the same bits as TL launches of
// jacobi_kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "jacobi_point.cuh"
#include "shg_host.h"
#include "thermal.h"

namespace shg {

namespace {

constexpr int kTbSide = 32;                    // staged tile side: a lane per column, a warp per row
constexpr int kTbThreads = kTbSide * kTbSide;  // one thread per staged column
constexpr int kTbSlots = 4;                    // staging ring of T and Q planes
constexpr int kTbAhead = 2;                    // planes in flight ahead of the one consumed

template <typename R, int TL>
struct TbCfg {
    static constexpr int A = 16 / (int)sizeof(R);    // TMA: x coordinate a multiple of 16 bytes
    static constexpr int HX = (TL + A - 1) / A * A;  // x halo: >= TL, a multiple of A
    static constexpr int TX = kTbSide - 2 * HX;      // output columns per tile
    static constexpr int TY = kTbSide - 2 * TL;      // output rows per tile
    static constexpr int PLANE = kTbSide * kTbSide;
    static constexpr int NPLANE = 2 * kTbSlots + 2 * (TL - 1);
    static constexpr size_t plane_bytes = sizeof(R) * PLANE;
    static constexpr size_t smem_bytes = plane_bytes * NPLANE + 8 * kTbSlots;
    static_assert(TL >= 2 && TX > 0 && TY > 0, "depth out of range");
    static_assert(TX % A == 0 && HX % A == 0, "every tile's x start must be 16-byte aligned");
    static_assert((kTbSide * sizeof(R)) % 16 == 0, "TMA box rows must be whole 16-byte units");
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase of parity `parity` of *b; false after `limit_ns` without completion.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, unsigned parity, uint64_t limit_ns) {
    if (mbar_try_wait(b, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(b, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

// 3D tiled TMA load of one box into shared memory, completing on *bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <typename R, int BOUND, int TL>
__global__ void __launch_bounds__(kTbThreads, 1)
    jacobi_tb_kernel(const __grid_constant__ CUtensorMap tmT, const __grid_constant__ CUtensorMap tmQ,
                     R* __restrict__ Tf, const JacobiCoef<R> k, int zc, unsigned* __restrict__ err, const TbWait w) {
    using Cfg = TbCfg<R, TL>;
    constexpr int W = kTbSide, PL = Cfg::PLANE;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R* sT = reinterpret_cast<R*>(smem_raw);  // kTbSlots staged T planes
    R* sQ = sT + kTbSlots * PL;              // kTbSlots staged Q planes
    R* sL = sQ + kTbSlots * PL;              // levels 1..TL-1, two planes each
    uint64_t* bar = reinterpret_cast<uint64_t*>(sL + 2 * (TL - 1) * PL);

    const int n = k.n, nz = k.nz;
    const int u = threadIdx.x % W, v = threadIdx.x / W;
    const int xs = (int)blockIdx.x * Cfg::TX - Cfg::HX, ys = (int)blockIdx.y * Cfg::TY - TL;
    const int gx = xs + u, gy = ys + v;
    const bool in_xy = gx >= 0 && gx < n && gy >= 0 && gy < n;
    const bool out_xy = u >= Cfg::HX && u < Cfg::HX + Cfg::TX;  // output column (rows: level TL's range)
    const int z0 = (int)blockIdx.z * zc, z1 = min(nz, z0 + zc);
    const int jb = max(0, z0 - TL), je = min(nz, z1 + TL), jl = z1 - 1 + TL;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTbSlots; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int j) {  // thread 0: stage plane j of T and of Q
        if (j == w.withhold) return;  // self-test: this plane's wait must run out
        const int s = (j - jb) % kTbSlots;
        mbar_expect_tx(&bar[s], 2u * (unsigned)Cfg::plane_bytes);
        tma_load_3d(sT + s * PL, &tmT, xs, ys, j, &bar[s]);
        tma_load_3d(sQ + s * PL, &tmQ, xs, ys, j, &bar[s]);
    };
    if (threadIdx.x == 0)
        for (int j = jb; j < min(je, jb + kTbAhead); ++j) issue(j);

    R ring[TL][3];  // own column, level l at planes (latest, latest - 1, latest - 2)
    R qr[TL + 1];   // own column, Q at planes j, j - 1, ..., j - TL
#pragma unroll
    for (int l = 0; l < TL; ++l) ring[l][0] = ring[l][1] = ring[l][2] = (R)0;
#pragma unroll
    for (int l = 0; l <= TL; ++l) qr[l] = (R)0;

    bool timed_out = false;
    int jstop = jl + 1;
    for (int j = jb; j <= jl; ++j) {
        if (threadIdx.x == 0 && j + kTbAhead < je) issue(j + kTbAhead);
#pragma unroll
        for (int l = 0; l < TL; ++l) {
            ring[l][2] = ring[l][1];
            ring[l][1] = ring[l][0];
        }
#pragma unroll
        for (int l = TL; l > 0; --l) qr[l] = qr[l - 1];
        if (j < je) {
            const int s = (j - jb) % kTbSlots;
            if (!mbar_wait_bounded(&bar[s], (unsigned)((j - jb) / kTbSlots) & 1u, w.limit_ns)) timed_out = true;
            ring[0][0] = sT[s * PL + v * W + u];
            qr[0] = sQ[s * PL + v * W + u];
        }
#pragma unroll
        for (int l = 1; l <= TL; ++l) {
            const int p = j - l;
            const int lo = max(0, z0 - (TL - l)), hi = min(nz, z1 + (TL - l));
            if (p < lo || p >= hi || v < l || v >= W - l) continue;  // uniform over the warp
            const R* nb = l == 1 ? sT + ((p - jb) % kTbSlots) * PL : sL + (2 * (l - 2) + ((p - jb) & 1)) * PL;
            R val = ring[l - 1][1];  // voxels the sweep does not write keep their value
            bool wr = false;
            if (in_xy && u >= l && u < W - l && (l < TL || out_xy)) {
                auto get = [&](int dx, int dy, int dz) -> R {
                    if (dz > 0) return ring[l - 1][0];
                    if (dz < 0) return ring[l - 1][2];
                    return nb[(v + dy) * W + (u + dx)];
                };
                R t;
                wr = jacobi_point<R, BOUND>(gx, gy, p, k, qr[l], get, &t);
                if (wr) val = t;
            }
            if (l < TL) {
                sL[(2 * (l - 1) + ((p - jb) & 1)) * PL + v * W + u] = val;
                ring[l][0] = val;
            } else if (wr) {
                Tf[(size_t)p * n * n + (size_t)gy * n + gx] = val;
            }
        }
        if (__syncthreads_or(timed_out)) {
            jstop = j;
            break;
        }
    }
    if (jstop <= jl && threadIdx.x == 0) {
        // a staged plane never arrived: report it, and give the loads still in flight a
        // bounded chance to land before the CTA's shared memory is released
        atomicOr(err, 1u);
        for (int jj = jstop; jj < min(je, jstop + kTbAhead + 1); ++jj)
            mbar_wait_bounded(&bar[(jj - jb) % kTbSlots], (unsigned)((jj - jb) / kTbSlots) & 1u, w.limit_ns / 4);
    }
}

// Driver entry point of cuTensorMapEncodeTiled, looked up once through the runtime (the
// library links only cudart).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

template <typename R, int BOUND, int TL>
cudaError_t launch_tb(const CUtensorMap& tmT, const CUtensorMap& tmQ, R* Tf, const JacobiCoef<R>& k, unsigned* err,
                      const TbWait& w, cudaStream_t s) {
    using Cfg = TbCfg<R, TL>;
    auto kern = jacobi_tb_kernel<R, BOUND, TL>;
    static PerDevice<int> state;  // kernel attributes and the SM count, once per device
    int sms = 0;
    const cudaError_t attr_err = state.get(
        [&](int dev, int& n) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem_bytes);
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
            return e;
        },
        &sms);
    if (attr_err != cudaSuccess) return attr_err;
    const int tx = (k.n + Cfg::TX - 1) / Cfg::TX, ty = (k.n + Cfg::TY - 1) / Cfg::TY;
    const int zc = jacobi_tb_chunk(tx * ty, k.nz, TL, sms);
    const dim3 grid(tx, ty, (k.nz + zc - 1) / zc);
    kern<<<grid, kTbThreads, Cfg::smem_bytes, s>>>(tmT, tmQ, Tf, k, zc, err, w);
    return cudaGetLastError();
}

}  // namespace

// z planes per CTA: the chunk that minimises (waves of CTAs) x (planes each CTA streams,
// its 2·TL halo planes included) for `tiles` tiles on `sms` SMs, one CTA per SM.
int jacobi_tb_chunk(int tiles, int nz, int depth, int sms) {
    int best_zc = nz;
    double best = 1e300;
    for (int c = 1; c <= std::min(nz, 64); ++c) {
        const int zc = (nz + c - 1) / c;
        const long ctas = (long)tiles * ((nz + zc - 1) / zc);
        const long waves = (ctas + sms - 1) / sms;
        const double cost = (double)waves * (zc + 2 * depth);
        if (cost < best * 0.999) {
            best = cost;
            best_zc = zc;
        }
    }
    return best_zc;
}

template <typename R>
shg_status make_tb_map(const R* base, int n, int nz, CUtensorMap* map) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) return fail(SHG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    if ((reinterpret_cast<uintptr_t>(base) & 15) || ((size_t)n * sizeof(R)) % 16)
        return fail(SHG_ERR_UNSUPPORTED, "temperature grid rows are not 16-byte aligned (side %d)", n);
    const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)n * sizeof(R), (cuuint64_t)n * n * sizeof(R)};
    const cuuint32_t box[3] = {(cuuint32_t)kTbSide, (cuuint32_t)kTbSide, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(map, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                           const_cast<R*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(SHG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SHG_OK;
}

template <typename R>
cudaError_t launch_jacobi_tb(const CUtensorMap& tmT, const CUtensorMap& tmQ, R* Tf, const JacobiCoef<R>& k,
                             int boundary, int depth, unsigned* err, cudaStream_t s, TbWait w) {
    if (boundary == SHG_BOUNDARY_OVEN_SURROUNDED) {
        switch (depth) {
            case 2: return launch_tb<R, SHG_BOUNDARY_OVEN_SURROUNDED, 2>(tmT, tmQ, Tf, k, err, w, s);
            case 3: return launch_tb<R, SHG_BOUNDARY_OVEN_SURROUNDED, 3>(tmT, tmQ, Tf, k, err, w, s);
            case 4: return launch_tb<R, SHG_BOUNDARY_OVEN_SURROUNDED, 4>(tmT, tmQ, Tf, k, err, w, s);
        }
    } else {
        switch (depth) {
            case 2: return launch_tb<R, SHG_BOUNDARY_TOP_OPEN, 2>(tmT, tmQ, Tf, k, err, w, s);
            case 3: return launch_tb<R, SHG_BOUNDARY_TOP_OPEN, 3>(tmT, tmQ, Tf, k, err, w, s);
            case 4: return launch_tb<R, SHG_BOUNDARY_TOP_OPEN, 4>(tmT, tmQ, Tf, k, err, w, s);
        }
    }
    return cudaErrorInvalidValue;
}

template shg_status make_tb_map<float>(const float*, int, int, CUtensorMap*);
template shg_status make_tb_map<double>(const double*, int, int, CUtensorMap*);
template cudaError_t launch_jacobi_tb<float>(const CUtensorMap&, const CUtensorMap&, float*, const JacobiCoef<float>&,
                                             int, int, unsigned*, cudaStream_t, TbWait);
template cudaError_t launch_jacobi_tb<double>(const CUtensorMap&, const CUtensorMap&, double*,
                                              const JacobiCoef<double>&, int, int, unsigned*, cudaStream_t, TbWait);

namespace {

// Self-test of the bounded staging wait: two blocked sweeps of a 64 x 64 x 32 grid whose
// plane `withhold` is never staged.
template <typename R>
shg_status selftest_wait(double wait_us, int withhold) {
    constexpr int n = 64, nz = 32;
    const size_t nt = (size_t)n * n * nz;
    shg_params p;
    shg_default_params(&p);
    p.nx = p.ny = n;
    p.nz = nz;
    p.precision = sizeof(R) == 8 ? 64 : 32;
    p.thermal = 1;
    const JacobiCoef<R> k = make_jacobi_coef<R>(p);
    char* buf = nullptr;
    cudaError_t e = cudaMalloc((void**)&buf, 3 * sizeof(R) * nt + 256);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    R* Ta = reinterpret_cast<R*>(buf);
    R* Tb = Ta + nt;
    R* Q = Tb + nt;
    unsigned* err = reinterpret_cast<unsigned*>(Q + nt);
    shg_status rc = SHG_OK;
    CUtensorMap mt, mq;
    do {
        if ((e = cudaMemset(buf, 0, 3 * sizeof(R) * nt + 256)) != cudaSuccess) { rc = cuda_fail(e, "cudaMemset"); break; }
        if ((rc = make_tb_map<R>(Ta, n, nz, &mt)) != SHG_OK || (rc = make_tb_map<R>(Q, n, nz, &mq)) != SHG_OK) break;
        TbWait w;
        w.limit_ns = (uint64_t)(wait_us * 1e3);
        w.withhold = withhold;
        if ((e = launch_jacobi_tb<R>(mt, mq, Tb, k, SHG_BOUNDARY_TOP_OPEN, 2, err, nullptr, w)) != cudaSuccess ||
            (e = cudaDeviceSynchronize()) != cudaSuccess) {
            rc = cuda_fail(e, "blocked sweeps");
            break;
        }
        unsigned h = 0;
        if ((e = cudaMemcpy(&h, err, sizeof(h), cudaMemcpyDeviceToHost)) != cudaSuccess) { rc = cuda_fail(e, "cudaMemcpy"); break; }
        if (h) rc = fail(SHG_ERR_CUDA, "a staged plane did not arrive within %g us (plane %d withheld)", wait_us, withhold);
    } while (0);
    cudaFree(buf);
    return rc;
}

}  // namespace

}  // namespace shg

extern "C" shg_status shg_selftest_bounded_wait(int32_t precision, double wait_us, int32_t withhold_plane) {
    using namespace shg;
    clear_error();
    if (precision != 32 && precision != 64) return fail(SHG_ERR_INVALID, "precision must be 32 or 64");
    if (!(wait_us > 0) || wait_us > 1e7) return fail(SHG_ERR_INVALID, "wait_us must be in (0, 1e7]");
    if (withhold_plane < -1 || withhold_plane >= 32) return fail(SHG_ERR_INVALID, "withhold_plane must be in -1..31");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    return precision == 64 ? selftest_wait<double>(wait_us, withhold_plane) : selftest_wait<float>(wait_us, withhold_plane);
}
