// ssfm_multipass.cuh — the SSFM march for grids whose two field planes do not fit in the
// shared memory of one thread-block cluster: 512 x 512 is 4 MB in FP32 and 8 MB in FP64,
// against 16 CTAs x 227 KB.  The planes stay in global memory (a few instances at a time
// stay resident in the 126 MB L2) and every SSFM step is two launches:
//
//   row pass     RB rows of both fields per CTA: inverse row transform, RK4 at the end of
//                step s, RK4 at the start of step s+1 (with the heat source, slice records and
//                outputs of boundary_point), forward row transform
//   column pass  CW columns of one field per CTA: forward column transform, propagator,
//                inverse column transform
//
// The transforms are the four-step FFT of the fused march (ssfm_plain.cuh) with N = 16 R2
// (R2 = 32 at N = 512): the same digit-reversed frequency order between the passes, the same
// twiddle and propagator tables, the same per-point arithmetic in the same order.  On a grid
// side both kernels are built for, the two agree up to where the compiler contracts a
// multiply and an add into one fused multiply-add differently (a last-bit effect).
//
// Reference counterparts as for the fused march: Solver::SSFM / CWES (src/headers/Solver.h:
// 267-308) with solverRK4 (:189-264) and diffraction (:153-186, cuFFT, kernelComplexProduct,
// cuFFTscale Efields.h:15-29).
#pragma once

#include "ssfm_plain.cuh"

namespace shg {

template <typename T, int N>
struct MpCfg {
    static constexpr int R2 = N / 16;
    static constexpr int SW = sizeof(T) == 4 ? 16 : 8;  // complex slots per 128 B
    static constexpr int RB = sizeof(T) == 4 ? 8 : 4;   // rows per row-pass CTA
    static constexpr int RNT = RB * 16;                  // row-pass threads: one (row, n1) job each
    static constexpr int CW = SW;                        // columns per column-pass CTA: one 128 B row segment
    static constexpr int CNT = 16 * CW;                  // column-pass threads: one (column, n1) job each
    static constexpr int RPART = N / RB;                 // row-pass CTAs per instance (power partials)
    // (FP32: plus the packed RK4 stage constants of the two steps, 6 Rk4Pack)
    static constexpr size_t row_smem = sizeof(cx<T>) * (2 * (size_t)RB * N + 12) + sizeof(mult<T>) * N +
                                       sizeof(double) * 2 * (RNT / 32) + (sizeof(T) == 4 ? 6 * sizeof(Rk4Pack) : 0);
    static constexpr size_t col_smem = sizeof(cx<T>) * (size_t)N * CW + sizeof(mult<T>) * (2 * (size_t)N + CW);
    // The thermal row pass gives each (row, n1) job several threads in its pointwise work (the
    // RK4 half steps with per-voxel coefficients, by far its longest part): a single instance
    // has only N x 16 jobs, and the pass otherwise lasts one thread's chain of R2 points.  Four
    // in FP32 (the kernel fits the 128 registers of a 512-thread block), two in FP64.
    __host__ __device__ static constexpr int row_px(bool therm) { return therm ? (sizeof(T) == 4 ? 4 : 2) : 1; }
    __host__ __device__ static constexpr int row_threads(bool therm) { return RNT * row_px(therm); }
    __host__ __device__ static constexpr size_t row_smem_for(bool therm) {
        return row_smem + sizeof(double) * 2 * (RNT / 32) * (row_px(therm) - 1);
    }
    static_assert(N % 16 == 0 && RB * RPART == N && N % CW == 0, "bad multi-pass split");
};

// Per-instance workspace in global memory, at base + inst * stride: the two field planes,
// the multiplier tables (twiddles tw, propagator factors pxp, pxs, pyp, pys: N each), the
// row-pass power partials, the running Δk prefix (thermal) and the step positions z_s.
struct MpLayout {
    char* base;
    size_t stride;
    size_t off_s, off_tab, off_part, off_dk, off_zs;
};

template <typename T, int N>
__host__ __device__ inline MpLayout mp_layout(char* base, int max_steps, bool thermal) {
    using Cfg = MpCfg<T, N>;
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    MpLayout L;
    L.base = base;
    const size_t plane = sizeof(cx<T>) * (size_t)N * N;
    L.off_s = up(plane);
    L.off_tab = L.off_s + up(plane);
    L.off_part = L.off_tab + up(sizeof(mult<T>) * 5 * (size_t)N);
    L.off_dk = L.off_part + up(sizeof(double) * 2 * Cfg::RPART);
    L.off_zs = L.off_dk + (thermal ? up(sizeof(double) * (size_t)N * N) : 0);
    L.stride = L.off_zs + up(sizeof(double) * ((size_t)max_steps + 1));
    return L;
}

// Tables and step positions of each instance (one block per instance).  z_s is accumulated
// like the fused march's z (+= dz per step), so both see the same stage phases.
template <typename T, int N>
__global__ void __launch_bounds__(256) mp_setup_kernel(const InstDesc* __restrict__ descs, MpLayout L) {
    const InstDesc d = descs[blockIdx.x];
    char* w = L.base + (size_t)blockIdx.x * L.stride;
    mult<T>* tab = reinterpret_cast<mult<T>*>(w + L.off_tab);
    init_tables<T, N>(d, tab, tab + N, tab + 2 * N, tab + 3 * N, tab + 4 * N, threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) {
        double* zs = reinterpret_cast<double*>(w + L.off_zs);
        double z = 0.0;
        zs[0] = z;
        for (int k = 0; k < d.nsteps; ++k) {
            z += d.dz;
            zs[k + 1] = z;
        }
    }
}

// The R2-point stage of the four-step transform on the elements n2 = 0..R2-1 of one n1:
// forward = DFT, then twiddle W_N^{n1 k}; inverse = conj(DFT(conj(x) W)).
template <typename T, int R2>
__device__ __forceinline__ void r2_stage(cx<T> (&v)[R2], const mult<T>* tw, int n1, bool inv) {
    auto cj = [](cx<T> a) { return mk<T>(a.x, -a.y); };
    if (inv) {
        v[0] = cj(v[0]);
#pragma unroll
        for (int k = 1; k < R2; ++k) v[k] = mulw(cj(v[k]), tw[k * 16 + n1]);
    }
    Dft<R2, -1, T>::run(v);
    if (inv) {
#pragma unroll
        for (int k = 0; k < R2; ++k) v[k] = cj(v[k]);
    } else {
#pragma unroll
        for (int k = 1; k < R2; ++k) v[k] = mulw(v[k], tw[k * 16 + n1]);
    }
}

// L2 prefetch of `bytes` of global memory from p, in 4 KB bulk prefetches issued by threads
// i, i + n, ... of the block; nothing when p or bytes is not a multiple of 16 (a bulk
// prefetch needs both).  A prefetch only warms L2: it never changes what a load returns.
__device__ __forceinline__ void l2_prefetch(const void* p, size_t bytes, int i, int n) {
    const char* c = reinterpret_cast<const char*>(p);
    if (((reinterpret_cast<uintptr_t>(c) | bytes) & 15) != 0) return;
    for (size_t o = (size_t)i * 4096; o < bytes; o += (size_t)n * 4096) {
        const unsigned b = (unsigned)(bytes - o < 4096 ? bytes - o : 4096);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c + o), "r"(b) : "memory");
    }
}

// Row pass of step s (s = -1: the first pass, which builds the initial fields; the pass with
// s + 1 = out_after writes the outputs and this CTA's power partials; s = nsteps-1 is the
// last).  Grid (N / RB, count).
template <typename T, int N, bool THERM>
__global__ void __launch_bounds__(MpCfg<T, N>::row_threads(THERM))
    mp_row_kernel(const InstDesc* __restrict__ descs, MpLayout L, int s) {
    using Cfg = MpCfg<T, N>;
    constexpr int R2 = Cfg::R2, RB = Cfg::RB, SW = Cfg::SW;
    constexpr int JOBS = Cfg::RNT, PX = Cfg::row_px(THERM), NT = JOBS * PX;
    using V = cx<T>;
    using W = mult<T>;
    const InstDesc d = descs[blockIdx.y];
    if (s >= d.nsteps) return;  // this instance has finished its march
    const int mode = s < 0 ? 0 : (s + 1 < d.nsteps ? 1 : 2);
    char* wbase = L.base + (size_t)blockIdx.y * L.stride;
    V* gP = reinterpret_cast<V*>(wbase);
    V* gS = reinterpret_cast<V*>(wbase + L.off_s);
    const W* gtab = reinterpret_cast<const W*>(wbase + L.off_tab);
    const double* zs = reinterpret_cast<const double*>(wbase + L.off_zs);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* Ps = reinterpret_cast<V*>(smem_raw);
    V* Ss = Ps + RB * N;
    V* coef = Ss + RB * N;  // [0..5] step s, [6..11] step s+1
    W* tw = reinterpret_cast<W*>(coef + 12);
    double* red = reinterpret_cast<double*>(tw + N);
    const int tid = threadIdx.x, y0 = blockIdx.x * RB;
    auto cj = [](V a) { return mk<T>(a.x, -a.y); };
    // FP32 plain: packed RK4 stage constants [2][3] (steps s, s + 1), after the reduction area
    constexpr bool PACK = !THERM && sizeof(T) == 4;
    Rk4Pack* kpk = reinterpret_cast<Rk4Pack*>(red + 2 * (NT / 32));

    if constexpr (THERM) {
        // step s reads slices s and s + 1 of the per-voxel optics; slice s + 1 is cold in
        // HBM. Warm this CTA's rows of slice s + 2 for the next row pass.
        if (s + 2 < d.nsteps) {
            const size_t off = (size_t)(s + 2) * N * N + (size_t)y0 * N, rb = sizeof(T) * RB * N;
            l2_prefetch(reinterpret_cast<const T*>(d.t_np) + off, rb, tid, NT);
            l2_prefetch(reinterpret_cast<const T*>(d.t_ns) + off, rb, tid, NT);
            l2_prefetch(reinterpret_cast<const T*>(d.t_dk) + off, rb, tid, NT);
        }
    }
    for (int j = tid; j < N; j += NT) tw[j] = gtab[j];
    if (!THERM && tid < 3) {
        if (mode == 0) {
            stage_coef<T>(d, 0, 0.0, tid, coef + 6);
        } else {
            stage_coef<T>(d, s, zs[s], tid, coef);
            if (mode == 1) stage_coef<T>(d, s + 1, zs[s + 1], tid, coef + 6);
            if constexpr (PACK) {
                if (mode == 1) {
                    stage_pack(coef, tid, kpk);
                    stage_pack(coef + 6, tid, kpk + 3);
                }
            }
        }
    }
    if (mode == 0) {
        // setPump (Efields.h:84-119); SH = 0 or the given field
        const V* sin_g = reinterpret_cast<const V*>(d.signal_in);
        for (int e = tid; e < RB * N; e += NT) {
            const int lr = e / N, x = e % N;
            const int y = y0 + lr;
            const double2 pv = pump_value(d, x, y, d.amp_re, d.amp_im, d.den_re, d.den_im);
            const V p0 = mk<T>((T)pv.x, (T)pv.y);
            const V s0 = d.has_signal_in ? sin_g[(size_t)y * N + x] : mk<T>((T)0, (T)0);
            Ps[sidx<N, R2, SW>(lr, x)] = p0;
            Ss[sidx<N, R2, SW>(lr, x)] = s0;
            if (d.slices_p) reinterpret_cast<V*>(d.slices_p)[(size_t)y * N + x] = p0;
            if (d.slices_s) reinterpret_cast<V*>(d.slices_s)[(size_t)y * N + x] = s0;
        }
    } else {
        for (int e = tid; e < RB * N; e += NT) {
            const int lr = e / N, x = e % N;
            const size_t g = (size_t)(y0 + lr) * N + x;
            Ps[sidx<N, R2, SW>(lr, x)] = gP[g];
            Ss[sidx<N, R2, SW>(lr, x)] = gS[g];
        }
    }
    __syncthreads();

    // 16-point stage over n1 of every (row, k2), both fields
    auto n1_pass = [&](bool inv) {
        for (int j = tid; j < RB * R2; j += NT) {
            const int k2 = j % R2, lr = j / R2;
#pragma unroll 1
            for (int f = 0; f < 2; ++f) {
                V* F = f ? Ss : Ps;
                V u[16];
#pragma unroll
                for (int n = 0; n < 16; ++n) {
                    u[n] = F[sidx<N, R2, SW>(lr, n + 16 * k2)];
                    if (inv) u[n] = cj(u[n]);
                }
                Dft<16, -1, T>::run(u);
#pragma unroll
                for (int n = 0; n < 16; ++n) F[sidx<N, R2, SW>(lr, n + 16 * k2)] = inv ? cj(u[n]) : u[n];
            }
        }
    };
    if (mode != 0) {
        n1_pass(true);
        __syncthreads();
    }

    const T hap = (T)d.hap, has = (T)d.has, qs = (T)d.qs, dz6 = (T)(d.dz / 6.0);
    double acc_s = 0.0, acc_p = 0.0;
    {
        // one (row, n1) job per JOBS threads; its R2 stages on the job's first thread, its
        // points shared by the job's PX threads (point k on thread part = k mod PX)
        const int job = tid % JOBS, part = tid / JOBS;
        const int n1 = job & 15, lr = job >> 4;
        double* dkint = THERM ? reinterpret_cast<double*>(wbase + L.off_dk) : nullptr;
        // the R2 stages of the job's two fields: on its first thread, or with several threads
        // per job one field each on the first two
#pragma unroll 1
        for (int f = PX > 1 ? part : 0; f < (PX > 1 ? part + 1 : 2) && f < 2 && mode != 0; ++f) {
            V* F = f ? Ss : Ps;
            V v[R2];
#pragma unroll
            for (int k = 0; k < R2; ++k) v[k] = F[sidx<N, R2, SW>(lr, n1 + 16 * k)];
            r2_stage<T, R2>(v, tw, n1, true);
#pragma unroll
            for (int k = 0; k < R2; ++k) F[sidx<N, R2, SW>(lr, n1 + 16 * k)] = v[k];
        }
        if constexpr (PX > 1) __syncthreads();
        int k0 = 0;
        if constexpr (PACK) {
            if (mode == 1 && s + 1 >= d.nslices) {
                // a middle step that records nothing: points k and k + 1 at once in packed
                // arithmetic (rk4_pair), the odd one out below
                const float2 nhap = bc2(-hap), nhas = bc2(-has), nqs = bc2(-qs), dzz = bc2(dz6);
#pragma unroll 1
                for (int k = 0; k + 1 < R2; k += 2) {
                    const int o0 = sidx<N, R2, SW>(lr, n1 + 16 * k), o1 = sidx<N, R2, SW>(lr, n1 + 16 * k + 16);
                    const V p0 = Ps[o0], q0 = Ss[o0], p1 = Ps[o1], q1 = Ss[o1];
                    Cx2 P{make_float2(p0.x, p1.x), make_float2(p0.y, p1.y)};
                    Cx2 S{make_float2(q0.x, q1.x), make_float2(q0.y, q1.y)};
                    rk4_pair(P, S, kpk, nhap, nhas, nqs, dzz);
                    rk4_pair(P, S, kpk + 3, nhap, nhas, nqs, dzz);
                    Ps[o0] = make_float2(P.r.x, P.i.x);
                    Ps[o1] = make_float2(P.r.y, P.i.y);
                    Ss[o0] = make_float2(S.r.x, S.i.x);
                    Ss[o1] = make_float2(S.r.y, S.i.y);
                }
                k0 = R2 & ~1;
            }
        }
        // thermal: each point's optics and Δk prefix are loaded before the previous point's
        // arithmetic (thermal_pre one point ahead)
        auto pre_of = [&](int k) {
            const size_t g = (size_t)(y0 + lr) * N + n1 + 16 * k;
            return thermal_pre<T, THERM>(d, mode, s, g, (size_t)N * N, THERM ? dkint + g : nullptr);
        };
        ThermPre<T> nxt = pre_of(k0 + part < R2 ? k0 + part : 0);
#pragma unroll 1
        for (int k = k0 + part; k < R2; k += PX) {
            const int x = n1 + 16 * k;
            const int o = sidx<N, R2, SW>(lr, x);
            const size_t g = (size_t)(y0 + lr) * N + x;
            const ThermPre<T> cur = nxt;
            if (k + PX < R2) nxt = pre_of(k + PX);
            V p = Ps[o], q = Ss[o];
            boundary_point<T, THERM>(d, mode, s, g, (size_t)N * N, p, q, coef, coef + 6, hap, has, qs, dz6,
                                     THERM ? dkint + g : nullptr, acc_s, acc_p, cur);
            if (mode != 2) {
                Ps[o] = p;
                Ss[o] = q;
            }
        }
        if constexpr (PX > 1) __syncthreads();
#pragma unroll 1
        for (int f = PX > 1 ? part : 0; f < (PX > 1 ? part + 1 : 2) && f < 2 && mode != 2; ++f) {
            V* F = f ? Ss : Ps;
            V v[R2];
#pragma unroll
            for (int k = 0; k < R2; ++k) v[k] = F[sidx<N, R2, SW>(lr, n1 + 16 * k)];
            r2_stage<T, R2>(v, tw, n1, false);
#pragma unroll
            for (int k = 0; k < R2; ++k) F[sidx<N, R2, SW>(lr, n1 + 16 * k)] = v[k];
        }
    }
    __syncthreads();
    if (s + 1 == d.out_after) {
        // the pass that wrote the outputs (the last step of a plain run, the one before the
        // last of a thermal run): this CTA's share of the SH and pump power sums,
        // block-reduced in a fixed order
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc_s += __shfl_down_sync(0xffffffffu, acc_s, o);
            acc_p += __shfl_down_sync(0xffffffffu, acc_p, o);
        }
        if ((tid & 31) == 0) {
            red[2 * (tid >> 5)] = acc_s;
            red[2 * (tid >> 5) + 1] = acc_p;
        }
        __syncthreads();
        if (tid == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < NT / 32; ++w) {
                a += red[2 * w];
                b += red[2 * w + 1];
            }
            double* part = reinterpret_cast<double*>(wbase + L.off_part);
            part[2 * blockIdx.x] = a;
            part[2 * blockIdx.x + 1] = b;
        }
    }
    if (mode != 2) {
        n1_pass(false);
        __syncthreads();
        for (int e = tid; e < RB * N; e += NT) {
            const int lr = e / N, x = e % N;
            const size_t g = (size_t)(y0 + lr) * N + x;
            gP[g] = Ps[sidx<N, R2, SW>(lr, x)];
            gS[g] = Ss[sidx<N, R2, SW>(lr, x)];
        }
    }
}

// Column pass of step s: the diffraction of one field over CW columns.  Grid (N / CW, 2
// fields, count).
template <typename T, int N>
__global__ void __launch_bounds__(MpCfg<T, N>::CNT)
    mp_col_kernel(const InstDesc* __restrict__ descs, MpLayout L, int s) {
    using Cfg = MpCfg<T, N>;
    constexpr int R2 = Cfg::R2, CW = Cfg::CW, NT = Cfg::CNT;
    using V = cx<T>;
    using W = mult<T>;
    if (s >= descs[blockIdx.z].nsteps) return;
    const int f = blockIdx.y;  // 0 pump, 1 SH
    char* wbase = L.base + (size_t)blockIdx.z * L.stride;
    V* F = reinterpret_cast<V*>(wbase + (f ? L.off_s : 0));
    const W* gtab = reinterpret_cast<const W*>(wbase + L.off_tab);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);  // element (y, c) at y * CW + c
    W* tw = reinterpret_cast<W*>(tile + N * CW);
    W* py = tw + N;  // y factor of this field's propagator, by frequency, × 1/N^2
    W* px = py + N;  // x factor of this field's propagator for the CTA's columns
    const int tid = threadIdx.x, x0 = blockIdx.x * CW;
    auto cj = [](V a) { return mk<T>(a.x, -a.y); };

    for (int j = tid; j < N; j += NT) {
        tw[j] = gtab[j];
        py[j] = gtab[(f ? 4 : 3) * N + j];
    }
    if (tid < CW) px[tid] = gtab[(f ? 2 : 1) * N + x0 + tid];
    for (int e = tid; e < N * CW; e += NT) {
        const int y = e / CW, c = e % CW;
        tile[e] = F[(size_t)y * N + x0 + c];
    }
    __syncthreads();
    auto col_stage = [&](bool inv) {  // R2-point stage over n2 of every (column, n1)
        const int c = tid % CW, n1 = tid / CW;
        V v[R2];
#pragma unroll
        for (int k = 0; k < R2; ++k) v[k] = tile[(n1 + 16 * k) * CW + c];
        r2_stage<T, R2>(v, tw, n1, inv);
#pragma unroll
        for (int k = 0; k < R2; ++k) tile[(n1 + 16 * k) * CW + c] = v[k];
    };
    col_stage(false);
    __syncthreads();
    // 16-point DFT over n1 of every (column, k2), propagator by frequency, inverse DFT
    for (int j = tid; j < R2 * CW; j += NT) {
        const int c = j % CW, k2 = j / CW;
        V u[16];
#pragma unroll
        for (int n = 0; n < 16; ++n) u[n] = tile[(n + 16 * k2) * CW + c];
#pragma unroll 1
        for (int it = 0; it < 2; ++it) {
            if (it) {
#pragma unroll
                for (int n = 0; n < 16; ++n) u[n] = cj(u[n]);
            }
            Dft<16, -1, T>::run(u);
            if (!it) {
#pragma unroll
                for (int k1 = 0; k1 < 16; ++k1) u[k1] = mulw(mulw(u[k1], py[k2 + R2 * k1]), px[c]);
            } else {
#pragma unroll
                for (int n = 0; n < 16; ++n) u[n] = cj(u[n]);
            }
        }
#pragma unroll
        for (int n = 0; n < 16; ++n) tile[(n + 16 * k2) * CW + c] = u[n];
    }
    __syncthreads();
    col_stage(true);
    __syncthreads();
    for (int e = tid; e < N * CW; e += NT) {
        const int y = e / CW, c = e % CW;
        F[(size_t)y * N + x0 + c] = tile[e];
    }
}

// SH and pump power of each instance from its row-pass partials, summed in a fixed order.
template <typename T, int N>
__global__ void mp_power_kernel(const InstDesc* __restrict__ descs, MpLayout L) {
    const InstDesc& d = descs[blockIdx.x];
    if (threadIdx.x != 0 || !d.power_out) return;
    const double* part = reinterpret_cast<const double*>(L.base + (size_t)blockIdx.x * L.stride + L.off_part);
    double a = 0.0, b = 0.0;
    for (int r = 0; r < MpCfg<T, N>::RPART; ++r) {
        a += part[2 * r];
        b += part[2 * r + 1];
    }
    d.power_out[0] = a * d.pw_s;
    d.power_out[1] = b * d.pw_p;
}

}  // namespace shg
