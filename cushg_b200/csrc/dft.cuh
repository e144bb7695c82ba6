// dft.cuh — register-resident small DFTs (2, 3, 4, 8, 12, 16, 32 points) used as the
// butterflies of the transverse 2D FFT of the SSFM step.
//
// All indices are compile-time constants after unrolling, so the arrays live in
// registers and every trivial twiddle (±1, ±i) is folded away.  SIGN = -1 is the
// forward kernel e^{-2πi jk/M}, SIGN = +1 the inverse (unnormalised), matching the
// convention of the cuFFT calls the reference makes (src/headers/Solver.h:161-178).
#pragma once

#include <cuda_runtime.h>

namespace shg {

template <typename T> struct cx_t;
template <> struct cx_t<float> { using type = float2; };
template <> struct cx_t<double> { using type = double2; };
template <typename T> using cx = typename cx_t<T>::type;

template <typename T> __device__ __forceinline__ cx<T> mk(T re, T im) { cx<T> c; c.x = re; c.y = im; return c; }
template <typename T> __device__ __forceinline__ cx<T> add(cx<T> a, cx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cx<T> sub(cx<T> a, cx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ cx<T> mul(cx<T> a, cx<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T> __device__ __forceinline__ cx<T> mulc(cx<T> a, cx<T> b) {
    return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T> __device__ __forceinline__ cx<T> scale(cx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }

// FP32 complex add / sub as one packed two-lane instruction each (sm_100 f32x2).  Both
// lanes round to nearest like the scalar pair; a - b is fma(b, -1, a), exact in the product.
template <> __device__ __forceinline__ float2 add<float>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 sub<float>(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}

// cos / sin of 2π m / 16 and 2π m / 12 as literals (m in [0, M)).
__host__ __device__ constexpr double cos16(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.923879532511286756128 : m == 2 ? 0.707106781186547524401
         : m == 3 ? 0.382683432365089771728 : m == 4 ? 0.0 : m == 5 ? -0.382683432365089771728
         : m == 6 ? -0.707106781186547524401 : m == 7 ? -0.923879532511286756128 : m == 8 ? -1.0
         : m == 9 ? -0.923879532511286756128 : m == 10 ? -0.707106781186547524401
         : m == 11 ? -0.382683432365089771728 : m == 12 ? 0.0 : m == 13 ? 0.382683432365089771728
         : m == 14 ? 0.707106781186547524401 : 0.923879532511286756128;
}
__host__ __device__ constexpr double sin16(int m) { return cos16((m + 12) & 15); }  // sin x = cos(x - π/2)
__host__ __device__ constexpr double cos12(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.866025403784438646764 : m == 2 ? 0.5 : m == 3 ? 0.0
         : m == 4 ? -0.5 : m == 5 ? -0.866025403784438646764 : m == 6 ? -1.0
         : m == 7 ? -0.866025403784438646764 : m == 8 ? -0.5 : m == 9 ? 0.0 : m == 10 ? 0.5
         : 0.866025403784438646764;
}
__host__ __device__ constexpr double sin12(int m) { return cos12((m + 9) % 12); }
// cos / sin of 2π m / 32 from the first octant (m in [0, 32))
__host__ __device__ constexpr double cos32q(int m) {  // m in [0, 8]
    return m == 0 ? 1.0 : m == 1 ? 0.980785280403230449126 : m == 2 ? 0.923879532511286756128
         : m == 3 ? 0.831469612302545237079 : m == 4 ? 0.707106781186547524401 : m == 5 ? 0.555570233019602224743
         : m == 6 ? 0.382683432365089771728 : m == 7 ? 0.195090322016128267848 : 0.0;
}
__host__ __device__ constexpr double cos32(int m) {
    return m <= 8 ? cos32q(m) : m <= 16 ? -cos32q(16 - m) : m <= 24 ? -cos32q(m - 16) : cos32q(32 - m);
}
__host__ __device__ constexpr double sin32(int m) { return cos32((m + 24) & 31); }  // sin x = cos(x - π/2)

// v * (c + i s) for a constant (c, s) known in double.  In float the constant is split
// into hi + lo parts and applied with fused multiply-adds, so its rounding does not
// bias the modulus of every transform by the same relative amount step after step (a
// coherent error that would grow linearly with the number of SSFM steps).
template <typename T>
__device__ __forceinline__ cx<T> rot_const(cx<T> v, double c, double s) {
    if constexpr (sizeof(T) == 8) {
        return mk<T>(v.x * c - v.y * s, v.x * s + v.y * c);
    } else {
        const float ch = (float)c, sh = (float)s;
        const float cl = (float)(c - (double)ch), sl = (float)(s - (double)sh);
        return mk<T>(fmaf(v.x, ch, fmaf(-v.y, sh, v.x * cl - v.y * sl)), fmaf(v.x, sh, fmaf(v.y, ch, v.x * sl + v.y * cl)));
    }
}

// v * e^{SIGN 2πi m / M} for M dividing 16, 12 or 32; m is a compile-time constant
// after unrolling, so the branches fold.
template <int M, int SIGN, typename T>
__device__ __forceinline__ cx<T> rot(cx<T> v, int m) {
    m = ((m % M) + M) % M;
    if (m == 0) return v;
    if (2 * m == M) return mk<T>(-v.x, -v.y);
    if (4 * m == M) return SIGN > 0 ? mk<T>(-v.y, v.x) : mk<T>(v.y, -v.x);
    if (4 * m == 3 * M) return SIGN > 0 ? mk<T>(v.y, -v.x) : mk<T>(-v.y, v.x);
    if (16 % M == 0) {
        const int q = m * (16 / M);
        return rot_const<T>(v, cos16(q), SIGN * sin16(q));
    } else if (32 % M == 0) {
        const int q = m * (32 / M);
        return rot_const<T>(v, cos32(q), SIGN * sin32(q));
    } else {
        const int q = m * (12 / M);
        return rot_const<T>(v, cos12(q), SIGN * sin12(q));
    }
}

// Constants of a precomputed multiplier table: double2 in FP64; in FP32 a float4
// (hi.x, hi.y, lo.x, lo.y) with hi + lo the double value.
template <typename T> struct mult_t;
template <> struct mult_t<double> { using type = double2; };
template <> struct mult_t<float> { using type = float4; };
template <typename T> using mult = typename mult_t<T>::type;

template <typename T> __host__ __device__ __forceinline__ mult<T> make_mult(double re, double im);
template <> __host__ __device__ __forceinline__ double2 make_mult<double>(double re, double im) {
    return make_double2(re, im);
}
template <> __host__ __device__ __forceinline__ float4 make_mult<float>(double re, double im) {
    const float hr = (float)re, hi = (float)im;
    return make_float4(hr, hi, (float)(re - (double)hr), (float)(im - (double)hi));
}

// v * w
__device__ __forceinline__ double2 mulw(double2 v, double2 w) {
    return make_double2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
}
__device__ __forceinline__ float2 mulw(float2 v, float4 w) {
    return make_float2(fmaf(v.x, w.x, fmaf(-v.y, w.y, v.x * w.z - v.y * w.w)),
                       fmaf(v.x, w.y, fmaf(v.y, w.x, v.x * w.w + v.y * w.z)));
}
// v * conj(w)
__device__ __forceinline__ double2 mulwc(double2 v, double2 w) {
    return make_double2(v.x * w.x + v.y * w.y, v.y * w.x - v.x * w.y);
}
__device__ __forceinline__ float2 mulwc(float2 v, float4 w) {
    return make_float2(fmaf(v.x, w.x, fmaf(v.y, w.y, v.x * w.z + v.y * w.w)),
                       fmaf(v.y, w.x, fmaf(-v.x, w.y, v.y * w.z - v.x * w.w)));
}

template <int M, int SIGN, typename T> struct Dft;

template <int SIGN, typename T> struct Dft<1, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&)[1]) {}
};

template <int SIGN, typename T> struct Dft<2, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[2]) {
        cx<T> a = v[0], b = v[1];
        v[0] = add<T>(a, b);
        v[1] = sub<T>(a, b);
    }
};

template <int SIGN, typename T> struct Dft<3, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[3]) {
        cx<T> t = add<T>(v[1], v[2]);
        cx<T> u = sub<T>(v[1], v[2]);
        cx<T> m = mk<T>(v[0].x - (T)0.5 * t.x, v[0].y - (T)0.5 * t.y);
        v[0] = add<T>(v[0], t);
        // X1 = m + SIGN*i*h*u, X2 = m - SIGN*i*h*u, h = sqrt(3)/2
        const cx<T> hu = rot_const<T>(u, 0.866025403784438646764, 0.0);
        cx<T> r = SIGN > 0 ? mk<T>(-hu.y, hu.x) : mk<T>(hu.y, -hu.x);
        v[1] = add<T>(m, r);
        v[2] = sub<T>(m, r);
    }
};

template <int SIGN, typename T> struct Dft<4, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[4]) {
        cx<T> t0 = add<T>(v[0], v[2]), t1 = sub<T>(v[0], v[2]);
        cx<T> t2 = add<T>(v[1], v[3]), d = sub<T>(v[1], v[3]);
        cx<T> t3 = SIGN > 0 ? mk<T>(-d.y, d.x) : mk<T>(d.y, -d.x);  // SIGN*i*d
        v[0] = add<T>(t0, t2);
        v[2] = sub<T>(t0, t2);
        v[1] = add<T>(t1, t3);
        v[3] = sub<T>(t1, t3);
    }
};

// Two-factor Cooley-Tukey: M = A*B, input index j = j0 + A*j1, output k = k1 + B*k0.
template <int A, int B, int SIGN, typename T>
__device__ __forceinline__ void dft_two_factor(cx<T> (&v)[A * B]) {
    constexpr int M = A * B;
    cx<T> y[A][B];
#pragma unroll
    for (int j0 = 0; j0 < A; ++j0) {
        cx<T> t[B];
#pragma unroll
        for (int j1 = 0; j1 < B; ++j1) t[j1] = v[j0 + A * j1];
        Dft<B, SIGN, T>::run(t);
#pragma unroll
        for (int k1 = 0; k1 < B; ++k1) y[j0][k1] = rot<M, SIGN, T>(t[k1], j0 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < B; ++k1) {
        cx<T> t[A];
#pragma unroll
        for (int j0 = 0; j0 < A; ++j0) t[j0] = y[j0][k1];
        Dft<A, SIGN, T>::run(t);
#pragma unroll
        for (int k0 = 0; k0 < A; ++k0) v[k1 + B * k0] = t[k0];
    }
}

template <int SIGN, typename T> struct Dft<6, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[6]) { dft_two_factor<2, 3, SIGN, T>(v); }
};
template <int SIGN, typename T> struct Dft<8, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[8]) { dft_two_factor<2, 4, SIGN, T>(v); }
};
template <int SIGN, typename T> struct Dft<12, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[12]) { dft_two_factor<4, 3, SIGN, T>(v); }
};
template <int SIGN, typename T> struct Dft<16, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[16]) { dft_two_factor<4, 4, SIGN, T>(v); }
};
template <int SIGN, typename T> struct Dft<32, SIGN, T> {
    static __device__ __forceinline__ void run(cx<T> (&v)[32]) { dft_two_factor<2, 16, SIGN, T>(v); }
};

}  // namespace shg
