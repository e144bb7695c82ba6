// heat_direct.cu — the steady temperature of the heat equation that the reference's Jacobi
// sweeps converge to (kernelHeatEquationTopOpen / OvenSurrounded, src/headers/Tfield.h:93-240;
// the loop Solver.h:339-355), computed directly instead of one sweep at a time.  No counterpart
// in the reference.
//
// The linear system.  Every update of Tfield.h:93-240 is one row of A T = b once the row is
// multiplied by its own scale: inner points by 1/L2 (Tfield.h:113-115), faces by 2/d^2 of their
// normal direction (Tfield.h:119-137, 229-236), edges by 4/(d_a d_b) (Tfield.h:143-177) and
// vertices by 2/(dx dy dz) (Tfield.h:181-196).  In that form every row is the sum of three
// one-dimensional parts, one per direction, each of which is
//   (2 u_i - u_{i-1} - u_{i+1}) / d^2                  inside the direction,
//   (2 (1 + Bi) u_0 - 2 u_1) / d^2  (right-hand 2 Bi T_inf / d^2)   at a Robin face,
//   and, next to a Dirichlet voxel g, the inside form with g moved to the right-hand side,
// plus Q / kappa on inner points only.  (The face, edge and vertex coefficients ax .. GV of
// the reference reduce exactly to these: e.g. the vertical edge's 0.5 (Bix + Biz) times
// 4/(dx dz) is 2 Bix / dx^2 + 2 Biz / dz^2.)  So A = Ax (+) Ay (+) Az, a Kronecker sum.
//
// The solve.  Ax and Ay are tridiagonal and similar to symmetric matrices (a diagonal scaling
// of the Robin end rows), whose eigendecomposition the host computes once per operator and
// device (implicit QL).  With the forward transforms F = V^T S and the inverse G = S^{-1} V:
//   1. b (FP64) from Q, the Dirichlet voxels and T_inf                        rhs_kernel
//   2. b <- b Fx^T (along x), then Fy b (along y)                            dgemm_kernel x2
//   3. for every mode (ky, kx): (Az + lambda_x + lambda_y) v = b along z       thomas_kernel
//   4. v <- Gy v, then v Gx^T                                                dgemm_kernel x2
//      (folded x transform: v's rows from their even and odd halves)           unfold_kernel
//   5. T <- v, with the FP64 residual of one Jacobi sweep of v and the change  finish_kernel
// Unknowns: TOP_OPEN, x 0..n-1 (Robin both ends), y 1..n-1 (y = 0 Dirichlet, Robin at n-1),
// z 0..nz-1 (Robin); OVEN_SURROUNDED, x and y 1..n-2 (Dirichlet both ends), z as above.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "jacobi_point.cuh"
#include "shg_host.h"
#include "thermal.h"

namespace shg {

namespace {

// One direction's operator: m unknowns at spacing d, each end Robin (with Biot number bi) or
// next to a Dirichlet voxel.
struct Op1D {
    int m = 0;
    double d = 0.0;
    int lo_robin = 0, hi_robin = 0;
    double bi = 0.0;
    bool operator==(const Op1D& o) const {
        return m == o.m && d == o.d && lo_robin == o.lo_robin && hi_robin == o.hi_robin && bi == o.bi;
    }
};

// Rows of the scaled operator: diagonal a, below-diagonal l (l[0] unused), above-diagonal r
// (r[m-1] unused).
void op_rows(const Op1D& op, std::vector<double>& a, std::vector<double>& l, std::vector<double>& r) {
    const int m = op.m;
    const double i2 = 1.0 / (op.d * op.d);
    a.assign(m, 2.0 * i2);
    l.assign(m, -i2);
    r.assign(m, -i2);
    l[0] = 0.0;
    r[m - 1] = 0.0;
    if (op.lo_robin) {
        a[0] = 2.0 * (1.0 + op.bi) * i2;
        if (m > 1) r[0] = -2.0 * i2;
    }
    if (op.hi_robin) {
        a[m - 1] = 2.0 * (1.0 + op.bi) * i2;
        if (m > 1) l[m - 1] = -2.0 * i2;
    }
}

// Eigenvalues and eigenvectors of the symmetric tridiagonal matrix with diagonal d[0..m) and
// off-diagonal e[0..m-1) (e[i] couples i and i+1): implicit QL iterations with Wilkinson
// shifts (Bowdler, Martin, Reinsch and Wilkinson, Numer. Math. 11, 293-306 (1968)).  On
// return d holds the eigenvalues and z (column-major: vector k is z[k*m .. k*m+m)) the
// orthonormal eigenvectors.  False if an eigenvalue took more than 64 iterations.
bool tridiag_eigen(int m, std::vector<double>& d, std::vector<double> e, std::vector<double>& z) {
    z.assign((size_t)m * m, 0.0);
    for (int k = 0; k < m; ++k) z[(size_t)k * m + k] = 1.0;
    e.resize(m);
    e[m - 1] = 0.0;
    for (int l = 0; l < m; ++l) {
        for (int iter = 0;; ++iter) {
            int j = l;
            for (; j < m - 1; ++j)  // first negligible off-diagonal at or after l
                if (std::fabs(e[j]) <= DBL_EPSILON * (std::fabs(d[j]) + std::fabs(d[j + 1]))) break;
            if (j == l) break;  // d[l] converged
            if (iter >= 64) return false;
            // shift: the eigenvalue of the leading 2x2 block nearer to d[l]
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[j] - d[l] + e[l] / (g + std::copysign(r, g));
            double s = 1.0, c = 1.0, p = 0.0;
            bool split = false;
            for (int i = j - 1; i >= l; --i) {  // chase the bulge from the bottom of the block up
                const double f = s * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {  // the block split: restart on the smaller one
                    d[i + 1] -= p;
                    e[j] = 0.0;
                    split = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                double* zi = &z[(size_t)i * m];
                double* zj = &z[(size_t)(i + 1) * m];
                for (int k = 0; k < m; ++k) {
                    const double t = zj[k];
                    zj[k] = s * zi[k] + c * t;
                    zi[k] = c * zi[k] - s * t;
                }
            }
            if (split) continue;
            d[l] -= p;
            e[l] = g;
            e[j] = 0.0;
        }
    }
    return true;
}

// Eigenvalues, forward transform F (row k: mode k) and inverse G (row i: point i) of one
// operator, all row-major m x m.  The operator M is similar to the symmetric B = S M S^{-1}
// with S = diag(s), s[i+1] = s[i] sqrt(r[i] / l[i+1]); B = V diag(lambda) V^T gives
// F = V^T S and G = S^{-1} V.
// An operator with the same kind of end at both sides and m even is symmetric under
// i -> m-1-i (B and S alike), and B splits into an even and an odd block of half size: for
// v = (w, +-J w) / sqrt(2) (J the reversal), B v = lambda v exactly when w is an eigenvector of
// the leading h x h block of B with its last diagonal entry d[h-1] +- e[h-1].  The modes are
// then built from the blocks' eigenvectors, even modes first (k < h), so that their parity is
// exact, which the folded transforms rely on; and the QL work is a quarter.
bool op_modes(const Op1D& op, std::vector<double>& lam, std::vector<double>& F, std::vector<double>& G) {
    const int m = op.m;
    std::vector<double> a, l, r;
    op_rows(op, a, l, r);
    std::vector<double> s(m, 1.0), e(m, 0.0);
    for (int i = 0; i + 1 < m; ++i) {
        s[i + 1] = s[i] * std::sqrt(r[i] / l[i + 1]);
        e[i] = -std::sqrt(r[i] * l[i + 1]);
    }
    std::vector<double> V;  // column-major: vector k at V[k*m .. k*m+m)
    if (op.lo_robin == op.hi_robin && m % 2 == 0 && m >= 2) {
        const int h = m / 2;
        V.assign((size_t)m * m, 0.0);
        lam.assign(m, 0.0);
        const double r2 = 1.0 / std::sqrt(2.0);
        for (int par = 0; par < 2; ++par) {  // 0: even, 1: odd
            std::vector<double> d(a.begin(), a.begin() + h), eh(e.begin(), e.begin() + h), W;
            d[h - 1] += par == 0 ? e[h - 1] : -e[h - 1];
            eh[h - 1] = 0.0;
            if (!tridiag_eigen(h, d, eh, W)) return false;
            for (int q = 0; q < h; ++q) {
                const int k = par * h + q;
                lam[k] = d[q];
                for (int i = 0; i < h; ++i) {
                    const double w = W[(size_t)q * h + i] * r2;
                    V[(size_t)k * m + i] = w;
                    V[(size_t)k * m + (m - 1 - i)] = par == 0 ? w : -w;
                }
            }
        }
    } else {
        lam = a;
        if (!tridiag_eigen(m, lam, e, V)) return false;
    }
    F.assign((size_t)m * m, 0.0);
    G.assign((size_t)m * m, 0.0);
    for (int k = 0; k < m; ++k)
        for (int i = 0; i < m; ++i) {
            const double v = V[(size_t)k * m + i];  // component i of eigenvector k
            F[(size_t)k * m + i] = v * s[i];
            G[(size_t)i * m + k] = v / s[i];
        }
    return true;
}

// Device copies of one operator's transforms: F and G row-major, their transposes, lambda.  The
// matrices' rows are ld = m rounded up to even doubles (zero-padded), so that every row starts
// on 16 bytes for the GEMM's copies.
struct OpMats {
    Op1D op;
    int dev = -1;
    int ld = 0;
    double *F = nullptr, *G = nullptr, *FT = nullptr, *GT = nullptr, *lam = nullptr;
    // Folded form, for an operator symmetric under i -> m-1-i (the same kind at both ends) with
    // m a multiple of 4: its modes are even or odd, so with s_i = b_i + b_{m-1-i} and
    // d_i = b_i - b_{m-1-i} (i < h = m/2) the even amplitudes are FeT-products of s and the odd
    // ones FoT-products of d, and back, P = GeT-products and Q = GoT-products give
    // u_i = P_i + Q_i, u_{m-1-i} = P_i - Q_i.  Half matrices h x h, row-major (ld = h, even),
    // laid out for C = A B like FT and GT; lamf the eigenvalues, even modes first.
    bool fold = false;
    double *FeT = nullptr, *FoT = nullptr, *GeT = nullptr, *GoT = nullptr, *lamf = nullptr;
};

// Process-wide cache of operator transforms, per device (an operator's eigendecomposition
// costs O(m^3) on the host: about 0.3 s at m = 512).
std::mutex g_ops_mu;
std::vector<OpMats*> g_ops;
constexpr size_t kMaxCachedOps = 64;

shg_status get_op(const Op1D& op, const OpMats** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_ops_mu);
    for (const OpMats* c : g_ops)
        if (c->dev == dev && c->op == op) {
            *out = c;
            return SHG_OK;
        }
    std::vector<double> lam, F, G;
    if (!op_modes(op, lam, F, G)) return fail(SHG_ERR_NOT_CONVERGED, "heat operator eigendecomposition (m = %d)", op.m);
    const int m = op.m, ld = m + (m & 1);
    const size_t mm = (size_t)m * ld;
    std::vector<double> Fp(mm, 0.0), Gp(mm, 0.0), FT(mm, 0.0), GT(mm, 0.0);
    for (int i = 0; i < m; ++i)
        for (int k = 0; k < m; ++k) {
            Fp[(size_t)k * ld + i] = F[(size_t)k * m + i];
            Gp[(size_t)i * ld + k] = G[(size_t)i * m + k];
            FT[(size_t)i * ld + k] = F[(size_t)k * m + i];
            GT[(size_t)k * ld + i] = G[(size_t)i * m + k];
        }
    // the folded form (op_modes gives a symmetric operator's even modes first, then its odd
    // ones, each of exact parity); m a multiple of 4 keeps the half rows 16-byte aligned
    const int h = m / 2;
    const bool fold = op.lo_robin == op.hi_robin && m % 4 == 0;
    const size_t hh = fold ? (size_t)h * h : 0;
    std::vector<double> FeT(hh), FoT(hh), GeT(hh), GoT(hh), lamf(fold ? m : 0);
    for (int a = 0; fold && a < h; ++a) {
        const int ke = a, ko = h + a;
        lamf[a] = lam[ke];
        lamf[h + a] = lam[ko];
        for (int i = 0; i < h; ++i) {
            FeT[(size_t)i * h + a] = F[(size_t)ke * m + i];  // B operand: rows i, columns modes
            FoT[(size_t)i * h + a] = F[(size_t)ko * m + i];
            GeT[(size_t)a * h + i] = G[(size_t)i * m + ke];  // B operand: rows modes, columns i
            GoT[(size_t)a * h + i] = G[(size_t)i * m + ko];
        }
    }
    if (g_ops.size() >= kMaxCachedOps) return fail(SHG_ERR_UNSUPPORTED, "more than %d heat operators cached", (int)kMaxCachedOps);
    double* buf = nullptr;
    if ((e = cudaMalloc((void**)&buf, sizeof(double) * (4 * mm + (m + (m & 1)) + 4 * hh + lamf.size()))) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc");
    OpMats* c = new OpMats;
    c->op = op;
    c->dev = dev;
    c->ld = ld;
    c->F = buf;
    c->G = buf + mm;
    c->FT = buf + 2 * mm;
    c->GT = buf + 3 * mm;
    c->lam = buf + 4 * mm;
    c->fold = fold;
    double* fb = c->lam + (m + (m & 1));  // 16-byte aligned (4 mm and the padded m are even)
    if (fold) {
        c->FeT = fb;
        c->FoT = fb + hh;
        c->GeT = fb + 2 * hh;
        c->GoT = fb + 3 * hh;
        c->lamf = fb + 4 * hh;
    }
    const double* src[10] = {Fp.data(), Gp.data(), FT.data(), GT.data(), lam.data(),
                             FeT.data(), FoT.data(), GeT.data(), GoT.data(), lamf.data()};
    double* dst[10] = {c->F, c->G, c->FT, c->GT, c->lam, c->FeT, c->FoT, c->GeT, c->GoT, c->lamf};
    const size_t cnt[10] = {mm, mm, mm, mm, (size_t)m, hh, hh, hh, hh, lamf.size()};
    for (int k = 0; k < 10 && e == cudaSuccess; ++k)
        if (cnt[k]) e = cudaMemcpy(dst[k], src[k], sizeof(double) * cnt[k], cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(buf);
        delete c;
        return cuda_fail(e, "heat operator upload");
    }
    g_ops.push_back(c);
    *out = c;
    return SHG_OK;
}

// The grid's three directions: unknown ranges and operators.
struct HeatGrid {
    int n = 0, nz = 0;
    int x0 = 0, y0 = 0, mx = 0, my = 0;  // first unknown and count along x and y
    Op1D ox, oy;
    double dx = 0, dy = 0, dz = 0, biz = 0;
};

HeatGrid heat_grid(const shg_params& p) {
    HeatGrid g;
    g.n = p.nx;
    g.nz = p.nz;
    g.dx = p.lx / (p.nx - 1);
    g.dy = p.ly / (p.ny - 1);
    g.dz = p.lz / (p.nz - 1);
    const double bix = p.h_conv * g.dx / p.kappa, biy = p.h_conv * g.dy / p.kappa;
    g.biz = p.h_conv * g.dz / p.kappa;
    if (p.boundary == SHG_BOUNDARY_TOP_OPEN) {
        g.x0 = 0;
        g.mx = g.n;
        g.ox = {g.mx, g.dx, 1, 1, bix};
        g.y0 = 1;
        g.my = g.n - 1;
        g.oy = {g.my, g.dy, 0, 1, biy};
    } else {
        g.x0 = g.y0 = 1;
        g.mx = g.my = g.n - 2;
        g.ox = {g.mx, g.dx, 0, 0, bix};
        g.oy = {g.my, g.dy, 0, 0, biy};
    }
    return g;
}

// What the kernels need of the grid and the model, in FP64.
struct HeatArgs {
    int n, nz, x0, y0, mx, my;
    int lo_x_robin, hi_x_robin, lo_y_robin, hi_y_robin;
    double idx2, idy2, idz2, iK, tinf, bix, biy, biz;
};

// Compact volume index c = (z * my + j) * mx + i of unknown (x0 + i, y0 + j, z).
// 1. Right-hand side of the scaled system: Q / kappa on inner points, 2 Bi T_inf / d^2 at each
//    Robin end, g / d^2 for each Dirichlet neighbour g (read from T).
template <typename R>
__device__ __forceinline__ double rhs_value(const R* __restrict__ T, const R* __restrict__ Q, const HeatArgs& a, int i,
                                            int j, int z) {
    const size_t nn = (size_t)a.n;
    const int x = a.x0 + i, y = a.y0 + j;
    const size_t v = ((size_t)z * nn + y) * nn + x;
    double s = 0.0;
    if (Q && x > 0 && x < a.n - 1 && y > 0 && y < a.n - 1 && z > 0 && z < a.nz - 1) s = (double)Q[v] * a.iK;
    if (i == 0) s += a.lo_x_robin ? 2.0 * a.bix * a.tinf * a.idx2 : (double)T[v - 1] * a.idx2;
    if (i == a.mx - 1) s += a.hi_x_robin ? 2.0 * a.bix * a.tinf * a.idx2 : (double)T[v + 1] * a.idx2;
    if (j == 0) s += a.lo_y_robin ? 2.0 * a.biy * a.tinf * a.idy2 : (double)T[v - nn] * a.idy2;
    if (j == a.my - 1) s += a.hi_y_robin ? 2.0 * a.biy * a.tinf * a.idy2 : (double)T[v + nn] * a.idy2;
    if (z == 0) s += 2.0 * a.biz * a.tinf * a.idz2;
    if (z == a.nz - 1) s += 2.0 * a.biz * a.tinf * a.idz2;
    return s;
}

// FOLD: each row holds s_i = b_i + b_{mx-1-i} at i < mx/2 and d_i = b_i - b_{mx-1-i} at mx/2 + i.
template <typename R, bool FOLD>
__global__ void rhs_kernel(const R* __restrict__ T, const R* __restrict__ Q, double* __restrict__ b, const HeatArgs a) {
    const int w = FOLD ? a.mx / 2 : a.mx;  // work items per row
    const size_t plane = (size_t)w * a.my, total = plane * a.nz;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < total; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % w), j = (int)((c / w) % a.my), z = (int)(c / plane);
        const size_t row = ((size_t)z * a.my + j) * a.mx;
        if (FOLD) {
            const double b1 = rhs_value<R>(T, Q, a, i, j, z), b2 = rhs_value<R>(T, Q, a, a.mx - 1 - i, j, z);
            b[row + i] = b1 + b2;
            b[row + w + i] = b1 - b2;
        } else {
            b[row + i] = rhs_value<R>(T, Q, a, i, j, z);
        }
    }
}

// A block computes a 128 x 128 tile of C with eight warps, each a 64 x 32 part of it as 4 x 4
// FP64 tensor-core products (mma.sync m16n8k4); k runs in 32-wide slices through a
// three-stage ring of cp.async copies.  Row pitches: A slices 36 doubles, B slices 132, so
// that the fragment reads of a half-warp (4 rows x 4 columns of A, 4 rows x 4 columns of B)
// fall in 16 different 8-byte bank pairs; every row starts on 16 bytes.
constexpr int kGemmBM = 128, kGemmBN = 128, kGemmBK = 32, kGemmThreads = 256, kGemmStages = 3;
constexpr int kGemmALd = kGemmBK + 4, kGemmBLd = kGemmBN + 4;
constexpr int kGemmStageDoubles = kGemmBM * kGemmALd + kGemmBK * kGemmBLd;
constexpr size_t kGemmSmem = sizeof(double) * kGemmStageDoubles * kGemmStages;  // 207 KB

// 16 bytes from global to shared memory, asynchronously; the bytes past `valid` (0..16) are
// zero-filled and not read.
__device__ __forceinline__ void cp_async16(double* dst, const double* src, int valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid) : "memory");
}

// c += A B for one 16 x 8 x 4 FP64 product held in the fragments of mma.sync m16n8k4: with
// g = lane / 4 and t = lane % 4, a0 = A[g][t], a1 = A[g + 8][t], b = B[t][g], and c = C[g][2t],
// C[g][2t + 1], C[g + 8][2t], C[g + 8][2t + 1].
__device__ __forceinline__ void mma_f64(double (&c)[4], double a0, double a1, double b) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b));
}

// 2, 4. C[b] = A[b] B[b] in FP64 for row-major A (M x K, lda), B (K x N, ldb) and C (M x N, ldc),
// batch b = blockIdx.z at element strides sA, sB, sC.  lda, ldb, ldc, the strides and the three
// base addresses are even (16-byte rows).  Copies past M, N and K are zero-filled.
__global__ void __launch_bounds__(kGemmThreads, 1) dgemm_kernel(const double* __restrict__ A, const double* __restrict__ B,
                                                             double* __restrict__ C, int M, int N, int K, int lda,
                                                             int ldb, int ldc, long long sA, long long sB, long long sC) {
    extern __shared__ __align__(16) double gsm[];
    A += blockIdx.z * sA;
    B += blockIdx.z * sB;
    C += blockIdx.z * sC;
    const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * kGemmBN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 64, wn = (warp >> 1) * 32;  // this warp's 64 x 32 part of the tile
    // k slice `tile` into stage st: A 128 x 32 and B 32 x 128, 2048 chunks of 16 bytes each
    auto load = [&](int tile, int st) {
        double* As = gsm + st * kGemmStageDoubles;
        double* Bs = As + kGemmBM * kGemmALd;
        const int k0 = tile * kGemmBK;
#pragma unroll
        for (int j = 0; j < kGemmBM * kGemmBK / 2 / kGemmThreads; ++j) {
            const int c = tid + j * kGemmThreads;
            const int row = c / (kGemmBK / 2), col = (c % (kGemmBK / 2)) * 2;
            const int gr = m0 + row, gc = k0 + col;
            const int valid = gr < M ? 8 * max(0, min(2, K - gc)) : 0;
            cp_async16(As + row * kGemmALd + col, valid ? A + (size_t)gr * lda + gc : A, valid);
        }
#pragma unroll
        for (int j = 0; j < kGemmBK * kGemmBN / 2 / kGemmThreads; ++j) {
            const int c = tid + j * kGemmThreads;
            const int row = c / (kGemmBN / 2), col = (c % (kGemmBN / 2)) * 2;
            const int gr = k0 + row, gc = n0 + col;
            const int valid = gr < K ? 8 * max(0, min(2, N - gc)) : 0;
            cp_async16(Bs + row * kGemmBLd + col, valid ? B + (size_t)gr * ldb + gc : B, valid);
        }
    };
    double acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
    const int tiles = (K + kGemmBK - 1) / kGemmBK;
#pragma unroll
    for (int st = 0; st < kGemmStages - 1; ++st) {
        if (st < tiles) load(st, st);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int tl = 0; tl < tiles; ++tl) {
        // this thread's copies of slice tl have landed; the barrier makes everyone's visible and
        // ends every read of the stage the next load overwrites (slice tl - 1's)
        asm volatile("cp.async.wait_group %0;" ::"n"(kGemmStages - 2) : "memory");
        __syncthreads();
        if (tl + kGemmStages - 1 < tiles) load(tl + kGemmStages - 1, (tl + kGemmStages - 1) % kGemmStages);
        asm volatile("cp.async.commit_group;" ::: "memory");
        const double* As = gsm + (tl % kGemmStages) * kGemmStageDoubles;
        const double* Bs = As + kGemmBM * kGemmALd;
#pragma unroll
        for (int kk = 0; kk < kGemmBK; kk += 4) {
            double a[4][2], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                a[i][0] = As[(wm + 16 * i + g) * kGemmALd + kk + t];
                a[i][1] = As[(wm + 16 * i + g + 8) * kGemmALd + kk + t];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[(kk + t) * kGemmBLd + wn + 8 * j + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_f64(acc[i][j], a[i][0], a[i][1], b[j]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int row = m0 + wm + 16 * i + g + 8 * h;
            if (row >= M) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = n0 + wn + 8 * j + 2 * t;  // even: 16-byte aligned in C
                double* out = C + (size_t)row * ldc + col;
                if (col + 1 < N) *reinterpret_cast<double2*>(out) = make_double2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
                else if (col < N) out[0] = acc[i][j][2 * h];
            }
        }
}

// 3. For every mode t = j * mx + i: (Az + lambda_x[i] + lambda_y[j]) u = f along z, Thomas
// elimination (the system is diagonally dominant: lambda_x + lambda_y > 0 whenever a direction
// has a Dirichlet end or a Robin end with Bi > 0, which every boundary model has).  f and then
// u in v; the eliminated upper diagonal in cp.  Both sweeps load kThomasChunk planes ahead of
// the dependent recurrence, so each thread keeps that many loads in flight.
constexpr int kThomasChunk = 4;

__global__ void thomas_kernel(double* __restrict__ v, double* __restrict__ cp, const double* __restrict__ lx,
                              const double* __restrict__ ly, int mx, int my, int nz, double idz2, double biz) {
    const size_t plane = (size_t)mx * my;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < plane; t += (size_t)gridDim.x * blockDim.x) {
        const double lam = lx[t % mx] + ly[t / mx];
        const double a_end = 2.0 * (1.0 + biz) * idz2 + lam;  // Robin rows z = 0, nz - 1
        const double a_in = 2.0 * idz2 + lam;
        double c = 0.0, d = 0.0;
        for (int z0 = 0; z0 < nz; z0 += kThomasChunk) {
            double f[kThomasChunk];
#pragma unroll
            for (int q = 0; q < kThomasChunk; ++q)
                if (z0 + q < nz) f[q] = v[(size_t)(z0 + q) * plane + t];
#pragma unroll
            for (int q = 0; q < kThomasChunk; ++q) {
                const int z = z0 + q;
                if (z >= nz) break;
                const bool first = z == 0, last = z == nz - 1;
                const double lo = first ? 0.0 : (last ? -2.0 * idz2 : -idz2);
                const double up = last ? 0.0 : (first ? -2.0 * idz2 : -idz2);
                const double r = 1.0 / ((first || last ? a_end : a_in) - lo * c);
                c = up * r;
                d = (f[q] - lo * d) * r;
                const size_t o = (size_t)z * plane + t;
                cp[o] = c;
                v[o] = d;
            }
        }
        double u = d;  // u at z = nz - 1
        for (int z1 = nz - 1; z1 > 0; z1 -= kThomasChunk) {  // z = z1 - 1 down to z1 - kThomasChunk
            double dv[kThomasChunk], cv[kThomasChunk];
#pragma unroll
            for (int q = 0; q < kThomasChunk; ++q) {
                const int z = z1 - 1 - q;
                if (z >= 0) {
                    dv[q] = v[(size_t)z * plane + t];
                    cv[q] = cp[(size_t)z * plane + t];
                }
            }
#pragma unroll
            for (int q = 0; q < kThomasChunk; ++q) {
                const int z = z1 - 1 - q;
                if (z < 0) break;
                u = dv[q] - cv[q] * u;
                v[(size_t)z * plane + t] = u;
            }
        }
    }
}

__device__ __forceinline__ double nan_max(double a, double b) { return (b > a || b != b) ? b : a; }

// 4'. Folded x transform: each row of the inverse transform's output holds P at i < mx/2 and Q
// at mx/2 + i; the solution row is u_i = P_i + Q_i, u_{mx-1-i} = P_i - Q_i.  One streaming pass
// into the other volume, so that the finishing pass reads one value per neighbour.
__global__ void unfold_kernel(const double* __restrict__ pq, double* __restrict__ u, size_t rows, int mx) {
    const int h = mx / 2;
    const size_t items = rows * (size_t)h;
    for (size_t it = blockIdx.x * (size_t)blockDim.x + threadIdx.x; it < items; it += (size_t)gridDim.x * blockDim.x) {
        const size_t r = it / h;
        const int i = (int)(it % h);
        const double* src = pq + r * mx;
        double* dst = u + r * mx;
        const double pv = src[i], qv = src[h + i];
        dst[i] = pv + qv;
        dst[mx - 1 - i] = pv - qv;
    }
}

// 5. T <- u (rounded to R) for every unknown, with four sums into out: [0] max |J(u) - u| and
// [1] sum (J(u) - u)^2 for one FP64 Jacobi sweep J of u (jacobi_point, coefficients in FP64),
// [2] max |u - T_before| and [3] sum (u - T_before)^2.  Maxima are kept as the bits of
// non-negative doubles (ordered like unsigned integers; a NaN wins).  A thread walks
// kFinishZ planes of one (x, y) column with u's z neighbours in registers, so every load of a
// plane is independent of the arithmetic; neighbours outside the unknowns are Dirichlet
// voxels of T, which nothing writes.
constexpr int kFinishZ = 16;

template <typename R, int BOUND>
__global__ void __launch_bounds__(256, 3) finish_kernel(R* __restrict__ T, const R* __restrict__ Q, const double* __restrict__ u,
                                                     const HeatArgs a, const JacobiCoef<double> k, double* __restrict__ out) {
    auto U = [&](size_t rowbase, int col) -> double { return u[rowbase + col]; };  // the solution
    const size_t plane = (size_t)a.mx * a.my, nn = (size_t)a.n, tplane = nn * nn;
    const int chunks = (a.nz + kFinishZ - 1) / kFinishZ;
    const size_t items = plane * chunks;
    double rmax = 0.0, rsum = 0.0, cmax = 0.0, csum = 0.0;
    for (size_t it = blockIdx.x * (size_t)blockDim.x + threadIdx.x; it < items; it += (size_t)gridDim.x * blockDim.x) {
        const size_t t = it % plane;
        const int z0 = (int)(it / plane) * kFinishZ, z1 = min(a.nz, z0 + kFinishZ);
        const int i = (int)(t % a.mx), j = (int)(t / a.mx);
        const int x = a.x0 + i, y = a.y0 + j;
        const bool uxm = i > 0, uxp = i + 1 < a.mx, uym = j > 0, uyp = j + 1 < a.my;
        const bool gxm = x > 0, gxp = x + 1 < a.n, gym = y > 0, gyp = y + 1 < a.n;
        size_t rb = (size_t)z0 * plane + (size_t)j * a.mx;  // this column's row in plane z
        size_t v = (size_t)z0 * tplane + (size_t)y * nn + x;
        double below = z0 > 0 ? U(rb - plane, i) : 0.0;
        double cur = U(rb, i);
#pragma unroll 2
        for (int z = z0; z < z1; ++z, rb += plane, v += tplane) {
            const double above = z + 1 < a.nz ? U(rb + plane, i) : 0.0;
            const double xm = uxm ? U(rb, i - 1) : (gxm ? (double)T[v - 1] : 0.0);
            const double xp = uxp ? U(rb, i + 1) : (gxp ? (double)T[v + 1] : 0.0);
            const double ym = uym ? U(rb - a.mx, i) : (gym ? (double)T[v - nn] : 0.0);
            const double yp = uyp ? U(rb + a.mx, i) : (gyp ? (double)T[v + nn] : 0.0);
            const double q = Q ? (double)Q[v] : 0.0;
            const double before = (double)T[v];
            auto get = [&](int dx, int dy, int dz) -> double {
                if (dz) return dz > 0 ? above : below;
                if (dy) return dy > 0 ? yp : ym;
                return dx > 0 ? xp : xm;
            };
            double w = cur;
            jacobi_point<double, BOUND>(x, y, z, k, q, get, &w);
            const double r = fabs(w - cur), dc = fabs(cur - before);
            rmax = nan_max(rmax, r);
            rsum += r * r;
            cmax = nan_max(cmax, dc);
            csum += dc * dc;
            T[v] = (R)cur;
            below = cur;
            cur = above;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        rmax = nan_max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        rsum += __shfl_xor_sync(0xffffffffu, rsum, o);
        cmax = nan_max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
        csum += __shfl_xor_sync(0xffffffffu, csum, o);
    }
    __shared__ double red[4][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][wid] = rmax;
        red[1][wid] = rsum;
        red[2][wid] = cmax;
        red[3][wid] = csum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2) {
            rmax = nan_max(rmax, red[0][w2]);
            rsum += red[1][w2];
            cmax = nan_max(cmax, red[2][w2]);
            csum += red[3][w2];
        }
        atomicMax(reinterpret_cast<unsigned long long*>(out), (unsigned long long)__double_as_longlong(rmax));
        atomicAdd(out + 1, rsum);
        atomicMax(reinterpret_cast<unsigned long long*>(out + 2), (unsigned long long)__double_as_longlong(cmax));
        atomicAdd(out + 3, csum);
    }
}

// C = A B over `batch` matrices (see dgemm_kernel); M is split into launches of at most 65535
// row tiles.
cudaError_t gemm(const double* A, const double* B, double* C, int M, int N, int K, int lda, int ldb, int ldc, int batch,
                 long long sA, long long sB, long long sC, cudaStream_t s) {
    static PerDevice<int> attr;  // the kernel's dynamic shared memory, once per device
    const cudaError_t ae = attr.get([](int, int&) {
        return cudaFuncSetAttribute(dgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
    });
    if (ae != cudaSuccess) return ae;
    const int max_rows = 65535 * kGemmBM;
    for (int r0 = 0; r0 < M; r0 += max_rows) {
        const int rows = std::min(M - r0, max_rows);
        const dim3 grid((unsigned)((N + kGemmBN - 1) / kGemmBN), (unsigned)((rows + kGemmBM - 1) / kGemmBM), (unsigned)batch);
        dgemm_kernel<<<grid, kGemmThreads, kGemmSmem, s>>>(A + (size_t)r0 * lda, B, C + (size_t)r0 * ldc, rows, N, K, lda, ldb,
                                                   ldc, sA, sB, sC);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int grid_for(size_t work, int threads) {
    return (int)std::max<size_t>(1, std::min<size_t>((work + threads - 1) / threads, (size_t)148 * 16));
}

}  // namespace

HeatDirect::~HeatDirect() {
    if (ws_) cudaFree(ws_);  // synchronous: nothing queued may still use it
}

void HeatDirect::release(cudaStream_t s) {
    if (ws_) cudaFreeAsync(ws_, s);
    ws_ = nullptr;
    cap_ = 0;
}

template <typename R>
shg_status HeatDirect::solve(const shg_params& p, R* T, const R* Q, double t_inf, cudaStream_t s) {
    const HeatGrid g = heat_grid(p);
    if (g.nz > 65535) return fail(SHG_ERR_UNSUPPORTED, "direct heat solve: nz = %d above 65535", g.nz);
    const OpMats *ox = nullptr, *oy = nullptr;
    shg_status rc;
    if ((rc = get_op(g.ox, &ox)) != SHG_OK || (rc = get_op(g.oy, &oy)) != SHG_OK) return rc;
    const size_t vol = (size_t)g.mx * g.my * g.nz;
    cudaError_t e;
    if (vol > cap_) {
        release(s);
        if ((e = dev_alloc((void**)&ws_, sizeof(double) * (2 * vol + 4), s)) != cudaSuccess) {
            ws_ = nullptr;
            return cuda_fail(e, "cudaMallocAsync");
        }
        cap_ = vol;
    }
    nt_ = (size_t)g.n * g.n * g.nz;
    double* X = ws_;
    double* Y = ws_ + cap_;
    double* out = ws_ + 2 * cap_;
    HeatArgs a;
    a.n = g.n;
    a.nz = g.nz;
    a.x0 = g.x0;
    a.y0 = g.y0;
    a.mx = g.mx;
    a.my = g.my;
    a.lo_x_robin = g.ox.lo_robin;
    a.hi_x_robin = g.ox.hi_robin;
    a.lo_y_robin = g.oy.lo_robin;
    a.hi_y_robin = g.oy.hi_robin;
    a.idx2 = 1.0 / (g.dx * g.dx);
    a.idy2 = 1.0 / (g.dy * g.dy);
    a.idz2 = 1.0 / (g.dz * g.dz);
    a.iK = 1.0 / p.kappa;
    a.tinf = t_inf;
    a.bix = g.ox.bi;
    a.biy = g.oy.bi;
    a.biz = g.biz;
    shg_params pk = p;
    pk.t_inf = t_inf;
    const JacobiCoef<double> k = make_jacobi_coef<double>(pk);
    const int mx = g.mx, my = g.my, nz = g.nz;
    const long long pl = (long long)mx * my;
    if ((e = cudaMemsetAsync(out, 0, 4 * sizeof(double), s)) != cudaSuccess) return cuda_fail(e, "memset");
    const bool fold = ox->fold;
    const int h = mx / 2;
    if (fold) rhs_kernel<R, true><<<grid_for(vol / 2, 256), 256, 0, s>>>(T, Q, X, a);
    else rhs_kernel<R, false><<<grid_for(vol, 256), 256, 0, s>>>(T, Q, X, a);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "heat right-hand side");
    // into mode space: along x (rows of X; folded, the even modes from the sums and the odd
    // ones from the differences, half the work), then along y (one product per z plane)
    // (folded: the even and odd halves as a batch of two, FoT = FeT + h*h)
    const long long hh = (long long)h * h;
    if (fold) {
        e = gemm(X, ox->FeT, Y, nz * my, h, h, mx, h, mx, 2, h, hh, h, s);
    } else {
        e = gemm(X, ox->FT, Y, nz * my, mx, mx, mx, ox->ld, mx, 1, 0, 0, 0, s);
    }
    if (e != cudaSuccess || (e = gemm(oy->F, Y, X, my, mx, my, oy->ld, mx, mx, nz, 0, pl, pl, s)) != cudaSuccess)
        return cuda_fail(e, "heat transform");
    thomas_kernel<<<grid_for((size_t)pl, 128), 128, 0, s>>>(X, Y, fold ? ox->lamf : ox->lam, oy->lam, mx, my, nz, a.idz2,
                                                             a.biz);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "heat tridiagonal solve");
    // back to voxels: along y, then along x (folded: P from the even modes, Q from the odd;
    // the finishing pass combines them)
    if ((e = gemm(oy->G, X, Y, my, mx, my, oy->ld, mx, mx, nz, 0, pl, pl, s)) != cudaSuccess)
        return cuda_fail(e, "heat transform");
    if (fold) {
        e = gemm(Y, ox->GeT, X, nz * my, h, h, mx, h, mx, 2, h, hh, h, s);
    } else {
        e = gemm(Y, ox->GT, X, nz * my, mx, mx, mx, ox->ld, mx, 1, 0, 0, 0, s);
    }
    if (e != cudaSuccess) return cuda_fail(e, "heat transform");
    const size_t fitems = (size_t)pl * ((nz + kFinishZ - 1) / kFinishZ);
    const int fb = grid_for(fitems, 256);
    const double* u = X;
    if (fold) {
        unfold_kernel<<<grid_for((size_t)nz * my * h, 256), 256, 0, s>>>(X, Y, (size_t)nz * my, mx);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "heat solution");
        u = Y;
    }
    if (p.boundary == SHG_BOUNDARY_TOP_OPEN)
        finish_kernel<R, SHG_BOUNDARY_TOP_OPEN><<<fb, 256, 0, s>>>(T, Q, u, a, k, out);
    else
        finish_kernel<R, SHG_BOUNDARY_OVEN_SURROUNDED><<<fb, 256, 0, s>>>(T, Q, u, a, k, out);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "heat solution");
    return SHG_OK;
}

shg_status HeatDirect::result(int rule, double* residual, double* change, cudaStream_t s) {
    if (!ws_) return fail(SHG_ERR_INVALID, "no heat solve to read");
    double h[4] = {0, 0, 0, 0};
    cudaError_t e;
    if ((e = cudaMemcpyAsync(h, ws_ + 2 * cap_, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(e, "heat solve result");
    const double nt = (double)nt_;
    if (residual) *residual = rule == SHG_CONV_REFERENCE ? std::sqrt(h[1]) / nt : h[0];
    if (change) *change = rule == SHG_CONV_REFERENCE ? std::sqrt(h[3]) / nt : h[2];
    return SHG_OK;
}

template shg_status HeatDirect::solve<float>(const shg_params&, float*, const float*, double, cudaStream_t);
template shg_status HeatDirect::solve<double>(const shg_params&, double*, const double*, double, cudaStream_t);

shg_status heat_steady_device(const shg_params& p, void* temperature, const void* q, double* residual,
                              cudaStream_t s) {
    HeatDirect h;
    shg_status rc = p.precision == 32
                        ? h.solve<float>(p, reinterpret_cast<float*>(temperature), reinterpret_cast<const float*>(q), p.t_inf, s)
                        : h.solve<double>(p, reinterpret_cast<double*>(temperature), reinterpret_cast<const double*>(q),
                                          p.t_inf, s);
    double r = 0.0;
    if (rc == SHG_OK) rc = h.result(SHG_CONV_MAXABS, &r, nullptr, s);
    h.release(s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "heat steady solve");
    if (rc == SHG_OK && !std::isfinite(r)) rc = fail(SHG_ERR_NONFINITE, "heat steady solve: residual %g", r);
    if (residual) *residual = r;
    return rc;
}

}  // namespace shg

extern "C" shg_status shg_heat_operator_modes(int32_t m, double d, int32_t lo_robin, int32_t hi_robin, double bi,
                                              double* lambda_out, double* forward_out, double* inverse_out) {
    using namespace shg;
    clear_error();
    if (m < 1 || m > 65536) return fail(SHG_ERR_INVALID, "m = %d must be in 1..65536", m);
    if (!(d > 0) || !std::isfinite(d) || !(bi >= 0) || !std::isfinite(bi))
        return fail(SHG_ERR_INVALID, "spacing must be > 0 and the Biot number >= 0, both finite");
    if (!lambda_out || !forward_out || !inverse_out) return fail(SHG_ERR_INVALID, "output pointer is NULL");
    Op1D op;
    op.m = m;
    op.d = d;
    op.lo_robin = lo_robin ? 1 : 0;
    op.hi_robin = hi_robin ? 1 : 0;
    op.bi = bi;
    std::vector<double> lam, F, G;
    if (!op_modes(op, lam, F, G)) return fail(SHG_ERR_NOT_CONVERGED, "heat operator eigendecomposition (m = %d)", m);
    std::memcpy(lambda_out, lam.data(), sizeof(double) * m);
    std::memcpy(forward_out, F.data(), sizeof(double) * F.size());
    std::memcpy(inverse_out, G.data(), sizeof(double) * G.size());
    return SHG_OK;
}
