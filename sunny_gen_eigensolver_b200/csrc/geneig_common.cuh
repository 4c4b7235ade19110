// Device helpers shared by the sm_100a eigensolver kernels: complex FP64
// arithmetic on double2, warp / column-group reductions, Givens rotations,
// the 2x2 symmetric eigenproblem and the resumable implicit QL/QR iteration
// on a real symmetric tridiagonal matrix.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace sgeig {

// ---------------------------------------------------------------- complex FP64
__device__ __forceinline__ double2 c2(double re, double im) { return make_double2(re, im); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return c2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return c2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return c2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return c2(a.x, -a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return c2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// acc + a*b
__device__ __forceinline__ double2 cfma(double2 acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc - a*b
__device__ __forceinline__ double2 cfms(double2 acc, double2 a, double2 b) {
    acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
// acc + conj(a)*b
__device__ __forceinline__ double2 cfmac(double2 acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
// acc - conj(a)*b
__device__ __forceinline__ double2 cfmsc(double2 acc, double2 a, double2 b) {
    acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc - a*conj(b)
__device__ __forceinline__ double2 cfms_bc(double2 acc, double2 a, double2 b) {
    acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
// Sum over the G consecutive lanes of one column group (G a power of two).
template <int G>
__device__ __forceinline__ double2 group_sum2(unsigned mask, double2 v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(mask, v.x, o, G);
        v.y += __shfl_xor_sync(mask, v.y, o, G);
    }
    return v;
}
template <int G>
__device__ __forceinline__ double2 group_bcast2(unsigned mask, double2 v, int src) {
    v.x = __shfl_sync(mask, v.x, src, G);
    v.y = __shfl_sync(mask, v.y, src, G);
    return v;
}

// First index i >= start with i % G == q.
template <int G>
__device__ __forceinline__ int first_in_class(int start, int q) {
    int d = q - (start % G);
    if (d < 0) d += G;
    return start + d;
}

// Total-order sort key for eigenvalues: NaN sorts after +inf, so that ranks
// computed as #{t : key_t < key_j or (key_t == key_j and t < j)} always form
// a permutation (they are used as indices).
__host__ __device__ __forceinline__ double order_key(double x) {
    return (x != x) ? __builtin_inf() : x;
}

// Reciprocal without a divide: the hardware's approximate FP64 reciprocal
// (PTX rcp.approx.ftz.f64) refined by two Newton-Raphson steps
// r <- r + r (1 - x r), each of which doubles the number of correct bits.
// Branch-free, so independent reciprocals pipeline, unlike IEEE division.
// Accuracy (checked against 1/x on the GPU by the self-test entry point):
// within 1 ulp for normal x; x = 0 or +-inf give NaN (callers never pass them).
__host__ __device__ __forceinline__ double fast_rcp(double x) {
#ifdef __CUDA_ARCH__
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
#else
    return 1.0 / x;
#endif
}

// ---------------------------------------------------------------- constants
// LAPACK dlamch conventions: eps = 2^-53 (relative machine precision),
// safmin = smallest normal double.
constexpr double kEps    = 1.1102230246251565e-16;
constexpr double kEps2   = kEps * kEps;
constexpr double kSafmin = 2.2250738585072014e-308;
constexpr double kSsfmax = 2.2346346549904327e+153;  // sqrt(1/safmin) / 3
constexpr double kSsfmin = 1.2101683706950478e-122;  // sqrt(safmin) / eps^2

// ---------------------------------------------------------------- rotations
// Plane rotation [c s; -s c] [f; g] = [r; 0] with c >= 0 and r carrying the
// sign of f (the convention of LAPACK 3.10+ dlartg). Inputs far from 1 in
// magnitude are rescaled first so that f^2 + g^2 neither overflows nor
// underflows.
__device__ __forceinline__ void givens(double f, double g, double& c, double& s, double& r) {
    if (g == 0.0) { c = 1.0; s = 0.0; r = f; return; }
    if (f == 0.0) { c = 0.0; s = copysign(1.0, g); r = fabs(g); return; }
    const double af = fabs(f), ag = fabs(g);
    const double mx = fmax(af, ag);
    if (mx > 1e150 || mx < 1e-150) {
        const double fs = f / mx, gs = g / mx;
        const double d = sqrt(fs * fs + gs * gs);
        c = fabs(fs) / d;
        const double rs = copysign(d, f);
        r = rs * mx;
        s = gs / rs;
    } else {
        const double d = sqrt(f * f + g * g);
        c = af / d;
        r = copysign(d, f);
        s = g / r;
    }
}

// Eigen-decomposition of the real symmetric 2x2 matrix [a b; b c]:
// rt1 is the eigenvalue of larger magnitude, rt2 the other, and (cs1, sn1)
// the unit eigenvector for rt1. This is the classical stable formulation
// (Wilkinson; the same method LAPACK documents for dlaev2): the larger root
// from the discriminant, the smaller from the determinant, the vector from
// the better-conditioned of the two component ratios.
__device__ __forceinline__ void sym_eig2(double a, double b, double c,
                                         double& rt1, double& rt2, double& cs1, double& sn1) {
    const double sm = a + c, df = a - c, adf = fabs(df), tb = b + b, ab = fabs(tb);
    double acmx, acmn;
    if (fabs(a) > fabs(c)) { acmx = a; acmn = c; } else { acmx = c; acmn = a; }
    double rt;
    if (adf > ab)      { const double t = ab / adf; rt = adf * sqrt(1.0 + t * t); }
    else if (adf < ab) { const double t = adf / ab; rt = ab * sqrt(1.0 + t * t); }
    else               { rt = ab * 1.4142135623730951; }
    int sgn1;
    if (sm < 0.0)      { rt1 = 0.5 * (sm - rt); sgn1 = -1; rt2 = (acmx / rt1) * acmn - (b / rt1) * b; }
    else if (sm > 0.0) { rt1 = 0.5 * (sm + rt); sgn1 = 1;  rt2 = (acmx / rt1) * acmn - (b / rt1) * b; }
    else               { rt1 = 0.5 * rt; rt2 = -0.5 * rt; sgn1 = 1; }
    int sgn2;
    double cs;
    if (df >= 0.0) { cs = df + rt; sgn2 = 1; } else { cs = df - rt; sgn2 = -1; }
    if (fabs(cs) > ab) {
        const double ct = -tb / cs;
        sn1 = 1.0 / sqrt(1.0 + ct * ct);
        cs1 = ct * sn1;
    } else if (ab == 0.0) {
        cs1 = 1.0; sn1 = 0.0;
    } else {
        const double tn = -cs / tb;
        cs1 = 1.0 / sqrt(1.0 + tn * tn);
        sn1 = tn * cs1;
    }
    if (sgn1 == sgn2) { const double tn = cs1; cs1 = -sn1; sn1 = tn; }
}

// ---------------------------------------------------------------- tridiagonal QL/QR
// Implicit-shift QL/QR on the real symmetric tridiagonal (d[0..n), e[0..n-1)),
// the method of LAPACK zsteqr/dsteqr (which zheev, and so zhegv, use):
// blocks split where |e| <= eps*sqrt(|d_i d_i+1|), each block is iterated
// with a Wilkinson-type shift, QL when its bottom diagonal entry is larger in
// magnitude and QR otherwise, 2x2 blocks are finished in closed form, at most
// 30*n sweeps in total, and blocks with extreme norms are scaled first.
//
// It is written as a resumable producer: each call runs until it has produced
// one sweep of plane rotations (rc[i], rs[i]) for column pairs (i, i+1),
// i in [lo, lo+count), and returns count (> 0); `backward` tells whether the
// rotations must be applied from the highest index down (QL) or upward (QR).
// Applying rotation (c, s) to columns (i, i+1) of Z means
//     z_{i+1} <- c z_{i+1} - s z_i,   z_i <- s z_{i+1} + c z_i.
// Returns 0 when the iteration has finished; `info` then holds the number of
// off-diagonal entries that failed to converge (0 on success).
struct TridiagQL {
    enum : int { kNewBlock = 0, kQL = 1, kQR = 2, kEndBlock = 3, kDone = 4 };
    int state, n, l1, l, lend, lsv, lendsv, jtot, nmaxit, iscale, info;
    double anorm;

    __device__ void init(int n_) {
        n = n_; state = kNewBlock; l1 = 0; l = lend = lsv = lendsv = 0;
        jtot = 0; nmaxit = 30 * n_; iscale = 0; info = 0; anorm = 0.0;
    }

    __device__ static void scale_block(double* d, double* e, int lo, int hi, double f) {
        for (int i = lo; i <= hi; ++i) d[i] *= f;
        for (int i = lo; i < hi; ++i) e[i] *= f;
    }

    __device__ int next(double* d, double* e, double* rc, double* rs, int& lo, bool& backward) {
        for (;;) {
            switch (state) {
            case kNewBlock: {
                if (l1 >= n) { state = kDone; return 0; }
                if (l1 > 0) e[l1 - 1] = 0.0;
                int m = n - 1;
                for (int mm = l1; mm <= n - 2; ++mm) {
                    const double tst = fabs(e[mm]);
                    if (tst == 0.0) { m = mm; break; }
                    if (tst <= (sqrt(fabs(d[mm])) * sqrt(fabs(d[mm + 1]))) * kEps) {
                        e[mm] = 0.0; m = mm; break;
                    }
                }
                l = l1; lsv = l; lend = m; lendsv = m; l1 = m + 1;
                if (lend == l) continue;
                double an = 0.0;
                for (int i = l; i <= lend; ++i) { const double v = fabs(d[i]); if (v > an || isnan(v)) an = v; }
                for (int i = l; i < lend; ++i)  { const double v = fabs(e[i]); if (v > an || isnan(v)) an = v; }
                anorm = an; iscale = 0;
                if (an == 0.0) continue;
                if (an > kSsfmax)      { iscale = 1; scale_block(d, e, l, lend, kSsfmax / an); }
                else if (an < kSsfmin) { iscale = 2; scale_block(d, e, l, lend, kSsfmin / an); }
                if (fabs(d[lend]) < fabs(d[l])) { lend = lsv; l = lendsv; }
                state = (lend > l) ? kQL : kQR;
                continue;
            }
            case kQL: {
                int m = lend;
                for (int mm = l; mm < lend; ++mm) {
                    const double tst = e[mm] * e[mm];
                    if (tst <= (kEps2 * fabs(d[mm])) * fabs(d[mm + 1]) + kSafmin) { m = mm; break; }
                }
                if (m < lend) e[m] = 0.0;
                double p = d[l];
                if (m == l) {
                    l += 1;
                    if (l > lend) state = kEndBlock;
                    continue;
                }
                if (m == l + 1) {
                    double rt1, rt2, c, s;
                    sym_eig2(d[l], e[l], d[l + 1], rt1, rt2, c, s);
                    rc[l] = c; rs[l] = s;
                    d[l] = rt1; d[l + 1] = rt2; e[l] = 0.0;
                    lo = l; backward = true;
                    l += 2;
                    if (l > lend) state = kEndBlock;
                    return 1;
                }
                if (jtot == nmaxit) { state = kEndBlock; continue; }
                ++jtot;
                double g = (d[l + 1] - p) / (2.0 * e[l]);
                double r = hypot(g, 1.0);
                g = d[m] - p + (e[l] / (g + copysign(r, g)));
                double s = 1.0, c = 1.0;
                p = 0.0;
                for (int i = m - 1; i >= l; --i) {
                    const double f = s * e[i], b = c * e[i];
                    givens(g, f, c, s, r);
                    if (i != m - 1) e[i + 1] = r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    rc[i] = c; rs[i] = -s;
                }
                d[l] -= p; e[l] = g;
                lo = l; backward = true;
                return m - l;
            }
            case kQR: {
                int m = lend;
                for (int mm = l; mm > lend; --mm) {
                    const double tst = e[mm - 1] * e[mm - 1];
                    if (tst <= (kEps2 * fabs(d[mm])) * fabs(d[mm - 1]) + kSafmin) { m = mm; break; }
                }
                if (m > lend) e[m - 1] = 0.0;
                double p = d[l];
                if (m == l) {
                    l -= 1;
                    if (l < lend) state = kEndBlock;
                    continue;
                }
                if (m == l - 1) {
                    double rt1, rt2, c, s;
                    sym_eig2(d[l - 1], e[l - 1], d[l], rt1, rt2, c, s);
                    rc[m] = c; rs[m] = s;
                    d[l - 1] = rt1; d[l] = rt2; e[l - 1] = 0.0;
                    lo = m; backward = false;
                    l -= 2;
                    if (l < lend) state = kEndBlock;
                    return 1;
                }
                if (jtot == nmaxit) { state = kEndBlock; continue; }
                ++jtot;
                double g = (d[l - 1] - p) / (2.0 * e[l - 1]);
                double r = hypot(g, 1.0);
                g = d[m] - p + (e[l - 1] / (g + copysign(r, g)));
                double s = 1.0, c = 1.0;
                p = 0.0;
                for (int i = m; i <= l - 1; ++i) {
                    const double f = s * e[i], b = c * e[i];
                    givens(g, f, c, s, r);
                    if (i != m) e[i - 1] = r;
                    g = d[i] - p;
                    r = (d[i + 1] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i] = g + p;
                    g = c * r - b;
                    rc[i] = c; rs[i] = s;
                }
                d[l] -= p; e[l - 1] = g;
                lo = m; backward = false;
                return l - m;
            }
            case kEndBlock: {
                if (iscale == 1)      scale_block(d, e, lsv, lendsv, anorm / kSsfmax);
                else if (iscale == 2) scale_block(d, e, lsv, lendsv, anorm / kSsfmin);
                iscale = 0;
                if (jtot < nmaxit) { state = kNewBlock; continue; }
                int cnt = 0;
                for (int i = 0; i < n - 1; ++i) if (e[i] != 0.0) ++cnt;
                info = cnt;
                state = kDone;
                return 0;
            }
            default:
                return 0;
            }
        }
    }
};

// Applies one sweep of rotations produced by TridiagQL::next to a row of Z
// whose element j sits at row[j * stride] (real part of a complex slot).
__device__ __forceinline__ void apply_sweep_row(double2* row, int stride, const double* rc,
                                                const double* rs, int lo, int count, bool backward) {
    if (backward) {
        const int top = lo + count;
        double carry = row[top * stride].x;
        for (int j = top - 1; j >= lo; --j) {
            const double c = rc[j], s = rs[j];
            const double zj = row[j * stride].x;
            row[(j + 1) * stride].x = c * carry - s * zj;
            carry = s * carry + c * zj;
        }
        row[lo * stride].x = carry;
    } else {
        double carry = row[lo * stride].x;
        for (int j = lo; j < lo + count; ++j) {
            const double c = rc[j], s = rs[j];
            const double zj1 = row[(j + 1) * stride].x;
            row[j * stride].x = s * zj1 + c * carry;
            carry = c * zj1 - s * carry;
        }
        row[(lo + count) * stride].x = carry;
    }
}

}  // namespace sgeig
