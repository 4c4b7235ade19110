// Divide-and-conquer eigensolver for the real symmetric tridiagonal matrix
// T = tridiag(e, d, e), one CTA, everything in shared memory.
//
// Method (Cuppen's divide and conquer with the Gu-Eisenstat correction, the
// algorithm of LAPACK dstedc / dlaed0-dlaed4):
//   * T is torn at every index k in [1, n): d[k-1] and d[k] each lose |e[k-1]|,
//     so that T = blockdiag(T1', T2') + |e| v v^T with v = e_{k-1} + sign(e) e_k.
//   * Leaves are 1x1 (Z = I). Blocks are merged bottom-up along a power-of-two
//     tree: level `half` merges [a, a+half) with [a+half, a+2*half).
//   * A merge forms z = (last row of Q1, sign(e) * first row of Q2)/sqrt(2),
//     rho = 2|e|, deflates entries with rho|z_j| <= tol and pairs of nearly
//     equal poles (Givens rotation of the two eigenvector columns), solves the
//     secular equation 1 + rho sum_j z_j^2/(d_j - lambda) = 0 for the K
//     remaining roots (one thread per root), recomputes z from the computed
//     roots with Loewner's formula so that the new eigenvectors are orthogonal
//     to working precision, and multiplies the old eigenvector columns by the
//     K x K eigenvector matrix of the rank-one problem.
// The secular solver is this file's own: each root is bracketed between its
// two poles, measured from the nearer pole (so that every d_j - lambda is
// formed without cancellation), and iterated with a two-pole rational model
// (fit value and slope of the left and right partial sums at the current
// point, solve the resulting quadratic), safeguarded by bisection.
//
// Output: Z (n x n, column slot j holds the eigenvector of w[j]); w[] in the
// caller's units. Eigenvalues are not sorted here.
//
// NMAX > 0 bounds n at compile time (Z, U in shared memory; merge products
// accumulate in registers). NMAX == 0 is the any-n form for matrices kept in
// global memory: merges wider than 32 columns are 16 x 16 FP64 tensor-core
// tiles written to the separate buffer Zo and copied back.
#pragma once

#include "geneig_common.cuh"

namespace sgeig {

struct DCShared {
    double* Z;  int ldz;    // eigenvectors
    double* U;  int ldu;    // K x K blocks of each merge at [a, a+K)^2
    double* Zo;             // NMAX == 0 only: n x ldz product buffer of the merge GEMMs
    double* d;  double* e;  // tridiagonal (modified)
    double* w;              // eigenvalue of column slot j
    double* z;              // merge z-vector by column slot
    double* dl;             // non-deflated poles [a, a+K)
    double* zz;             // their z
    double* zh;             // Loewner z-hat
    double* rt;             // root offsets from their origin pole
    int* org;               // origin pole (merge-local index) of each root
    int* nd;                // non-deflated column slots [a, a+K)
    int* perm;              // ascending order of the merge's eigenvalues
    int* kcnt;              // K per merge, indexed by a
    double* rho;            // rho per merge, indexed by a
    double* scal;           // [0] = scale applied to T
};

// Largest power of two strictly below x (x >= 2).
__host__ __device__ constexpr int top_bit(int x) { return (x & (x - 1)) ? top_bit(x & (x - 1)) : x; }
__host__ __device__ constexpr int pow2_below(int x) { return (x & (x - 1)) ? top_bit(x) : x / 2; }
static_assert(pow2_below(48) == 32 && pow2_below(64) == 32 && pow2_below(32) == 16 && pow2_below(16) == 8, "pow2_below");

// Number of doubles / ints of scratch DCShared needs for size n (excluding Z, U).
__host__ __device__ inline int dc_vec_doubles(int n) { return 8 * n + 2; }
__host__ __device__ inline int dc_vec_ints(int n) { return 4 * n; }

// Sum over the P consecutive lanes that share one root (P = 1, 2 or 4); on
// the host (P = 1) it is the identity. Every lane ends with the same value
// (the butterfly adds the same pairs in the same order up to commutation).
template <int P>
__host__ __device__ __forceinline__ double lanes_sum(double v, unsigned mask) {
#ifdef __CUDA_ARCH__
    if (P >= 2) v += __shfl_xor_sync(mask, v, 1);
    if (P >= 4) v += __shfl_xor_sync(mask, v, 2);
#else
    (void)mask;
#endif
    return v;
}
template <int P>
__host__ __device__ __forceinline__ double lanes_prod(double v, unsigned mask) {
#ifdef __CUDA_ARCH__
    if (P >= 2) v *= __shfl_xor_sync(mask, v, 1);
    if (P >= 4) v *= __shfl_xor_sync(mask, v, 2);
#else
    (void)mask;
#endif
    return v;
}

// Root i (0-based) of 1 + rho sum_j zz_j^2 / (dl_j - x) = 0 with dl ascending,
// rho > 0, computed by P lanes together (lane qq sums the terms j = qq mod P).
// Returns the offset tau of the root from pole `org`; the return value is the
// number of iterations taken.
template <int P>
__host__ __device__ inline int secular_root_p(int i, int K, const double* dl, const double* zz, double rho,
                                              int qq, unsigned mask, double& tau_out, int& org_out) {
    if (K == 1) { org_out = 0; tau_out = rho * zz[0] * zz[0]; return 0; }
    int o;
    double lo, hi, tau;
    if (i < K - 1) {
        const double gap = dl[i + 1] - dl[i];
        const double mid = 0.5 * gap;
        double gs = 0.0;
#pragma unroll 4
        for (int j = qq; j < K; j += P) {
            const double del = (dl[j] - dl[i]) - mid;
            gs = fma(rho * zz[j], zz[j] * fast_rcp(del), gs);
        }
        const double g = 1.0 + lanes_sum<P>(gs, mask);
        if (g >= 0.0) { o = i;     lo = 0.0;  hi = mid; tau = mid; }
        else          { o = i + 1; lo = -mid; hi = 0.0; tau = -mid; }
        // Starting point: the two nearest poles' terms exactly, the others
        // frozen at their midpoint value c (the fixed-weight start), i.e. the
        // root of c + a/(p - x) + b/(q - x) in origin coordinates, taken when
        // it lies inside the bracket (otherwise the midpoint stays).
        const double a = rho * zz[i] * zz[i], b = rho * zz[i + 1] * zz[i + 1];
        const double rm = fast_rcp(mid);
        const double c = g + (a - b) * rm;
        const double p0 = dl[i] - dl[o], q0 = dl[i + 1] - dl[o];
        const double B = -(c * (p0 + q0) + a + b), C = a * q0 + b * p0;
        if (c != 0.0) {
            double disc = B * B - 4.0 * c * C;
            if (disc < 0.0) disc = 0.0;
            const double qq2 = -0.5 * (B + copysign(sqrt(disc), B));
            const double x1 = qq2 * fast_rcp(c), x2 = (qq2 != 0.0) ? C * fast_rcp(qq2) : x1;
            if (x1 > lo && x1 < hi) tau = x1;
            else if (x2 > lo && x2 < hi) tau = x2;
        }
    } else {
        double ss = 0.0;
        for (int j = qq; j < K; j += P) ss += zz[j] * zz[j];
        o = K - 1; lo = 0.0; hi = rho * lanes_sum<P>(ss, mask); tau = hi;
        // Starting point: the last pole's term exactly, the others frozen at
        // the bracket's midpoint m (c = f(m) - b / (-m)): the root of
        // c + b / (-x) = 0, x = b / c, when it lies inside the bracket.
        const double m = 0.5 * hi;
        if (m > 0.0) {
            double gs = 0.0;
#pragma unroll 4
            for (int j = qq; j < K; j += P) {
                const double del = (dl[j] - dl[K - 1]) - m;
                gs = fma(rho * zz[j], zz[j] * fast_rcp(del), gs);
            }
            const double b = rho * zz[K - 1] * zz[K - 1];
            const double c = 1.0 + lanes_sum<P>(gs, mask) + b * fast_rcp(m);
            if (c > 0.0) {
                const double x = b * fast_rcp(c);
                if (x > lo && x < hi) tau = x;
            }
        }
    }
    const double dlo = dl[o];
    const double p = dl[i] - dlo;
    const double q = (i < K - 1) ? dl[i + 1] - dlo : 0.0;
    int it = 0;
    for (; it < 80; ++it) {
        double psi = 0.0, dpsi = 0.0, phi = 0.0, dphi = 0.0, erra = 0.0;
#pragma unroll 4
        for (int j = qq; j < K; j += P) {
            const double del = (dl[j] - dlo) - tau;
            const double t = zz[j] * fast_rcp(del);
            const double term = rho * zz[j] * t;
            const double dterm = rho * t * t;
            const bool left = j <= i;       // poles left of the root go to psi
            psi += left ? term : 0.0;
            dpsi += left ? dterm : 0.0;
            phi += left ? 0.0 : term;
            dphi += left ? 0.0 : dterm;
            erra += fabs(term);
        }
        psi = lanes_sum<P>(psi, mask);
        dpsi = lanes_sum<P>(dpsi, mask);
        phi = lanes_sum<P>(phi, mask);
        dphi = lanes_sum<P>(dphi, mask);
        erra = lanes_sum<P>(erra, mask);
        const double g = 1.0 + psi + phi;
        const double err = kEps * (2.0 + 8.0 * erra + 3.0 * fabs(tau) * (dpsi + dphi));
        if (fabs(g) <= err) break;
        if (g < 0.0) lo = tau; else hi = tau;
        if (hi - lo <= 2.0 * kEps * fmax(fabs(lo), fabs(hi))) break;
        double tn;
        if (i < K - 1) {
            const double bpsi = dpsi * (p - tau) * (p - tau);
            const double apsi = psi - dpsi * (p - tau);
            const double bphi = dphi * (q - tau) * (q - tau);
            const double aphi = phi - dphi * (q - tau);
            const double c = 1.0 + apsi + aphi;
            // c + bpsi/(p - x) + bphi/(q - x) = 0 in origin coordinates
            // (one of p, q is 0, so p q = 0):
            //   c x^2 - (c (p + q) + bpsi + bphi) x + (bpsi q + bphi p) = 0
            const double B = -(c * (p + q) + bpsi + bphi);
            const double C = bpsi * q + bphi * p;
            tn = lo - 1.0;
            if (c == 0.0) {
                tn = -C * fast_rcp(B);
            } else {
                double disc = B * B - 4.0 * c * C;
                if (disc < 0.0) disc = 0.0;
                const double qq2 = -0.5 * (B + copysign(sqrt(disc), B));
                const double x1 = qq2 * fast_rcp(c), x2 = (qq2 != 0.0) ? C * fast_rcp(qq2) : x1;
                tn = (x1 > lo && x1 < hi) ? x1 : x2;
            }
        } else {
            const double bpsi = dpsi * (p - tau) * (p - tau);
            const double apsi = psi - dpsi * (p - tau);
            const double den = 1.0 + apsi;
            tn = (den > 0.0) ? p + bpsi * fast_rcp(den) : lo - 1.0;
        }
        // converged when the model step is within a few ulps of the iterate
        // (it may then round just outside the bracket)
        if (fabs(tn - tau) <= 4.0 * kEps * fabs(tau)) {
            if (tn > lo && tn < hi) tau = tn;
            break;
        }
        if (!(tn > lo && tn < hi) || it >= 30) tn = 0.5 * (lo + hi);
        if (tn == tau) break;
        tau = tn;
    }
    tau_out = tau;
    org_out = o;
    return it;
}

// Single-lane form (host tests and callers without lane groups).
__host__ __device__ inline int secular_root(int i, int K, const double* dl, const double* zz, double rho,
                                            double& tau_out, int& org_out) {
    return secular_root_p<1>(i, K, dl, zz, rho, 0, 0u, tau_out, org_out);
}

// Phase E of a level whose single merge covers [0, n): 8x8 output tiles on
// the FP64 tensor cores (mma.m8n8k4.f64), one warp per tile, accumulators in
// registers (n <= NMAX); all reads finish before the barrier, then the tiles
// are written back to the gathered columns.
template <int NT, int NMAX, int BLOCK = NT>
__device__ __forceinline__ void dc_merge_top_regs(int n, const DCShared& s) {
    const int lane = team_tid<NT, BLOCK>() & 31, warp = team_tid<NT, BLOCK>() >> 5;
    constexpr int NW = NT / 32;
    const int K = s.kcnt[0];
    const int tm = (n + 7) >> 3, tn = (K + 7) >> 3;
    constexpr int MAXT = ((NMAX / 8) * (NMAX / 8) + NW - 1) / NW;
    double acc[MAXT][2];
#pragma unroll
    for (int u = 0; u < MAXT; ++u) {
        acc[u][0] = acc[u][1] = 0.0;
        const int t = warp + NW * u;
        if (K == 0 || t >= tm * tn) continue;
        const int ti = t / tn, tj = t - ti * tn;
        const int ia = 8 * ti + (lane >> 2), jb = 8 * tj + (lane >> 2);
        for (int k = 0; k < K; k += 4) {
            const int ka = k + (lane & 3);
            const double av = (ia < n && ka < K) ? s.Z[ia + (size_t)s.nd[ka] * s.ldz] : 0.0;
            const double bv = (ka < K && jb < K) ? s.U[ka + (size_t)jb * s.ldu] : 0.0;
            asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                : "+d"(acc[u][0]), "+d"(acc[u][1]) : "d"(av), "d"(bv));
        }
    }
    team_sync<NT, BLOCK>();
#pragma unroll
    for (int u = 0; u < MAXT; ++u) {
        const int t = warp + NW * u;
        if (K == 0 || t >= tm * tn) continue;
        const int ti = t / tn, tj = t - ti * tn;
        const int r = 8 * ti + (lane >> 2), j = 8 * tj + 2 * (lane & 3);
        if (r < n && j < K) s.Z[r + (size_t)s.nd[j] * s.ldz] = acc[u][0];
        if (r < n && j + 1 < K) s.Z[r + (size_t)s.nd[j + 1] * s.ldz] = acc[u][1];
    }
}

// Phase E of a level of merges at most 4 * UMAX columns wide: four lanes per
// row, lane q accumulating output columns j = q + 4u in registers. A row's
// reads and writes stay within its quad, so no barrier is needed between them.
template <int NT, int UMAX, int BLOCK = NT>
__device__ __forceinline__ void dc_merge_rows_regs(int n, int half, int span, const DCShared& s) {
    for (int p0 = 0; p0 < 4 * n; p0 += NT) {
        const int pidx = p0 + team_tid<NT, BLOCK>();
        const int r = pidx >> 2, part = pidx & 3;
        const int a = (r < n) ? r - r % span : n;
        const bool active = r < n && a + half < n && s.kcnt[a] > 0;
        const int K = active ? s.kcnt[a] : 0;
        double acc[UMAX];
#pragma unroll
        for (int u = 0; u < UMAX; ++u) acc[u] = 0.0;
        for (int l = 0; l < K; ++l) {
            const double x = s.Z[r + (size_t)s.nd[a + l] * s.ldz];
            const double* ur = s.U + (a + l) + (size_t)(a + part) * s.ldu;
#pragma unroll
            for (int u = 0; u < UMAX; ++u)
                if (part + 4 * u < K) acc[u] = fma(x, ur[(size_t)(4 * u) * s.ldu], acc[u]);
        }
        __syncwarp();
#pragma unroll
        for (int u = 0; u < UMAX; ++u) {
            const int j = part + 4 * u;
            if (j < K) s.Z[r + (size_t)s.nd[a + j] * s.ldz] = acc[u];
        }
    }
}

// Phase E for any merge width (NMAX == 0): for every merge [a, a+m) of the
// level, the m x K product Z(a:a+m, nd) * U on the FP64 tensor cores in
// 16 x 16 warp tiles (2 x 2 mma.m8n8k4 tiles), rows outside [a, a+m) being
// zero in those columns. Tiles are dealt round-robin to the warps across all
// merges of the level; products go to Zo, then back into Z after a barrier.
template <int NT, int BLOCK = NT>
__device__ __forceinline__ void dc_merge_tiled(int n, int half, int span, const DCShared& s) {
    const int lane = team_tid<NT, BLOCK>() & 31, warp = team_tid<NT, BLOCK>() >> 5;
    constexpr int NW = NT / 32;
    int dealt = 0;
    for (int a = 0; a + half < n; a += span) {
        const int K = s.kcnt[a];
        if (K == 0) continue;
        const int m = min(span, n - a);
        const int tn = (K + 15) >> 4, T = ((m + 15) >> 4) * tn;
        const int* nd = s.nd + a;
        const double* Ub = s.U + a + (size_t)a * s.ldu;
        int t = (warp - dealt % NW + NW) % NW;
        for (; t < T; t += NW) {
            const int ti = t / tn, tj = t - ti * tn;
            const int r0 = 16 * ti + (lane >> 2), j0 = 16 * tj + (lane >> 2);
            double acc[2][2][2];
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int g = 0; g < 2; ++g) acc[h][g][0] = acc[h][g][1] = 0.0;
#pragma unroll 4
            for (int k = 0; k < K; k += 4) {
                const int ka = k + (lane & 3);
                const bool kin = ka < K;
                const double* zc = s.Z + a + (size_t)(kin ? nd[ka] : 0) * s.ldz;
                double av[2], bv[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    av[h] = (kin && r0 + 8 * h < m) ? zc[r0 + 8 * h] : 0.0;
                    bv[h] = (kin && j0 + 8 * h < K) ? Ub[ka + (size_t)(j0 + 8 * h) * s.ldu] : 0.0;
                }
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int g = 0; g < 2; ++g)
                        asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                            : "+d"(acc[h][g][0]), "+d"(acc[h][g][1]) : "d"(av[h]), "d"(bv[g]));
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = 16 * ti + 8 * h + (lane >> 2);
                if (r >= m) continue;
#pragma unroll
                for (int g = 0; g < 2; ++g) {
                    const int j = 16 * tj + 8 * g + 2 * (lane & 3);
                    if (j < K) s.Zo[a + r + (size_t)nd[j] * s.ldz] = acc[h][g][0];
                    if (j + 1 < K) s.Zo[a + r + (size_t)nd[j + 1] * s.ldz] = acc[h][g][1];
                }
            }
        }
        dealt += T;
    }
    team_sync<NT, BLOCK>();
    const int width = min(span, n);
    for (int idx = team_tid<NT, BLOCK>(); idx < n * width; idx += NT) {
        const int jj = idx / n, r = idx - jj * n;
        const int a = r - r % span;
        if (a + half >= n || jj >= s.kcnt[a]) continue;
        const size_t o = r + (size_t)s.nd[a + jj] * s.ldz;
        s.Z[o] = s.Zo[o];
    }
}

// All NT threads of the CTA call this. n >= 1. On return Z, w hold the
// eigen-decomposition of the tridiagonal (d, e) given on entry.
template <int NT, int NMAX, int BLOCK = NT>
__device__ void tridiag_dc(int n, DCShared s) {
    const int tid = team_tid<NT, BLOCK>(), lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;

    // ---- scale T by a power of two so that max |T_ij| is in [0.5, 1)
    if (tid < 32) {
        double mx = 0.0;
        for (int i = lane; i < n; i += 32) mx = fmax(mx, fabs(s.d[i]));
        for (int i = lane; i < n - 1; i += 32) mx = fmax(mx, fabs(s.e[i]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) {
            int ex = 0;
            double sc = 1.0;
            if (mx > 0.0 && isfinite(mx)) { frexp(mx, &ex); sc = ldexp(1.0, -ex); }
            s.scal[0] = sc;
        }
    }
    team_sync<NT, BLOCK>();
    const double sc = s.scal[0];
    // ---- scale, tear at every split, leaves: Z = I, w = d
    for (int i = tid; i < n; i += NT) {
        double di = s.d[i] * sc;
        if (i > 0) di -= fabs(s.e[i - 1] * sc);
        if (i < n - 1) di -= fabs(s.e[i] * sc);
        s.w[i] = di;
    }
    team_sync<NT, BLOCK>();   // every unscaled e[] read above before it is scaled in place
    for (int i = tid; i < n - 1; i += NT) s.e[i] *= sc;
    for (int idx = tid; idx < n * n; idx += NT) {
        const int j = idx / n, i = idx - j * n;
        s.Z[i + j * s.ldz] = (i == j) ? 1.0 : 0.0;
    }
    team_sync<NT, BLOCK>();
    phase_mark(10);

    for (int half = 1; half < n; half <<= 1) {
        const int span = half << 1;
        // ---- phase A: one warp per merge: z, order, deflation
        for (int a = warp * span; a < n; a += NW * span) {
            const int k = a + half;
            if (k >= n) { if (lane == 0) s.kcnt[a] = 0; continue; }
            const int b = min(a + span, n);
            const int m = b - a;
            const double er = s.e[k - 1];
            if (er == 0.0) { if (lane == 0) s.kcnt[a] = 0; continue; }
            const double sgn = er < 0.0 ? -1.0 : 1.0;
            const double rho = 2.0 * fabs(er);
            double zmax = 0.0, dmax = 0.0;
            for (int j = a + lane; j < b; j += 32) {
                const double zj = (j < k ? s.Z[(k - 1) + j * s.ldz] : sgn * s.Z[k + j * s.ldz]) * 0.70710678118654752440;
                s.z[j] = zj;
                zmax = fmax(zmax, fabs(zj));
                dmax = fmax(dmax, fabs(s.w[j]));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                zmax = fmax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
                dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
            }
            const double tol = 8.0 * kEps * fmax(dmax, zmax);
            for (int j = a + lane; j < b; j += 32) {
                const double wj = order_key(s.w[j]);
                int r = 0;
                for (int t = a; t < b; ++t) {
                    const double wt = order_key(s.w[t]);
                    r += (wt < wj) || (wt == wj && t < j);
                }
                s.perm[a + r] = j;   // r in [0, m): the keys are totally ordered
            }
            __syncwarp();
            // fast path: keep entries with rho|z| > tol, in ascending order
            int base = 0;
            for (int t0 = 0; t0 < m; t0 += 32) {
                const int t = t0 + lane;
                int j = -1;
                bool keep = false;
                if (t < m) { j = s.perm[a + t]; keep = rho * fabs(s.z[j]) > tol; }
                const unsigned mask = __ballot_sync(0xffffffffu, keep);
                const int pos = base + __popc(mask & ((1u << lane) - 1u));
                if (keep) { s.nd[a + pos] = j; s.dl[a + pos] = s.w[j]; s.zz[a + pos] = s.z[j]; }
                base += __popc(mask);
            }
            __syncwarp();
            const int K0 = base;
            bool close = false;
            for (int p = 1 + lane; p < K0; p += 32) {
                const double T = s.dl[a + p] - s.dl[a + p - 1];
                const double zn = s.zz[a + p], zp = s.zz[a + p - 1];
                close |= fabs(T) * fabs(zn * zp) <= tol * (zn * zn + zp * zp);
            }
            close = __any_sync(0xffffffffu, close);
            if (close && lane == 0) {
                // sequential deflation with rotations of nearly equal poles
                int K = 0, pj = -1;
                for (int t = 0; t < m; ++t) {
                    const int nj = s.perm[a + t];
                    if (!(rho * fabs(s.z[nj]) > tol)) continue;
                    if (pj < 0) { pj = nj; continue; }
                    const double T = s.w[nj] - s.w[pj];
                    const double zn = s.z[nj], zp = s.z[pj];
                    const double t2 = zn * zn + zp * zp;
                    if (fabs(T) * fabs(zn * zp) <= tol * t2) {
                        const double ta = sqrt(t2);
                        const double c = zn / ta, sn = -zp / ta;
                        s.z[nj] = ta; s.z[pj] = 0.0;
                        for (int r = a; r < b; ++r) {
                            const double x = s.Z[r + pj * s.ldz], y = s.Z[r + nj * s.ldz];
                            s.Z[r + pj * s.ldz] = c * x + sn * y;
                            s.Z[r + nj * s.ldz] = c * y - sn * x;
                        }
                        const double wp = s.w[pj], wn = s.w[nj];
                        s.w[pj] = wp * c * c + wn * sn * sn;
                        s.w[nj] = wp * sn * sn + wn * c * c;
                        pj = nj;
                    } else {
                        s.nd[a + K] = pj; s.dl[a + K] = s.w[pj]; s.zz[a + K] = s.z[pj]; ++K;
                        pj = nj;
                    }
                }
                if (pj >= 0) { s.nd[a + K] = pj; s.dl[a + K] = s.w[pj]; s.zz[a + K] = s.z[pj]; ++K; }
                s.kcnt[a] = K;
                s.rho[a] = rho;
            } else if (lane == 0) {
                s.kcnt[a] = K0;
                s.rho[a] = rho;
            }
        }
        team_sync<NT, BLOCK>();
        phase_mark(11);
        // ---- phase B: secular roots, four lanes per root (root slot = tid / 4)
        for (int p0 = 0; p0 < 4 * n; p0 += NT) {
            const int pidx = (p0 + tid) >> 2, qq = tid & 3;
            const unsigned qmask = 0xFu << (lane & ~3);
            if (pidx >= n) continue;
            const int a = pidx - pidx % span;
            if (a + half >= n) continue;
            const int i = pidx - a, K = s.kcnt[a];
            if (i >= K) continue;
            double t; int o;
            const int its = secular_root_p<4>(i, K, s.dl + a, s.zz + a, s.rho[a], qq, qmask, t, o);
            if (qq == 0) {
                s.rt[pidx] = t; s.org[pidx] = o;
                phase_count(27, (unsigned long long)its);
                phase_count(29, 1);
                phase_level_max((unsigned)its);
            }
        }
        team_sync<NT, BLOCK>();
        phase_mark(12);
        phase_level_flush(28);
        // ---- phase C: Loewner z-hat, four lanes per root
        for (int p0 = 0; p0 < 4 * n; p0 += NT) {
            const int pidx = (p0 + tid) >> 2, qq = tid & 3;
            const unsigned qmask = 0xFu << (lane & ~3);
            if (pidx >= n) continue;
            const int a = pidx - pidx % span;
            if (a + half >= n) continue;
            const int i = pidx - a, K = s.kcnt[a];
            if (i >= K) continue;
            const double* dl = s.dl + a;
            const double dli = dl[i];
            double W = (qq == 0) ? (dli - dl[s.org[a + i]]) - s.rt[a + i] : 1.0;
            for (int j = qq; j < K; j += 4) {
                if (j == i) continue;
                const double del = (dli - dl[s.org[a + j]]) - s.rt[a + j];
                W *= del * fast_rcp(dli - dl[j]);
            }
            W = lanes_prod<4>(W, qmask);
            if (qq == 0) s.zh[pidx] = copysign(sqrt(fmax(-W, 0.0)), s.zz[pidx]);
        }
        team_sync<NT, BLOCK>();
        phase_mark(13);
        // ---- phase D: eigenvector columns of the rank-one problem (four lanes
        // per column), new eigenvalues
        for (int p0 = 0; p0 < 4 * n; p0 += NT) {
            const int pidx = (p0 + tid) >> 2, qq = tid & 3;
            const unsigned qmask = 0xFu << (lane & ~3);
            if (pidx >= n) continue;
            const int a = pidx - pidx % span;
            if (a + half >= n) continue;
            const int j = pidx - a, K = s.kcnt[a];
            if (j >= K) continue;
            const double* dl = s.dl + a;
            const double base = dl[s.org[a + j]], tj = s.rt[a + j];
            double* ucol = s.U + a + (size_t)(a + j) * s.ldu;
            double nrm = 0.0;
            for (int l = qq; l < K; l += 4) {
                const double v = s.zh[a + l] * fast_rcp((dl[l] - base) - tj);
                ucol[l] = v;
                nrm = fma(v, v, nrm);
            }
            const double inv = rsqrt(lanes_sum<4>(nrm, qmask));
            for (int l = qq; l < K; l += 4) ucol[l] *= inv;
            if (qq == 0) s.w[s.nd[a + j]] = base + tj;
        }
        team_sync<NT, BLOCK>();
        phase_mark(14);
        // ---- phase E: Z(:, nd) <- Z(:, nd) * U.
        if constexpr (NMAX > 0) {
            if (span >= n) dc_merge_top_regs<NT, NMAX, BLOCK>(n, s);
            else dc_merge_rows_regs<NT, pow2_below(NMAX) / 4, BLOCK>(n, half, span, s);
        } else {
            if (span <= 32) dc_merge_rows_regs<NT, 8, BLOCK>(n, half, span, s);
            else dc_merge_tiled<NT, BLOCK>(n, half, span, s);
        }
        team_sync<NT, BLOCK>();
        phase_mark(15);
    }
    // ---- back to the caller's units
    const double inv = 1.0 / sc;
    for (int i = tid; i < n; i += NT) s.w[i] *= inv;
    team_sync<NT, BLOCK>();
}

}  // namespace sgeig
