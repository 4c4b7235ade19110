// Per-pencil body of the tiled (l2-slot) solver, shared by its own kernel
// (geneig_tiled.cu) and the persistent uneven-size kernel (geneig_uneven.cu).
// The stage chain is described in geneig_tiled.cu.
#pragma once

// How the per-pencil body is compiled into its callers: inlined into the
// size's own kernel; a caller that dispatches several bodies (the persistent
// uneven-size kernel) may define it as __noinline__ before including, so
// that each body keeps its own register allocation.
#ifndef SGEIG_TILED_BODY_INLINE
#define SGEIG_TILED_BODY_INLINE __forceinline__
#endif

#include "geneig_common.cuh"
#include "geneig_dc.cuh"
#include "geneig_kernels.h"
namespace sgeig {
namespace tiled {

constexpr int kNT = 256;          // threads per CTA
constexpr int kNW = kNT / 32;     // warps per CTA
// Below this n the per-column (unblocked) Householder reduction is faster on
// B200 than the 16-column panels (fewer barriers per column); above it the
// panels' halved trailing-matrix traffic wins (measured crossover ~90).
constexpr int kBlockedHetrdMinN = 96;
// Up to this n the blocked reduction forms y = A v column by column with
// per-warp partial vectors in shared memory (8 n complex entries, which keep
// two CTAs per SM up to here); above it, a warp per row item.
constexpr int kColMatvecMaxN = 352;

struct TiledArgs {
    const double2* __restrict__ H;
    const double2* __restrict__ S;
    double*  W;
    double2* U;
    int*     info;
    double2* scratch;
    long long batch;
    int n, ld, stage;
    int sigma;      // H = diag(I_{n/2}, -I_{n/2}), not read from memory
    int mixed;      // FP32 Householder reduction + FP64 refinement
    int refine_max; // mixed: refinement steps before the FP64 fallback
};

// Ogita-Aishima refinement of the mixed form: it stops as soon as the current
// estimate V is orthonormal and diagonalises C to rounding level
// (||I - V^H V||_F and ||V^H C V - diag(lam)||_F / max|lam| both <= 16 eps n,
// checked directly: the correction alone can look converged while vectors
// of a tight pair stay mixed), after at most TiledArgs::refine_max
// corrections (default kRefineMaxIters). Widely spread spectra (cond(S) =
// 1e5 makes C's small eigenvalues nearly clustered against ||C||) need more
// steps from the FP32 start; a pencil that has not converged by then is
// solved again in FP64.

// ---------------------------------------------------------------- complex FP32
__device__ __forceinline__ float2 f2(float re, float im) { return make_float2(re, im); }
__device__ __forceinline__ float2 fcmul(float2 a, float2 b) {
    return f2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// acc + conj(a) * b
__device__ __forceinline__ float2 fcfmac(float2 acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x); acc.x = fmaf(a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y); acc.y = fmaf(-a.y, b.x, acc.y);
    return acc;
}
// acc + a * b
__device__ __forceinline__ float2 fcfma(float2 acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x); acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y); acc.y = fmaf(a.y, b.x, acc.y);
    return acc;
}
// acc - a * conj(b)
__device__ __forceinline__ float2 fcfms_bc(float2 acc, float2 a, float2 b) {
    acc.x = fmaf(-a.x, b.x, acc.x); acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y); acc.y = fmaf(-a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float2 warp_sum2f(float2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ double2 f2d(float2 a) { return c2((double)a.x, (double)a.y); }

// Shared-memory vectors of one CTA.
struct TVec {
    double2* tau;   // n    Householder scalars
    double2* vb;    // n    current Householder vector (v[k+1] = 1)
    double2* pb;    // n    tau * A22 * v
    double2* red;   // 32   reduction scratch
    double2* tb;    // 256  T factor of the current WY block (16 x 16, column-major)
    double2* part;  // tiled_part_elems(n): per-warp partials of the blocked y = A v
    double2* gb;    // 512  Y^H Y of the current WY block: two partial sums, then their sum
    double*  d;     // n    tridiagonal diagonal
    double*  e;     // n    tridiagonal off-diagonal
    double*  rdg;   // n    1 / L_kk
    double*  dcd;   // divide-and-conquer doubles (dc_vec_doubles(n)); eigenvalues first
    int*     rank;  // n    ascending position of eigenvalue j
    int*     ctl;   // 8    control words
    int*     dci;   // divide-and-conquer ints (dc_vec_ints(n))
};

__host__ __device__ inline size_t tiled_part_elems(int n) {
    return (n >= kBlockedHetrdMinN && n <= kColMatvecMaxN) ? (size_t)8 * n : 0;
}

__device__ inline TVec tcarve(unsigned char* p, int n) {
    TVec v;
    v.tau = reinterpret_cast<double2*>(p);
    v.vb  = v.tau + n;
    v.pb  = v.vb + n;
    v.red = v.pb + n;
    v.tb  = v.red + 32;
    v.gb  = v.tb + 256;
    v.part = v.gb + 512;
    v.d   = reinterpret_cast<double*>(v.part + tiled_part_elems(n));
    v.e   = v.d + n;
    v.rdg = v.e + n;
    v.dcd = v.rdg + n;
    v.rank = reinterpret_cast<int*>(v.dcd + dc_vec_doubles(n));
    v.ctl  = v.rank + n;
    v.dci  = v.ctl + 8;
    return v;
}

__device__ __forceinline__ double2 cneg(double2 a) { return c2(-a.x, -a.y); }

// ---------------------------------------------------------------- 16x16 complex MMA tiles
// D(8x8) += A(8x4) B(4x8) in FP64 on the tensor cores. Fragments: lane l
// holds A(l/4, l%4), B(l%4, l/4) and D(l/4, 2(l%4) + {0, 1}).
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b));
}

// A warp's 16 x 16 complex accumulator: 2 x 2 subtiles of 8 x 8, real and
// imaginary parts apart. Element [h][g][e] is row i0 + 8h + lane/4, column
// j0 + 8g + 2(lane%4) + e.
struct Z16 {
    double re[2][2][2];
    double im[2][2][2];
};

__device__ __forceinline__ void z16_zero(Z16& c) {
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int g = 0; g < 2; ++g)
#pragma unroll
            for (int e = 0; e < 2; ++e) c.re[h][g][e] = c.im[h][g][e] = 0.0;
}

// f(i, j) -> double2 for every element of the tile at (i0, j0)
template <class F>
__device__ __forceinline__ void z16_load(Z16& c, int i0, int j0, F f) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int g = 0; g < 2; ++g)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const double2 x = f(i0 + 8 * h + (lane >> 2), j0 + 8 * g + 2 * (lane & 3) + e);
                c.re[h][g][e] = x.x;
                c.im[h][g][e] = x.y;
            }
}

// f(i, j, value) for every element of the tile at (i0, j0)
template <class F>
__device__ __forceinline__ void z16_store(const Z16& c, int i0, int j0, F f) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int g = 0; g < 2; ++g)
#pragma unroll
            for (int e = 0; e < 2; ++e)
                f(i0 + 8 * h + (lane >> 2), j0 + 8 * g + 2 * (lane & 3) + e, c2(c.re[h][g][e], c.im[h][g][e]));
}

// c += A(i0:i0+16, k0:k1) B(k0:k1, j0:j0+16); a_at(i, k) and b_at(k, j)
// return the operand elements (they must return 0 outside the operands;
// k < k1 is checked here).
template <class FA, class FB>
__device__ __forceinline__ void z16_mma(Z16& c, int i0, int j0, int k0, int k1, FA a_at, FB b_at) {
    const int lane = threadIdx.x & 31;
    const int ar = i0 + (lane >> 2), bc = j0 + (lane >> 2), kq = lane & 3;
#pragma unroll 4
    for (int k = k0; k < k1; k += 4) {
        const int kk = k + kq;
        double2 a[2], b[2];
        if (kk < k1) {
            a[0] = a_at(ar, kk);
            a[1] = a_at(ar + 8, kk);
            b[0] = b_at(kk, bc);
            b[1] = b_at(kk, bc + 8);
        } else {
            a[0] = a[1] = b[0] = b[1] = c2(0.0, 0.0);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                dmma(c.re[h][g], a[h].x, b[g].x);
                dmma(c.re[h][g], -a[h].y, b[g].y);
                dmma(c.im[h][g], a[h].x, b[g].y);
                dmma(c.im[h][g], a[h].y, b[g].x);
            }
    }
}

// t -> (ti, tj) with ti >= tj, enumerating the lower triangle row by row.
__device__ __forceinline__ void tri_tile(int t, int& ti, int& tj) {
    int r = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    ti = r;
    tj = t - r * (r + 1) / 2;
}

// One pencil b, solved end to end by the whole CTA in its global-memory
// slot `slot` (tiled_slot_elems(n, mixed) complex entries) with the
// launch's dynamic shared memory as the vector area.
__device__ SGEIG_TILED_BODY_INLINE void tiled_solve(const TiledArgs& a, long long b, double2* slot,
                                            unsigned char* smem_raw) {
    const int n = a.n, ld = a.ld;
    const size_t mat = (size_t)n * ld;
    const bool mixed = a.mixed != 0;
    double2* M0 = slot;
    double2* M1 = M0 + mat;
    double2* M2 = M1 + mat;
    double2* M3 = mixed ? M2 + mat : nullptr;       // mixed only
    double2* zob = mixed ? M3 + mat : M2 + mat;
    double*  Zo = reinterpret_cast<double*>(zob);
    double2* Wsc = zob;                      // WY scratch (16 x n), shares Zo's storage
    // mixed only: FP32 copy of C after Zo; after the back-transform Zo and
    // it together hold one more n x ld complex matrix (M4)
    float2*  C32 = reinterpret_cast<float2*>(zob + tiled_zo_elems(n));
    double2* M4 = zob;
    TVec v = tcarve(smem_raw, n);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tn = (n + 15) >> 4;
    const size_t nn = (size_t)n * n;
    const double2 zero = c2(0.0, 0.0);
    const double2* Hb = a.H + (size_t)b * nn;
    const double2* Sb = a.S + (size_t)b * nn;
    double*  Wb = a.W + (size_t)b * n;
    double2* Ub = a.U + (size_t)b * nn;

    __syncthreads();  // previous pencil fully consumed
    phase_mark(24);
    // ---- a1: S (lower triangle and diagonal) -> M0
    for (int idx = tid; idx < (int)nn; idx += kNT) {
        const int j = idx / n, i = idx - j * n;
        if (i >= j) M0[i + (size_t)j * ld] = __ldg(Sb + idx);
    }
    if (tid < 8) v.ctl[tid] = 0;
    __syncthreads();
    phase_mark(16);

    // ---- a2: blocked Cholesky (lower). The pivot test is the same as
    // potrf's (not > 0, NaN included), taken in column order.
    int fail = 0;
    for (int p = 0; p < n && !fail; p += 16) {
        const int pe = min(p + 16, n);
        for (int c = p; c < pe; ++c) {
            const double piv = M0[c + (size_t)c * ld].x;
            if (!(piv > 0.0)) { fail = c + 1; break; }
            const double lc = sqrt(piv), r = 1.0 / lc;
            double2* lcol = M0 + (size_t)c * ld;
            for (int i = c + 1 + tid; i < n; i += kNT) lcol[i] = cscale(lcol[i], r);
            __syncthreads();
            if (tid == 0) { lcol[c] = c2(lc, 0.0); v.rdg[c] = r; }
            // rank-1 update of the panel columns right of c
            const int wc = pe - c - 1, rows = n - c - 1;
            for (int idx = tid; idx < rows * wc; idx += kNT) {
                const int cc = c + 1 + idx / rows, i = c + 1 + idx % rows;
                if (i >= cc) {
                    double2* x = M0 + i + (size_t)cc * ld;
                    *x = cfms_bc(*x, lcol[i], lcol[cc]);
                }
            }
            __syncthreads();
        }
        if (fail) break;
        // trailing lower tiles: C -= L_p L_p^H over columns [p, pe)
        const int m2 = n - pe;
        if (m2 > 0) {
            const int tm = (m2 + 15) >> 4, T = tm * (tm + 1) / 2;
            for (int t = warp; t < T; t += kNW) {
                int ti, tj;
                tri_tile(t, ti, tj);
                const int i0 = pe + 16 * ti, j0 = pe + 16 * tj;
                Z16 acc;
                z16_load(acc, i0, j0, [&](int i, int j) { return (i < n && j < n) ? M0[i + (size_t)j * ld] : zero; });
                z16_mma(acc, i0, j0, p, pe,
                        [&](int i, int k) { return i < n ? cneg(M0[i + (size_t)k * ld]) : zero; },
                        [&](int k, int j) { return j < n ? cconj(M0[j + (size_t)k * ld]) : zero; });
                z16_store(acc, i0, j0, [&](int i, int j, double2 x) {
                    if (i < n && j < n && i >= j) M0[i + (size_t)j * ld] = x;
                });
            }
        }
        __syncthreads();
    }
    int code = fail ? n + fail : 0;   // zhegv: info = n + order of the failing minor
    phase_mark(17);

    if (!code && a.stage >= 2) {
        // ---- a3: X = L^-1 -> M1, block row r0..re at a time
        for (int r0 = 0; r0 < n; r0 += 16) {
            const int re = min(r0 + 16, n);
            for (int t = warp; t < (r0 >> 4); t += kNW) {
                const int j0 = 16 * t;
                Z16 acc;
                z16_zero(acc);
                z16_mma(acc, r0, j0, j0, r0,
                        [&](int i, int k) { return i < n ? M0[i + (size_t)k * ld] : zero; },
                        [&](int k, int j) { return k >= j ? M1[k + (size_t)j * ld] : zero; });
                z16_store(acc, r0, j0, [&](int i, int j, double2 x) { if (i < n) M1[i + (size_t)j * ld] = x; });
            }
            __syncthreads();
            for (int c = tid; c < re; c += kNT) {
                double2 x[16];
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const int i = r0 + r;
                    x[r] = (i < re) ? ((c < r0) ? cneg(M1[i + (size_t)c * ld]) : c2(i == c ? 1.0 : 0.0, 0.0))
                                    : zero;
                }
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const int i = r0 + r;
                    if (i < re) {
                        double2 s = x[r];
#pragma unroll
                        for (int q = 0; q < r; ++q) s = cfms(s, M0[i + (size_t)(r0 + q) * ld], x[q]);
                        x[r] = cscale(s, v.rdg[i]);
                    }
                }
#pragma unroll
                for (int r = 0; r < 16; ++r)
                    if (r0 + r < re) M1[r0 + r + (size_t)c * ld] = x[r];
            }
            __syncthreads();
        }
        phase_mark(18);
    }

    if (!code && a.stage == 1) {
        for (int idx = tid; idx < (int)nn; idx += kNT) {
            const int j = idx / n, i = idx - j * n;
            Ub[idx] = (i >= j) ? M0[i + (size_t)j * ld] : zero;
        }
        if (tid == 0) a.info[b] = 0;
        return;
    }

    if (!code) {
        // ---- a4: T = H X^H -> M2, T(i, j) = sum_{k <= j} H(i, k) conj(X(j, k))
        if (a.sigma) {
            const int m = n >> 1;
            for (int idx = tid; idx < (int)nn; idx += kNT) {
                const int j = idx / n, i = idx - j * n;
                const double2 x = (i <= j) ? cconj(M1[j + (size_t)i * ld]) : zero;
                M2[i + (size_t)j * ld] = (i < m) ? x : cneg(x);
            }
        } else {
            for (int t = warp; t < tn * tn; t += kNW) {
                const int ti = t / tn, tj = t - ti * tn, i0 = 16 * ti, j0 = 16 * tj;
                Z16 acc;
                z16_zero(acc);
                z16_mma(acc, i0, j0, 0, min(n, j0 + 16),
                        [&](int i, int k) { return i < n ? __ldg(Hb + i + (size_t)k * n) : zero; },
                        [&](int k, int j) { return (j < n && k <= j) ? cconj(M1[j + (size_t)k * ld]) : zero; });
                z16_store(acc, i0, j0, [&](int i, int j, double2 x) {
                    if (i < n && j < n) M2[i + (size_t)j * ld] = x;
                });
            }
        }
        __syncthreads();
        // C = X T, lower tiles; each lower element is written with its
        // mirror so that C is exactly Hermitian. L in M0 is dead by now.
        for (int t = warp; t < tn * (tn + 1) / 2; t += kNW) {
            int ti, tj;
            tri_tile(t, ti, tj);
            const int i0 = 16 * ti, j0 = 16 * tj;
            Z16 acc;
            z16_zero(acc);
            z16_mma(acc, i0, j0, 0, min(n, i0 + 16),
                    [&](int i, int k) { return (i < n && k <= i) ? M1[i + (size_t)k * ld] : zero; },
                    [&](int k, int j) { return j < n ? M2[k + (size_t)j * ld] : zero; });
            z16_store(acc, i0, j0, [&](int i, int j, double2 x) {
                if (i < n && j < n && i >= j) {
                    if (i == j) x.y = 0.0;
                    M0[i + (size_t)j * ld] = x;
                    M0[j + (size_t)i * ld] = cconj(x);
                }
            });
        }
        __syncthreads();
        phase_mark(19);
    }

    if (!code && a.stage == 2) {
        for (int idx = tid; idx < (int)nn; idx += kNT) {
            const int j = idx / n, i = idx - j * n;
            Ub[idx] = M0[i + (size_t)j * ld];
        }
        if (tid == 0) a.info[b] = 0;
        return;
    }

    // The mixed form tries the FP32 reduction first; a pencil whose
    // refinement does not converge goes round once more in FP64.
    bool use32 = mixed;
    for (;;) {
        if (!code) {
            // ---- a5a: Householder tridiagonalisation of C (lower). Reflector
            // k: I - tau_k v v^H on rows k+1.., v[k+1] = 1, v[k+2..] stored in
            // column k of M0 below the subdiagonal. Small n: one rank-2
            // update of the trailing matrix per column. Larger n: blocked as
            // LAPACK's zhetrd/zlatrd, panels of up to 16 columns reduced
            // against the panel-start trailing matrix A with the corrections
            // of the panel's earlier columns (V = reflectors, W = their
            // update vectors, W kept in M2 whose product T is dead by now),
            // then A -= V W^H + W V^H on tensor-core tiles.
            if (use32) {
                // Mixed form: the unblocked reduction in FP32 on a
                // single-precision copy of C (reflectors kept in its columns;
                // tau, d, e widened to FP64). C itself stays in M0 for the
                // refinement. The vectors live in pb's storage as float2.
                for (int idx = tid; idx < (int)nn; idx += kNT) {
                    const int j = idx / n, i = idx - j * n;
                    const double2 x = M0[i + (size_t)j * ld];
                    C32[i + (size_t)j * ld] = f2((float)x.x, (float)x.y);
                }
                float2* vbf = reinterpret_cast<float2*>(v.pb);
                float2* pbf = vbf + n;
                const float2 fz = f2(0.0f, 0.0f);
                __syncthreads();
                for (int k = 0; k < n - 1; ++k) {
                    float2* ck = C32 + (size_t)k * ld;
                    if (warp == 0) {
                        float ss = 0.0f;
                        for (int i = k + 2 + lane; i < n; i += 32) { const float2 x = ck[i]; ss = fmaf(x.x, x.x, fmaf(x.y, x.y, ss)); }
                        ss = warp_sumf(ss);
                        const float2 alpha = ck[k + 1];
                        float2 taui = fz, scal = fz;
                        float beta;
                        if (ss == 0.0f && alpha.y == 0.0f) {
                            beta = alpha.x;
                        } else {
                            beta = -copysignf(sqrtf(alpha.x * alpha.x + alpha.y * alpha.y + ss), alpha.x);
                            taui = f2((beta - alpha.x) / beta, -alpha.y / beta);
                            const float2 z = f2(alpha.x - beta, alpha.y);
                            const float inv = 1.0f / (z.x * z.x + z.y * z.y);
                            scal = f2(z.x * inv, -z.y * inv);
                        }
                        for (int i = k + 2 + lane; i < n; i += 32) {
                            const float2 vi = fcmul(ck[i], scal);
                            vbf[i] = vi;
                            ck[i] = vi;
                        }
                        if (lane == 0) {
                            vbf[k + 1] = f2(1.0f, 0.0f);
                            v.tau[k] = f2d(taui);
                            v.d[k] = (double)ck[k].x;
                            v.e[k] = (double)beta;
                        }
                    }
                    __syncthreads();
                    const float2 taui = f2((float)v.tau[k].x, (float)v.tau[k].y);
                    if (taui.x == 0.0f && taui.y == 0.0f) continue;
                    for (int i = k + 1 + warp; i < n; i += kNW) {
                        const float2* ci = C32 + (size_t)i * ld;
                        float2 acc = fz;
#pragma unroll 4
                        for (int j = k + 1 + lane; j < n; j += 32) acc = fcfmac(acc, ci[j], vbf[j]);
                        acc = warp_sum2f(acc);
                        if (lane == 0) pbf[i] = fcmul(taui, acc);
                    }
                    __syncthreads();
                    if (warp == 0) {
                        float2 dot = fz;
                        for (int i = k + 1 + lane; i < n; i += 32) dot = fcfmac(dot, pbf[i], vbf[i]);
                        dot = warp_sum2f(dot);
                        if (lane == 0) { const float2 t = fcmul(taui, dot); v.red[0] = c2(-0.5 * t.x, -0.5 * t.y); }
                    }
                    __syncthreads();
                    const float2 alpha2 = f2((float)v.red[0].x, (float)v.red[0].y);
                    for (int j = k + 1 + warp; j < n; j += kNW) {
                        float2* cj = C32 + (size_t)j * ld;
                        // w = p + alpha2 v
                        const float2 vj = vbf[j], wj = fcfma(pbf[j], alpha2, vj);
#pragma unroll 4
                        for (int i = k + 1 + lane; i < n; i += 32) {
                            const float2 vi = vbf[i], wi = fcfma(pbf[i], alpha2, vi);
                            float2 x = cj[i];
                            x = fcfms_bc(x, vi, wj);
                            x = fcfms_bc(x, wi, vj);
                            cj[i] = x;
                        }
                    }
                    __syncthreads();
                }
                if (tid == 0) {
                    v.d[n - 1] = (double)C32[(n - 1) + (size_t)(n - 1) * ld].x;
                    if (n == 1) v.tau[0] = zero;
                }
                __syncthreads();
            } else if (n < kBlockedHetrdMinN) {
                for (int k = 0; k < n - 1; ++k) {
                    double2* ck = M0 + (size_t)k * ld;
                    if (warp == 0) {
                        double ss = 0.0;
                        for (int i = k + 2 + lane; i < n; i += 32) { const double2 x = ck[i]; ss = fma(x.x, x.x, fma(x.y, x.y, ss)); }
                        ss = warp_sum(ss);
                        const double2 alpha = ck[k + 1];
                        double2 taui, scal = zero;
                        double beta;
                        if (ss == 0.0 && alpha.y == 0.0) {
                            taui = zero;
                            beta = alpha.x;
                        } else {
                            beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + ss), alpha.x);
                            const double rb = fast_rcp(beta);
                            taui = c2((beta - alpha.x) * rb, -alpha.y * rb);
                            const double2 z = c2(alpha.x - beta, alpha.y);
                            const double inv = fast_rcp(z.x * z.x + z.y * z.y);
                            scal = c2(z.x * inv, -z.y * inv);
                        }
                        for (int i = k + 2 + lane; i < n; i += 32) {
                            const double2 vi = cmul(ck[i], scal);
                            v.vb[i] = vi;
                            ck[i] = vi;
                        }
                        if (lane == 0) {
                            v.vb[k + 1] = c2(1.0, 0.0);
                            v.tau[k] = taui;
                            v.d[k] = ck[k].x;
                            v.e[k] = beta;
                        }
                    }
                    __syncthreads();
                    const double2 taui = v.tau[k];
                    if (taui.x == 0.0 && taui.y == 0.0) continue;
                    // p = tau A22 v = tau sum_j v_j A(:, j) (A22 is kept as a full
                    // Hermitian matrix): warp w takes the contiguous columns
                    // j = k+1+w, +8, ..., lane l the rows k+1+l, +32, +64 (n < 96),
                    // so each lane has a load per column in flight and no
                    // shuffles; the 8 per-warp partials meet in shared memory (tb
                    // and gb, contiguous, hold 768 >= 8 n entries) and warp 0 adds
                    // them in a fixed order, then forms p^H v.
                    double2* part = v.tb;
                    {
                        double2 acc[3] = {zero, zero, zero};
    #pragma unroll 2
                        for (int j = k + 1 + warp; j < n; j += kNW) {
                            const double2* cj = M0 + (size_t)j * ld;
                            const double2 vj = v.vb[j];
    #pragma unroll
                            for (int r = 0; r < 3; ++r) {
                                const int i = k + 1 + lane + 32 * r;
                                if (i < n) acc[r] = cfma(acc[r], cj[i], vj);
                            }
                        }
    #pragma unroll
                        for (int r = 0; r < 3; ++r) {
                            const int i = k + 1 + lane + 32 * r;
                            if (i < n) part[warp * n + i] = acc[r];
                        }
                    }
                    __syncthreads();
                    if (warp == 0) {
                        double2 dot = zero;
                        for (int i = k + 1 + lane; i < n; i += 32) {
                            double2 sp = zero;
    #pragma unroll
                            for (int w = 0; w < kNW; ++w) sp = cadd(sp, part[w * n + i]);
                            const double2 pi = cmul(taui, sp);
                            v.pb[i] = pi;
                            dot = cfmac(dot, pi, v.vb[i]);
                        }
                        dot = warp_sum2(dot);
                        if (lane == 0) v.red[0] = cscale(cmul(taui, dot), -0.5);
                    }
                    __syncthreads();
                    const double2 alpha2 = v.red[0];
                    // A22 -= v w^H + w v^H, w = p + alpha2 v; a warp per column,
                    // four columns per pass so that their loads are in flight together
                    for (int j0 = k + 1 + warp; j0 < n; j0 += 4 * kNW) {
                        double2 vj[4], wj[4];
    #pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int j = j0 + u * kNW;
                            vj[u] = j < n ? v.vb[j] : zero;
                            wj[u] = j < n ? cfma(v.pb[j], alpha2, vj[u]) : zero;
                        }
                        for (int i = k + 1 + lane; i < n; i += 32) {
                            const double2 vi = v.vb[i], wi = cfma(v.pb[i], alpha2, vi);
                            double2 x[4];
    #pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int j = j0 + u * kNW;
                                x[u] = j < n ? M0[i + (size_t)j * ld] : zero;
                            }
    #pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int j = j0 + u * kNW;
                                if (j < n) M0[i + (size_t)j * ld] = cfms_bc(cfms_bc(x[u], vi, wj[u]), wi, vj[u]);
                            }
                        }
                    }
                    __syncthreads();
                }
            } else {
                double2* Wp = M2;
                for (int p = 0; p < n - 1; p += 16) {
                    const int w = min(16, n - 1 - p);
                    // V(i, c) = v_{p+c}(i) for rows i > p + c
                    auto Vp = [&](int i, int c) -> double2 {
                        const int k = p + c;
                        return (i <= k) ? zero : (i == k + 1) ? c2(1.0, 0.0) : M0[i + (size_t)k * ld];
                    };
                    for (int c = 0; c < w; ++c) {
                        const int k = p + c;
                        double2* ck = M0 + (size_t)k * ld;
                        // (1) a_k(k:n) -= V(k:n, 0:c) W(k, 0:c)^H + W(k:n, 0:c) V(k, 0:c)^H
                        if (c > 0) {
                            for (int i = k + tid; i < n; i += kNT) {
                                double2 x = ck[i];
                                for (int cc = 0; cc < c; ++cc) {
                                    x = cfms_bc(x, Vp(i, cc), Wp[k + (size_t)cc * ld]);
                                    x = cfms_bc(x, Wp[i + (size_t)cc * ld], Vp(k, cc));
                                }
                                ck[i] = x;
                            }
                            __syncthreads();
                        }
                        // (2) reflector from a_k(k+1:n), warp 0
                        if (warp == 0) {
                            double ss = 0.0;
                            for (int i = k + 2 + lane; i < n; i += 32) { const double2 x = ck[i]; ss = fma(x.x, x.x, fma(x.y, x.y, ss)); }
                            ss = warp_sum(ss);
                            const double2 alpha = ck[k + 1];
                            double2 taui, scal = zero;
                            double beta;
                            if (ss == 0.0 && alpha.y == 0.0) {
                                taui = zero;
                                beta = alpha.x;
                            } else {
                                beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + ss), alpha.x);
                                const double rb = fast_rcp(beta);
                                taui = c2((beta - alpha.x) * rb, -alpha.y * rb);
                                const double2 z = c2(alpha.x - beta, alpha.y);
                                const double inv = fast_rcp(z.x * z.x + z.y * z.y);
                                scal = c2(z.x * inv, -z.y * inv);
                            }
                            for (int i = k + 2 + lane; i < n; i += 32) {
                                const double2 vi = cmul(ck[i], scal);
                                v.vb[i] = vi;
                                ck[i] = vi;
                            }
                            if (lane == 0) {
                                v.vb[k + 1] = c2(1.0, 0.0);
                                v.tau[k] = taui;
                                v.d[k] = ck[k].x;
                                v.e[k] = beta;
                            }
                        }
                        __syncthreads();
                        const double2 taui = v.tau[k];
                        // (3) y = A v (A: panel-start trailing matrix), t1 = W^H v and
                        // t2 = V^H v over rows k+1..n. Up to kColMatvecMaxN, y is
                        // formed column by column: warp w takes the contiguous
                        // columns j = k+1+w, +8, ..., its lanes 4 rows each per
                        // pass, so every lane keeps a load per row in flight and no
                        // shuffles are needed; the 8 partials per row are added in
                        // (4) in a fixed order. Above it, and for t1 / t2, one warp
                        // per item reads down a column (y_i = sum_j conj(A(j, i)) v_j).
                        const int m = n - k - 1;
                        const bool colmv = n <= kColMatvecMaxN;
                        if (colmv) {
                            double2* part = v.part;
                            for (int r0 = k + 1; r0 < n; r0 += 128) {
                                double2 acc[4] = {zero, zero, zero, zero};
    #pragma unroll 2
                                for (int j = k + 1 + warp; j < n; j += kNW) {
                                    const double2* cj = M0 + (size_t)j * ld;
                                    const double2 vj = v.vb[j];
    #pragma unroll
                                    for (int u = 0; u < 4; ++u) {
                                        const int i = r0 + lane + 32 * u;
                                        if (i < n) acc[u] = cfma(acc[u], cj[i], vj);
                                    }
                                }
    #pragma unroll
                                for (int u = 0; u < 4; ++u) {
                                    const int i = r0 + lane + 32 * u;
                                    if (i < n) part[warp * n + i] = acc[u];
                                }
                            }
                        }
                        for (int it = (colmv ? m : 0) + warp; it < m + 2 * c; it += kNW) {
                            double2 acc = zero;
                            if (it < m) {
                                const int i = k + 1 + it;
                                const double2* ci = M0 + (size_t)i * ld;
    #pragma unroll 4
                                for (int j = k + 1 + lane; j < n; j += 32) acc = cfmac(acc, ci[j], v.vb[j]);
                            } else if (it < m + c) {
                                const double2* wc = Wp + (size_t)(it - m) * ld;
                                for (int j = k + 1 + lane; j < n; j += 32) acc = cfmac(acc, wc[j], v.vb[j]);
                            } else {
                                const int cc = it - m - c;
                                for (int j = k + 1 + lane; j < n; j += 32) acc = cfmac(acc, Vp(j, cc), v.vb[j]);
                            }
                            acc = warp_sum2(acc);
                            if (lane == 0) {
                                if (it < m) v.pb[k + 1 + it] = acc;
                                else v.red[it - m] = acc;      // t1 at red[0..c), t2 at red[c..2c)
                            }
                        }
                        __syncthreads();
                        // (4) w = tau (y - V t1 - W t2) on rows k+1..n: the
                        // current trailing matrix is A - V W^H - W V^H
                        for (int i = k + 1 + tid; i < n; i += kNT) {
                            double2 x = v.pb[i];
                            if (colmv) {
                                x = zero;
    #pragma unroll
                                for (int w = 0; w < kNW; ++w) x = cadd(x, v.part[w * n + i]);
                            }
                            for (int cc = 0; cc < c; ++cc) {
                                x = cfms(x, Vp(i, cc), v.red[cc]);
                                x = cfms(x, Wp[i + (size_t)cc * ld], v.red[c + cc]);
                            }
                            v.pb[i] = cmul(taui, x);
                        }
                        __syncthreads();
                        // (5) alpha2 = -tau/2 (w^H v)
                        if (warp == 0) {
                            double2 dot = zero;
                            for (int i = k + 1 + lane; i < n; i += 32) dot = cfmac(dot, v.pb[i], v.vb[i]);
                            dot = warp_sum2(dot);
                            if (lane == 0) v.gb[0] = cscale(cmul(taui, dot), -0.5);
                        }
                        __syncthreads();
                        // (6) W(:, c) = w + alpha2 v on rows k+1..n, zero above
                        const double2 alpha2 = v.gb[0];
                        for (int i = tid; i < n; i += kNT)
                            Wp[i + (size_t)c * ld] = (i > k) ? cfma(v.pb[i], alpha2, v.vb[i]) : zero;
                        __syncthreads();
                    }
                    // trailing update A(q:n, q:n) -= V W^H + W V^H, q = p + w (all tiles)
                    const int q = p + w, mq = n - q;
                    if (mq > 0) {
                        const int tq = (mq + 15) >> 4;
                        for (int t = warp; t < tq * tq; t += kNW) {
                            const int ti = t / tq, tj = t - ti * tq, i0 = q + 16 * ti, j0 = q + 16 * tj;
                            Z16 acc;
                            z16_load(acc, i0, j0, [&](int i, int j) { return (i < n && j < n) ? M0[i + (size_t)j * ld] : zero; });
                            z16_mma(acc, i0, j0, 0, w,
                                    [&](int i, int cc) { return i < n ? cneg(Vp(i, cc)) : zero; },
                                    [&](int cc, int j) { return j < n ? cconj(Wp[j + (size_t)cc * ld]) : zero; });
                            z16_mma(acc, i0, j0, 0, w,
                                    [&](int i, int cc) { return i < n ? cneg(Wp[i + (size_t)cc * ld]) : zero; },
                                    [&](int cc, int j) { return j < n ? cconj(Vp(j, cc)) : zero; });
                            z16_store(acc, i0, j0, [&](int i, int j, double2 x) {
                                if (i < n && j < n) M0[i + (size_t)j * ld] = x;
                            });
                        }
                    }
                    __syncthreads();
                }
            }
            if (!use32 && tid == 0) {
                v.d[n - 1] = M0[(n - 1) + (size_t)(n - 1) * ld].x;
                if (n == 1) v.tau[0] = zero;
            }
            __syncthreads();
            phase_mark(20);

            // ---- a5b: divide and conquer on T: Z in M2 (real), its merge
            // workspace after it, merge products through Zo
            DCShared dc;
            dc.Z = reinterpret_cast<double*>(M2); dc.ldz = ld;
            dc.U = dc.Z + mat;                    dc.ldu = ld;
            dc.Zo = Zo;
            dc.d = v.d; dc.e = v.e;
            dc.w = v.dcd; dc.z = dc.w + n; dc.dl = dc.z + n; dc.zz = dc.dl + n; dc.zh = dc.zz + n;
            dc.rt = dc.zh + n; dc.rho = dc.rt + n; dc.scal = dc.rho + n;
            dc.org = v.dci; dc.nd = dc.org + n; dc.perm = dc.nd + n; dc.kcnt = dc.perm + n;
            tridiag_dc<kNT, 0>(n, dc);
            if (tid == 0) {
                bool bad = false;
                for (int i = 0; i < n; ++i) bad |= !isfinite(dc.w[i]);
                v.ctl[4] = bad ? kEigFailCode : 0;
            }
            __syncthreads();
            code = v.ctl[4];
            if (!code) {
                for (int j = tid; j < n; j += kNT) {
                    const double dj = order_key(v.dcd[j]);
                    int r = 0;
                    for (int k2 = 0; k2 < n; ++k2) {
                        const double dk = order_key(v.dcd[k2]);
                        r += (dk < dj) || (dk == dj && k2 < j);
                    }
                    v.rank[j] = r;
                }
            }
            __syncthreads();
            phase_mark(21);
        }

        if (code) break;

        // ---- a5c: V = Q Z in the output, columns in ascending eigenvalue order
        {
            const double* Z = reinterpret_cast<const double*>(M2);
            for (int idx = tid; idx < (int)nn; idx += kNT) {
                const int j = idx / n, i = idx - j * n;
                Ub[i + (size_t)v.rank[j] * n] = c2(Z[i + (size_t)j * ld], 0.0);
            }
            for (int j = tid; j < n; j += kNT) Wb[v.rank[j]] = v.dcd[j];
        }
        __syncthreads();
        const int nref = n - 1;
        for (int kb = nref > 0 ? ((nref - 1) / 16) * 16 : -1; kb >= 0; kb -= 16) {
            const int w = min(16, nref - kb);
            // Y(i, c) = v_{kb+c}(i): 0 above row kb+c+1, 1 there, stored below
            auto Y = [&](int i, int c) -> double2 {
                if (c >= w || i >= n) return zero;
                const int k = kb + c;
                return (i <= k) ? zero : (i == k + 1) ? c2(1.0, 0.0)
                     : use32 ? f2d(C32[i + (size_t)k * ld]) : M0[i + (size_t)k * ld];
            };
            v.tb[tid] = zero;   // kNT == 256 == 16 x 16
            // G = Y^H Y: warps 0 and 1 each sum half of the rows, and the two
            // halves are added in a fixed order (results are bitwise
            // reproducible from launch to launch)
            if (warp < 2) {
                const int r0 = kb + 1, rows = n - r0;
                const int per = ((rows + 7) / 8) * 4;
                const int k0 = r0 + warp * per, k1 = min(n, k0 + per);
                Z16 acc;
                z16_zero(acc);
                z16_mma(acc, 0, 0, k0, k1, [&](int c, int i) { return cconj(Y(i, c)); },
                        [&](int i, int c) { return Y(i, c); });
                z16_store(acc, 0, 0, [&](int i, int j, double2 x) { v.gb[256 * warp + i + 16 * j] = x; });
            }
            __syncthreads();
            v.gb[tid] = cadd(v.gb[tid], v.gb[256 + tid]);
            __syncthreads();
            // T_b (upper triangular, forward column-wise): T(j, j) = tau_j,
            // T(0:j, j) = T(0:j, 0:j) (-tau_j G(0:j, j))
            if (warp == 0) {
                for (int j = 0; j < w; ++j) {
                    const double2 tj = v.tau[kb + j];
                    const double2 y = (lane < j) ? cneg(cmul(tj, v.gb[lane + 16 * j])) : zero;
                    double2 s = zero;
                    for (int l = 0; l < j; ++l) {
                        const double2 yl = c2(__shfl_sync(0xffffffffu, y.x, l), __shfl_sync(0xffffffffu, y.y, l));
                        if (lane <= l) s = cfma(s, v.tb[lane + 16 * l], yl);
                    }
                    if (lane < j) v.tb[lane + 16 * j] = s;
                    if (lane == j) v.tb[j + 16 * j] = tj;
                    __syncwarp();
                }
            }
            __syncthreads();
            // W1 = Y^H V (16 x n) then W2 = T_b W1 in place, one column tile per warp
            for (int t = warp; t < tn; t += kNW) {
                const int j0 = 16 * t;
                Z16 acc;
                z16_zero(acc);
                z16_mma(acc, 0, j0, kb + 1, n, [&](int c, int i) { return cconj(Y(i, c)); },
                        [&](int i, int j) { return j < n ? Ub[i + (size_t)j * n] : zero; });
                z16_store(acc, 0, j0, [&](int c, int j, double2 x) { if (j < n) Wsc[c + 16 * j] = x; });
                __syncwarp();
                Z16 acc2;
                z16_zero(acc2);
                z16_mma(acc2, 0, j0, 0, 16, [&](int c, int l) { return v.tb[c + 16 * l]; },
                        [&](int l, int j) { return j < n ? Wsc[l + 16 * j] : zero; });
                __syncwarp();
                z16_store(acc2, 0, j0, [&](int c, int j, double2 x) { if (j < n) Wsc[c + 16 * j] = x; });
            }
            __syncthreads();
            // V -= Y W2 on rows kb+1..n
            const int rt0 = (kb + 1) >> 4, T = (tn - rt0) * tn;
            for (int t = warp; t < T; t += kNW) {
                const int ti = rt0 + t / tn, tj = t % tn, i0 = 16 * ti, j0 = 16 * tj;
                Z16 acc;
                z16_load(acc, i0, j0, [&](int i, int j) { return (i < n && j < n) ? Ub[i + (size_t)j * n] : zero; });
                z16_mma(acc, i0, j0, 0, 16, [&](int i, int c) { return cneg(Y(i, c)); },
                        [&](int c, int j) { return j < n ? Wsc[c + 16 * j] : zero; });
                z16_store(acc, i0, j0, [&](int i, int j, double2 x) {
                    if (i < n && j < n) Ub[i + (size_t)j * n] = x;
                });
            }
            __syncthreads();
        }

        if (use32) {
            // ---- a5d: Ogita-Aishima refinement in FP64 of the eigenpairs of
            // C (M0) from the estimate V (columns in the output):
            //   R = I - V^H V, P = C V, Sm = V^H P, lam_i = Sm_ii / (1 - R_ii),
            //   delta = 2 (||Sm - diag(lam)||_F + max|lam| ||R||_F),
            //   E_ij = (Sm_ij + lam_j R_ij) / (lam_j - lam_i) if |lam_j - lam_i| > delta,
            //          R_ij / 2 otherwise (and on the diagonal),
            //   V <- V + V E,
            // until V passes the convergence test above. R / E in M2, P in
            // the next-estimate buffer, Sm in M4.
            double* lam = v.dcd + n;
            double2* Vh = Ub;  int ldh = n;
            double2* Vn = M3;  int ldn = ld;
            const int tl = tn * (tn + 1) / 2;
            bool conv = false;
            for (int it = 0;; ++it) {
                for (int t = warp; t < tl + tn * tn; t += kNW) {
                    Z16 acc;
                    z16_zero(acc);
                    if (t < tl) {
                        int ti, tj;
                        tri_tile(t, ti, tj);
                        const int i0 = 16 * ti, j0 = 16 * tj;
                        z16_mma(acc, i0, j0, 0, n, [&](int i, int k) { return i < n ? cconj(Vh[k + (size_t)i * ldh]) : zero; },
                                [&](int k, int j) { return j < n ? Vh[k + (size_t)j * ldh] : zero; });
                        z16_store(acc, i0, j0, [&](int i, int j, double2 x) {
                            if (i < n && j < n && i >= j) {
                                x = c2((i == j ? 1.0 : 0.0) - x.x, i == j ? 0.0 : -x.y);
                                M2[i + (size_t)j * ld] = x;
                                M2[j + (size_t)i * ld] = cconj(x);
                            }
                        });
                    } else {
                        const int t2 = t - tl, ti = t2 / tn, tj = t2 - ti * tn, i0 = 16 * ti, j0 = 16 * tj;
                        z16_mma(acc, i0, j0, 0, n, [&](int i, int k) { return i < n ? M0[i + (size_t)k * ld] : zero; },
                                [&](int k, int j) { return j < n ? Vh[k + (size_t)j * ldh] : zero; });
                        z16_store(acc, i0, j0, [&](int i, int j, double2 x) { if (i < n && j < n) Vn[i + (size_t)j * ldn] = x; });
                    }
                }
                __syncthreads();
                for (int t = warp; t < tl; t += kNW) {
                    int ti, tj;
                    tri_tile(t, ti, tj);
                    const int i0 = 16 * ti, j0 = 16 * tj;
                    Z16 acc;
                    z16_zero(acc);
                    z16_mma(acc, i0, j0, 0, n, [&](int i, int k) { return i < n ? cconj(Vh[k + (size_t)i * ldh]) : zero; },
                            [&](int k, int j) { return j < n ? Vn[k + (size_t)j * ldn] : zero; });
                    z16_store(acc, i0, j0, [&](int i, int j, double2 x) {
                        if (i < n && j < n && i >= j) {
                            if (i == j) x.y = 0.0;
                            M4[i + (size_t)j * ld] = x;
                            M4[j + (size_t)i * ld] = cconj(x);
                        }
                    });
                }
                __syncthreads();
                for (int i = tid; i < n; i += kNT) lam[i] = M4[i + (size_t)i * ld].x / (1.0 - M2[i + (size_t)i * ld].x);
                __syncthreads();
                {
                    double sS = 0.0, sR = 0.0, lmax = 0.0;
                    for (int idx = tid; idx < (int)nn; idx += kNT) {
                        const int j = idx / n, i = idx - j * n;
                        double2 x = M4[i + (size_t)j * ld];
                        if (i == j) x.x -= lam[i];
                        sS = fma(x.x, x.x, fma(x.y, x.y, sS));
                        const double2 r = M2[i + (size_t)j * ld];
                        sR = fma(r.x, r.x, fma(r.y, r.y, sR));
                    }
                    for (int i = tid; i < n; i += kNT) lmax = fmax(lmax, fabs(lam[i]));
                    sS = warp_sum(sS);
                    sR = warp_sum(sR);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
                    if (lane == 0) { v.red[warp] = c2(sS, sR); v.gb[warp] = c2(lmax, 0.0); }
                    __syncthreads();
                    if (tid == 0) {
                        double a1 = 0.0, a2 = 0.0, mx = 0.0;
                        for (int w8 = 0; w8 < kNW; ++w8) { a1 += v.red[w8].x; a2 += v.red[w8].y; mx = fmax(mx, v.gb[w8].x); }
                        v.gb[16] = c2(2.0 * (sqrt(a1) + mx * sqrt(a2)), 0.0);
                        // converged: V orthonormal and C V = V diag(lam) to rounding level
                        const double tol = 16.0 * kEps * n;
                        v.gb[17] = c2((sqrt(a2) <= tol && sqrt(a1) <= tol * mx) ? 1.0 : 0.0, 0.0);
                    }
                    __syncthreads();
                }
                if (v.gb[17].x != 0.0) { conv = true; break; }
                if (it == a.refine_max) break;
                const double delta = v.gb[16].x;
                for (int idx = tid; idx < (int)nn; idx += kNT) {
                    const int j = idx / n, i = idx - j * n;
                    const double2 r = M2[i + (size_t)j * ld];
                    double2 e = cscale(r, 0.5);
                    if (i != j) {
                        const double g = lam[j] - lam[i];
                        if (fabs(g) > delta) e = cscale(cadd(M4[i + (size_t)j * ld], cscale(r, lam[j])), 1.0 / g);
                    }
                    M2[i + (size_t)j * ld] = e;
                }
                __syncthreads();
                for (int t = warp; t < tn * tn; t += kNW) {
                    const int ti = t / tn, tj = t - ti * tn, i0 = 16 * ti, j0 = 16 * tj;
                    Z16 acc;
                    z16_load(acc, i0, j0, [&](int i, int j) { return (i < n && j < n) ? Vh[i + (size_t)j * ldh] : zero; });
                    z16_mma(acc, i0, j0, 0, n, [&](int i, int k) { return i < n ? Vh[i + (size_t)k * ldh] : zero; },
                            [&](int k, int j) { return j < n ? M2[k + (size_t)j * ld] : zero; });
                    z16_store(acc, i0, j0, [&](int i, int j, double2 x) { if (i < n && j < n) Vn[i + (size_t)j * ldn] = x; });
                }
                __syncthreads();
                double2* tp = Vh; Vh = Vn; Vn = tp;
                const int tld = ldh; ldh = ldn; ldn = tld;
            }
            if (!conv) {
                // no convergence from the FP32 start (possible when C's
                // spectrum is spread over many orders of magnitude): redo
                // this pencil's eigensolve in FP64 from C, still intact in M0
                use32 = false;
                continue;
            }
            if (Vh != Ub) {   // an odd number of steps left the estimate in M3
                for (int idx = tid; idx < (int)nn; idx += kNT) {
                    const int j = idx / n, i = idx - j * n;
                    Ub[idx] = Vh[i + (size_t)j * ldh];
                }
                __syncthreads();
            }
            // new ascending order of the refined eigenvalues
            for (int j = tid; j < n; j += kNT) {
                const double dj = order_key(lam[j]);
                int r = 0;
                for (int k2 = 0; k2 < n; ++k2) {
                    const double dk = order_key(lam[k2]);
                    r += (dk < dj) || (dk == dj && k2 < j);
                }
                v.rank[j] = r;
            }
            __syncthreads();
            for (int j = tid; j < n; j += kNT) Wb[v.rank[j]] = lam[j];
            if (a.stage == 3) {
                for (int idx = tid; idx < (int)nn; idx += kNT) {
                    const int j = idx / n, i = idx - j * n;
                    M2[i + (size_t)v.rank[j] * ld] = Ub[idx];
                }
                __syncthreads();
                for (int idx = tid; idx < (int)nn; idx += kNT) {
                    const int j = idx / n, i = idx - j * n;
                    Ub[idx] = M2[i + (size_t)j * ld];
                }
            }
        }

        break;
    }
    phase_mark(22);
    if (code) {
        const double qnan = __longlong_as_double(0x7ff8000000000000LL);
        for (int idx = tid; idx < (int)nn; idx += kNT) Ub[idx] = c2(qnan, qnan);
        if (a.stage >= 3) for (int i = tid; i < n; i += kNT) Wb[i] = qnan;
        if (tid == 0) a.info[b] = code == kEigFailCode ? eig_fail_info(n) : code;
        return;
    }

    if (tid == 0) a.info[b] = 0;
    if (a.stage == 3) return;

    // ---- a6: U = X^H V -> M2, U(i, j) = sum_{k >= i} conj(X(k, i)) V(k, j); then to the output
    for (int t = warp; t < tn * tn; t += kNW) {
        const int ti = t / tn, tj = t - ti * tn, i0 = 16 * ti, j0 = 16 * tj;
        Z16 acc;
        z16_zero(acc);
        z16_mma(acc, i0, j0, i0, n,
                [&](int i, int k) { return (i < n && k >= i) ? cconj(M1[k + (size_t)i * ld]) : zero; },
                [&](int k, int j) { return j < n ? Ub[k + (size_t)j * n] : zero; });
        z16_store(acc, i0, j0, [&](int i, int j, double2 x) { if (i < n && j < n) M2[i + (size_t)j * ld] = x; });
    }
    __syncthreads();
    phase_mark(23);
    for (int idx = tid; idx < (int)nn; idx += kNT) {
        const int j = idx / n, i = idx - j * n;
        Ub[i + (size_t)(use32 ? v.rank[j] : j) * n] = M2[i + (size_t)j * ld];
    }
}

}  // namespace tiled
}  // namespace sgeig
