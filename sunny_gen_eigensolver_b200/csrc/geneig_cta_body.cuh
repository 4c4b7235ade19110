// Per-pencil body of the shared-memory (smem-cta) solver, shared by its own
// kernel (geneig_cta.cu) and the persistent uneven-size kernel
// (geneig_uneven.cu). The stage chain is described in geneig_cta.cu.
#pragma once

// How the per-pencil body is compiled into its callers: inlined into the
// size's own kernel; a caller that dispatches several bodies (the persistent
// uneven-size kernel) may define it as __noinline__ before including, so
// that each body keeps its own register allocation.
#ifndef SGEIG_CTA_BODY_INLINE
#define SGEIG_CTA_BODY_INLINE __forceinline__
#endif

#include "geneig_common.cuh"
#include "geneig_dc.cuh"
#include "geneig_kernels.h"

#include <cmath>
namespace sgeig {
namespace cta {

constexpr int kNT = 256;
constexpr int kG = 4;
// stage number of the intensity form (the spin-wave metric solve that
// reduces U to S(q, E) on the device instead of storing it)
constexpr int kStageIntensity = 5;

struct CtaArgs {
    const double2* __restrict__ H;
    const double2* __restrict__ S;
    double*  W;
    double2* U;
    int*     info;
    long long batch;
    int n, ld, stage;
    int sigma;      // H = diag(I_{n/2}, -I_{n/2}), not read from memory
    // stage kStageIntensity (spin-wave intensities in place of U):
    const double2* O;        // 3 x n observable matrix per problem (column-major)
    const double*  qhat;     // 3 per problem
    const double*  energies; // ne
    double*        spec;     // ne per problem
    int            ne;
    double         gnorm;    // Gaussian normalisation 1 / (sigma sqrt(2 pi))
    double         ginv2;    // 1 / (2 sigma^2)
};

// S assembled on the device instead of loaded (the FS form of cta_solve):
// S(q)_e = sum_{t in [start[e], start[e+1])} coef[t] exp(2 pi i q . disp[3t..3t+2])
// for the lower-triangle entries e = row + n col (row >= col), q = q[3b..3b+2].
struct CtaFourier {
    const int*     start;   // n*n + 1
    const double2* coef;
    const double*  disp;
    const double*  q;
    int            nterms;  // terms are read only from [0, nterms)
};

struct CtaVec {
    double2* tau;   // n   Householder scalars
    double2* vb;    // n   Householder vector of even steps
    double2* vb2;   // n   Householder vector of odd steps (written one step ahead)
    double2* pb;    // n   tau * A22 * v
    double2* wred;  // 8   per-warp partial dots
    double2* colv;  // 2n  column k of the Cholesky working matrix (double-buffered)
    double2* rowv;  // 2n  row k of the inverse accumulator (double-buffered)
    double*  d;     // n
    double*  e;     // n
    double*  rdg;   // n   1 / L_kk
    double*  dcd;   // D&C doubles
    int*     dci;   // D&C ints
    int*     rank;  // n
    int*     ctl;   // 8
};

__host__ __device__ inline size_t cta_vec_bytes(int n) {
    return (size_t)n * 16 * 8 + 8 * 16 + (size_t)n * 8 * 3 + (size_t)dc_vec_doubles(n) * 8 +
           (size_t)dc_vec_ints(n) * 4 + (size_t)n * 4 + 8 * 4;
}

// Shared-memory bytes of one pencil's team (both matrices and the vector
// area), rounded up to 16 so that consecutive teams stay aligned.
__host__ __device__ inline size_t cta_team_bytes(int n) {
    return ((size_t)2 * n * (n | 1) * 16 + cta_vec_bytes(n) + 15) & ~(size_t)15;
}

__device__ inline CtaVec cta_carve(unsigned char* p, int n) {
    CtaVec v;
    v.tau  = reinterpret_cast<double2*>(p);
    v.vb   = v.tau + n;
    v.vb2  = v.vb + n;
    v.pb   = v.vb2 + n;
    v.wred = v.pb + n;
    v.colv = v.wred + 8;
    v.rowv = v.colv + 2 * n;
    v.d    = reinterpret_cast<double*>(v.rowv + 2 * n);
    v.e    = v.d + n;
    v.rdg  = v.e + n;
    v.dcd  = v.rdg + n;
    v.dci  = reinterpret_cast<int*>(v.dcd + dc_vec_doubles(n));
    v.rank = v.dci + dc_vec_ints(n);
    v.ctl  = v.rank + n;
    return v;
}

// One FP64 tensor-core step D += A B on an 8x8x4 tile (mma.m8n8k4.f64).
// Fragments: lane l holds A(l/4, l%4), B(l%4, l/4) and D(l/4, 2(l%4)+{0,1}).
__device__ __forceinline__ void mma884(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// Complex product on 8x8 output tiles, one warp per tile (round robin over
// the CTA's warps), four real MMAs per 8x8x4 step:
//   Dr += Ar Br - Ai Bi,  Di += Ar Bi + Ai Br.
// fa(i, k) / fb(k, j) return the operands (zero outside their nonzero
// pattern and outside the matrix); kr(ti, tj, k0, k1) bounds the k loop of
// tile (ti, tj); keep(ti, tj) selects the tiles to compute. The results stay
// in registers (acc) so that the caller can barrier before overwriting an
// operand, then call `put` for every computed element.
template <int MAXT>
struct ZTiles {
    double re[MAXT][2], im[MAXT][2];
};

template <int MAXT, int NT, int BLOCK, class FA, class FB, class FK, class FKeep>
__device__ __forceinline__ void ztiles_compute(ZTiles<MAXT>& acc, int tm, int tn, FA fa, FB fb, FK kr, FKeep keep) {
    const int lane = team_tid<NT, BLOCK>() & 31, warp = team_tid<NT, BLOCK>() >> 5;
    constexpr int NW = NT / 32;
#pragma unroll
    for (int u = 0; u < MAXT; ++u) {
        acc.re[u][0] = acc.re[u][1] = acc.im[u][0] = acc.im[u][1] = 0.0;
        const int t = warp + NW * u;
        if (t >= tm * tn) continue;
        const int ti = t / tn, tj = t - ti * tn;
        if (!keep(ti, tj)) continue;
        int k0, k1;
        kr(ti, tj, k0, k1);
        const int ia = 8 * ti + (lane >> 2), ka = lane & 3;   // A fragment element
        const int kb = lane & 3, jb = 8 * tj + (lane >> 2);   // B fragment element
        for (int k = k0; k < k1; k += 4) {
            const double2 av = fa(ia, k + ka);
            const double2 bv = fb(k + kb, jb);
            mma884(acc.re[u][0], acc.re[u][1], av.x, bv.x);
            mma884(acc.re[u][0], acc.re[u][1], -av.y, bv.y);
            mma884(acc.im[u][0], acc.im[u][1], av.x, bv.y);
            mma884(acc.im[u][0], acc.im[u][1], av.y, bv.x);
        }
    }
}

template <int MAXT, int NT, int BLOCK, class FKeep, class FPut>
__device__ __forceinline__ void ztiles_store(const ZTiles<MAXT>& acc, int tm, int tn, FKeep keep, FPut put) {
    const int lane = team_tid<NT, BLOCK>() & 31, warp = team_tid<NT, BLOCK>() >> 5;
    constexpr int NW = NT / 32;
#pragma unroll
    for (int u = 0; u < MAXT; ++u) {
        const int t = warp + NW * u;
        if (t >= tm * tn) continue;
        const int ti = t / tn, tj = t - ti * tn;
        if (!keep(ti, tj)) continue;
        const int i = 8 * ti + (lane >> 2), j = 8 * tj + 2 * (lane & 3);
        put(i, j, c2(acc.re[u][0], acc.im[u][0]));
        put(i, j + 1, c2(acc.re[u][1], acc.im[u][1]));
    }
}

// One pencil b, solved end to end by a team of NT threads (every thread of
// the team calls this with the same b and the team's shared memory): the
// whole CTA when BLOCK == NT, else one of the BLOCK / NT teams of a CTA of
// BLOCK threads. NT >= 4 NMAX: the Cholesky gives each row a column group
// of four lanes. FS: S is assembled from the Fourier terms `fs` instead of
// loaded (a separate instantiation, so that the plain solve's register
// allocation is untouched).
template <int NMAX, int NT = kNT, int BLOCK = NT, bool FS = false>
__device__ SGEIG_CTA_BODY_INLINE void cta_solve(const CtaArgs& a, long long b, unsigned char* smem_raw,
                                                const CtaFourier* fs = nullptr) {
    constexpr int R = NMAX / kG;    // rows per lane in a column group
    constexpr int NW = NT / 32;     // warps
    constexpr int NG = NT / kG;     // column groups
    constexpr int TR = NT / 16;     // thread rows of the 16-wide copy loops
    static_assert(NG >= NMAX && NW >= 2 && NW <= 8 && NT % 32 == 0, "CTA shape");
    const int n = a.n, ld = a.ld;
    const size_t mat = (size_t)n * ld;
    double2* A = reinterpret_cast<double2*>(smem_raw);
    double2* B = A + mat;
    CtaVec v = cta_carve(reinterpret_cast<unsigned char*>(B + mat), n);

    // (threadIdx.x read here directly: through team_tid the register
    // allocation of the 56- and 64-row kernels spilled 300+ bytes)
    const int tid = BLOCK == NT ? (int)threadIdx.x : (int)(threadIdx.x % NT), lane = tid & 31, warp = tid >> 5;
    const int tr = tid >> 4, tc = tid & 15;
    const int g = tid >> 2, q = tid & 3;
    const unsigned gmask = 0xFu << (lane & ~3);
    const size_t nn = (size_t)n * n;

    const double2* Hb = a.H + (size_t)b * nn;
    const double2* Sb = a.S + (size_t)b * nn;
    double*  Wb = a.W + (size_t)b * n;
    double2* Ub = a.U + (size_t)b * nn;

    team_sync<NT, BLOCK>();
    phase_mark(8);
    // ---- a1: load (rows by tc so that global reads are contiguous)
    if constexpr (FS) {
        // S(q) from its Fourier terms, lower triangle (the only part the
        // Cholesky reads); the terms are shared by all pencils (L1/L2-resident).
        // Term values first, one term per thread (coalesced, independent
        // loads), into B, which the metric solve leaves free until a3; then
        // each lower entry sums its terms in table order.
        const double q0 = __ldg(fs->q + 3 * b), q1 = __ldg(fs->q + 3 * b + 1), q2 = __ldg(fs->q + 3 * b + 2);
        const int nt = fs->nterms;
        auto term = [&](int t) {
            const double x = fma(q0, __ldg(fs->disp + 3 * t),
                             fma(q1, __ldg(fs->disp + 3 * t + 1), q2 * __ldg(fs->disp + 3 * t + 2)));
            double sn, cs;
            sincospi(2.0 * x, &sn, &cs);
            return cmul(__ldg(fs->coef + t), c2(cs, sn));
        };
        const bool staged = nt <= n * ld;
        if (staged) {
            for (int t = tid; t < nt; t += NT) B[t] = term(t);
            team_sync<NT, BLOCK>();
        }
        for (int idx = tid; idx < n * n; idx += NT) {
            const int j = idx / n, i = idx - j * n;
            if (i < j) continue;
            double2 acc = c2(0.0, 0.0);
            const int t1 = min(__ldg(fs->start + idx + 1), nt);
            for (int t = max(__ldg(fs->start + idx), 0); t < t1; ++t) acc = cadd(acc, staged ? B[t] : term(t));
            A[i + (size_t)j * ld] = acc;
        }
    } else {
        for (int j = tr; j < n; j += TR)
            for (int i = tc; i < n; i += 16) {
                A[i + (size_t)j * ld] = __ldg(Sb + i + (size_t)j * n);
                if (!a.sigma) B[i + (size_t)j * ld] = __ldg(Hb + i + (size_t)j * n);
            }
    }
    if (tid < 8) v.ctl[tid] = 0;

    // ---- a2: Cholesky S = L L^H fused with X = L^-1, in registers.
    // Group g owns row i = g; lane q holds slots j = q + 4t (t < R). Slot j
    // holds the Cholesky working value a_ij while j > k and, from step j
    // on, the inverse accumulator acc(i, j), so that at the end
    // X(i, j) = acc(i, j) r_i with r_k = 1/sqrt(a_kk). Step k reads, from
    // shared memory, column k (colv: a_jk, final after step k-1) and row k
    // of acc (rowv: acc(k, j), j < k), and for i > k applies
    //   a_ij -= a_ik conj(a_jk) r_k^2           k < j <= i
    //   acc(i, j) -= a_ik r_k^2 acc(k, j)       j < k
    //   acc(i, k) = -a_ik r_k^2
    // then publishes column k+1 and row k+1 into the other buffers; one
    // barrier per step. The step loop is unrolled so that slot k is a
    // register known at compile time.
    int fail = 0;
    team_sync<NT, BLOCK>();   // the loads above are complete
    phase_mark(0);
    {
        const int i = g;
        double2 x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) {
            const int j = q + kG * t;
            x[t] = (i < n && j <= i) ? A[i + (size_t)j * ld] : c2(0.0, 0.0);
        }
        if (i < n && q == 0) v.colv[i] = x[0];   // column 0, buffer 0
        double ri = 0.0;
#pragma unroll
        for (int k = 0; k < NMAX; ++k) {
            if (k >= n) break;
            team_sync<NT, BLOCK>();
            const double2* colk = v.colv + (k & 1) * n;
            const double2* rowk = v.rowv + (k & 1) * n;
            double2* coln = v.colv + ((k + 1) & 1) * n;
            double2* rown = v.rowv + ((k + 1) & 1) * n;
            const double akk = colk[k].x;
            if (!(akk > 0.0)) { fail = k + 1; break; }   // uniform: every thread reads akk
            const double r = rsqrt(akk);
            const double r2 = r * r;
            if (i == k) ri = r;
            if (tid == 0) v.rdg[k] = r;
            if (a.stage == 1) {   // stage-wise output: column k of L
                for (int jj = k + tid; jj < n; jj += NT)
                    A[jj + (size_t)k * ld] = (jj == k) ? c2(1.0 / r, 0.0) : cscale(colk[jj], r);
            }
            if (i > k && i < n) {
                const double2 aik = cscale(colk[i], r2);
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    const int j = q + kG * t;
                    if (j > k && j <= i) x[t] = cfms_bc(x[t], aik, colk[j]);
                    else if (j < k) x[t] = cfms(x[t], aik, rowk[j]);
                }
                if (q == (k & 3)) x[k >> 2] = cscale(aik, -1.0);
            }
            // publish column k+1 (rows >= k+1) and row k+1 of acc (j <= k)
            if (k + 1 < n) {
                if (i >= k + 1 && i < n && q == ((k + 1) & 3)) coln[i] = x[(k + 1) >> 2];
                if (i == k + 1) {
#pragma unroll
                    for (int t = 0; t < R; ++t) {
                        const int j = q + kG * t;
                        if (j <= k) rown[j] = x[t];
                    }
                }
            }
        }
        team_sync<NT, BLOCK>();
        if (!fail && a.stage >= 2 && i < n) {
            // X(i, j) = acc(i, j) r_i, X(i, i) = r_i, into A's lower triangle
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int j = q + kG * t;
                if (j < i) A[i + (size_t)j * ld] = cscale(x[t], ri);
                else if (j == i) A[i + (size_t)i * ld] = c2(ri, 0.0);
            }
        }
    }
    team_sync<NT, BLOCK>();
    phase_mark(1);
    int code = fail ? n + fail : 0;   // zhegv: info = n + order of the failing minor

    if (!code && a.stage == 1) {
        for (int j = tr; j < n; j += TR)
            for (int i = tc; i < n; i += 16)
                Ub[i + (size_t)j * n] = (i >= j) ? A[i + (size_t)j * ld] : c2(0.0, 0.0);
        if (tid == 0) a.info[b] = 0;
        return;
    }

    if (!code) {
        // A now holds X = L^-1 in its lower triangle (diagonal real).
        // ---- a3: T = H X^H, T(i, j) = sum_{k <= j} H(i, k) conj(X(j, k)),
        // FP64 tensor-core tiles; T overwrites H after the barrier.
        constexpr int MAXT = ((NMAX / 8) * (NMAX / 8) + NW - 1) / NW;
        const int tn8 = (n + 7) >> 3;
        if (a.sigma) {
            // H = diag(I, -I): T(i, j) = sigma_i conj(X(j, i)), no product needed
            const int m = n >> 1;
            for (int j = tr; j < n; j += TR)
                for (int i = tc; i < n; i += 16) {
                    const double2 x = (i <= j) ? cconj(A[j + (size_t)i * ld]) : c2(0.0, 0.0);
                    B[i + (size_t)j * ld] = (i < m) ? x : c2(-x.x, -x.y);
                }
            team_sync<NT, BLOCK>();
        } else {
            ZTiles<MAXT> acc;
            ztiles_compute<MAXT, NT, BLOCK>(acc, tn8, tn8,
                [&](int i, int k) { return (i < n && k < n) ? B[i + (size_t)k * ld] : c2(0.0, 0.0); },
                [&](int k, int j) { return (j < n && k <= j) ? cconj(A[j + (size_t)k * ld]) : c2(0.0, 0.0); },
                [&](int, int tj, int& k0, int& k1) { k0 = 0; k1 = min(n, 8 * tj + 8); },
                [](int, int) { return true; });
            team_sync<NT, BLOCK>();
            ztiles_store<MAXT, NT, BLOCK>(acc, tn8, tn8, [](int, int) { return true; },
                [&](int i, int j, double2 c) { if (i < n && j < n) B[i + (size_t)j * ld] = c; });
            team_sync<NT, BLOCK>();
        }
        phase_mark(2);
        // ---- a4: C = X T, C(i, j) = sum_{k <= i} X(i, k) T(k, j); lower
        // tiles only, each lower element written with its mirror, so that
        // C is exactly Hermitian.
        {
            ZTiles<MAXT> acc;
            ztiles_compute<MAXT, NT, BLOCK>(acc, tn8, tn8,
                [&](int i, int k) { return (i < n && k <= i) ? A[i + (size_t)k * ld] : c2(0.0, 0.0); },
                [&](int k, int j) { return (k < n && j < n) ? B[k + (size_t)j * ld] : c2(0.0, 0.0); },
                [&](int ti, int, int& k0, int& k1) { k0 = 0; k1 = min(n, 8 * ti + 8); },
                [](int ti, int tj) { return ti >= tj; });
            team_sync<NT, BLOCK>();
            ztiles_store<MAXT, NT, BLOCK>(acc, tn8, tn8, [](int ti, int tj) { return ti >= tj; },
                [&](int i, int j, double2 c) {
                    if (i < n && j < n && i >= j) {
                        if (i == j) c.y = 0.0;
                        B[i + (size_t)j * ld] = c;
                        B[j + (size_t)i * ld] = cconj(c);
                    }
                });
            team_sync<NT, BLOCK>();
            phase_mark(3);
        }
    }

    if (!code && a.stage == 2) {
        for (int j = tr; j < n; j += TR)
            for (int i = tc; i < n; i += 16) Ub[i + (size_t)j * n] = B[i + (size_t)j * ld];
        if (tid == 0) a.info[b] = 0;
        return;
    }

    if (!code) {
        // ---- a5a: Householder tridiagonalisation of C (lower). Reflector k:
        // I - tau_k v v^H on rows k+1.., v[k+1] = 1, v[k+2..] kept in A's
        // strict upper triangle (row k), tau_k in v.tau. Look-ahead: during
        // the rank-2 update of step k, warp 0 updates column k+1 first and
        // computes reflector k+1 (into the other vector buffer) while the
        // other warps update the rest, so each step needs two barriers.
        auto reflect = [&](int k, double2* vbuf) {   // warp 0
            const double2* bk = B + (size_t)k * ld;
            double ss = 0.0;
            for (int i = k + 2 + lane; i < n; i += 32) { const double2 x = bk[i]; ss = fma(x.x, x.x, fma(x.y, x.y, ss)); }
            ss = warp_sum(ss);
            const double2 alpha = bk[k + 1];
            double2 taui, scal = c2(0.0, 0.0);
            double beta;
            if (ss == 0.0 && alpha.y == 0.0) {
                taui = c2(0.0, 0.0);
                beta = alpha.x;
            } else {
                beta = -copysign(sqrt(fma(alpha.x, alpha.x, fma(alpha.y, alpha.y, ss))), alpha.x);
                const double rb = fast_rcp(beta);
                taui = c2((beta - alpha.x) * rb, -alpha.y * rb);
                const double2 z = c2(alpha.x - beta, alpha.y);
                const double inv = fast_rcp(fma(z.x, z.x, z.y * z.y));
                scal = c2(z.x * inv, -z.y * inv);
            }
            for (int i = k + 2 + lane; i < n; i += 32) {
                const double2 vi = cmul(bk[i], scal);
                vbuf[i] = vi;
                A[k + (size_t)i * ld] = vi;
            }
            if (lane == 0) {
                vbuf[k + 1] = c2(1.0, 0.0);
                v.tau[k] = taui;
                v.d[k] = bk[k].x;
                v.e[k] = beta;
            }
        };
        if (n >= 2 && warp == 0) reflect(0, v.vb);
        team_sync<NT, BLOCK>();
        for (int k = 0; k < n - 1; ++k) {
            double2* vk = (k & 1) ? v.vb2 : v.vb;
            double2* vn = (k & 1) ? v.vb : v.vb2;
            const double2 taui = v.tau[k];
            const bool has = !(taui.x == 0.0 && taui.y == 0.0);
            if (has) {
                // p = tau A22 v: four lanes per row; per-warp partial of p^H v
                double2 dotp = c2(0.0, 0.0);
                for (int i = k + 1 + g; i < n; i += NG) {
                    double2 acc = c2(0.0, 0.0);
                    for (int j = k + 1 + q; j < n; j += kG) acc = cfma(acc, B[i + (size_t)j * ld], vk[j]);
                    acc = group_sum2<kG>(gmask, acc);
                    const double2 pi = cmul(taui, acc);
                    if (q == 0) { v.pb[i] = pi; dotp = cfmac(dotp, pi, vk[i]); }
                }
                dotp = warp_sum2(dotp);
                if (lane == 0) v.wred[warp] = dotp;
                team_sync<NT, BLOCK>();
            }
            // A22 -= v w^H + w v^H, w = p + alpha2 v, alpha2 = -tau/2 (p^H v)
            double2 alpha2 = c2(0.0, 0.0);
            if (has) {
                double2 dot = c2(0.0, 0.0);
#pragma unroll
                for (int w = 0; w < NW; ++w) dot = cadd(dot, v.wred[w]);
                alpha2 = cscale(cmul(taui, dot), -0.5);
            }
            if (warp == 0) {
                if (has) {
                    const int j = k + 1;
                    const double2 vj = vk[j];
                    const double2 wj = cfma(v.pb[j], alpha2, vj);
                    for (int i = j + lane; i < n; i += 32) {
                        const double2 vi = vk[i];
                        const double2 wi = cfma(v.pb[i], alpha2, vi);
                        double2* p = B + i + (size_t)j * ld;
                        *p = cfms_bc(cfms_bc(*p, vi, wj), wi, vj);
                    }
                    __syncwarp();
                }
                if (k + 1 < n - 1) reflect(k + 1, vn);
            } else if (has) {
                // group g - 8 of warps 1.. takes rows k+1+(g-8), + NG-8, ...;
                // its lanes take columns j = k+2+q step 4 (column k+1 is warp 0's)
                for (int i = k + 1 + (g - 8); i < n; i += NG - 8) {
                    const double2 vi = vk[i];
                    const double2 wi = cfma(v.pb[i], alpha2, vi);
                    double2* bi = B + i;
                    int j = k + 2 + q;
                    for (; j + 4 < n; j += 8) {
                        const double2 x0 = bi[(size_t)j * ld], x1 = bi[(size_t)(j + 4) * ld];
                        const double2 v0 = vk[j], v1 = vk[j + 4];
                        const double2 w0 = cfma(v.pb[j], alpha2, v0), w1 = cfma(v.pb[j + 4], alpha2, v1);
                        bi[(size_t)j * ld] = cfms_bc(cfms_bc(x0, vi, w0), wi, v0);
                        bi[(size_t)(j + 4) * ld] = cfms_bc(cfms_bc(x1, vi, w1), wi, v1);
                    }
                    if (j < n) {
                        const double2 v0 = vk[j];
                        const double2 w0 = cfma(v.pb[j], alpha2, v0);
                        bi[(size_t)j * ld] = cfms_bc(cfms_bc(bi[(size_t)j * ld], vi, w0), wi, v0);
                    }
                }
            }
            team_sync<NT, BLOCK>();
        }
        if (tid == 0) v.d[n - 1] = B[(n - 1) + (size_t)(n - 1) * ld].x;
        team_sync<NT, BLOCK>();
        phase_mark(4);
        // ---- a5b: divide and conquer; Z (real) and its workspace in B
        DCShared dc;
        dc.Z = reinterpret_cast<double*>(B); dc.ldz = ld;
        dc.U = dc.Z + (size_t)n * ld;        dc.ldu = ld;
        dc.d = v.d; dc.e = v.e;
        dc.w = v.dcd; dc.z = dc.w + n; dc.dl = dc.z + n; dc.zz = dc.dl + n; dc.zh = dc.zz + n;
        dc.rt = dc.zh + n; dc.rho = dc.rt + n; dc.scal = dc.rho + n;
        dc.org = v.dci; dc.nd = dc.org + n; dc.perm = dc.nd + n; dc.kcnt = dc.perm + n;
        tridiag_dc<NT, NMAX, BLOCK>(n, dc);
        if (tid == 0) {
            bool bad = false;
            for (int i = 0; i < n; ++i) bad |= !isfinite(dc.w[i]);
            v.ctl[4] = bad ? kEigFailCode : 0;
        }
        team_sync<NT, BLOCK>();
        phase_mark(5);
        if (v.ctl[4]) code = v.ctl[4];
    }

    if (code) {
        const double qnan = __longlong_as_double(0x7ff8000000000000LL);
        if (a.stage == kStageIntensity) {
            for (int e = tid; e < a.ne; e += NT) a.spec[(size_t)b * a.ne + e] = qnan;
        } else {
            for (size_t idx = tid; idx < nn; idx += NT) Ub[idx] = c2(qnan, qnan);
        }
        if (a.stage >= 3) for (int i = tid; i < n; i += NT) Wb[i] = qnan;
        if (tid == 0) a.info[b] = code == kEigFailCode ? eig_fail_info(n) : code;
        return;
    }

    // ---- ascending rank of each eigenvalue
    for (int j = tid; j < n; j += NT) {
        const double dj = order_key(v.dcd[j]);
        int r = 0;
        for (int k2 = 0; k2 < n; ++k2) {
            const double dk = order_key(v.dcd[k2]);
            r += (dk < dj) || (dk == dj && k2 < j);
        }
        v.rank[j] = r;
        Wb[r] = v.dcd[j];
    }
    // ---- a5c: V = Q Z with Q = H_0 H_1 ... H_{n-2} in compact-WY blocks of
    // 16 reflectors on the FP64 tensor cores. Block c (reflectors 16c ..,
    // m_c of them) is Q_c = I - Y_c T_c Y_c^H (the zlarft forward,
    // columnwise T: T(l, l) = tau_l, T(0:l, l) = -tau_l T(0:l, 0:l) Y^H y_l),
    // and V = Q_0 (Q_1 (... Q_last Z)). Steps:
    //   1. G_c = Y_c^H Y_c (MMA tiles, upper 8x8 tiles), packed into the
    //      vector area (free from here on); Z (real) into registers.
    //   2. V = Z as complex in B; T_c by its column recurrence, one warp per
    //      block, written over G_c column by column.
    //   3. warp p owns columns [8p, 8p+8) of V and applies the blocks, last
    //      first, with no CTA barrier: W1 = Y_c^H V_p, W2 = T_c W1,
    //      V_p -= Y_c W2, the 8-column intermediates passed between MMA
    //      fragment layouts by shuffles.
    {
        const int nref = n - 1;                      // reflectors 0 .. n-2
        const int nblk = (nref + 15) >> 4;
        double2* tpk = v.vb;                         // packed upper T_c (G_c before)
        auto tidx = [](int c, int l, int i) { return 136 * c + ((i * (i + 1)) >> 1) + l; };
        // Y_c(r, l): reflector k = 16c + l, v_k[k+1] = 1, v_k[r] in A's row k
        auto yv = [&](int c, int r, int l) -> double2 {
            const int k = 16 * c + l;
            if (k >= nref || r <= k || r >= n) return c2(0.0, 0.0);
            return (r == k + 1) ? c2(1.0, 0.0) : A[k + (size_t)r * ld];
        };
        // 1. Gram blocks: tiles (c, hr, hc) with hr <= hc, dealt to the warps
        for (int t = warp; t < 3 * nblk; t += NW) {
            const int c = t / 3, hh = t - 3 * c;
            const int hr = hh == 2 ? 1 : 0, hc = hh == 0 ? 0 : 1;
            double gr[2] = {0.0, 0.0}, gi[2] = {0.0, 0.0};
            const int la = 8 * hr + (lane >> 2), lb = 8 * hc + (lane >> 2);
            for (int k0 = 16 * c; k0 < n; k0 += 4) {
                const int r = k0 + (lane & 3);
                const double2 ya = yv(c, r, la);   // A(l, r) = conj(Y(r, l))
                const double2 yb = yv(c, r, lb);   // B(r, l') = Y(r, l')
                mma884(gr[0], gr[1], ya.x, yb.x);
                mma884(gr[0], gr[1], ya.y, yb.y);
                mma884(gi[0], gi[1], ya.x, yb.y);
                mma884(gi[0], gi[1], -ya.y, yb.x);
            }
            const int l = 8 * hr + (lane >> 2);
#pragma unroll
            for (int e2 = 0; e2 < 2; ++e2) {
                const int i = 8 * hc + 2 * (lane & 3) + e2;
                if (l < i && 16 * c + i < nref) tpk[tidx(c, l, i)] = c2(gr[e2], gi[e2]);
            }
        }
        // Z (real) into registers, then V = Z as complex in place
        constexpr int ZR = (NMAX * NMAX + NT - 1) / NT;
        double zr[ZR];
        const double* Z = reinterpret_cast<const double*>(B);
#pragma unroll
        for (int u = 0; u < ZR; ++u) {
            const int idx = tid + NT * u, j = idx / n, i = idx - j * n;
            zr[u] = (idx < n * n) ? Z[i + (size_t)j * ld] : 0.0;
        }
        team_sync<NT, BLOCK>();
#pragma unroll
        for (int u = 0; u < ZR; ++u) {
            const int idx = tid + NT * u, j = idx / n, i = idx - j * n;
            if (idx < n * n) B[i + (size_t)j * ld] = c2(zr[u], 0.0);
        }
        // 2. T_c: lane l of warp c holds row l of T_c; column i needs
        // T(l, m < i) and G(m, i) (l <= m < i); every lane reads column i of
        // G before any lane overwrites it with column i of T.
        for (int c = warp; c < nblk; c += NW) {
            const int l = lane;
            const int mc = min(16, nref - 16 * c);
            double2 trow[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                trow[i] = c2(0.0, 0.0);
                if (i < mc && l < 16 && l <= i) {
                    const double2 ti = v.tau[16 * c + i];
                    if (l == i) {
                        trow[i] = ti;
                    } else {
                        double2 s0 = c2(0.0, 0.0), s1 = c2(0.0, 0.0);
#pragma unroll
                        for (int m = 0; m < i; ++m) {
                            if (m < l) continue;
                            const double2 gm = tpk[tidx(c, m, i)];
                            if (m & 1) s1 = cfma(s1, trow[m], gm); else s0 = cfma(s0, trow[m], gm);
                        }
                        trow[i] = cscale(cmul(ti, cadd(s0, s1)), -1.0);
                    }
                }
                __syncwarp();
                if (i < mc && l < 16 && l <= i) tpk[tidx(c, l, i)] = trow[i];
                __syncwarp();
            }
        }
        team_sync<NT, BLOCK>();
        // 3. per-warp panels: columns [8p, 8p+8), p = warp, warp + NW, ...
        for (int p = warp; 8 * p < n; p += NW) {
            const int jb = 8 * p + (lane >> 2);   // B-fragment column of this lane
            // W (16 x 8, accumulator layout: rows 8h + lane/4, columns
            // 2(lane%4) + e) -> B-fragment layout for k-step s: element
            // (4s + lane%4, lane/4), returned as (re, im) scaled by `sgn`
            auto to_bfrag = [&](const double (&wr)[2][2], const double (&wi)[2][2], int s, double sgn,
                                double& br, double& bi) {
                const int src = 16 * (s & 1) + 4 * (lane & 3) + (lane >> 3);
                const int h = s >> 1, e2 = (lane >> 2) & 1;
                const double r0 = __shfl_sync(0xffffffffu, wr[h][0], src);
                const double r1 = __shfl_sync(0xffffffffu, wr[h][1], src);
                const double i0 = __shfl_sync(0xffffffffu, wi[h][0], src);
                const double i1 = __shfl_sync(0xffffffffu, wi[h][1], src);
                br = sgn * (e2 ? r1 : r0);
                bi = sgn * (e2 ? i1 : i0);
            };
            for (int c = nblk - 1; c >= 0; --c) {
                // W1 = Y_c^H V_p  (16 x 8, K = rows 16c .. n-1)
                double w1r[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, w1i[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
                for (int k0 = 16 * c; k0 < n; k0 += 4) {
                    const int r = k0 + (lane & 3);
                    const double2 vb_ = (r < n && jb < n) ? B[r + (size_t)jb * ld] : c2(0.0, 0.0);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const double2 ya = yv(c, r, 8 * h + (lane >> 2));
                        mma884(w1r[h][0], w1r[h][1], ya.x, vb_.x);
                        mma884(w1r[h][0], w1r[h][1], ya.y, vb_.y);
                        mma884(w1i[h][0], w1i[h][1], ya.x, vb_.y);
                        mma884(w1i[h][0], w1i[h][1], -ya.y, vb_.x);
                    }
                }
                // W2 = T_c W1 (T upper, K = 16), negated for the update
                double w2r[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, w2i[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    double br, bi;
                    to_bfrag(w1r, w1i, s, -1.0, br, bi);
                    const int kk = 4 * s + (lane & 3);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int l = 8 * h + (lane >> 2);
                        const double2 ta = (l <= kk && 16 * c + kk < nref) ? tpk[tidx(c, l, kk)] : c2(0.0, 0.0);
                        mma884(w2r[h][0], w2r[h][1], ta.x, br);
                        mma884(w2r[h][0], w2r[h][1], -ta.y, bi);
                        mma884(w2i[h][0], w2i[h][1], ta.x, bi);
                        mma884(w2i[h][0], w2i[h][1], ta.y, br);
                    }
                }
                // V_p += Y_c (-W2) on row tiles from 2c (rows < 16c + 1 get 0)
                double bfr[4], bfi[4];
#pragma unroll
                for (int s = 0; s < 4; ++s) to_bfrag(w2r, w2i, s, 1.0, bfr[s], bfi[s]);
                const int j0 = 8 * p + 2 * (lane & 3);
                for (int t = 2 * c; 8 * t < n; ++t) {
                    const int r = 8 * t + (lane >> 2);
                    double ar[2], ai[2];
#pragma unroll
                    for (int e2 = 0; e2 < 2; ++e2) {
                        const double2 x = (r < n && j0 + e2 < n) ? B[r + (size_t)(j0 + e2) * ld] : c2(0.0, 0.0);
                        ar[e2] = x.x; ai[e2] = x.y;
                    }
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const double2 ya = yv(c, r, 4 * s + (lane & 3));   // A(r, l) = Y(r, l)
                        mma884(ar[0], ar[1], ya.x, bfr[s]);
                        mma884(ar[0], ar[1], -ya.y, bfi[s]);
                        mma884(ai[0], ai[1], ya.x, bfi[s]);
                        mma884(ai[0], ai[1], ya.y, bfr[s]);
                    }
#pragma unroll
                    for (int e2 = 0; e2 < 2; ++e2)
                        if (r < n && j0 + e2 < n) B[r + (size_t)(j0 + e2) * ld] = c2(ar[e2], ai[e2]);
                }
                __syncwarp();
            }
        }
    }
    team_sync<NT, BLOCK>();
    phase_mark(6);
    if (a.stage == 3) {
        for (int jj = tr; jj < n; jj += TR) {
            double2* uo = Ub + (size_t)v.rank[jj] * n;
            for (int i = tc; i < n; i += 16) uo[i] = B[i + (size_t)jj * ld];
        }
        if (tid == 0) a.info[b] = 0;
        return;
    }
    // ---- a6: U = X^H V, U(i, j) = sum_{k >= i} conj(X(k, i)) V(k, j), FP64
    // tensor-core tiles; U overwrites V after the barrier.
    {
        constexpr int MAXT = ((NMAX / 8) * (NMAX / 8) + NW - 1) / NW;
        const int tn8 = (n + 7) >> 3;
        ZTiles<MAXT> acc;
        ztiles_compute<MAXT, NT, BLOCK>(acc, tn8, tn8,
            [&](int i, int k) { return (i < n && k >= i && k < n) ? cconj(A[k + (size_t)i * ld]) : c2(0.0, 0.0); },
            [&](int k, int j) { return (k < n && j < n) ? B[k + (size_t)j * ld] : c2(0.0, 0.0); },
            [&](int ti, int, int& k0, int& k1) { k0 = 8 * ti; k1 = n; },
            [](int, int) { return true; });
        team_sync<NT, BLOCK>();
        ztiles_store<MAXT, NT, BLOCK>(acc, tn8, tn8, [](int, int) { return true; },
            [&](int i, int j, double2 c) { if (i < n && j < n) B[i + (size_t)j * ld] = c; });
        team_sync<NT, BLOCK>();
        phase_mark(7);
    }
    if (a.stage == kStageIntensity) {
        // ---- spin-wave intensities from U (in B, column jj = eigenvalue
        // dcd[jj]) without storing U: for each positive eigenvalue lambda,
        // t = u / sqrt(lambda) is the Bogoliubov vector of the mode of
        // energy omega = 1 / lambda; Y = O t (3 components) and
        // I = sum_ab (delta_ab - q_a q_b) conj(Y_a) Y_b = |Y|^2 - |q . Y|^2;
        // then S(E_e) = sum_modes I g(E_e - omega) with the Gaussian g.
        // A (X) is free after a6 and takes O (3 n <= n ld for even n);
        // the modes go to the dead Householder vector pb.
        const double2* Ob = a.O + (size_t)b * 3 * n;
        double2* Os = A;
        double* om = reinterpret_cast<double*>(v.pb);
        double* it = om + n;
        for (int idx = tid; idx < 3 * n; idx += NT) Os[idx] = __ldg(Ob + idx);
        const double q0 = __ldg(a.qhat + 3 * b), q1 = __ldg(a.qhat + 3 * b + 1), q2 = __ldg(a.qhat + 3 * b + 2);
        team_sync<NT, BLOCK>();
        for (int jj = g; jj < n; jj += NG) {
            const double lam = v.dcd[jj];
            double2 y0 = c2(0.0, 0.0), y1 = c2(0.0, 0.0), y2 = c2(0.0, 0.0);
            for (int i = q; i < n; i += kG) {
                const double2 u = B[i + (size_t)jj * ld];
                y0 = cfma(y0, Os[3 * i], u);
                y1 = cfma(y1, Os[3 * i + 1], u);
                y2 = cfma(y2, Os[3 * i + 2], u);
            }
            const unsigned gm = 0xFu << (lane & ~3);
            y0 = group_sum2<kG>(gm, y0);
            y1 = group_sum2<kG>(gm, y1);
            y2 = group_sum2<kG>(gm, y2);
            if (q == 0) {
                const double yy = fma(y0.x, y0.x, fma(y0.y, y0.y, fma(y1.x, y1.x, fma(y1.y, y1.y,
                                  fma(y2.x, y2.x, y2.y * y2.y)))));
                const double2 qy = c2(fma(q0, y0.x, fma(q1, y1.x, q2 * y2.x)), fma(q0, y0.y, fma(q1, y1.y, q2 * y2.y)));
                const bool pos = lam > 0.0;
                om[jj] = pos ? 1.0 / lam : -1.0;
                it[jj] = pos ? (yy - fma(qy.x, qy.x, qy.y * qy.y)) / lam : 0.0;
            }
        }
        team_sync<NT, BLOCK>();
        for (int e = tid; e < a.ne; e += NT) {
            const double E = __ldg(a.energies + e);
            double acc = 0.0;
            for (int jj = 0; jj < n; ++jj) {
                if (!(om[jj] > 0.0)) continue;
                const double x = E - om[jj];
                acc = fma(it[jj], exp(-x * x * a.ginv2), acc);
            }
            a.spec[(size_t)b * a.ne + e] = acc * a.gnorm;
        }
        if (tid == 0) a.info[b] = 0;
        return;
    }
    // ---- a7: store U, column j to position rank[j]
    for (int jj = tr; jj < n; jj += TR) {
        double2* uo = Ub + (size_t)v.rank[jj] * n;
        for (int i = tc; i < n; i += 16) uo[i] = B[i + (size_t)jj * ld];
    }
    if (tid == 0) a.info[b] = 0;
}

}  // namespace cta
}  // namespace sgeig
