// FP64 batched generalized Hermitian-definite eigensolver for sm_100a, the
// "smem-wide" regime (N too large for the register-resident smem-cta kernel,
// small enough for both working matrices to fit one CTA's shared memory).
//
// One CTA solves one matrix pair at a time (persistent over the batch):
//   a1  load S -> A, H^H -> B                     (kernel_source.hpp:233-242)
//   a2  A <- L, S = L L^H (lower Cholesky)        (:244)
//   a3  B <- L^-1 H                               (:246)
//   a4  B <- B L^-H = C   (done as L^-1 (L^-1 H)^H, same value)  (:248)
//   a5  C = Q T Q^H (Householder, lower), T = Z diag(w) Z^T by divide and
//       conquer, V = Q Z                          (:250)
//   a6  U = L^-H V                                (:252)
//   a7  store W (ascending) and U                 (:268-276)
// Column work (a3, a4, a6 and the back-transform of a5) is owned by groups
// of G = 4 lanes per column, which synchronise with warp shuffles only; the
// Cholesky and Householder steps use CTA barriers. A and B are n x ld
// complex, ld odd so that row walks are bank-conflict free.
//
// This file also holds the regime choice (plain_plan), the launch dispatch
// and the allocation-free entry point, which runs the tiled kernel.

#include "geneig_common.cuh"
#include "geneig_dc.cuh"
#include "geneig_kernels.h"
#include "sunny_geneig.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>

namespace sgeig {
namespace {

constexpr int kG  = 4;     // lanes per column group
constexpr int kNT = 256;   // threads per CTA

struct PlainArgs {
    const double2* __restrict__ H;
    const double2* __restrict__ S;
    double*  W;
    double2* U;
    int*     info;
    double2* scratch;
    long long batch;
    int n, ld, stage;
    int sigma;      // H = diag(I_{n/2}, -I_{n/2}), not read from memory
};

// Shared-memory vector area (after the matrices in the SmemCta regime).
struct VecArea {
    double2* tau;   // n   Householder scalars
    double2* vb;    // n   current Householder vector (v[k+1] = 1)
    double2* pb;    // n   tau * A22 * v
    double2* red;   // 32  reduction scratch
    double*  d;     // n   tridiagonal diagonal / eigenvalues
    double*  e;     // n   tridiagonal off-diagonal
    double*  rdg;   // n   1 / L_kk
    int*     rank;  // n   ascending position of eigenvalue j
    int*     ctl;   // 8   control words
    double*  dcd;   // divide-and-conquer doubles (dc_vec_doubles(n))
    int*     dci;   // divide-and-conquer ints (dc_vec_ints(n))
};

__host__ __device__ inline size_t vec_area_bytes(int n) {
    return (size_t)n * 16 * 3 + 32 * 16 + (size_t)n * 8 * 3 + (size_t)n * 4 + 8 * 4 +
           (size_t)dc_vec_doubles(n) * 8 + (size_t)dc_vec_ints(n) * 4;
}

__device__ inline VecArea carve(unsigned char* p, int n) {
    VecArea v;
    v.tau = reinterpret_cast<double2*>(p);
    v.vb  = v.tau + n;
    v.pb  = v.vb + n;
    v.red = v.pb + n;
    v.d   = reinterpret_cast<double*>(v.red + 32);
    v.e   = v.d + n;
    v.rdg = v.e + n;
    v.dcd  = v.rdg + n;
    v.rank = reinterpret_cast<int*>(v.dcd + dc_vec_doubles(n));
    v.ctl  = v.rank + n;
    v.dci  = v.ctl + 8;
    return v;
}

// X <- L^-1 X for the columns of X owned by this group (rows split by lane).
__device__ __forceinline__ void group_forward_solve(const double2* A, const double* rdg, double2* X,
                                                    int n, int ld, int g, int q, unsigned gmask) {
    constexpr int NG = kNT / kG;
    for (int j = g; j < n; j += NG) {
        double2* x = X + (size_t)j * ld;
        for (int k = 0; k < n; ++k) {
            double2 xk = c2(0.0, 0.0);
            const int owner = k % kG;
            if (q == owner) { xk = cscale(x[k], rdg[k]); x[k] = xk; }
            xk = group_bcast2<kG>(gmask, xk, owner);
            const double2* lk = A + (size_t)k * ld;
            for (int i = first_in_class<kG>(k + 1, q); i < n; i += kG) x[i] = cfms(x[i], lk[i], xk);
        }
    }
}

template <int NMAX>
__global__ void __launch_bounds__(kNT, 1) geneig_plain_kernel(PlainArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, ld = a.ld;
    const size_t mat = (size_t)n * ld;

    double2* A = reinterpret_cast<double2*>(smem_raw);
    double2* B = A + mat;
    VecArea v = carve(reinterpret_cast<unsigned char*>(B + mat), n);

    const int tid  = threadIdx.x;
    const int g    = tid / kG;
    const int q    = tid % kG;
    const int lane = tid & 31;
    const unsigned gmask = ((1u << kG) - 1u) << (lane & ~(kG - 1));
    constexpr int NG = kNT / kG;
    const size_t nn = (size_t)n * n;

    for (long long b = blockIdx.x; b < a.batch; b += gridDim.x) {
        const double2* Hb = a.H + (size_t)b * nn;
        const double2* Sb = a.S + (size_t)b * nn;
        double*  Wb = a.W + (size_t)b * n;
        double2* Ub = a.U + (size_t)b * nn;

        __syncthreads();  // previous matrix fully consumed
        // ---- a1: load. A(i,j) = S(i,j); B(i,j) = conj(H(j,i)), so that
        // L^-1 (L^-1 H^H)^H = L^-1 H L^-H for any H (reads both triangles).
        for (int idx = tid; idx < (int)nn; idx += kNT) {
            const int j = idx / n, i = idx - j * n;
            A[i + (size_t)j * ld] = __ldg(Sb + idx);
            if (a.sigma) {
                B[j + (size_t)i * ld] = c2(i != j ? 0.0 : (2 * i < n ? 1.0 : -1.0), 0.0);
            } else {
                const double2 h = __ldg(Hb + idx);
                B[j + (size_t)i * ld] = cconj(h);
            }
        }
        if (tid < 8) v.ctl[tid] = 0;
        __syncthreads();

        // ---- a2: Cholesky (lower). Column k is finalised by its owner group,
        // then every group applies it to the columns it owns.
        for (int k = 0; k < n; ++k) {
            if (k % NG == g) {
                __syncwarp(gmask);
                double2* ak = A + (size_t)k * ld;
                const double akk = ak[k].x;
                __syncwarp(gmask);          // every lane has read the pivot before it is overwritten
                if (akk > 0.0) {            // false for NaN, as LAPACK's potrf test
                    const double lk = sqrt(akk), r = 1.0 / lk;
                    for (int i = first_in_class<kG>(k + 1, q); i < n; i += kG) ak[i] = cscale(ak[i], r);
                    if (q == k % kG) { ak[k] = c2(lk, 0.0); v.rdg[k] = r; }
                } else if (q == 0) {
                    v.ctl[0] = k + 1;
                }
            }
            __syncthreads();
            if (v.ctl[0]) break;
            const double2* ak = A + (size_t)k * ld;
            int j = g;
            while (j <= k) j += NG;
            for (; j < n; j += NG) {
                const double2 ljk = ak[j];
                double2* aj = A + (size_t)j * ld;
                for (int i = first_in_class<kG>(j, q); i < n; i += kG) aj[i] = cfms_bc(aj[i], ak[i], ljk);
            }
        }

        int code = v.ctl[0] ? (n + v.ctl[0]) : 0;   // zhegv: info = n + order of failing minor
        if (!code && a.stage >= 2) {
            // ---- a3: B <- L^-1 H^H
            group_forward_solve(A, v.rdg, B, n, ld, g, q, gmask);
            __syncthreads();
            // ---- a4: B <- L^-1 B^H  (= L^-1 H L^-H)
            for (int idx = tid; idx < (int)nn; idx += kNT) {
                const int j = idx / n, i = idx - j * n;
                if (i > j) {
                    const double2 x = B[i + (size_t)j * ld], y = B[j + (size_t)i * ld];
                    B[i + (size_t)j * ld] = cconj(y);
                    B[j + (size_t)i * ld] = cconj(x);
                } else if (i == j) {
                    B[i + (size_t)i * ld].y = -B[i + (size_t)i * ld].y;
                }
            }
            __syncthreads();
            group_forward_solve(A, v.rdg, B, n, ld, g, q, gmask);
            __syncthreads();
            // C is taken from its lower triangle, as a lower-fill heev does.
            for (int idx = tid; idx < (int)nn; idx += kNT) {
                const int j = idx / n, i = idx - j * n;
                if (i > j) B[j + (size_t)i * ld] = cconj(B[i + (size_t)j * ld]);
                else if (i == j) B[i + (size_t)i * ld].y = 0.0;
            }
            __syncthreads();
        }

        if (!code && a.stage >= 3) {
            // ---- a5a: Householder tridiagonalisation (lower), C = Q T Q^H.
            // Reflector k: H_k = I - tau_k v v^H on rows k+1..n-1, v[k+1] = 1.
            // v[k+2..n) is kept in A's strict upper triangle, row k, and tau_k
            // at A(k, k+1) (that triangle is unused by the Cholesky factor).
            for (int k = 0; k < n - 1; ++k) {
                double2* bk = B + (size_t)k * ld;
                if (tid < 32) {
                    double ss = 0.0;
                    for (int i = k + 2 + tid; i < n; i += 32) { const double2 x = bk[i]; ss = fma(x.x, x.x, fma(x.y, x.y, ss)); }
                    ss = warp_sum(ss);
                    const double2 alpha = bk[k + 1];
                    double2 taui, scal = c2(0.0, 0.0);
                    double beta;
                    if (ss == 0.0 && alpha.y == 0.0) {
                        taui = c2(0.0, 0.0);
                        beta = alpha.x;
                    } else {
                        beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + ss), alpha.x);
                        taui = c2((beta - alpha.x) / beta, -alpha.y / beta);
                        const double2 z = c2(alpha.x - beta, alpha.y);
                        const double inv = 1.0 / (z.x * z.x + z.y * z.y);
                        scal = c2(z.x * inv, -z.y * inv);
                    }
                    for (int i = k + 2 + tid; i < n; i += 32) {
                        const double2 vi = cmul(bk[i], scal);
                        v.vb[i] = vi;
                        A[k + (size_t)i * ld] = vi;
                    }
                    if (tid == 0) {
                        v.vb[k + 1] = c2(1.0, 0.0);
                        v.tau[k] = taui;
                        A[k + (size_t)(k + 1) * ld] = taui;
                        v.d[k] = bk[k].x;
                        v.e[k] = beta;
                    }
                }
                __syncthreads();
                const double2 taui = v.tau[k];
                if (taui.x == 0.0 && taui.y == 0.0) continue;
                // p = tau * A22 * v (A22 kept as a full Hermitian matrix)
                for (int i = k + 1 + g; i < n; i += NG) {
                    double2 acc = c2(0.0, 0.0);
                    for (int j = k + 1 + q; j < n; j += kG) acc = cfma(acc, B[i + (size_t)j * ld], v.vb[j]);
                    acc = group_sum2<kG>(gmask, acc);
                    if (q == 0) v.pb[i] = cmul(taui, acc);
                }
                __syncthreads();
                if (tid < 32) {
                    double2 dot = c2(0.0, 0.0);
                    for (int i = k + 1 + tid; i < n; i += 32) dot = cfmac(dot, v.pb[i], v.vb[i]);
                    dot = warp_sum2(dot);
                    if (tid == 0) v.red[0] = cscale(cmul(taui, dot), -0.5);
                }
                __syncthreads();
                const double2 alpha2 = v.red[0];
                // A22 -= v w^H + w v^H,  w = p + alpha2 v
                const int m = n - k - 1;
                for (int idx = tid; idx < m * m; idx += kNT) {
                    const int jj = idx / m, ii = idx - jj * m;
                    const int i = k + 1 + ii, j = k + 1 + jj;
                    const double2 vi = v.vb[i], vj = v.vb[j];
                    const double2 wi = cfma(v.pb[i], alpha2, vi), wj = cfma(v.pb[j], alpha2, vj);
                    double2 x = B[i + (size_t)j * ld];
                    x = cfms_bc(x, vi, wj);
                    x = cfms_bc(x, wi, vj);
                    B[i + (size_t)j * ld] = x;
                }
                __syncthreads();
            }
            if (tid == 0) {
                v.d[n - 1] = B[(n - 1) + (size_t)(n - 1) * ld].x;
                if (n == 1) v.tau[0] = c2(0.0, 0.0);
            }
            __syncthreads();
            // ---- a5b: divide and conquer on T; Z (real) and its merge
            // workspace share B's storage, eigenvalues land in dcd[0..n).
            {
                DCShared dc;
                dc.Z = reinterpret_cast<double*>(B); dc.ldz = ld;
                dc.U = dc.Z + (size_t)n * ld;        dc.ldu = ld;
                dc.Zo = nullptr;
                dc.d = v.d; dc.e = v.e;
                dc.w = v.dcd; dc.z = dc.w + n; dc.dl = dc.z + n; dc.zz = dc.dl + n; dc.zh = dc.zz + n;
                dc.rt = dc.zh + n; dc.rho = dc.rt + n; dc.scal = dc.rho + n;
                dc.org = v.dci; dc.nd = dc.org + n; dc.perm = dc.nd + n; dc.kcnt = dc.perm + n;
                tridiag_dc<kNT, NMAX>(n, dc);
                if (tid == 0) {
                    bool bad = false;
                    for (int i = 0; i < n; ++i) bad |= !isfinite(dc.w[i]);
                    v.ctl[4] = bad ? kEigFailCode : 0;
                }
                __syncthreads();
                if (v.ctl[4]) code = v.ctl[4];
            }
            // ascending rank of each eigenvalue
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
        }

        // ---- outputs
        if (code) {
            const double qnan = __longlong_as_double(0x7ff8000000000000LL);
            for (int idx = tid; idx < (int)nn; idx += kNT) Ub[idx] = c2(qnan, qnan);
            if (a.stage >= 3) for (int i = tid; i < n; i += kNT) Wb[i] = qnan;
            if (tid == 0) a.info[b] = code == kEigFailCode ? eig_fail_info(n) : code;
            continue;
        }
        if (tid == 0) a.info[b] = 0;
        if (a.stage == 1) {
            for (int idx = tid; idx < (int)nn; idx += kNT) {
                const int j = idx / n, i = idx - j * n;
                Ub[idx] = (i >= j) ? A[i + (size_t)j * ld] : c2(0.0, 0.0);
            }
            continue;
        }
        if (a.stage == 2) {
            for (int idx = tid; idx < (int)nn; idx += kNT) {
                const int j = idx / n, i = idx - j * n;
                Ub[idx] = B[i + (size_t)j * ld];
            }
            continue;
        }
        {
            // a5c + a6 + a7 in registers, one column per group (rows i = q + G t):
            // x = Q z_j, then L^H u = x, then store u as column rank[j].
            constexpr int R = NMAX / kG;
            const double* Z = reinterpret_cast<const double*>(B);
            for (int j = g; j < n; j += NG) {
                double2 x[R];
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    const int i = q + kG * t;
                    x[t] = c2(i < n ? Z[i + (size_t)j * ld] : 0.0, 0.0);
                }
                for (int k = n - 2; k >= 0; --k) {
                    const double2 tk = v.tau[k];
                    if (tk.x == 0.0 && tk.y == 0.0) continue;
                    const double2* vk = A + k;   // v_k[i] = vk[i * ld] for i >= k+2, v_k[k+1] = 1
                    double2 s = c2(0.0, 0.0);
#pragma unroll
                    for (int t = 0; t < R; ++t) {
                        const int i = q + kG * t;
                        if (i > k && i < n) {
                            const double2 vi = (i == k + 1) ? c2(1.0, 0.0) : vk[(size_t)i * ld];
                            s = cfmac(s, vi, x[t]);
                        }
                    }
                    s = group_sum2<kG>(gmask, s);
                    const double2 ts = cmul(tk, s);
#pragma unroll
                    for (int t = 0; t < R; ++t) {
                        const int i = q + kG * t;
                        if (i > k && i < n) {
                            const double2 vi = (i == k + 1) ? c2(1.0, 0.0) : vk[(size_t)i * ld];
                            x[t] = cfms(x[t], ts, vi);
                        }
                    }
                }
                if (a.stage >= 4) {
                    // back substitution, row i = qq + G tt from the bottom up
#pragma unroll
                    for (int tt = R - 1; tt >= 0; --tt) {
#pragma unroll
                        for (int qq = kG - 1; qq >= 0; --qq) {
                            const int i = qq + kG * tt;
                            if (i >= n) continue;
                            double2 ui = c2(0.0, 0.0);
                            if (q == qq) { ui = cscale(x[tt], v.rdg[i]); x[tt] = ui; }
                            ui = group_bcast2<kG>(gmask, ui, qq);
#pragma unroll
                            for (int t = 0; t <= tt; ++t) {
                                const int kr = q + kG * t;
                                if (kr < i) x[t] = cfmsc(x[t], A[i + (size_t)kr * ld], ui);
                            }
                        }
                    }
                }
                const int r = v.rank[j];
                double2* uo = Ub + (size_t)r * n;
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    const int i = q + kG * t;
                    if (i < n) uo[i] = x[t];
                }
                if (q == 0) Wb[r] = v.dcd[j];
            }
        }
    }
}

int g_smem_optin = -1;

constexpr int kWideNmax = 96;

}  // namespace

int smem_cta_max_n() {
    // largest n with 2*n*ld*16 + vectors <= 227 KB (ld = n | 1)
    int best = 0;
    for (int n = 1; n <= kMaxN; ++n) {
        const int ld = n | 1;
        const size_t bytes = (size_t)2 * n * ld * 16 + vec_area_bytes(n);
        if (bytes <= 232448) best = n;
    }
    return best;
}

bool plain_plan(int n, int device, PlainPlan* plan, std::string* err, bool mixed, const char* regime,
                int slots_per_sm, int pencils_per_cta) {
    if (n < 1 || n > kMaxN) {
        *err = "matrix size out of range [1, " + std::to_string(kMaxN) + "]";
        return false;
    }
    int optin = 0, sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) { *err = std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e); return false; }
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) { *err = std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e); return false; }
    g_smem_optin = optin;

    // Optional override for measurements: SUNNY_GENEIG_REGIME = smem-cta |
    // smem-wide | l2-slot picks that regime wherever it can hold n.
    const bool asked = regime != nullptr && regime[0] != '\0';
    const char* force = asked ? regime : std::getenv("SUNNY_GENEIG_REGIME");
    const std::string want = force ? force : "";
    if (asked && want != "smem-cta" && want != "smem-wide" && want != "l2-slot") {
        *err = "unknown regime '" + want + "' (smem-cta, smem-wide or l2-slot)";
        return false;
    }
    if (slots_per_sm != 0 && slots_per_sm != 1 && slots_per_sm != 2) {
        *err = "slots_per_sm must be 0 (default), 1 or 2";
        return false;
    }
    PlainPlan p;
    p.n = n;
    p.ld = n | 1;
    p.threads = kNT;
    // Each kernel's dynamic shared-memory limit is set to the device maximum
    // (not to this n's need), so that creating a handle for a smaller n never
    // lowers the limit under a live handle for a larger one.
    // Measured on B200 (solves/s, batch 32768): the tiled kernel overtakes the
    // register-resident smem-cta kernel between n = 60 and n = 62 and runs
    // about 2x the smem-wide kernel at n = 66..80, so smem-wide is only used
    // when asked for.
    const size_t smem_wide = (size_t)2 * n * p.ld * 16 + vec_area_bytes(n);
    const bool cta_ok = n <= kCtaMaxN && cta_smem_bytes(n) <= (size_t)optin;
    const bool wide_ok = smem_wide <= (size_t)optin && n <= kWideNmax;
    p.mixed = mixed;
    if (asked && ((want == "smem-cta" && (mixed || !cta_ok)) || (want == "smem-wide" && (mixed || !wide_ok)))) {
        *err = "regime " + want + " cannot hold n=" + std::to_string(n) + (mixed ? " in the mixed form" : "");
        return false;
    }
    // SUNNY_GENEIG_MIXED_REFINE_MAX caps the mixed form's refinement steps
    // (0..32); pencils that have not converged by then are solved in FP64.
    if (const char* rm = std::getenv("SUNNY_GENEIG_MIXED_REFINE_MAX")) {
        const int v = std::atoi(rm);
        p.refine_max = v < 0 ? 0 : v > 32 ? 32 : v;
    }
    if (!mixed && cta_ok && ((want.empty() && n <= kCtaPreferredMaxN) || want == "smem-cta")) {
        p.regime = Regime::SmemCta;
        p.nmax = cta_nmax_for(n);
        const int want_teams = pencils_per_cta > 0 ? pencils_per_cta : cta_default_teams(p.nmax);
        int teams = 1;
        while (teams * 2 <= want_teams && teams * 2 <= cta_max_teams(p.nmax) &&
               cta_teams_smem_bytes(n, teams * 2) <= (size_t)optin)
            teams *= 2;
        p.teams = teams;
        p.smem = cta_teams_smem_bytes(n, teams);
        p.threads = teams * cta_threads_for(p.nmax);
        e = cta_set_attributes(p.nmax, (size_t)optin);
    } else if (!mixed && wide_ok && want == "smem-wide") {
        p.regime = Regime::SmemWide;
        p.smem = smem_wide;
        p.nmax = kWideNmax;
        e = cudaFuncSetAttribute(geneig_plain_kernel<kWideNmax>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    } else {
        p.regime = Regime::L2Slot;
        p.smem = tiled_vec_bytes(n);
        // resident CTAs (and scratch slots) per SM: SUNNY_GENEIG_SLOTS_PER_SM
        // = 1 or 2 (default 2, the kernel's occupancy limit)
        int per_sm = 2;
        if (slots_per_sm != 0) per_sm = slots_per_sm;
        else if (const char* ps = std::getenv("SUNNY_GENEIG_SLOTS_PER_SM")) per_sm = std::atoi(ps) == 1 ? 1 : 2;
        p.slots = per_sm * sms;
        p.scratch_bytes = (size_t)p.slots * tiled_slot_bytes(n, mixed);
        e = tiled_set_attributes((size_t)optin);
    }
    if (e != cudaSuccess) { *err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e); return false; }
    *plan = p;
    return true;
}

cudaError_t plain_launch(const PlainPlan& plan, int stage, const void* H, const void* S, double* W,
                         void* U, int* info, long long batch, void* scratch, cudaStream_t stream, bool sigma) {
    if (batch <= 0) return cudaSuccess;
    PlainArgs a;
    a.H = static_cast<const double2*>(H);
    a.S = static_cast<const double2*>(S);
    a.W = W;
    a.U = static_cast<double2*>(U);
    a.info = info;
    a.scratch = static_cast<double2*>(scratch);
    a.batch = batch;
    a.n = plan.n;
    a.ld = plan.ld;
    a.stage = stage;
    a.sigma = sigma ? 1 : 0;
    if (plan.regime == Regime::SmemCta)
        return cta_launch(plan.n, plan.nmax, plan.smem, stage, H, S, W, U, info, batch, stream, sigma, plan.teams);
    if (plan.regime == Regime::L2Slot)
        return tiled_launch(plan.n, plan.slots, plan.smem, stage, H, S, W, U, info, batch, scratch, stream, sigma,
                            plan.mixed, plan.refine_max);
    const long long grid = batch < 0x7fffffffLL ? batch : 0x7fffffffLL;
    geneig_plain_kernel<kWideNmax><<<(unsigned)grid, kNT, plan.smem, stream>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free entry point (no counterpart in the reference).
//
// Callers that cannot allocate device memory -- code running inside another
// framework's memory pool or under a strict no-allocation policy, plugins
// whose host forbids cudaMalloc on its streams, and graph-replay setups that
// must not touch the allocator -- get, for n up to the smem-cta limit, the
// shared-memory kernel, which needs no scratch at all, and above it the
// L2-slot kernel with its per-CTA scratch slots taken from the fixed array
// below instead of a cudaMalloc'd buffer. The array is sized once
// (kNoAllocScratchBytes) and every GPU that loads the library keeps it for
// the life of the process. It holds floor(32 MiB / slot) slots, so the
// number of resident CTAs, and with it the throughput, falls with n: 161
// CTAs at n = 61, 12 at n = 216, 2 at n = 512 (the regular launch keeps
// 2 per SM, 296 on B200).
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;   // 32 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocDevice {
    bool ready = false;
    void* scratch = nullptr;   // device address of g_noalloc_scratch on this device
    int sms = 0;
    int optin = 0;             // largest dynamic shared memory per CTA
};
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// Once per device, with that device current: resolve the array's device
// address (the host-side symbol is only a stand-in and must never be handed
// to a kernel) and set the kernels' shared-memory limits.
cudaError_t noalloc_setup(int dev, NoAllocDevice** out, std::string* err) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) { *err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return e; }
        e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) { *err = std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e); return e; }
        int optin = 0;
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) { *err = std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e); return e; }
        e = tiled_set_attributes((size_t)optin);
        for (int nmax : {16, 24, 32, 40, 48, 56, 64})
            if (e == cudaSuccess) e = cta_set_attributes(nmax, (size_t)optin);
        if (e != cudaSuccess) { *err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e); return e; }
        d.optin = optin;
        d.scratch = ptr;
        d.ready = true;
    }
    *out = &d;
    return cudaSuccess;
}

}  // namespace
}  // namespace sgeig

#pragma GCC visibility push(default)
extern "C" sunny_geneig_status_t sunny_geneig_launch_noalloc(int n, uintptr_t d_H, uintptr_t d_S, uintptr_t d_W,
                                                             uintptr_t d_U, uintptr_t d_info, int batch_size,
                                                             uintptr_t stream) {
    using namespace sgeig;
    api_clear_error();
    const size_t slot = (n >= 1 && n <= kMaxN) ? tiled_slot_bytes(n) : 0;
    if (n < 1 || n > kMaxN || slot > kNoAllocScratchBytes) {
        api_set_error("sunny_geneig_launch_noalloc: n=" + std::to_string(n) + " outside [1, " +
                      std::to_string(kMaxN) + "] (the static scratch holds " +
                      std::to_string(kNoAllocScratchBytes >> 20) + " MiB)");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (batch_size < 0) { api_set_error("sunny_geneig_launch_noalloc: batch_size < 0"); return SUNNY_GENEIG_INVALID_ARG; }
    if (batch_size == 0) return SUNNY_GENEIG_OK;
    if (!d_H || !d_S || !d_W || !d_U || !d_info) {
        api_set_error("sunny_geneig_launch_noalloc: NULL device buffer");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (d_H % 16 || d_S % 16 || d_U % 16 || d_W % 8 || d_info % 4) {
        api_set_error("sunny_geneig_launch_noalloc: misaligned device buffer (H, S, U need 16 B; W 8 B; info 4 B)");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        api_set_error(std::string("sunny_geneig_launch_noalloc: no usable current device: ") + cudaGetErrorString(e));
        return SUNNY_GENEIG_DEVICE_ERROR;
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        api_set_error("sunny_geneig_launch_noalloc: current device index " + std::to_string(dev) +
                      " is beyond this entry point's limit of " + std::to_string(kNoAllocMaxDevices) + " devices");
        return SUNNY_GENEIG_DEVICE_ERROR;
    }
    NoAllocDevice* d = nullptr;
    std::string err;
    if (noalloc_setup(dev, &d, &err) != cudaSuccess) {
        api_set_error("sunny_geneig_launch_noalloc: " + err);
        return SUNNY_GENEIG_DEVICE_ERROR;
    }
    if (n <= kCtaPreferredMaxN && cta_smem_bytes(n) <= (size_t)d->optin) {
        // the shared-memory kernel keeps everything on chip: no scratch at all
        const int nmax = cta_nmax_for(n), teams = cta_default_teams(nmax);
        e = cta_launch(n, nmax, cta_teams_smem_bytes(n, teams), 4, reinterpret_cast<const void*>(d_H),
                       reinterpret_cast<const void*>(d_S), reinterpret_cast<double*>(d_W),
                       reinterpret_cast<void*>(d_U), reinterpret_cast<int*>(d_info), batch_size,
                       reinterpret_cast<cudaStream_t>(stream), false, teams);
        if (e != cudaSuccess) {
            api_set_error(std::string("sunny_geneig_launch_noalloc: kernel launch failed: ") + cudaGetErrorString(e));
            return SUNNY_GENEIG_LAUNCH_ERROR;
        }
        return SUNNY_GENEIG_OK;
    }
    const long long fit = (long long)(kNoAllocScratchBytes / slot);
    const int slots = (int)(fit < 2LL * d->sms ? fit : 2LL * d->sms);
    e = tiled_launch(n, slots, tiled_vec_bytes(n), 4, reinterpret_cast<const void*>(d_H),
                     reinterpret_cast<const void*>(d_S), reinterpret_cast<double*>(d_W), reinterpret_cast<void*>(d_U),
                     reinterpret_cast<int*>(d_info), batch_size, d->scratch, reinterpret_cast<cudaStream_t>(stream),
                     false);
    if (e != cudaSuccess) {
        api_set_error(std::string("sunny_geneig_launch_noalloc: kernel launch failed: ") + cudaGetErrorString(e));
        return SUNNY_GENEIG_LAUNCH_ERROR;
    }
    return SUNNY_GENEIG_OK;
}
#pragma GCC visibility pop
