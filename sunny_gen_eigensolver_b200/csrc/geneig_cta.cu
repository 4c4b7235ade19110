// Batched generalized Hermitian-definite eigensolver, shared-memory regime
// (N <= 64): a team of NT threads (64 to 256 by N) holds one matrix pair in
// shared memory and solves it end to end; a CTA is one team or, with
// several pencils per CTA, up to four, each with its own named barrier and
// shared-memory slice; CTAs loop over the batch. A second kernel form
// assembles S(q) from Fourier terms in the load stage (the metric solve of
// a spin-wave dynamical matrix that never exists in memory).
//
// Stage chain (reference: src/unified/kernel_source.hpp:233-276):
//   a1  load S -> A, H -> B                                   (:233-242)
//   a2  Cholesky S = L L^H fused with X = L^-1: each row lives in the
//       registers of a four-lane group, one barrier per column   (:244)
//   a3+a4  C = L^-1 H L^-H as two complex GEMMs on the FP64 tensor cores
//       (mma.m8n8k4.f64): T = H X^H, then C = X T (lower tiles, mirrored);
//       H is read in full, as the reference's two triangular solves do (:246-248)
//   a5  Householder tridiagonalisation (lower, look-ahead reflector, two
//       barriers per step), divide and conquer on the tridiagonal,
//       back-transform V = Q Z in compact-WY blocks of 16 reflectors on the
//       FP64 tensor cores, one 8-column panel of V per warp          (:250)
//   a6  U = L^-H V = X^H V on the FP64 tensor cores            (:252)
//   a7  W (ascending) and U, columns permuted by eigenvalue rank (:268-276)
//
// Thread layouts (NT threads): groups of four lanes (g = tid / 4, q = tid % 4)
// owning one row or one column for the Cholesky/inverse and the Householder
// updates; warps owning 8x8 output tiles or 8-column panels for the
// tensor-core GEMMs; an NT/16 x 16 grid (tr, tc) for the copies.
//
// A variant that kept C in registers for the Householder steps (16 x 16
// thread grid, rank-2 updates in registers) was measured slower on B200 at
// N = 24 and 54 (80 K vs 75 K and 365 K vs 229 K cycles per solve): the
// per-warp redundant reflector arithmetic and whole-block predicated
// updates cost more issue slots than the shared-memory traffic they saved.

#include "geneig_cta_body.cuh"

namespace sgeig {
using namespace cta;
namespace {

// Threads per pencil (one pencil per CTA) and CTAs per SM that the register
// allocation is sized for, by row bound (at least 4 NMAX threads: the
// Cholesky gives each row a four-lane group). Small pencils run on narrow
// CTAs, several resident per SM: their steps are latency chains (a barrier
// per Cholesky column, two per Householder step), so more pencils in flight
// raise throughput more than more threads per pencil. Measured on B200
// (solves/s at batch 65,536, against 256 threads and 2-3 CTAs/SM):
//   NMAX 16: 64 x 8   N=16 9.09 M (3.80 M); 64 x 16 (spills) 7.36 M
//   NMAX 24: 128 x 4  N=24 4.45 M (2.42 M); 96 x 4 4.39 M, 128 x 6 2.85 M
//   NMAX 32: 128 x 4  N=32 2.26 M (1.96 M); 128 x 5 2.09 M
//   NMAX 40: 256 x 3  N=40 1.36 M; 160 x 3 1.31 M, 192 x 3 1.34 M
//   NMAX 48: 192 x 2  N=44 1.16 M (1.08 M); N=48 0.97 M either way
//   NMAX 56: 256 x 2  N=54 832 K; 224 x 2 748 K
template <int NMAX> struct CtaShape { static constexpr int nt = kNT, minb = 2; };
template <> struct CtaShape<16> { static constexpr int nt = 64, minb = 8; };
template <> struct CtaShape<24> { static constexpr int nt = 128, minb = 4; };
template <> struct CtaShape<32> { static constexpr int nt = 128, minb = 4; };
template <> struct CtaShape<40> { static constexpr int nt = kNT, minb = 3; };
template <> struct CtaShape<48> { static constexpr int nt = 192, minb = 2; };

// TEAMS pencils per CTA at a time (the reference's batches per block): the
// CTA has TEAMS teams of CtaShape<NMAX>::nt threads, each with its own
// barrier and shared-memory slice, team t taking pencils TEAMS * cta + t,
// then a grid's stride on. TEAMS = 1 is the default launch.
template <int NMAX, int TEAMS>
__global__ void __launch_bounds__(CtaShape<NMAX>::nt * TEAMS, (CtaShape<NMAX>::minb + TEAMS - 1) / TEAMS)
geneig_cta_kernel(CtaArgs a) {
    constexpr int NT = CtaShape<NMAX>::nt;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    phase_start();
    if constexpr (TEAMS == 1) {
        for (long long b = blockIdx.x; b < a.batch; b += gridDim.x) cta_solve<NMAX, NT, NT>(a, b, smem_raw);
    } else {
        const int t = (int)(threadIdx.x / NT);
        unsigned char* sm = smem_raw + (size_t)t * cta_team_bytes(a.n);
        for (long long b = (long long)blockIdx.x * TEAMS + t; b < a.batch; b += (long long)gridDim.x * TEAMS)
            cta_solve<NMAX, NT, NT * TEAMS>(a, b, sm);
    }
}

// S assembled on the device from Fourier terms (one pencil per CTA).
template <int NMAX>
__global__ void __launch_bounds__(CtaShape<NMAX>::nt, CtaShape<NMAX>::minb)
geneig_cta_fourier_kernel(CtaArgs a, CtaFourier f) {
    constexpr int NT = CtaShape<NMAX>::nt;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    phase_start();
    for (long long b = blockIdx.x; b < a.batch; b += gridDim.x) cta_solve<NMAX, NT, NT, true>(a, b, smem_raw, &f);
}

}  // namespace

size_t cta_smem_bytes(int n) { return (size_t)2 * n * (n | 1) * 16 + cta_vec_bytes(n); }

// Compile-time row bounds: the register arrays and unrolled loops are sized by
// NMAX, so a bound close above n wastes less (56 covers the N=54 workload).
int cta_nmax_for(int n) {
    return n <= 16 ? 16 : n <= 24 ? 24 : n <= 32 ? 32 : n <= 40 ? 40 : n <= 48 ? 48 : n <= 56 ? 56 : 64;
}

using CtaKernelFn = void (*)(CtaArgs);
static CtaKernelFn cta_kernel_for(int nmax, int teams) {
    switch (nmax) {
        case 16: return teams == 4 ? geneig_cta_kernel<16, 4> : teams == 2 ? geneig_cta_kernel<16, 2>
                                                                          : geneig_cta_kernel<16, 1>;
        case 24: return teams == 2 ? geneig_cta_kernel<24, 2> : geneig_cta_kernel<24, 1>;
        case 32: return teams == 2 ? geneig_cta_kernel<32, 2> : geneig_cta_kernel<32, 1>;
        case 40: return geneig_cta_kernel<40, 1>;
        case 48: return geneig_cta_kernel<48, 1>;
        case 56: return geneig_cta_kernel<56, 1>;
        default: return geneig_cta_kernel<64, 1>;
    }
}

// The assembled-S (Fourier) form, one pencil per CTA.
using CtaFourierKernelFn = void (*)(CtaArgs, CtaFourier);
static CtaFourierKernelFn cta_fourier_kernel_for(int nmax) {
    switch (nmax) {
        case 16: return geneig_cta_fourier_kernel<16>;
        case 24: return geneig_cta_fourier_kernel<24>;
        case 32: return geneig_cta_fourier_kernel<32>;
        case 40: return geneig_cta_fourier_kernel<40>;
        case 48: return geneig_cta_fourier_kernel<48>;
        case 56: return geneig_cta_fourier_kernel<56>;
        default: return geneig_cta_fourier_kernel<64>;
    }
}

int cta_max_teams(int nmax) { return nmax <= 16 ? 4 : nmax <= 32 ? 2 : 1; }

// Default pencils per CTA, measured on B200 (solves/s at batch 65,536, one
// pencil per CTA -> default): N=12 12.4 M -> 14.4 M, N=16 9.3 M -> 11.9 M
// (4 teams of 64); N=32 2.2 M -> 3.0 M (2 of 128); N=24 stays at one
// (4.4 M; 3.95 M with 2 teams). Two teams of the 48- and 56-row kernels
// (384- and 512-thread CTAs, one per SM) were not kept: N=44 1.14 M vs
// 1.16 M, N=48 1.05 M vs 0.98 M, N=54 810 K vs 836 K.
int cta_default_teams(int nmax) { return nmax <= 16 ? 4 : nmax == 32 ? 2 : 1; }

size_t cta_teams_smem_bytes(int n, int teams) { return teams <= 1 ? cta_smem_bytes(n) : teams * cta_team_bytes(n); }

int cta_threads_for(int nmax) {
    switch (nmax) {
        case 16: return CtaShape<16>::nt;
        case 24: return CtaShape<24>::nt;
        case 32: return CtaShape<32>::nt;
        case 40: return CtaShape<40>::nt;
        case 48: return CtaShape<48>::nt;
        case 56: return CtaShape<56>::nt;
        default: return CtaShape<64>::nt;
    }
}

// `smem` is the per-CTA shared-memory limit; the kernel's own static shared
// memory (profiling builds have some) comes off the dynamic allowance.
cudaError_t cta_set_attributes(int nmax, size_t smem) {
    {
        cudaFuncAttributes fa{};
        cudaError_t e = cudaFuncGetAttributes(&fa, cta_fourier_kernel_for(nmax));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(cta_fourier_kernel_for(nmax), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(smem - fa.sharedSizeBytes));
        if (e != cudaSuccess) return e;
    }
    for (int teams = 1; teams <= cta_max_teams(nmax); teams *= 2) {
        cudaFuncAttributes fa{};
        cudaError_t e = cudaFuncGetAttributes(&fa, cta_kernel_for(nmax, teams));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(cta_kernel_for(nmax, teams), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(smem - fa.sharedSizeBytes));
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t cta_launch(int n, int nmax, size_t smem, int stage, const void* H, const void* S, double* W, void* U,
                       int* info, long long batch, cudaStream_t stream, bool sigma, int teams) {
    CtaArgs a{};
    a.H = static_cast<const double2*>(H);
    a.S = static_cast<const double2*>(S);
    a.W = W;
    a.U = static_cast<double2*>(U);
    a.info = info;
    a.batch = batch;
    a.n = n;
    a.ld = n | 1;
    a.stage = stage;
    a.sigma = sigma ? 1 : 0;
    a.O = nullptr;
    a.qhat = a.energies = nullptr;
    a.spec = nullptr;
    a.ne = 0;
    a.gnorm = a.ginv2 = 0.0;
    const long long ctas = (batch + teams - 1) / teams;
    const long long grid = ctas < 0x7fffffffLL ? ctas : 0x7fffffffLL;
    cta_kernel_for(nmax, teams)<<<(unsigned)grid, teams * cta_threads_for(nmax), smem, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t cta_launch_intensity(int n, int nmax, size_t smem, const void* S, const void* O, const double* qhat,
                                 const double* energies, int ne, double fwhm, double* W, double* spec, int* info,
                                 long long batch, cudaStream_t stream, int teams) {
    CtaArgs a{};
    a.H = nullptr;
    a.S = static_cast<const double2*>(S);
    a.W = W;
    a.U = nullptr;
    a.info = info;
    a.batch = batch;
    a.n = n;
    a.ld = n | 1;
    a.stage = kStageIntensity;
    a.sigma = 1;
    a.O = static_cast<const double2*>(O);
    a.qhat = qhat;
    a.energies = energies;
    a.spec = spec;
    a.ne = ne;
    const double sigma_e = fwhm / (2.0 * std::sqrt(2.0 * std::log(2.0)));
    a.gnorm = 1.0 / (sigma_e * std::sqrt(2.0 * M_PI));
    a.ginv2 = 1.0 / (2.0 * sigma_e * sigma_e);
    const long long ctas = (batch + teams - 1) / teams;
    const long long grid = ctas < 0x7fffffffLL ? ctas : 0x7fffffffLL;
    cta_kernel_for(nmax, teams)<<<(unsigned)grid, teams * cta_threads_for(nmax), smem, stream>>>(a);
    return cudaGetLastError();
}


cudaError_t cta_launch_fourier(int n, int nmax, const FourierTerms& ft, const double* q,
                               const void* O, const double* qhat, const double* energies, int ne, double fwhm,
                               double* W, void* U, double* spec, int* info, long long batch, cudaStream_t stream) {
    CtaArgs a{};
    a.W = W;
    a.U = static_cast<double2*>(U);
    a.info = info;
    a.batch = batch;
    a.n = n;
    a.ld = n | 1;
    a.sigma = 1;
    CtaFourier f{};
    f.start = ft.start;
    f.coef = static_cast<const double2*>(ft.coef);
    f.disp = ft.disp;
    f.q = q;
    f.nterms = ft.nterms;
    if (O) {
        a.stage = kStageIntensity;
        a.O = static_cast<const double2*>(O);
        a.qhat = qhat;
        a.energies = energies;
        a.spec = spec;
        a.ne = ne;
        const double sigma_e = fwhm / (2.0 * std::sqrt(2.0 * std::log(2.0)));
        a.gnorm = 1.0 / (sigma_e * std::sqrt(2.0 * M_PI));
        a.ginv2 = 1.0 / (2.0 * sigma_e * sigma_e);
    } else {
        a.stage = 4;
    }
    const long long grid = batch < 0x7fffffffLL ? batch : 0x7fffffffLL;
    cta_fourier_kernel_for(nmax)<<<(unsigned)grid, cta_threads_for(nmax), cta_smem_bytes(n), stream>>>(a, f);
    return cudaGetLastError();
}

}  // namespace sgeig

#ifdef SGEIG_PHASE_TIMERS
// Profiling builds only: copies the per-phase cycle counters of the
// smem-cta kernel (see phase_mark in geneig_common.cuh) to `out` and, when
// `reset` is nonzero, clears them. Not part of the product library's ABI.
#pragma GCC visibility push(default)
extern "C" int sunny_geneig_phase_cycles(unsigned long long* out, int count, int reset) {
    if (count > sgeig::kPhaseSlots) count = sgeig::kPhaseSlots;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && out && count > 0)
        e = cudaMemcpyFromSymbol(out, sgeig::g_phase_cycles, sizeof(unsigned long long) * count);
    if (e == cudaSuccess && reset) {
        static const unsigned long long zeros[sgeig::kPhaseSlots] = {};
        e = cudaMemcpyToSymbol(sgeig::g_phase_cycles, zeros, sizeof(zeros));
    }
    if (e == cudaSuccess && out && count > 0) e = sgeig::tiled_phase_cycles(out, count, reset != 0);
    return e == cudaSuccess ? 0 : -1;
}
#pragma GCC visibility pop
#endif

