// Tiled FP64 batched generalized Hermitian-definite eigensolver for sm_100a,
// for matrices too large to keep in one CTA's shared memory (the "l2-slot"
// regime). One CTA solves one pencil at a time, persistent over the batch;
// its working matrices live in a per-CTA global-memory slot
//     M0, M1, M2: n x ld complex,  Zo: n x ld real (at least 16 n complex)
// and every O(n^3) step except the Householder matrix-vector products is a complex GEMM
// on the FP64 tensor cores (mma.sync.m8n8k4.f64; a complex 8x8x4 step is four
// real MMAs), one 16 x 16 output tile per warp at a time:
//
//   a1  M0 <- S (lower triangle)                      (kernel_source.hpp:233-242)
//   a2  blocked Cholesky S = L L^H in M0: 16-column panels factored column
//       by column, trailing lower tiles updated as C -= L_p L_p^H   (:244)
//   a3  X = L^-1 in M1, one 16-row block at a time: R = L_rk X_kc (GEMM),
//       X_r = L_rr^-1 (e_r - R) (one thread per column)            (:246)
//   a4  T = H X^H in M2, C = X T in M0 (lower tiles, mirrored), so that
//       C = L^-1 H L^-H; for the spin-wave metric H = diag(I, -I) the first
//       product is a sign flip of X^H                              (:248)
//   a5  C = Q T Q^H (Householder, lower; v_k kept in column k of M0 below
//       the subdiagonal; for n >= 96 in 16-column panels whose trailing
//       update A -= V W^H + W V^H is a GEMM), T = Z diag(w) Z^T by divide and conquer (Z and its
//       merge workspace in M2, merge products through Zo), V = Q Z with
//       compact-WY blocks of 16 reflectors, Q_b = I - Y T_b Y^H:
//       W1 = Y^H V, W2 = T_b W1, V -= Y W2 (all GEMMs), V in the output U   (:250)
//   a6  U = X^H V into M2, copied to the output                   (:252)
//   a7  W ascending, U columns in the same order                  (:268-276)
//
// Stage-wise outputs (stage 1: L, 2: C, 3: W and V) follow the reference's
// static kernels in src/geneig_fixed.cu.
//
// Mixed-precision form (kernel mode MIXED): the Householder reduction runs in
// FP32 on a single-precision copy of C (reflectors stored in FP32); divide
// and conquer, the back-transform and everything else stay FP64; then
// Ogita-Aishima refinement steps (FP64 tensor-core GEMMs against the FP64 C,
// repeated until the correction is negligible) recover FP64 eigenpairs of C
// before U = X^H V.

#include "geneig_tiled_body.cuh"
#include "sunny_geneig.h"

namespace sgeig {
using namespace tiled;
namespace {

__global__ void __launch_bounds__(kNT, 2) geneig_tiled_kernel(TiledArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* slot = a.scratch + (size_t)blockIdx.x * tiled_slot_elems(a.n, a.mixed != 0);
    phase_start();
    for (long long b = blockIdx.x; b < a.batch; b += gridDim.x) tiled_solve(a, b, slot, smem_raw);
}

}  // namespace

size_t tiled_vec_bytes(int n) {
    return (size_t)n * 16 * 3 + 32 * 16 + 3 * 256 * 16 + tiled_part_elems(n) * 16 + (size_t)n * 8 * 3 +
           (size_t)dc_vec_doubles(n) * 8 + (size_t)n * 4 + 8 * 4 + (size_t)dc_vec_ints(n) * 4;
}

// `smem` is the per-CTA shared-memory limit; the kernel's own static shared
// memory (profiling builds have some) comes off the dynamic allowance.
cudaError_t tiled_set_attributes(size_t smem) {
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, geneig_tiled_kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(geneig_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(smem - fa.sharedSizeBytes));
}

cudaError_t tiled_launch(int n, int slots, size_t smem, int stage, const void* H, const void* S, double* W, void* U,
                         int* info, long long batch, void* scratch, cudaStream_t stream, bool sigma, bool mixed,
                         int refine_max) {
    if (batch <= 0) return cudaSuccess;
    TiledArgs a;
    a.H = static_cast<const double2*>(H);
    a.S = static_cast<const double2*>(S);
    a.W = W;
    a.U = static_cast<double2*>(U);
    a.info = info;
    a.scratch = static_cast<double2*>(scratch);
    a.batch = batch;
    a.n = n;
    a.ld = n | 1;
    a.stage = stage;
    a.sigma = sigma ? 1 : 0;
    a.mixed = mixed ? 1 : 0;
    a.refine_max = refine_max;
    const long long grid = batch < slots ? batch : slots;
    geneig_tiled_kernel<<<(unsigned)grid, kNT, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace sgeig

#ifdef SGEIG_PHASE_TIMERS
namespace sgeig {
// Profiling builds only: this translation unit's phase counters (the tiled
// kernel's marks), added into `out` by sunny_geneig_phase_cycles.
cudaError_t tiled_phase_cycles(unsigned long long* out, int count, bool reset) {
    unsigned long long mine[kPhaseSlots] = {};
    cudaError_t e = cudaMemcpyFromSymbol(mine, g_phase_cycles, sizeof(mine));
    for (int i = 0; e == cudaSuccess && i < count && i < kPhaseSlots; ++i) out[i] += mine[i];
    if (e == cudaSuccess && reset) {
        static const unsigned long long zeros[kPhaseSlots] = {};
        e = cudaMemcpyToSymbol(g_phase_cycles, zeros, sizeof(zeros));
    }
    return e;
}
}  // namespace sgeig
#endif

