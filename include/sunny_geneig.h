/*
 * sunny_geneig.h -- C ABI of libsunny_geneig.so, the B200 (sm_100a) batched
 * complex Hermitian-definite generalized eigensolver  H u = lambda S u.
 *
 * Drop-in for the reference's src/common/c_api.h: every type, enum value and
 * function signature below that carries a "replaces" note has the same name,
 * argument meaning and error behaviour as the reference entry point it names.
 * Entry points marked "extension" have no counterpart in the reference.
 *
 * Buffers (all device pointers passed as uintptr_t, caller-owned):
 *   d_H, d_S : complex128, column-major N x N per matrix, batch-contiguous
 *              (element (i,j) of matrix b at b*N*N + j*N + i). Read only.
 *              H is read in full (both triangles); S only in its lower triangle.
 *   d_W      : float64 N x batch; ascending eigenvalues of matrix b at b*N.
 *   d_U      : complex128 N x N x batch; column k of matrix b is the eigenvector
 *              for W[b*N + k], normalised so that U^H S U = I.
 *   d_info   : int32[batch]; 0 on success; N + k when the leading minor of
 *              order k of S is not positive definite (LAPACK zhegv convention;
 *              a NaN pivot counts as not positive definite, as in reference
 *              LAPACK's zpotrf); N - 1 when the tridiagonal eigensolve fails on
 *              non-finite values (zhegv's count of unconverged off-diagonals;
 *              0 for N <= 2, as zhegv). W and U of a failed matrix are NaN.
 * Launches are asynchronous on `stream` (0 = legacy default stream); the
 * library never synchronises the host inside a launch.
 * Alignment: d_H, d_S, d_U 16-byte, d_W 8-byte, d_info 4-byte aligned.
 */
#ifndef SUNNY_GENEIG_H
#define SUNNY_GENEIG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* replaces src/common/c_api.h:22 (opaque handle) */
typedef struct sunny_geneig_solver* sunny_geneig_solver_t;

/* replaces src/common/c_api.h:24-30 */
typedef enum {
    SUNNY_GENEIG_OK            =  0,
    SUNNY_GENEIG_INVALID_ARG   = -1,
    SUNNY_GENEIG_DEVICE_ERROR  = -2,
    SUNNY_GENEIG_COMPILE_ERROR = -3,
    SUNNY_GENEIG_LAUNCH_ERROR  = -4
} sunny_geneig_status_t;

/* replaces src/common/c_api.h:32-36. Kernels here are compiled ahead of
 * time, so the cache holds the autotuner's choices only (see
 * SUNNY_GENEIG_TUNING_AUTOTUNE): AUTO keeps them in the process and in the
 * table tune_v1.tsv under $SUNNY_GENEIG_CACHE_DIR (else
 * $XDG_CACHE_HOME/sunny_geneig, $HOME/.cache/sunny_geneig,
 * /tmp/sunny_geneig), NODISK in the process only, NOCACHE nowhere. */
typedef enum {
    SUNNY_GENEIG_CACHE_AUTO    = 0,
    SUNNY_GENEIG_CACHE_NODISK  = 1,
    SUNNY_GENEIG_CACHE_NOCACHE = 2
} sunny_geneig_cache_mode_t;

/* replaces src/common/c_api.h:38-41. SUGGESTED: the execution
 * configuration is chosen by N from measured crossovers. AUTOTUNE: create
 * times every configuration that can hold N (smem-cta, smem-wide, l2-slot
 * with 1 or 2 CTAs per SM) on a seeded synthetic batch on the device and
 * keeps the fastest (cached per N, kernel mode, device and library build
 * as the cache mode says); the mixed form has a single configuration. */
typedef enum {
    SUNNY_GENEIG_TUNING_SUGGESTED = 0,
    SUNNY_GENEIG_TUNING_AUTOTUNE  = 1
} sunny_geneig_tuning_mode_t;

/* replaces src/common/c_api.h:43-46. UNIFIED and HYBRID both select the
 * plain FP64 sm_100a kernel (no cuSolverDx / cuSOLVER / cuBLAS here).
 * MIXED is an extension: FP32 tridiagonal stage plus FP64 refinement. */
typedef enum {
    SUNNY_GENEIG_KERNEL_UNIFIED = 0,
    SUNNY_GENEIG_KERNEL_HYBRID  = 1,
    SUNNY_GENEIG_KERNEL_MIXED   = 2
} sunny_geneig_kernel_mode_t;

/* replaces src/common/c_api.h:50-55 (impl c_api.cpp:76-107).
 * Returns NULL on failure (message in sunny_geneig_last_error()).
 * batches_per_block_request: matrix pairs one CTA solves at a time. 0:
 * automatic (4 for N <= 16, 2 for N = 25..32, else 1: the fastest measured
 * on B200). 1: one per CTA. 2 or more: 2 for N <= 32, 4 for N <= 16 (the
 * largest form at or below the request that the shared-memory kernel has;
 * 1 otherwise and in the global-memory regime).
 * sunny_geneig_batches_per_block reports the choice. */
sunny_geneig_solver_t sunny_geneig_create(
    int                         n,
    int                         device_id,
    int                         batches_per_block_request,
    sunny_geneig_tuning_mode_t  tuning_mode,
    sunny_geneig_cache_mode_t   cache_mode);

/* replaces src/common/c_api.h:63-69 (impl c_api.cpp:109-137) */
sunny_geneig_solver_t sunny_geneig_create_ex(
    int                         n,
    int                         device_id,
    int                         batches_per_block_request,
    sunny_geneig_tuning_mode_t  tuning_mode,
    sunny_geneig_cache_mode_t   cache_mode,
    sunny_geneig_kernel_mode_t  kernel_mode);

/* replaces src/common/c_api.h:72 (impl c_api.cpp:139-145). NULL is a no-op. */
void sunny_geneig_destroy(sunny_geneig_solver_t solver);

/* replaces src/common/c_api.h:77-85 (impl c_api.cpp:147-186).
 * INVALID_ARG for a NULL solver, batch_size < 0, a NULL or misaligned
 * buffer with batch_size > 0; batch_size == 0 is a no-op returning OK;
 * LAUNCH_ERROR when the CUDA launch itself fails. One handle may be used
 * from several streams: for sizes whose solver keeps scratch slots (the
 * "l2-slot" regime) a launch on a different stream than the previous one
 * waits for it on the device, so launches of one such handle never overlap.
 * That ordering covers normal launches only: a launch captured into a CUDA
 * graph uses the same scratch slots when the graph is replayed, so the
 * caller must order each replay against other launches and replays of the
 * same handle (same stream, or an event recorded after one and waited for
 * before the other); inside one graph, capture each such handle's launches
 * on one stream. smem-cta handles keep no scratch and need none of this. */
sunny_geneig_status_t sunny_geneig_launch(
    sunny_geneig_solver_t solver,
    uintptr_t             d_H,
    uintptr_t             d_S,
    uintptr_t             d_W,
    uintptr_t             d_U,
    uintptr_t             d_info,
    int                   batch_size,
    uintptr_t             stream);

/* replace src/common/c_api.h:88-91 (impl c_api.cpp:188-208).
 * -1 (0 for shared_mem_bytes) when solver is NULL. */
int          sunny_geneig_matrix_size      (sunny_geneig_solver_t solver);
int          sunny_geneig_batches_per_block(sunny_geneig_solver_t solver);
int          sunny_geneig_block_dim_x      (sunny_geneig_solver_t solver);
unsigned int sunny_geneig_shared_mem_bytes (sunny_geneig_solver_t solver);

/* replaces src/common/c_api.h:95 (impl c_api.cpp:210-212). Thread-local,
 * never NULL, "" when no error was recorded on the calling thread. */
const char*  sunny_geneig_last_error(void);

/* replace src/common/c_api.h:100-101 (impl c_api.cpp:214-220).
 * path_name: "unified", "hybrid" or "mixed" ("" for NULL). */
const char*                sunny_geneig_path_name  (sunny_geneig_solver_t solver);
sunny_geneig_kernel_mode_t sunny_geneig_kernel_mode(sunny_geneig_solver_t solver);

/* ---- extensions (no counterpart in the reference's C ABI) ---------------- */

/* Stage-wise launch for parity tests; the stages follow the reference's
 * static kernels in src/geneig_fixed.cu:
 *   stage 1: Cholesky only (chol_n54_kernel :106-132). U <- L (lower, upper
 *            triangle zero). W untouched.
 *   stage 2: reduction (geneig_reduce_n54_kernel :166-206). U <- C =
 *            L^-1 H L^-H, full Hermitian matrix.
 *   stage 3: reduction + eigensolve (geneig_reduce_eig_n54_kernel :247-300).
 *            W <- ascending eigenvalues of C, U <- orthonormal eigenvectors V.
 *   stage 4: the full solve, identical to sunny_geneig_launch. */
sunny_geneig_status_t sunny_geneig_launch_stage(
    sunny_geneig_solver_t solver,
    int                   stage,
    uintptr_t             d_H,
    uintptr_t             d_S,
    uintptr_t             d_W,
    uintptr_t             d_U,
    uintptr_t             d_info,
    int                   batch_size,
    uintptr_t             stream);

/* Spin-wave metric solve (no counterpart in the reference's C ABI): the
 * batch of pencils (Sigma, S) with Sigma = diag(I_{n/2}, -I_{n/2}), the
 * para-unitary metric of linear spin-wave theory, where S is the dynamical
 * matrix (Hermitian positive definite). Sunny calls its generalized solver in
 * this pattern (Sigma u = lambda S u). H is implied and never read, so one
 * matrix per problem less crosses HBM and the step T = H X^H of the
 * reduction becomes a sign flip. n must be even. Same W/U/info layouts,
 * info codes and error behaviour as sunny_geneig_launch. */
sunny_geneig_status_t sunny_geneig_launch_sigma(
    sunny_geneig_solver_t solver,
    uintptr_t             d_S,
    uintptr_t             d_W,
    uintptr_t             d_U,
    uintptr_t             d_info,
    int                   batch_size,
    uintptr_t             stream);

/* Spin-wave intensities (no counterpart in the reference's C ABI; the step
 * Sunny runs after the solve, the reference's benchmarks/sw08_baseline.jl:
 * 99-103): the metric solve of sunny_geneig_launch_sigma, with each problem's
 * eigenvectors reduced on the device to its spectrum on an energy grid, so
 * that U (16 N^2 bytes per problem) never leaves the chip. For the positive
 * eigenvalues lambda_k, t_k = u_k / sqrt(lambda_k) is the Bogoliubov vector
 * of the mode of energy omega_k = 1 / lambda_k; with Y = O t_k,
 *   I_k = sum_ab (delta_ab - qhat_a qhat_b) conj(Y_a) Y_b,
 *   spec[b * n_energies + e] = sum_k I_k g(energies[e] - omega_k),
 * g the normalised Gaussian of full width at half maximum fwhm.
 *   d_O        complex128 3 x N per problem, column-major (element (a, j) of
 *              problem b at b*3N + 3j + a): the one-body observable matrix
 *   d_qhat     float64 3 per problem: unit scattering direction
 *   d_energies float64 n_energies: the energy grid (shared by all problems)
 *   d_W        float64 N per problem: ascending eigenvalues, as for launch
 *   d_spec     float64 n_energies per problem
 * Needs a plain solver in the smem-cta regime (even N <= 64); INVALID_ARG
 * otherwise, for n_energies < 1 or fwhm <= 0. A failed problem gets its info
 * code and NaN W and spec. */
sunny_geneig_status_t sunny_geneig_launch_sigma_intensity(
    sunny_geneig_solver_t solver,
    uintptr_t             d_S,
    uintptr_t             d_O,
    uintptr_t             d_qhat,
    uintptr_t             d_energies,
    int                   n_energies,
    double                fwhm,
    uintptr_t             d_W,
    uintptr_t             d_spec,
    uintptr_t             d_info,
    int                   batch_size,
    uintptr_t             stream);

/* Spin-wave metric solve with the metric-side matrix assembled on the device
 * (Sunny's dynamical_matrix! step, which the reference's caller runs before
 * sunny_geneig_launch: julia/SunnyGeneigBench/scripts/setup_sw08.jl:103),
 * so that S never passes through device memory. For problem b with
 * wavevector q = d_q[3b .. 3b+2] (reciprocal-lattice units), entry
 * e = row + N col of the lower triangle (row >= col) of S is
 *   S(q)_e = sum_{t = start[e]}^{start[e+1]-1} coef[t] exp(2 pi i q . disp[3t .. 3t+2]);
 * upper-triangle entries are not read (S is Hermitian). Then exactly
 * sunny_geneig_launch_sigma: H = diag(I_{N/2}, -I_{N/2}), W, U and info as
 * for sunny_geneig_launch.
 *   d_start   int32 N*N + 1, nondecreasing: entry e's terms are
 *             [start[e], start[e+1]); indices outside [0, n_terms) are never
 *             read (the sum is clipped to that range)
 *   d_coef    complex128 n_terms; d_disp float64 3 per term (lattice units)
 *   d_q       float64 3 per problem
 * Needs a plain solver in the smem-cta regime (even N <= 64); INVALID_ARG
 * otherwise. `sunny_gen_eigensolver_b200.lswt` builds the terms of a linear
 * spin-wave model (sites, spin directions, exchange bonds, fields). */
sunny_geneig_status_t sunny_geneig_launch_fourier_sigma(
    sunny_geneig_solver_t solver,
    uintptr_t             d_start,
    uintptr_t             d_coef,
    uintptr_t             d_disp,
    int                   n_terms,
    uintptr_t             d_q,
    uintptr_t             d_W,
    uintptr_t             d_U,
    uintptr_t             d_info,
    int                   batch_size,
    uintptr_t             stream);

/* The same assembly feeding the intensity form of
 * sunny_geneig_launch_sigma_intensity (W and spec per problem, no U):
 * assembly, solve and S(q, E) in one launch. */
sunny_geneig_status_t sunny_geneig_launch_fourier_sigma_intensity(
    sunny_geneig_solver_t solver,
    uintptr_t             d_start,
    uintptr_t             d_coef,
    uintptr_t             d_disp,
    int                   n_terms,
    uintptr_t             d_q,
    uintptr_t             d_O,
    uintptr_t             d_qhat,
    uintptr_t             d_energies,
    int                   n_energies,
    double                fwhm,
    uintptr_t             d_W,
    uintptr_t             d_spec,
    uintptr_t             d_info,
    int                   batch_size,
    uintptr_t             stream);

/* Create with an explicit execution configuration (no counterpart in the
 * reference; its NVRTC autotuner picked launch shapes inside create).
 * `regime` is "smem-cta", "smem-wide" or "l2-slot" (NULL or "" = the default
 * choice by N); `slots_per_sm` is 1 or 2 resident CTAs per SM for the
 * l2-slot regime (0 = default). A configuration that cannot hold n returns
 * NULL with the reason in sunny_geneig_last_error(). The uneven-batch
 * autotuner times the candidates per N through this call. */
sunny_geneig_solver_t sunny_geneig_create_config(int n, int device_id, sunny_geneig_kernel_mode_t kernel_mode,
                                                 const char* regime, int slots_per_sm);

/* Persistent solver for batches of uneven sizes (no counterpart in the
 * reference's C ABI). One launch solves problems of up to 8 different sizes,
 * each size's problems in their own buffers with the layouts, info codes and
 * NaN fill of sunny_geneig_launch: a device work counter hands out work
 * items, largest N first, to a grid of 2 CTAs per SM, each item solved by
 * the same per-problem code as that size's own kernel (results are bitwise
 * those of per-size launches in the same regime). A work item is one
 * problem in the l2-slot regime and `per_item` problems in the smem-cta
 * regime.
 *   create: sizes[i] distinct, 1 <= sizes[i] <= sunny_geneig_max_matrix_size();
 *     regimes[i] (NULL = all 0): 0 the default choice by N, 1 smem-cta
 *     (N <= 64), 2 l2-slot; per_item[i] (NULL or <= 0 = default: 4 in
 *     smem-cta, 1 in l2-slot). Reserves the l2-slot scratch for the largest
 *     such size and the work counter. NULL on failure (last_error).
 *   launch: arrays indexed like `sizes`; counts[i] >= 0 problems of size
 *     sizes[i] (0 skips the size, its buffers may then be NULL). The launch
 *     resets the counter on `stream` first (a memset node when captured).
 *     Launches on different streams are ordered on the device; replays of a
 *     captured launch must be ordered by the caller, as for sunny_geneig_launch.
 *   shape: writes the groups in work order (descending N): size, regime (1
 *     smem-cta, 2 l2-slot) and problems per item; returns their number. */
typedef struct sunny_geneig_uneven* sunny_geneig_uneven_t;
sunny_geneig_uneven_t sunny_geneig_uneven_create(int num_sizes, const int* sizes, const int* regimes,
                                                 const int* per_item, int device_id);
sunny_geneig_status_t sunny_geneig_uneven_launch(sunny_geneig_uneven_t solver, const uintptr_t* d_H,
                                                 const uintptr_t* d_S, const uintptr_t* d_W,
                                                 const uintptr_t* d_U, const uintptr_t* d_info,
                                                 const int* counts, uintptr_t stream);
void sunny_geneig_uneven_destroy(sunny_geneig_uneven_t solver);
int  sunny_geneig_uneven_shape(sunny_geneig_uneven_t solver, int* sizes, int* regimes, int* per_item);

/* Largest N this build accepts in sunny_geneig_create. */
int sunny_geneig_max_matrix_size(void);

/* Name of the execution regime chosen at create time, e.g. "smem-cta"
 * (both matrices resident in one CTA's shared memory) or "l2-slot"
 * (matrices in a per-CTA global-memory slot). "" for NULL. */
const char* sunny_geneig_regime_name(sunny_geneig_solver_t solver);

/* Self-test of the device reciprocal the eigensolver uses in place of FP64
 * division (hardware approximation + two Newton-Raphson steps):
 * out[i] = 1 / x[i] for n device doubles, asynchronously on `stream`. */
sunny_geneig_status_t sunny_geneig_selftest_reciprocal(uintptr_t d_x, uintptr_t d_out, int n,
                                                       uintptr_t stream);

/* Allocation-free solve (no counterpart in the reference's C ABI).
 * For callers that cannot allocate device memory: code running inside
 * another framework's memory pool or under a no-allocation policy, hosts
 * that forbid cudaMalloc from plugins, graph-replay setups that must not
 * touch the allocator. Same buffers, layouts, info codes and error
 * behaviour as sunny_geneig_launch, on the calling thread's current device,
 * with no handle. For n <= 60 it runs the shared-memory kernel, which needs
 * no scratch at all; above that, the L2-slot kernel with its per-CTA scratch
 * taken from a fixed 32 MiB device array built into the library (held by
 * every GPU that loads the library until the process exits), so it
 * allocates nothing. The array holds floor(32 MiB / slot) slots, so the
 * number of CTAs in flight, and with it the throughput, falls as n grows:
 * 161 at n = 61, 12 at n = 216, 2 at n = 512 (a regular handle keeps two
 * per SM). n outside [1, 512] is rejected with INVALID_ARG. The first call
 * on a device resolves the array's address and sets the kernels'
 * shared-memory limits; make that first call before any stream capture.
 * All calls share the one array: calls whose kernels overlap on the GPU
 * (other streams, other host threads) race on it and must be serialised by
 * the caller. */
sunny_geneig_status_t sunny_geneig_launch_noalloc(
    int                   n,
    uintptr_t             d_H,
    uintptr_t             d_S,
    uintptr_t             d_W,
    uintptr_t             d_U,
    uintptr_t             d_info,
    int                   batch_size,
    uintptr_t             stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* SUNNY_GENEIG_H */
