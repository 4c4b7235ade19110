// Internal launcher interface between the C ABI shim (c_api.cpp) and the
// sm_100a kernels. Not installed; callers use include/sunny_geneig.h.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <string>
#include <utility>
#include <vector>

namespace sgeig {

// Largest N accepted at create time.
constexpr int kMaxN = 512;
// Largest N whose two working matrices fit one CTA's shared memory.
int smem_cta_max_n();

// How one solve is laid out on the device.
// Default choice by N: SmemCta up to 60, L2Slot above (measured crossovers);
// SmemWide only when asked for.
enum class Regime : int {
    SmemCta  = 0,  // N <= 64: both matrices in one CTA's shared memory, register/MMA kernel
    SmemWide = 1,  // N <= ~80: both matrices in shared memory, column-group kernel
    L2Slot   = 2,  // any N: working matrices in a per-CTA global-memory slot, tiled MMA kernel
};

// Shared-memory kernel for N <= 64 (geneig_cta.cu); chosen by default up to
// kCtaPreferredMaxN (measured crossover with the l2-slot kernel on B200).
constexpr int kCtaMaxN = 64;
constexpr int kCtaPreferredMaxN = 60;
size_t cta_smem_bytes(int n);
int cta_nmax_for(int n);
int cta_threads_for(int nmax);   // threads per pencil (per team) of that row bound's kernel
// Pencils per CTA at a time (teams) that row bound's kernels exist for: 4 for
// nmax <= 16, 2 for nmax <= 32, else 1; and the dynamic shared memory of a
// CTA of `teams` teams.
int cta_max_teams(int nmax);
int cta_default_teams(int nmax);   // pencils per CTA when none is requested
size_t cta_teams_smem_bytes(int n, int teams);
cudaError_t cta_set_attributes(int nmax, size_t smem);   // every teams form of the row bound
// `sigma`: H is the metric diag(I_{n/2}, -I_{n/2}) and is not read (H may be NULL).
// `teams`: pencils per CTA (1, or up to cta_max_teams(nmax)); smem from
// cta_teams_smem_bytes.
cudaError_t cta_launch(int n, int nmax, size_t smem, int stage, const void* H, const void* S, double* W, void* U,
                       int* info, long long batch, cudaStream_t stream, bool sigma = false, int teams = 1);

// Spin-wave metric solve that reduces the eigenvectors to the spectrum
// S(q, E) on the device (no U output): O is 3 x n complex per problem,
// qhat 3 doubles per problem, energies ne doubles, spec ne doubles per
// problem; Gaussian broadening of full width at half maximum fwhm.
cudaError_t cta_launch_intensity(int n, int nmax, size_t smem, const void* S, const void* O, const double* qhat,
                                 const double* energies, int ne, double fwhm, double* W, double* spec, int* info,
                                 long long batch, cudaStream_t stream, int teams = 1);

// Spin-wave metric solve with S assembled on the device from Fourier terms
// (no S in memory): entry e = row + n col of the lower triangle is
// S(q)_e = sum_{t in [start[e], start[e+1])} coef[t] exp(2 pi i q . disp[3t..3t+2]),
// start int32[n*n + 1], coef complex128, disp 3 doubles per term, q 3
// doubles per problem. O == NULL: W and U as cta_launch (stage 4); else the
// intensity form of cta_launch_intensity (W and spec, no U). One pencil per
// CTA (its own kernel instantiation), dynamic smem cta_smem_bytes(n).
struct FourierTerms {
    const int*    start  = nullptr;
    const void*   coef   = nullptr;
    const double* disp   = nullptr;
    int           nterms = 0;   // terms outside [0, nterms) are never read
};
cudaError_t cta_launch_fourier(int n, int nmax, const FourierTerms& ft, const double* q,
                               const void* O, const double* qhat, const double* energies, int ne, double fwhm,
                               double* W, void* U, double* spec, int* info, long long batch, cudaStream_t stream);

// Tiled kernel for the L2Slot regime (geneig_tiled.cu). A CTA's slot holds,
// in double2 units, three n x ld complex matrices (four in the mixed form)
// and an n x ld real one (at least 16 n complex); the mixed form adds an
// n x ld single-precision complex copy of C.
__host__ __device__ inline size_t tiled_zo_elems(int n) {
    const size_t mat = (size_t)n * (size_t)(n | 1);
    return (mat + 1) / 2 > (size_t)16 * n ? (mat + 1) / 2 : (size_t)16 * n;
}
__host__ __device__ inline size_t tiled_slot_elems(int n, bool mixed = false) {
    const size_t mat = (size_t)n * (size_t)(n | 1);
    return (mixed ? 4 : 3) * mat + tiled_zo_elems(n) + (mixed ? (mat + 1) / 2 : 0);
}
__host__ __device__ inline size_t tiled_slot_bytes(int n, bool mixed = false) {
    return tiled_slot_elems(n, mixed) * 16;
}
size_t tiled_vec_bytes(int n);
cudaError_t tiled_set_attributes(size_t smem);
// `mixed`: FP32 Householder reduction, FP64 refinement (see geneig_tiled.cu).
// `refine_max`: mixed form's refinement steps before it falls back to FP64.
constexpr int kRefineMaxIters = 8;
cudaError_t tiled_launch(int n, int slots, size_t smem, int stage, const void* H, const void* S, double* W, void* U,
                         int* info, long long batch, void* scratch, cudaStream_t stream, bool sigma,
                         bool mixed = false, int refine_max = kRefineMaxIters);

struct PlainPlan {
    int    n        = 0;
    int    ld       = 0;      // leading dimension of the working matrices (odd)
    int    threads  = 0;      // CTA size
    size_t smem     = 0;      // dynamic shared memory per CTA
    Regime regime   = Regime::SmemCta;
    int    nmax     = 0;      // SmemCta: compile-time row bound of the register arrays
    int    teams    = 1;      // SmemCta: pencils per CTA at a time (threads / teams each)
    int    slots    = 0;      // L2Slot: number of resident CTAs (= scratch slots)
    size_t scratch_bytes = 0; // L2Slot: bytes of device scratch needed
    bool   mixed    = false;  // mixed-precision form (always the L2Slot regime)
    int    refine_max = kRefineMaxIters;  // mixed: refinement steps before the FP64 fallback
};

// Picks the regime and launch shape for size n on `device` and sets the
// kernel attributes it needs. Returns false with a message on failure.
// `mixed` selects the mixed-precision form (FP32 Householder reduction plus
// FP64 eigenpair refinement), which runs in the L2Slot regime for every n.
// `regime` (smem-cta | smem-wide | l2-slot) and `slots_per_sm` (1 or 2, the
// l2-slot CTAs per SM) request a configuration explicitly; a request that
// cannot hold n fails with a message. NULL / "" and 0 keep the default
// choice (or the SUNNY_GENEIG_REGIME / SUNNY_GENEIG_SLOTS_PER_SM overrides).
// `pencils_per_cta` (the reference's batches per block request): 0 the
// measured default (cta_default_teams), 1 one pencil per CTA, 2 or 4 that
// many pencils per CTA at a time where the smem-cta kernel has that form
// (N <= 32 for 2, N <= 16 for 4), else the largest form below the request
// (plan->teams says which).
bool plain_plan(int n, int device, PlainPlan* plan, std::string* err, bool mixed = false,
                const char* regime = nullptr, int slots_per_sm = 0, int pencils_per_cta = 0);

// Enqueues one launch of `stage` (1..4) over `batch` matrices on `stream`.
// `scratch` must hold plan.scratch_bytes when plan.regime == L2Slot.
// `sigma`: H is diag(I_{n/2}, -I_{n/2}) (n even) and is not read.
cudaError_t plain_launch(const PlainPlan& plan, int stage,
                         const void* H, const void* S, double* W, void* U,
                         int* info, long long batch, void* scratch,
                         cudaStream_t stream, bool sigma = false);

#ifdef SGEIG_PHASE_TIMERS
// Profiling builds only: adds the tiled kernel's phase counters into out.
cudaError_t tiled_phase_cycles(unsigned long long* out, int count, bool reset);
#endif

// Thread-local last-error text of the C ABI (defined in c_api.cpp), for
// entry points implemented in other translation units.
void api_set_error(const std::string& msg);
void api_clear_error();

// Autotuner behind TUNING_AUTOTUNE (tune.cu). tune_key names a (size, kernel
// mode, device, library build) pair; tune_lookup / tune_store read and write
// the cached choice ("regime:slots_per_sm") under `cache_mode` (the C ABI's
// sunny_geneig_cache_mode_t: 0 memory + disk, 1 memory only, 2 none);
// tune_pick times the candidate configurations on a synthetic batch on the
// current device and returns the index of the fastest (-1 if none ran).
std::string tune_key(int n, int mode, int device);
bool tune_lookup(const std::string& key, int cache_mode, std::string* config);
void tune_store(const std::string& key, int cache_mode, const std::string& config);
int tune_pick(int n, int device, const std::vector<std::pair<std::string, int>>& cands, std::string* err);

// Persistent uneven-size kernel (geneig_uneven.cu). One launch solves up to
// kUnevenMaxGroups size groups, given in the order their work is handed out
// (descending N); kind is uneven_kind(n, l2slot): 0..4 the smem-cta row
// bound 16/32/48/56/64, 5 the l2-slot body; per_item pencils make one work
// item. `head` is a device counter (reset by the launch), `scratch` holds
// `grid` slots of slot_elems complex entries when any group is l2-slot.
constexpr int kUnevenMaxGroups = 8;
struct UnevenLaunch {
    int ngroups = 0;
    int n[kUnevenMaxGroups] = {};
    int kind[kUnevenMaxGroups] = {};
    int per_item[kUnevenMaxGroups] = {};
    long long count[kUnevenMaxGroups] = {};
    const void* H[kUnevenMaxGroups] = {};
    const void* S[kUnevenMaxGroups] = {};
    double* W[kUnevenMaxGroups] = {};
    void* U[kUnevenMaxGroups] = {};
    int* info[kUnevenMaxGroups] = {};
};
int uneven_kind(int n, bool l2slot);
size_t uneven_smem_bytes(int n, int kind);
cudaError_t uneven_set_attributes(size_t smem);
cudaError_t uneven_launch(const UnevenLaunch& L, unsigned long long* head, void* scratch, size_t slot_elems,
                          int grid, size_t smem, cudaStream_t stream);

}  // namespace sgeig
