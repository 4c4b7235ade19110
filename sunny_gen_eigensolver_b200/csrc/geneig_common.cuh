// Device helpers shared by the sm_100a eigensolver kernels: complex FP64
// arithmetic on double2, warp / column-group reductions, the total order used
// to rank eigenvalues, and the fast FP64 reciprocal.
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

// ---------------------------------------------------------------- teams
// The NT threads that solve one pencil in a CTA of BLOCK threads: the whole
// CTA when BLOCK == NT, else one of its BLOCK / NT teams of consecutive whole
// warps (several pencils per CTA). team_sync is the team's barrier:
// __syncthreads for a whole-CTA team, named barrier 1 + team otherwise
// (barrier 0 stays the CTA's own).
template <int NT, int BLOCK>
__device__ __forceinline__ unsigned team_tid() {
    if constexpr (BLOCK == NT) return threadIdx.x;
    else return threadIdx.x % NT;
}
template <int NT, int BLOCK>
__device__ __forceinline__ void team_sync() {
    static_assert(NT % 32 == 0 && BLOCK % NT == 0 && BLOCK / NT <= 15, "team shape");
    if constexpr (BLOCK == NT) __syncthreads();
    else asm volatile("bar.sync %0, %1;" :: "r"(1 + (int)(threadIdx.x / NT)), "n"(NT) : "memory");
}

// ---------------------------------------------------------------- constants
// LAPACK dlamch convention: eps = 2^-53 (relative machine precision).
constexpr double kEps    = 1.1102230246251565e-16;

// ---------------------------------------------------------------- failure codes
// Internal marker of a failed tridiagonal eigensolve (non-finite values):
// distinct from every info code (0, 1..n, n+1..2n).
constexpr int kEigFailCode = -1;
// The info such a pencil reports, LAPACK zhegv's for the same input: its
// tridiagonal QR counts the n - 1 off-diagonal elements that did not
// converge, and for n <= 2 it returns 0 with NaN eigenvalues (W and U are
// NaN-filled here in every case).
__host__ __device__ __forceinline__ int eig_fail_info(int n) { return n >= 3 ? n - 1 : 0; }

// ---------------------------------------------------------------- phase timers
// Profiling builds only (-DSGEIG_PHASE_TIMERS, built as a separate library by
// build.py --phase-timers): thread 0 of every CTA adds the clock64 cycles
// since its previous mark to the counter of the phase that just ended. Marks
// sit right after CTA barriers, so a counter divided by the number of solves
// is the CTA time per solve spent in that phase (with the SM shared by the
// other resident CTAs, as in a normal run). The product library compiles
// every mark to nothing.
constexpr int kPhaseSlots = 32;
#ifdef SGEIG_PHASE_TIMERS
static __device__ unsigned long long g_phase_cycles[kPhaseSlots];
__device__ __forceinline__ long long& phase_prev() {
    __shared__ long long t;
    return t;
}
__device__ __forceinline__ unsigned& phase_level();
__device__ __forceinline__ void phase_start() {
    if (threadIdx.x == 0) { phase_prev() = clock64(); phase_level() = 0; }
}
__device__ __forceinline__ void phase_mark(int slot) {
    if (threadIdx.x == 0) {
        const long long t = clock64();
        atomicAdd(&g_phase_cycles[slot], (unsigned long long)(t - phase_prev()));
        phase_prev() = t;
    }
}
// Event counters in the same array (profiling builds): phase_count adds v
// to a slot; phase_level_max keeps the largest v seen since the last
// phase_level_flush, which (thread 0, after a barrier) adds it to a slot.
__device__ __forceinline__ unsigned& phase_level() {
    __shared__ unsigned m;
    return m;
}
__device__ __forceinline__ void phase_count(int slot, unsigned long long v) { atomicAdd(&g_phase_cycles[slot], v); }
__device__ __forceinline__ void phase_level_max(unsigned v) { atomicMax(&phase_level(), v); }
__device__ __forceinline__ void phase_level_flush(int slot) {
    if (threadIdx.x == 0) {
        atomicAdd(&g_phase_cycles[slot], (unsigned long long)phase_level());
        phase_level() = 0;
    }
}
#else
__device__ __forceinline__ void phase_start() {}
__device__ __forceinline__ void phase_mark(int) {}
__device__ __forceinline__ void phase_count(int, unsigned long long) {}
__device__ __forceinline__ void phase_level_max(unsigned) {}
__device__ __forceinline__ void phase_level_flush(int) {}
#endif

}  // namespace sgeig
