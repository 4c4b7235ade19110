// Persistent kernel for batches of pencils of uneven sizes (one launch for
// the whole mix). The host groups the problems by size N (up to kMaxGroups
// sizes, each group batch-contiguous in its own buffers, the layouts of
// sunny_geneig_launch) and orders the groups by descending N. The groups are
// cut into work items: one pencil for sizes in the l2-slot regime, `per_item`
// pencils for sizes in the smem-cta regime. Every CTA of the persistent grid
// (2 per SM) takes the next item index from a device counter (atomicAdd,
// reset to 0 by the host before each launch), so the largest problems start
// first and the small ones fill the tail, and solves it with the same
// per-pencil body as the size's own kernel (cta_solve / tiled_solve), so the
// results are bitwise those of per-size launches. An l2-slot body uses the
// CTA's own global-memory slot, sized for the largest l2-slot N of the mix.
// Small pencils are solved several per CTA at a time: an item of N <= 16
// goes to four 64-thread teams and one of N <= 32 to two 128-thread teams,
// each team with its own barrier and shared-memory slice, taking the item's
// pencils in turn (the thread counts of the sizes' own kernels).

// The smem-cta bodies are called, each with its own register allocation
// (inlining all of them with the tiled body into one function made the
// register allocator spill); the tiled body is inlined into the kernel.
#define SGEIG_CTA_BODY_INLINE __noinline__
#include "geneig_cta_body.cuh"
#include "geneig_tiled_body.cuh"

namespace sgeig {
namespace {

constexpr int kTeams16 = 4;   // 64-thread teams per CTA for N <= 16
constexpr int kTeams32 = 2;   // 128-thread teams per CTA for N <= 32

size_t team_slice(int n) { return (cta_smem_bytes(n) + 15) & ~(size_t)15; }

struct UnevenGroup {
    const double2* H;
    const double2* S;
    double*  W;
    double2* U;
    int*     info;
    long long count;        // pencils in the group
    long long first_item;   // global index of the group's first item
    int n;
    int kind;               // 0..4: smem-cta row bound 16/32/48/56/64; 5: l2-slot
    int per_item;           // pencils per work item
    size_t slice;           // kinds 0, 1: shared-memory bytes of one team
};

struct UnevenArgs {
    UnevenGroup g[kUnevenMaxGroups];
    int ngroups;
    long long nitems;
    unsigned long long* head;   // work counter
    double2* scratch;           // one l2-slot slot per CTA
    size_t slot_elems;
};

__global__ void __launch_bounds__(256, 2) geneig_uneven_kernel(UnevenArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long s_item;
    double2* slot = a.scratch ? a.scratch + (size_t)blockIdx.x * a.slot_elems : nullptr;
    phase_start();
    for (;;) {
        __syncthreads();                       // everyone has read the previous s_item
        if (threadIdx.x == 0) s_item = atomicAdd(a.head, 1ULL);
        __syncthreads();
        const long long it = (long long)s_item;
        if (it >= a.nitems) break;
        int gi = 0;
        while (gi + 1 < a.ngroups && it >= a.g[gi + 1].first_item) ++gi;
        const UnevenGroup& G = a.g[gi];
        const long long b0 = (it - G.first_item) * G.per_item;
        const long long b1 = b0 + G.per_item < G.count ? b0 + G.per_item : G.count;
        if (G.kind == 5) {
            tiled::TiledArgs t;
            t.H = G.H; t.S = G.S; t.W = G.W; t.U = G.U; t.info = G.info;
            t.scratch = a.scratch; t.batch = G.count;
            t.n = G.n; t.ld = G.n | 1; t.stage = 4; t.sigma = 0; t.mixed = 0; t.refine_max = 0;
            for (long long b = b0; b < b1; ++b) tiled::tiled_solve(t, b, slot, smem_raw);
        } else {
            cta::CtaArgs c;
            c.H = G.H; c.S = G.S; c.W = G.W; c.U = G.U; c.info = G.info;
            c.batch = G.count; c.n = G.n; c.ld = G.n | 1; c.stage = 4; c.sigma = 0;
            c.O = nullptr; c.qhat = nullptr; c.energies = nullptr; c.spec = nullptr; c.ne = 0;
            c.gnorm = 0.0; c.ginv2 = 0.0;
            switch (G.kind) {
                case 0: {
                    const int t = threadIdx.x / 64;
                    for (long long b = b0 + t; b < b1; b += kTeams16)
                        cta::cta_solve<16, 64, 256>(c, b, smem_raw + t * G.slice);
                    break;
                }
                case 1: {
                    const int t = threadIdx.x / 128;
                    for (long long b = b0 + t; b < b1; b += kTeams32)
                        cta::cta_solve<32, 128, 256>(c, b, smem_raw + t * G.slice);
                    break;
                }
                case 2: for (long long b = b0; b < b1; ++b) cta::cta_solve<48>(c, b, smem_raw); break;
                case 3: for (long long b = b0; b < b1; ++b) cta::cta_solve<56>(c, b, smem_raw); break;
                default: for (long long b = b0; b < b1; ++b) cta::cta_solve<64>(c, b, smem_raw); break;
            }
        }
    }
}

}  // namespace

cudaError_t uneven_set_attributes(size_t smem) {
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, geneig_uneven_kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(geneig_uneven_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(smem - fa.sharedSizeBytes));
}

int uneven_kind(int n, bool l2slot) {
    if (l2slot) return 5;
    return n <= 16 ? 0 : n <= 32 ? 1 : n <= 48 ? 2 : n <= 56 ? 3 : 4;
}

size_t uneven_smem_bytes(int n, int kind) {
    return kind == 5 ? tiled_vec_bytes(n)
         : kind == 0 ? kTeams16 * team_slice(n)
         : kind == 1 ? kTeams32 * team_slice(n)
         : cta_smem_bytes(n);
}

cudaError_t uneven_launch(const UnevenLaunch& L, unsigned long long* head, void* scratch, size_t slot_elems,
                          int grid, size_t smem, cudaStream_t stream) {
    UnevenArgs a{};
    long long first = 0;
    int ng = 0;
    for (int i = 0; i < L.ngroups; ++i) {
        if (L.count[i] <= 0) continue;
        UnevenGroup& G = a.g[ng++];
        G.H = static_cast<const double2*>(L.H[i]);
        G.S = static_cast<const double2*>(L.S[i]);
        G.W = L.W[i];
        G.U = static_cast<double2*>(L.U[i]);
        G.info = L.info[i];
        G.count = L.count[i];
        G.n = L.n[i];
        G.kind = L.kind[i];
        G.per_item = L.per_item[i] > 0 ? L.per_item[i] : 1;
        G.slice = team_slice(G.n);
        G.first_item = first;
        first += (G.count + G.per_item - 1) / G.per_item;
    }
    if (ng == 0) return cudaSuccess;
    a.ngroups = ng;
    a.nitems = first;
    a.head = head;
    a.scratch = static_cast<double2*>(scratch);
    a.slot_elems = slot_elems;
    cudaError_t e = cudaMemsetAsync(head, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    const long long g = first < grid ? first : grid;
    geneig_uneven_kernel<<<(unsigned)g, 256, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace sgeig
