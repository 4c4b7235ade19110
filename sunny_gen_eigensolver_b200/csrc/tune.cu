// Launch-configuration autotuner behind the C ABI's tuning and cache modes
// (the reference's autotune sweep and its disk cache:
// src/unified/unified_solver.cpp:649-925 and :403-597, mapped from the C ABI
// in src/common/c_api.cpp:76-107).
//
// TUNING_AUTOTUNE: every execution configuration this build can run for n
// (smem-cta, smem-wide, l2-slot with 1 or 2 CTAs per SM; the plain form
// only, the mixed form has one configuration) is timed on a seeded synthetic
// batch of that size, generated on the device, and the fastest is kept.
// Its name is cached under the key (n, kernel mode, device name, SM count,
// library build): CACHE_AUTO keeps it in this process and in an on-disk table
// ($SUNNY_GENEIG_CACHE_DIR, else $XDG_CACHE_HOME/sunny_geneig, else
// $HOME/.cache/sunny_geneig, else /tmp/sunny_geneig; file tune_v1.tsv, one
// "key<TAB>config" line per entry, rewritten atomically), CACHE_NODISK in
// this process only, CACHE_NOCACHE nowhere (every create tunes again).
// TUNING_SUGGESTED never tunes and never reads the cache: the default choice
// by n is used.

#include "geneig_common.cuh"
#include "geneig_kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

namespace sgeig {
namespace {

// SplitMix64: a fixed, portable hash of (seed, index) for the synthetic inputs.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double unit(unsigned long long h) {   // [-0.5, 0.5)
    return (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

// H Hermitian with real and imaginary parts in [-0.5, 0.5); S = n I + E with
// E Hermitian of the same kind, so S is Hermitian positive definite by
// Gershgorin (each off-diagonal |E_ij| < 1/sqrt(2), so a row's off-diagonal
// sum is below (n - 1) / sqrt(2) < n - 1/2 <= the smallest diagonal entry).
__global__ void tune_inputs_kernel(double2* H, double2* S, int n, long long batch, unsigned long long seed) {
    const long long nn = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nn * batch;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long b = idx / nn;
        const int r = (int)(idx - b * nn), j = r / n, i = r - j * n;
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const unsigned long long key = seed ^ ((unsigned long long)b << 24) ^ ((unsigned long long)lo << 12) ^ hi;
        double hr = unit(mix64(key * 4 + 0)), him = unit(mix64(key * 4 + 1));
        double sr = unit(mix64(key * 4 + 2)), sim = unit(mix64(key * 4 + 3));
        if (i == j) { him = 0.0; sim = 0.0; sr += (double)n; }
        else if (i < j) { him = -him; sim = -sim; }      // (i, j) = conj((j, i))
        H[idx] = c2(hr, him);
        S[idx] = c2(sr, sim);
    }
}

std::mutex g_tune_mu;
std::map<std::string, std::string> g_tune_mem;   // key -> config name

std::string cache_dir() {
    if (const char* e = std::getenv("SUNNY_GENEIG_CACHE_DIR")) return e;
    if (const char* x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/sunny_geneig";
    if (const char* h = std::getenv("HOME")) return std::string(h) + "/.cache/sunny_geneig";
    return "/tmp/sunny_geneig";
}

void mkdirs(const std::string& path) {
    std::string cur = (!path.empty() && path[0] == '/') ? "/" : "";
    std::stringstream ss(path);
    std::string part;
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
}

// One "key<TAB>config" entry per line; lines without a tab are skipped.
std::map<std::string, std::string> read_table(const std::string& file) {
    std::map<std::string, std::string> t;
    std::ifstream f(file);
    std::string line;
    while (std::getline(f, line)) {
        const size_t tab = line.find('\t');
        if (tab == std::string::npos || tab == 0 || tab + 1 >= line.size()) continue;
        t[line.substr(0, tab)] = line.substr(tab + 1);
    }
    return t;
}

void write_table(const std::string& dir, const std::string& file, const std::map<std::string, std::string>& t) {
    mkdirs(dir);
    const std::string tmp = file + ".tmp." + std::to_string((long long)getpid());
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return;
        for (const auto& kv : t) f << kv.first << '\t' << kv.second << '\n';
        if (!f) { std::remove(tmp.c_str()); return; }
    }
    std::rename(tmp.c_str(), file.c_str());   // atomic on POSIX
}

}  // namespace

std::string tune_key(int n, int mode, int device) {
    cudaDeviceProp p{};
    cudaGetDeviceProperties(&p, device);
    std::ostringstream k;
    k << "n=" << n << ";mode=" << mode << ";dev=" << p.name << ";sms=" << p.multiProcessorCount
      << ";build=" << __DATE__ << " " << __TIME__;
    return k.str();
}

bool tune_lookup(const std::string& key, int cache_mode, std::string* config) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    if (cache_mode == 2) return false;   // NOCACHE
    auto it = g_tune_mem.find(key);
    if (it != g_tune_mem.end()) { *config = it->second; return true; }
    if (cache_mode == 1) return false;   // NODISK
    const auto t = read_table(cache_dir() + "/tune_v1.tsv");
    auto jt = t.find(key);
    if (jt == t.end()) return false;
    g_tune_mem[key] = jt->second;
    *config = jt->second;
    return true;
}

void tune_store(const std::string& key, int cache_mode, const std::string& config) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    if (cache_mode == 2) return;
    g_tune_mem[key] = config;
    if (cache_mode == 1) return;
    const std::string dir = cache_dir(), file = dir + "/tune_v1.tsv";
    auto t = read_table(file);
    t[key] = config;
    write_table(dir, file, t);
}

// Times each candidate configuration (regime name, l2-slot CTAs per SM) for
// size n on a synthetic batch on `device` (current) and returns the index of
// the fastest, or -1 when none could run. The batch is sized for about 20 ms
// per launch at a tenth of the FP64 peak, between 2 x SMs and 4096 problems.
int tune_pick(int n, int device, const std::vector<std::pair<std::string, int>>& cands, std::string* err) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const double flops = 68.0 / 3.0 * (double)n * n * n;
    long long batch = (long long)(0.02 * 3.5e12 / flops);
    batch = std::max<long long>(2LL * sms, std::min<long long>(4096, batch));
    const size_t nn = (size_t)n * n;
    double2 *H = nullptr, *S = nullptr, *U = nullptr;
    double* W = nullptr;
    int* info = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto release = [&]() {
        if (st) cudaStreamSynchronize(st);
        cudaFree(H); cudaFree(S); cudaFree(U); cudaFree(W); cudaFree(info);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
    };
    if (cudaMalloc(&H, nn * batch * 16) != cudaSuccess || cudaMalloc(&S, nn * batch * 16) != cudaSuccess ||
        cudaMalloc(&U, nn * batch * 16) != cudaSuccess || cudaMalloc(&W, (size_t)n * batch * 8) != cudaSuccess ||
        cudaMalloc(&info, (size_t)batch * 4) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        *err = "autotune: could not allocate the tuning batch";
        cudaGetLastError();
        release();
        return -1;
    }
    const unsigned long long seed = 0xA5A5A5A5A5A5A5A5ULL ^ ((unsigned long long)n << 16);
    tune_inputs_kernel<<<2 * sms, 256, 0, st>>>(H, S, n, batch, seed);
    int best = -1;
    float best_ms = 1e30f;
    for (size_t c = 0; c < cands.size(); ++c) {
        PlainPlan plan;
        std::string perr;
        if (!plain_plan(n, device, &plan, &perr, false, cands[c].first.c_str(), cands[c].second)) continue;
        void* scratch = nullptr;
        if (plan.scratch_bytes && cudaMalloc(&scratch, plan.scratch_bytes) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        bool ok = plain_launch(plan, 4, H, S, W, U, info, batch, scratch, st) == cudaSuccess;   // warm-up
        float ms = 1e30f;
        for (int rep = 0; ok && rep < 3; ++rep) {
            ok = cudaEventRecord(e0, st) == cudaSuccess &&
                 plain_launch(plan, 4, H, S, W, U, info, batch, scratch, st) == cudaSuccess &&
                 cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
            float t = 0.0f;
            if (ok && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) ms = std::min(ms, t);
        }
        cudaStreamSynchronize(st);
        cudaFree(scratch);
        if (ok && ms < best_ms) { best_ms = ms; best = (int)c; }
    }
    if (best < 0) *err = "autotune: no configuration could run n=" + std::to_string(n);
    release();
    return best;
}

}  // namespace sgeig
