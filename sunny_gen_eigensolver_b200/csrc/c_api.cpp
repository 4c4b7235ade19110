// C ABI of libsunny_geneig.so (declared in include/sunny_geneig.h).
//
// Same contract as the reference's src/common/c_api.cpp: nothrow at the
// boundary, exceptions and CUDA errors become status codes, the last message
// is kept per thread, device pointers travel as uintptr_t. Behind it there is
// no runtime compilation: the sm_100a kernels are compiled ahead of time and
// `create` only picks a launch plan and reserves the scratch that plan needs.

#include "sunny_geneig.h"
#include "geneig_kernels.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

struct sunny_geneig_solver {
    int n = 0;
    int device = 0;
    sunny_geneig_kernel_mode_t mode = SUNNY_GENEIG_KERNEL_UNIFIED;
    sunny_geneig_tuning_mode_t tuning = SUNNY_GENEIG_TUNING_SUGGESTED;
    sunny_geneig_cache_mode_t cache = SUNNY_GENEIG_CACHE_AUTO;
    int bpb = 1;
    bool tuned = false;          // configuration chosen by the autotuner
    sgeig::PlainPlan plan;
    void* scratch = nullptr;
    // Scratch ordering across streams: a launch that uses the handle's
    // scratch slots waits for the previous such launch when that one went to
    // another stream (launches on one stream are ordered by the stream).
    cudaEvent_t scratch_done = nullptr;
    uintptr_t last_stream = 0;
    bool scratch_used = false;
    std::mutex scratch_mu;
};

// Handle of the persistent uneven-size solver (sunny_geneig_uneven_*).
struct sunny_geneig_uneven {
    int device = 0;
    int ngroups = 0;
    int order[sgeig::kUnevenMaxGroups] = {};   // caller's index of group g (groups by descending n)
    int n[sgeig::kUnevenMaxGroups] = {};
    int kind[sgeig::kUnevenMaxGroups] = {};
    int per_item[sgeig::kUnevenMaxGroups] = {};
    size_t smem = 0;
    int grid = 0;
    size_t slot_elems = 0;
    void* scratch = nullptr;
    unsigned long long* head = nullptr;
    cudaEvent_t done = nullptr;
    uintptr_t last_stream = 0;
    bool used = false;
    std::mutex mu;
};

namespace {

thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

// Runs `fn` with `device` current on the calling thread and restores the
// caller's current device afterwards.
template <typename F>
cudaError_t with_device(int device, F&& fn) {
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    if (prev != device) {
        e = cudaSetDevice(device);
        if (e != cudaSuccess) return e;
    }
    e = fn();
    if (prev != device) cudaSetDevice(prev);
    return e;
}

bool aligned(uintptr_t p, uintptr_t a) { return (p % a) == 0; }

// NVTX range around each entry point (header-only NVTX v3: a no-op unless a
// profiler such as nsys or ncu --nvtx is attached), so that a timeline or an
// ncu --nvtx-include filter can pick out the solver's calls by name.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

sunny_geneig_solver_t create_impl(int n, int device_id, int bpb_request,
                                  sunny_geneig_tuning_mode_t tuning,
                                  sunny_geneig_cache_mode_t cache,
                                  sunny_geneig_kernel_mode_t mode, const char* fn,
                                  const char* regime = nullptr, int slots_per_sm = 0) {
    NvtxRange range(fn);
    clear_error();
    if (n < 1 || n > sgeig::kMaxN) {
        set_error(std::string(fn) + ": n=" + std::to_string(n) + " outside [1, " +
                  std::to_string(sgeig::kMaxN) + "]");
        return nullptr;
    }
    if (mode != SUNNY_GENEIG_KERNEL_UNIFIED && mode != SUNNY_GENEIG_KERNEL_HYBRID &&
        mode != SUNNY_GENEIG_KERNEL_MIXED) {
        set_error(std::string(fn) + ": unsupported kernel_mode " + std::to_string((int)mode));
        return nullptr;
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        set_error(std::string(fn) + ": no CUDA device available (" +
                  (e != cudaSuccess ? cudaGetErrorString(e) : "device count 0") + ")");
        return nullptr;
    }
    if (device_id < 0 || device_id >= count) {
        set_error(std::string(fn) + ": device_id " + std::to_string(device_id) + " out of range");
        return nullptr;
    }
    sunny_geneig_solver* s = nullptr;
    try {
        s = new sunny_geneig_solver();
    } catch (const std::bad_alloc&) {
        set_error(std::string("out of memory in ") + fn);
        return nullptr;
    }
    s->n = n;
    s->device = device_id;
    s->mode = mode;
    s->tuning = tuning;
    s->cache = cache;
    s->bpb = 1;
    std::string err;
    std::string tuned_regime;
    e = with_device(device_id, [&]() -> cudaError_t {
        // TUNING_AUTOTUNE (plain form, no explicit configuration): time every
        // configuration that can hold n, or take the cached choice
        if (tuning == SUNNY_GENEIG_TUNING_AUTOTUNE && mode != SUNNY_GENEIG_KERNEL_MIXED &&
            (regime == nullptr || regime[0] == '\0') && slots_per_sm == 0) {
            const std::string key = sgeig::tune_key(n, (int)mode, device_id);
            std::string cfg;
            if (!sgeig::tune_lookup(key, (int)cache, &cfg)) {
                const std::vector<std::pair<std::string, int>> cands = {
                    {"smem-cta", 0}, {"smem-wide", 0}, {"l2-slot", 1}, {"l2-slot", 2}};
                const int pick = sgeig::tune_pick(n, device_id, cands, &err);
                if (pick < 0) return cudaErrorInvalidValue;
                cfg = cands[pick].first + ":" + std::to_string(cands[pick].second);
                sgeig::tune_store(key, (int)cache, cfg);
            }
            const size_t colon = cfg.find(':');
            tuned_regime = cfg.substr(0, colon);
            slots_per_sm = colon == std::string::npos ? 0 : std::atoi(cfg.c_str() + colon + 1);
            regime = tuned_regime.c_str();
            s->tuned = true;
        }
        if (!sgeig::plain_plan(n, device_id, &s->plan, &err, mode == SUNNY_GENEIG_KERNEL_MIXED, regime,
                               slots_per_sm, bpb_request)) {
            // a cached choice this build cannot run any more: the default choice
            if (!s->tuned || !sgeig::plain_plan(n, device_id, &s->plan, &err, false, nullptr, 0, bpb_request))
                return cudaErrorInvalidValue;
            s->tuned = false;
        }
        // batches per block: the pencils one CTA solves at a time
        s->bpb = s->plan.regime == sgeig::Regime::SmemCta ? s->plan.teams : 1;
        if (s->plan.scratch_bytes) {
            cudaError_t ea = cudaMalloc(&s->scratch, s->plan.scratch_bytes);
            if (ea != cudaSuccess) { err = std::string("cudaMalloc scratch: ") + cudaGetErrorString(ea); return ea; }
            ea = cudaEventCreateWithFlags(&s->scratch_done, cudaEventDisableTiming);
            if (ea != cudaSuccess) { err = std::string("cudaEventCreate: ") + cudaGetErrorString(ea); return ea; }
        }
        return cudaSuccess;
    });
    if (e != cudaSuccess) {
        set_error(std::string(fn) + ": " + (err.empty() ? cudaGetErrorString(e) : err));
        if (s->scratch) with_device(device_id, [&]() { return cudaFree(s->scratch); });
        if (s->scratch_done) with_device(device_id, [&]() { return cudaEventDestroy(s->scratch_done); });
        delete s;
        return nullptr;
    }
    return s;
}

sunny_geneig_status_t launch_impl(sunny_geneig_solver_t s, int stage, uintptr_t d_H, uintptr_t d_S,
                                  uintptr_t d_W, uintptr_t d_U, uintptr_t d_info, int batch,
                                  uintptr_t stream, const char* fn, bool sigma = false) {
    NvtxRange range(fn);
    clear_error();
    if (!s) { set_error(std::string(fn) + ": solver is NULL"); return SUNNY_GENEIG_INVALID_ARG; }
    if (batch < 0) { set_error(std::string(fn) + ": batch_size < 0"); return SUNNY_GENEIG_INVALID_ARG; }
    if (stage < 1 || stage > 4) { set_error(std::string(fn) + ": stage must be 1..4"); return SUNNY_GENEIG_INVALID_ARG; }
    if (sigma && (s->n & 1)) {
        set_error(std::string(fn) + ": n must be even for the metric diag(I, -I)");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (batch == 0) return SUNNY_GENEIG_OK;
    if (sigma) d_H = d_S;   // never read; stands in for the checks below
    if (!d_H || !d_S || !d_W || !d_U || !d_info) {
        set_error(std::string(fn) + ": NULL device buffer");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (!aligned(d_H, 16) || !aligned(d_S, 16) || !aligned(d_U, 16) || !aligned(d_W, 8) || !aligned(d_info, 4)) {
        set_error(std::string(fn) + ": misaligned device buffer (H, S, U need 16 B; W 8 B; info 4 B)");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    try {
        auto run = [&]() {
            return sgeig::plain_launch(s->plan, stage, reinterpret_cast<const void*>(d_H),
                                       reinterpret_cast<const void*>(d_S), reinterpret_cast<double*>(d_W),
                                       reinterpret_cast<void*>(d_U), reinterpret_cast<int*>(d_info), batch,
                                       s->scratch, reinterpret_cast<cudaStream_t>(stream), sigma);
        };
        cudaError_t e;
        if (s->scratch) {
            std::lock_guard<std::mutex> lock(s->scratch_mu);
            e = with_device(s->device, [&]() {
                const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
                cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
                if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
                    return run();   // graph replays are ordered by the caller (see sunny_geneig_launch)
                if (s->scratch_used && s->last_stream != stream) {
                    cudaError_t w = cudaStreamWaitEvent(st, s->scratch_done, 0);
                    if (w != cudaSuccess) return w;
                }
                cudaError_t l = run();
                if (l != cudaSuccess) return l;
                l = cudaEventRecord(s->scratch_done, st);
                if (l == cudaSuccess) { s->scratch_used = true; s->last_stream = stream; }
                return l;
            });
        } else {
            e = with_device(s->device, run);
        }
        if (e != cudaSuccess) {
            set_error(std::string(fn) + ": kernel launch failed: " + cudaGetErrorString(e));
            return SUNNY_GENEIG_LAUNCH_ERROR;
        }
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return SUNNY_GENEIG_LAUNCH_ERROR;
    } catch (...) {
        set_error(std::string("unknown C++ exception in ") + fn);
        return SUNNY_GENEIG_LAUNCH_ERROR;
    }
    return SUNNY_GENEIG_OK;
}

}  // namespace

namespace sgeig {
void api_set_error(const std::string& msg) { set_error(msg); }
void api_clear_error() { clear_error(); }
}  // namespace sgeig

namespace {
// Shared body of the two fused-assembly entry points (d_O == 0: W and U).
sunny_geneig_status_t fourier_impl(const char* fn, sunny_geneig_solver_t solver, uintptr_t d_start,
                                   uintptr_t d_coef, uintptr_t d_disp, int n_terms, uintptr_t d_q, uintptr_t d_O,
                                   uintptr_t d_qhat, uintptr_t d_energies, int n_energies, double fwhm,
                                   uintptr_t d_W, uintptr_t d_U, uintptr_t d_spec, uintptr_t d_info,
                                   int batch_size, uintptr_t stream) {
    NvtxRange range(fn);
    clear_error();
    const bool intensity = d_O != 0 || d_spec != 0;
    if (!solver) { set_error(std::string(fn) + ": solver is NULL"); return SUNNY_GENEIG_INVALID_ARG; }
    if (batch_size < 0) { set_error(std::string(fn) + ": batch_size < 0"); return SUNNY_GENEIG_INVALID_ARG; }
    if (n_terms < 0) { set_error(std::string(fn) + ": n_terms < 0"); return SUNNY_GENEIG_INVALID_ARG; }
    if (solver->n & 1) { set_error(std::string(fn) + ": n must be even"); return SUNNY_GENEIG_INVALID_ARG; }
    if (solver->plan.regime != sgeig::Regime::SmemCta || solver->plan.mixed) {
        set_error(std::string(fn) + ": needs a plain solver in the smem-cta regime (n <= " +
                  std::to_string(sgeig::kCtaMaxN) + ")");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (intensity && (n_energies < 1 || !(fwhm > 0.0))) {
        set_error(std::string(fn) + ": n_energies must be >= 1 and fwhm > 0");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (batch_size == 0) return SUNNY_GENEIG_OK;
    if (!d_start || !d_q || !d_W || !d_info || (n_terms > 0 && (!d_coef || !d_disp)) ||
        (intensity ? (!d_O || !d_qhat || !d_energies || !d_spec) : !d_U)) {
        set_error(std::string(fn) + ": NULL device buffer");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (!aligned(d_start, 4) || !aligned(d_coef, 16) || !aligned(d_disp, 8) || !aligned(d_q, 8) ||
        !aligned(d_W, 8) || !aligned(d_info, 4) || !aligned(d_U, 16) || !aligned(d_O, 16) ||
        !aligned(d_qhat, 8) || !aligned(d_energies, 8) || !aligned(d_spec, 8)) {
        set_error(std::string(fn) + ": misaligned device buffer (coef, U, O need 16 B; start, info 4 B; "
                  "disp, q, W, qhat, energies, spec 8 B)");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    try {
        const sgeig::PlainPlan& p = solver->plan;
        sgeig::FourierTerms ft;
        ft.start = reinterpret_cast<const int*>(d_start);
        ft.coef = reinterpret_cast<const void*>(d_coef);
        ft.disp = reinterpret_cast<const double*>(d_disp);
        ft.nterms = n_terms;
        cudaError_t e = with_device(solver->device, [&]() {
            return sgeig::cta_launch_fourier(p.n, p.nmax, ft, reinterpret_cast<const double*>(d_q),
                                             intensity ? reinterpret_cast<const void*>(d_O) : nullptr,
                                             reinterpret_cast<const double*>(d_qhat),
                                             reinterpret_cast<const double*>(d_energies), n_energies, fwhm,
                                             reinterpret_cast<double*>(d_W), reinterpret_cast<void*>(d_U),
                                             reinterpret_cast<double*>(d_spec), reinterpret_cast<int*>(d_info),
                                             batch_size, reinterpret_cast<cudaStream_t>(stream));
        });
        if (e != cudaSuccess) {
            set_error(std::string(fn) + ": kernel launch failed: " + cudaGetErrorString(e));
            return SUNNY_GENEIG_LAUNCH_ERROR;
        }
    } catch (...) {
        set_error(std::string("unknown C++ exception in ") + fn);
        return SUNNY_GENEIG_LAUNCH_ERROR;
    }
    return SUNNY_GENEIG_OK;
}
}  // namespace

#pragma GCC visibility push(default)
extern "C" {

sunny_geneig_solver_t sunny_geneig_create(int n, int device_id, int batches_per_block_request,
                                          sunny_geneig_tuning_mode_t tuning_mode,
                                          sunny_geneig_cache_mode_t cache_mode) {
    try {
        return create_impl(n, device_id, batches_per_block_request, tuning_mode, cache_mode,
                           SUNNY_GENEIG_KERNEL_UNIFIED, "sunny_geneig_create");
    } catch (...) {
        set_error("unknown C++ exception in sunny_geneig_create");
        return nullptr;
    }
}

sunny_geneig_solver_t sunny_geneig_create_ex(int n, int device_id, int batches_per_block_request,
                                             sunny_geneig_tuning_mode_t tuning_mode,
                                             sunny_geneig_cache_mode_t cache_mode,
                                             sunny_geneig_kernel_mode_t kernel_mode) {
    try {
        return create_impl(n, device_id, batches_per_block_request, tuning_mode, cache_mode, kernel_mode,
                           "sunny_geneig_create_ex");
    } catch (...) {
        set_error("unknown C++ exception in sunny_geneig_create_ex");
        return nullptr;
    }
}

void sunny_geneig_destroy(sunny_geneig_solver_t solver) {
    if (!solver) return;
    try {
        if (solver->scratch) {
            const int dev = solver->device;
            void* p = solver->scratch;
            cudaEvent_t ev = solver->scratch_done;
            with_device(dev, [&]() {
                if (ev) cudaEventSynchronize(ev);   // no launch may still use the slots
                if (ev) cudaEventDestroy(ev);
                return cudaFree(p);
            });
        }
        delete solver;
    } catch (...) {
    }
}

sunny_geneig_solver_t sunny_geneig_create_config(int n, int device_id, sunny_geneig_kernel_mode_t kernel_mode,
                                                 const char* regime, int slots_per_sm) {
    try {
        return create_impl(n, device_id, 0, SUNNY_GENEIG_TUNING_SUGGESTED, SUNNY_GENEIG_CACHE_AUTO, kernel_mode,
                           "sunny_geneig_create_config", regime, slots_per_sm);
    } catch (...) {
        set_error("unknown C++ exception in sunny_geneig_create_config");
        return nullptr;
    }
}

sunny_geneig_status_t sunny_geneig_launch(sunny_geneig_solver_t solver, uintptr_t d_H, uintptr_t d_S,
                                          uintptr_t d_W, uintptr_t d_U, uintptr_t d_info, int batch_size,
                                          uintptr_t stream) {
    return launch_impl(solver, 4, d_H, d_S, d_W, d_U, d_info, batch_size, stream, "sunny_geneig_launch");
}

sunny_geneig_status_t sunny_geneig_launch_stage(sunny_geneig_solver_t solver, int stage, uintptr_t d_H,
                                                uintptr_t d_S, uintptr_t d_W, uintptr_t d_U, uintptr_t d_info,
                                                int batch_size, uintptr_t stream) {
    return launch_impl(solver, stage, d_H, d_S, d_W, d_U, d_info, batch_size, stream,
                       "sunny_geneig_launch_stage");
}

sunny_geneig_status_t sunny_geneig_launch_sigma(sunny_geneig_solver_t solver, uintptr_t d_S, uintptr_t d_W,
                                                uintptr_t d_U, uintptr_t d_info, int batch_size, uintptr_t stream) {
    return launch_impl(solver, 4, 0, d_S, d_W, d_U, d_info, batch_size, stream, "sunny_geneig_launch_sigma",
                       true);
}

sunny_geneig_status_t sunny_geneig_launch_fourier_sigma(sunny_geneig_solver_t solver, uintptr_t d_start,
                                                        uintptr_t d_coef, uintptr_t d_disp, int n_terms,
                                                        uintptr_t d_q, uintptr_t d_W, uintptr_t d_U,
                                                        uintptr_t d_info, int batch_size, uintptr_t stream) {
    return fourier_impl("sunny_geneig_launch_fourier_sigma", solver, d_start, d_coef, d_disp, n_terms, d_q, 0, 0,
                        0, 0, 0.0, d_W, d_U, 0, d_info, batch_size, stream);
}

sunny_geneig_status_t sunny_geneig_launch_fourier_sigma_intensity(
    sunny_geneig_solver_t solver, uintptr_t d_start, uintptr_t d_coef, uintptr_t d_disp, int n_terms, uintptr_t d_q,
    uintptr_t d_O, uintptr_t d_qhat, uintptr_t d_energies, int n_energies, double fwhm, uintptr_t d_W,
    uintptr_t d_spec, uintptr_t d_info, int batch_size, uintptr_t stream) {
    const char* fn = "sunny_geneig_launch_fourier_sigma_intensity";
    if (solver && batch_size > 0 && (!d_O || !d_spec)) {
        clear_error();
        set_error(std::string(fn) + ": NULL device buffer");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    return fourier_impl(fn, solver, d_start, d_coef, d_disp, n_terms, d_q, d_O, d_qhat, d_energies,
                        n_energies, fwhm, d_W, 0, d_spec, d_info, batch_size, stream);
}

sunny_geneig_status_t sunny_geneig_launch_sigma_intensity(sunny_geneig_solver_t solver, uintptr_t d_S,
                                                          uintptr_t d_O, uintptr_t d_qhat, uintptr_t d_energies,
                                                          int n_energies, double fwhm, uintptr_t d_W,
                                                          uintptr_t d_spec, uintptr_t d_info, int batch_size,
                                                          uintptr_t stream) {
    const char* fn = "sunny_geneig_launch_sigma_intensity";
    NvtxRange range(fn);
    clear_error();
    if (!solver) { set_error(std::string(fn) + ": solver is NULL"); return SUNNY_GENEIG_INVALID_ARG; }
    if (batch_size < 0) { set_error(std::string(fn) + ": batch_size < 0"); return SUNNY_GENEIG_INVALID_ARG; }
    if (solver->n & 1) { set_error(std::string(fn) + ": n must be even"); return SUNNY_GENEIG_INVALID_ARG; }
    if (solver->plan.regime != sgeig::Regime::SmemCta || solver->plan.mixed) {
        set_error(std::string(fn) + ": needs a plain solver in the smem-cta regime (n <= " +
                  std::to_string(sgeig::kCtaMaxN) + ")");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (n_energies < 1 || !(fwhm > 0.0)) {
        set_error(std::string(fn) + ": n_energies must be >= 1 and fwhm > 0");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (batch_size == 0) return SUNNY_GENEIG_OK;
    if (!d_S || !d_O || !d_qhat || !d_energies || !d_W || !d_spec || !d_info) {
        set_error(std::string(fn) + ": NULL device buffer");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    if (!aligned(d_S, 16) || !aligned(d_O, 16) || !aligned(d_qhat, 8) || !aligned(d_energies, 8) ||
        !aligned(d_W, 8) || !aligned(d_spec, 8) || !aligned(d_info, 4)) {
        set_error(std::string(fn) + ": misaligned device buffer (S, O need 16 B; qhat, energies, W, spec 8 B)");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    try {
        const sgeig::PlainPlan& p = solver->plan;
        cudaError_t e = with_device(solver->device, [&]() {
            return sgeig::cta_launch_intensity(p.n, p.nmax, p.smem, reinterpret_cast<const void*>(d_S),
                                               reinterpret_cast<const void*>(d_O),
                                               reinterpret_cast<const double*>(d_qhat),
                                               reinterpret_cast<const double*>(d_energies), n_energies, fwhm,
                                               reinterpret_cast<double*>(d_W), reinterpret_cast<double*>(d_spec),
                                               reinterpret_cast<int*>(d_info), batch_size,
                                               reinterpret_cast<cudaStream_t>(stream), p.teams);
        });
        if (e != cudaSuccess) {
            set_error(std::string(fn) + ": kernel launch failed: " + cudaGetErrorString(e));
            return SUNNY_GENEIG_LAUNCH_ERROR;
        }
    } catch (...) {
        set_error(std::string("unknown C++ exception in ") + fn);
        return SUNNY_GENEIG_LAUNCH_ERROR;
    }
    return SUNNY_GENEIG_OK;
}

sunny_geneig_uneven_t sunny_geneig_uneven_create(int num_sizes, const int* sizes, const int* regimes,
                                                 const int* per_item, int device_id) {
    const char* fn = "sunny_geneig_uneven_create";
    clear_error();
    try {
        if (num_sizes < 1 || num_sizes > sgeig::kUnevenMaxGroups || !sizes) {
            set_error(std::string(fn) + ": num_sizes must be 1.." + std::to_string(sgeig::kUnevenMaxGroups));
            return nullptr;
        }
        for (int i = 0; i < num_sizes; ++i) {
            if (sizes[i] < 1 || sizes[i] > sgeig::kMaxN) {
                set_error(std::string(fn) + ": size " + std::to_string(sizes[i]) + " outside [1, " +
                          std::to_string(sgeig::kMaxN) + "]");
                return nullptr;
            }
            for (int j = 0; j < i; ++j)
                if (sizes[j] == sizes[i]) {
                    set_error(std::string(fn) + ": size " + std::to_string(sizes[i]) + " given twice");
                    return nullptr;
                }
            const int r = regimes ? regimes[i] : 0;
            if (r < 0 || r > 2) {
                set_error(std::string(fn) + ": regime code must be 0 (default), 1 (smem-cta) or 2 (l2-slot)");
                return nullptr;
            }
            if (r == 1 && sizes[i] > sgeig::kCtaMaxN) {
                set_error(std::string(fn) + ": smem-cta cannot hold n=" + std::to_string(sizes[i]));
                return nullptr;
            }
        }
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device_id < 0 || device_id >= count) {
            set_error(std::string(fn) + ": device_id " + std::to_string(device_id) + " out of range");
            return nullptr;
        }
        auto* h = new sunny_geneig_uneven();
        h->device = device_id;
        h->ngroups = num_sizes;
        for (int i = 0; i < num_sizes; ++i) h->order[i] = i;
        std::sort(h->order, h->order + num_sizes, [&](int x, int y) { return sizes[x] > sizes[y]; });
        std::string err;
        cudaError_t e = with_device(device_id, [&]() -> cudaError_t {
            int optin = 0, sms = 0;
            cudaError_t ea = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_id);
            if (ea == cudaSuccess) ea = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_id);
            if (ea != cudaSuccess) return ea;
            size_t slot = 0;
            for (int g = 0; g < num_sizes; ++g) {
                const int i = h->order[g], n = sizes[i];
                const int r = regimes ? regimes[i] : 0;
                const bool l2 = r == 2 || (r == 0 && n > sgeig::kCtaPreferredMaxN);
                h->n[g] = n;
                h->kind[g] = sgeig::uneven_kind(n, l2);
                h->per_item[g] = (per_item && per_item[i] > 0) ? per_item[i] : (l2 ? 1 : 4);
                h->smem = std::max(h->smem, sgeig::uneven_smem_bytes(n, h->kind[g]));
                if (l2) slot = std::max(slot, sgeig::tiled_slot_elems(n));
            }
            if (h->smem > (size_t)optin) { err = "the mix needs more shared memory than a CTA has"; return cudaErrorInvalidValue; }
            ea = sgeig::uneven_set_attributes((size_t)optin);
            if (ea != cudaSuccess) { err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ea); return ea; }
            h->grid = 2 * sms;
            h->slot_elems = slot;
            if (slot) {
                ea = cudaMalloc(&h->scratch, (size_t)h->grid * slot * 16);
                if (ea != cudaSuccess) { err = std::string("cudaMalloc scratch: ") + cudaGetErrorString(ea); return ea; }
            }
            ea = cudaMalloc(reinterpret_cast<void**>(&h->head), sizeof(unsigned long long));
            if (ea != cudaSuccess) { err = std::string("cudaMalloc counter: ") + cudaGetErrorString(ea); return ea; }
            return cudaEventCreateWithFlags(&h->done, cudaEventDisableTiming);
        });
        if (e != cudaSuccess) {
            set_error(std::string(fn) + ": " + (err.empty() ? cudaGetErrorString(e) : err));
            with_device(device_id, [&]() {
                cudaFree(h->scratch);
                cudaFree(h->head);
                if (h->done) cudaEventDestroy(h->done);
                return cudaSuccess;
            });
            delete h;
            return nullptr;
        }
        return h;
    } catch (...) {
        set_error(std::string("unknown C++ exception in ") + fn);
        return nullptr;
    }
}

sunny_geneig_status_t sunny_geneig_uneven_launch(sunny_geneig_uneven_t h, const uintptr_t* d_H,
                                                 const uintptr_t* d_S, const uintptr_t* d_W,
                                                 const uintptr_t* d_U, const uintptr_t* d_info,
                                                 const int* counts, uintptr_t stream) {
    const char* fn = "sunny_geneig_uneven_launch";
    NvtxRange range(fn);
    clear_error();
    if (!h) { set_error(std::string(fn) + ": handle is NULL"); return SUNNY_GENEIG_INVALID_ARG; }
    if (!d_H || !d_S || !d_W || !d_U || !d_info || !counts) {
        set_error(std::string(fn) + ": NULL array argument");
        return SUNNY_GENEIG_INVALID_ARG;
    }
    sgeig::UnevenLaunch L;
    L.ngroups = h->ngroups;
    for (int g = 0; g < h->ngroups; ++g) {
        const int i = h->order[g];
        if (counts[i] < 0) { set_error(std::string(fn) + ": negative count"); return SUNNY_GENEIG_INVALID_ARG; }
        if (counts[i] > 0) {
            if (!d_H[i] || !d_S[i] || !d_W[i] || !d_U[i] || !d_info[i]) {
                set_error(std::string(fn) + ": NULL device buffer for size " + std::to_string(h->n[g]));
                return SUNNY_GENEIG_INVALID_ARG;
            }
            if (!aligned(d_H[i], 16) || !aligned(d_S[i], 16) || !aligned(d_U[i], 16) || !aligned(d_W[i], 8) ||
                !aligned(d_info[i], 4)) {
                set_error(std::string(fn) + ": misaligned device buffer (H, S, U need 16 B; W 8 B; info 4 B)");
                return SUNNY_GENEIG_INVALID_ARG;
            }
        }
        L.n[g] = h->n[g];
        L.kind[g] = h->kind[g];
        L.per_item[g] = h->per_item[g];
        L.count[g] = counts[i];
        L.H[g] = reinterpret_cast<const void*>(d_H[i]);
        L.S[g] = reinterpret_cast<const void*>(d_S[i]);
        L.W[g] = reinterpret_cast<double*>(d_W[i]);
        L.U[g] = reinterpret_cast<void*>(d_U[i]);
        L.info[g] = reinterpret_cast<int*>(d_info[i]);
    }
    try {
        std::lock_guard<std::mutex> lock(h->mu);
        cudaError_t e = with_device(h->device, [&]() {
            const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            const bool capturing = cudaStreamIsCapturing(st, &cs) == cudaSuccess &&
                                   cs == cudaStreamCaptureStatusActive;
            if (!capturing && h->used && h->last_stream != stream) {
                cudaError_t w = cudaStreamWaitEvent(st, h->done, 0);
                if (w != cudaSuccess) return w;
            }
            cudaError_t l = sgeig::uneven_launch(L, h->head, h->scratch, h->slot_elems, h->grid, h->smem, st);
            if (l != cudaSuccess || capturing) return l;
            l = cudaEventRecord(h->done, st);
            if (l == cudaSuccess) { h->used = true; h->last_stream = stream; }
            return l;
        });
        if (e != cudaSuccess) {
            set_error(std::string(fn) + ": launch failed: " + cudaGetErrorString(e));
            return SUNNY_GENEIG_LAUNCH_ERROR;
        }
    } catch (...) {
        set_error(std::string("unknown C++ exception in ") + fn);
        return SUNNY_GENEIG_LAUNCH_ERROR;
    }
    return SUNNY_GENEIG_OK;
}

void sunny_geneig_uneven_destroy(sunny_geneig_uneven_t h) {
    if (!h) return;
    try {
        with_device(h->device, [&]() {
            if (h->done) { cudaEventSynchronize(h->done); cudaEventDestroy(h->done); }
            cudaFree(h->scratch);
            cudaFree(h->head);
            return cudaSuccess;
        });
        delete h;
    } catch (...) {
    }
}

int sunny_geneig_uneven_shape(sunny_geneig_uneven_t h, int* sizes, int* regimes, int* per_item) {
    if (!h) return -1;
    for (int g = 0; g < h->ngroups; ++g) {
        if (sizes) sizes[g] = h->n[g];
        if (regimes) regimes[g] = h->kind[g] == 5 ? 2 : 1;
        if (per_item) per_item[g] = h->per_item[g];
    }
    return h->ngroups;
}

int sunny_geneig_matrix_size(sunny_geneig_solver_t solver) { return solver ? solver->n : -1; }
int sunny_geneig_batches_per_block(sunny_geneig_solver_t solver) { return solver ? solver->bpb : -1; }
int sunny_geneig_block_dim_x(sunny_geneig_solver_t solver) { return solver ? solver->plan.threads : -1; }
unsigned int sunny_geneig_shared_mem_bytes(sunny_geneig_solver_t solver) {
    return solver ? static_cast<unsigned int>(solver->plan.smem) : 0u;
}

const char* sunny_geneig_last_error(void) { return g_last_error.c_str(); }

const char* sunny_geneig_path_name(sunny_geneig_solver_t solver) {
    if (!solver) return "";
    switch (solver->mode) {
        case SUNNY_GENEIG_KERNEL_HYBRID: return "hybrid";
        case SUNNY_GENEIG_KERNEL_MIXED:  return "mixed";
        default:                         return "unified";
    }
}

sunny_geneig_kernel_mode_t sunny_geneig_kernel_mode(sunny_geneig_solver_t solver) {
    if (!solver) return static_cast<sunny_geneig_kernel_mode_t>(-1);
    return solver->mode;
}

int sunny_geneig_max_matrix_size(void) { return sgeig::kMaxN; }

const char* sunny_geneig_regime_name(sunny_geneig_solver_t solver) {
    if (!solver) return "";
    switch (solver->plan.regime) {
        case sgeig::Regime::SmemCta:  return "smem-cta";
        case sgeig::Regime::SmemWide: return "smem-wide";
        default:                      return "l2-slot";
    }
}

}  // extern "C"
#pragma GCC visibility pop
