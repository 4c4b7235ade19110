// Self-test kernels for the device arithmetic helpers the solver relies on,
// exposed through sunny_geneig_selftest_reciprocal so that a GPU test can
// compare them with CUDA's own correctly rounded operations.
#include "geneig_common.cuh"
#include "sunny_geneig.h"

#include <cuda_runtime.h>

namespace {

__global__ void reciprocal_kernel(const double* __restrict__ x, double* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = sgeig::fast_rcp(x[i]);
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" sunny_geneig_status_t sunny_geneig_selftest_reciprocal(uintptr_t d_x, uintptr_t d_out, int n,
                                                                  uintptr_t stream) {
    if (n < 0 || (n > 0 && (!d_x || !d_out))) return SUNNY_GENEIG_INVALID_ARG;
    if (n == 0) return SUNNY_GENEIG_OK;
    reciprocal_kernel<<<(n + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const double*>(d_x), reinterpret_cast<double*>(d_out), n);
    return cudaGetLastError() == cudaSuccess ? SUNNY_GENEIG_OK : SUNNY_GENEIG_LAUNCH_ERROR;
}
#pragma GCC visibility pop
