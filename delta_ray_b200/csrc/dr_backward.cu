// Backward pass kernels (placeholder until the adjoint kernels land).
#include "dr_kernels.h"

cudaError_t dr_launch_backward(const DevScene &, int, int, int, int, uint64_t, const float *, float *, float *,
                               long long, int, const BackwardWorkspace &, cudaStream_t, int *) {
    return cudaErrorNotSupported;
}
