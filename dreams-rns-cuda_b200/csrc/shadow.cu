// Instantiations of the FP64 shadow kernels (see shadow_impl.cuh).
#include "instances.h"
#include "launch.h"
#include "shadow_impl.cuh"

namespace dr {

cudaError_t shadow_interp_dispatch(uint32_t m, int grid, int block, size_t smem, cudaStream_t st,
                                   const ShadowArgs& a, int* occ) {
    switch (m) {
#define DR_X(M_, D_) \
    case M_: return run_kernel(k_shadow_interp<M_>, grid, block, smem, st, a, occ);
        DR_INTERP_INSTANCES(DR_X)
#undef DR_X
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t shadow_fd_dispatch(uint32_t cls, uint32_t m, uint32_t D, int grid, int block,
                               size_t smem, cudaStream_t st, const ShadowArgs& a, int* occ) {
    if (cls == CLS_COMPANION) {
        switch (m * 100 + D) {
#define DR_X(M_, D_) \
    case M_ * 100 + D_: return run_kernel(k_shadow_intfd<CLS_COMPANION, M_, D_>, grid, block, smem, st, a, occ);
            DR_COMPANION_INSTANCES(DR_X)
#undef DR_X
            default: return cudaErrorInvalidValue;
        }
    }
    if (cls == CLS_DENSE) {
        switch (m * 100 + D) {
#define DR_X(M_, D_) \
    case M_ * 100 + D_: return run_kernel(k_shadow_intfd<CLS_DENSE, M_, D_>, grid, block, smem, st, a, occ);
            DR_DENSE_INSTANCES(DR_X)
#undef DR_X
            default: return cudaErrorInvalidValue;
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace dr
