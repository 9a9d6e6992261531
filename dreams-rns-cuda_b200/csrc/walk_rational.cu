// Instantiations of the rational walk kernel (see walk_impl.cuh).
#include "instances.h"
#include "launch.h"
#include "walk_impl.cuh"

namespace dr {

cudaError_t walk_dispatch_rational(uint32_t m, uint32_t D, int grid, int block, size_t smem,
                                 cudaStream_t st, const WalkArgs& a, int* occ) {
    switch (m * 100 + D) {
#define DR_X(M_, D_) \
    case M_ * 100 + D_: return run_kernel(k_walk<CLS_RATIONAL, M_, D_>, grid, block, smem, st, a, occ);
        DR_RATIONAL_INSTANCES(DR_X)
#undef DR_X
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace dr
