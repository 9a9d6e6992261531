// Instantiations of the per-step interpreter walk kernel (see walk_impl.cuh).
#include "instances.h"
#include "launch.h"
#include "walk_impl.cuh"

namespace dr {

cudaError_t walk_dispatch_interp(uint32_t m, int grid, int block, size_t smem, cudaStream_t st,
                                 const WalkArgs& a, int* occ) {
    switch (m) {
#define DR_X(M_, D_) \
    case M_: return run_kernel(k_walk<CLS_INTERP, M_, 0>, grid, block, smem, st, a, occ);
        DR_INTERP_INSTANCES(DR_X)
#undef DR_X
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t walk_dispatch(uint32_t cls, uint32_t m, uint32_t D, int grid, int block, size_t smem,
                          cudaStream_t st, const WalkArgs& a, int* occ) {
    switch (cls) {
        case CLS_COMPANION: return walk_dispatch_companion(m, D, grid, block, smem, st, a, occ);
        case CLS_RATIONAL: return walk_dispatch_rational(m, D, grid, block, smem, st, a, occ);
        case CLS_DENSE: return walk_dispatch_dense(m, D, grid, block, smem, st, a, occ);
        default: return walk_dispatch_interp(m, grid, block, smem, st, a, occ);
    }
}

}  // namespace dr
