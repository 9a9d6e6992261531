// Instantiations of the FP64 shadow kernels (see shadow_impl.cuh).
#include <algorithm>

#include "instances.h"
#include "launch.h"
#include "shadow_impl.cuh"

namespace dr {

cudaError_t shadow_eval_dispatch(uint32_t U, int grid, int block, size_t smem, cudaStream_t st,
                                 const ShadowArgs& a, int* occ) {
    switch (U) {
        case 1: return run_kernel(k_shadow_eval<1>, grid, block, smem, st, a, occ);
        case 2: return run_kernel(k_shadow_eval<2>, grid, block, smem, st, a, occ);
        case 4: return run_kernel(k_shadow_eval<4>, grid, block, smem, st, a, occ);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t shadow_chain_dispatch(uint32_t m, uint32_t flags, int grid, int block, size_t smem,
                                  cudaStream_t st, const ShadowArgs& a, int* occ) {
    // flags bit 2: the lean instantiation (exact steps) for co-located chains
    switch (m * 8 + (flags & 3u) + (a.lean ? 4u : 0u)) {
#define DR_X(M_, D_) \
    case M_ * 8: return run_kernel(k_shadow_chain<M_, 0>, grid, block, smem, st, a, occ, true); \
    case M_ * 8 + 1: return run_kernel(k_shadow_chain<M_, 1>, grid, block, smem, st, a, occ, true); \
    case M_ * 8 + 2: return run_kernel(k_shadow_chain<M_, 2>, grid, block, smem, st, a, occ, true); \
    case M_ * 8 + 3: return run_kernel(k_shadow_chain<M_, 3>, grid, block, smem, st, a, occ, true); \
    case M_ * 8 + 4: return run_kernel(k_shadow_chain<M_, 4>, grid, block, smem, st, a, occ, true); \
    case M_ * 8 + 5: return run_kernel(k_shadow_chain<M_, 5>, grid, block, smem, st, a, occ, true); \
    case M_ * 8 + 6: return run_kernel(k_shadow_chain<M_, 6>, grid, block, smem, st, a, occ, true); \
    case M_ * 8 + 7: return run_kernel(k_shadow_chain<M_, 7>, grid, block, smem, st, a, occ, true);
        DR_INTERP_INSTANCES(DR_X)
#undef DR_X
        default: return cudaErrorInvalidValue;
    }
}

size_t shadow_chain_smem(uint32_t m, bool comp) {
    const int ne = (int)shadow_entries(m, comp);
    return (size_t)chain_buffers(ne) * chain_chunk_steps(ne) * ne * 32 * sizeof(double);
}

cudaError_t shadow_fd_dispatch(uint32_t cls, uint32_t m, uint32_t D, int grid, int block,
                               size_t smem, cudaStream_t st, const ShadowArgs& a, int* occ) {
    if (cls == CLS_COMPANION) {
        switch (m * 100 + D) {
#define DR_X(M_, D_) \
    case M_ * 100 + D_: \
        return a.lean ? run_kernel(k_shadow_intfd<CLS_COMPANION, M_, D_, true>, grid, block, smem, st, a, occ) \
                      : run_kernel(k_shadow_intfd<CLS_COMPANION, M_, D_, false>, grid, block, smem, st, a, occ);
            DR_COMPANION_INSTANCES(DR_X)
#undef DR_X
            default: return cudaErrorInvalidValue;
        }
    }
    if (cls == CLS_DENSE) {
        switch (m * 100 + D) {
#define DR_X(M_, D_) \
    case M_ * 100 + D_: \
        return a.lean ? run_kernel(k_shadow_intfd<CLS_DENSE, M_, D_, true>, grid, block, smem, st, a, occ) \
                      : run_kernel(k_shadow_intfd<CLS_DENSE, M_, D_, false>, grid, block, smem, st, a, occ);
            DR_DENSE_INSTANCES(DR_X)
#undef DR_X
            default: return cudaErrorInvalidValue;
        }
    }
    return cudaErrorInvalidValue;
}

bool shadow_split_supported(uint32_t cls, uint32_t m, uint32_t D) {
    if (cls != CLS_COMPANION) return false;
    switch (m * 100 + D) {
#define DR_X(M_, D_) case M_ * 100 + D_: return true;
        DR_SPLIT_INSTANCES(DR_X)
#undef DR_X
        default: return false;
    }
}

cudaError_t shadow_split_dispatch(uint32_t cls, uint32_t m, uint32_t D, int grid, int block, size_t smem,
                                  cudaStream_t st, const ShadowArgs& a, int* occ) {
    if (cls != CLS_COMPANION) return cudaErrorInvalidValue;
    switch (m * 100 + D) {
#define DR_X(M_, D_) \
    case M_ * 100 + D_: return run_kernel(k_shadow_split<CLS_COMPANION, M_, D_>, grid, block, smem, st, a, occ, true);
        DR_SPLIT_INSTANCES(DR_X)
#undef DR_X
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace dr

namespace dr {

// Test hook: the shadow's rescale division, one quotient per thread.
__global__ void k_debug_rescale(const double* x, const double* b, int n, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double P[1][1] = {{x[i]}};
    rescale<1>(P, b[i]);
    out[i] = P[0][0];
}

// Latency floor of the m = 2 chain: one warp runs the companion fast step
// on PCF step matrices computed in registers (b(n) cubic, a(n) linear), so
// nothing but the step itself is on its dependency chain.
__global__ void k_chain_floor(int steps, double* sink) {
    const int lane = threadIdx.x & 31;
    FChain<2> ch;
    DevWalk W{};
    W.flags = DR_WALK_INIT_PCF;
    W.a0 = 1 + lane % 3;
    ch.init(W);
    const double b3 = -(1 + lane % 4), b1 = lane % 7 - 3, a1 = 1 + lane % 5;
    bool out = false;
    for (int s = 0; s < steps; s += 8) {
#pragma unroll 2
        for (int t = 0; t < 8; ++t) {
            const double n = (double)(s + t + 1);
            double c[2] = {(b3 * n * n + b1) * n + 5.0, a1 * n + 2.0};
            ch.step_companion_fast(c, out);
        }
        ch.renorm();
    }
    sink[lane] = ch.P[0][1] + ch.sc_m + (out ? 1.0 : 0.0);
}

}  // namespace dr

extern "C" int dr_bench_chain_step(int32_t steps, double* ns_per_step) {
    using namespace dr;
    if (steps < 8 || !ns_per_step) return DR_ERR_ARG;
    double* d = nullptr;
    if (cudaMalloc(&d, 32 * sizeof(double)) != cudaSuccess) return DR_ERR_NOMEM;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        e = cudaEventRecord(e0);
        if (e == cudaSuccess) {
            k_chain_floor<<<1, 32>>>(steps, d);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(e1);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess) best = std::min(best, ms);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d);
    if (e != cudaSuccess) return DR_ERR_CUDA;
    *ns_per_step = (double)best * 1e6 / steps;
    return DR_OK;
}

extern "C" int dr_debug_rescale(const double* x, const double* b, int32_t n, double* out) {
    using namespace dr;
    if (n < 0 || (n > 0 && (!x || !b || !out))) return DR_ERR_ARG;
    if (n == 0) return DR_OK;
    double* d = nullptr;
    const size_t bytes = 8ull * n;
    if (cudaMalloc(&d, 3 * bytes) != cudaSuccess) return DR_ERR_NOMEM;
    cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + n, b, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_debug_rescale<<<(n + 255) / 256, 256>>>(d, d + n, n, d + 2 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? DR_OK : DR_ERR_CUDA;
}
