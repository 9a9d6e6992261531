// Integer-pipe peak microbenchmarks: the denominators of the walk kernels'
// roofline, one per instruction class the Montgomery step uses.  Each thread
// runs 8 independent dependency chains so issue, not latency, is the limit;
// one launch fills every SM with 2048 threads.
//   kind 0: 32x32->64 wide multiply-add (mad.wide.u32), the Montgomery product
//   kind 1: 32-bit add + unsigned min, the modular addition
//   kind 2: 1:2 mix of kind 0 and kind 1 instructions
//   kind 3: 32-bit low multiply-add (mad.lo.u32), the Montgomery quotient
//   kind 4: unsigned min alone (plus one add per 8 mins for a varying operand)
// Reports lane-instructions per second (kind 4 counts its mins only).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dreams_b200.h"
#include "../../include/dreams_b200_debug.h"
#include "host_common.h"

namespace dr {

template <int KIND>
__global__ void __launch_bounds__(256) k_int_peak(uint32_t* out, int iters, uint32_t seed) {
    const uint32_t t = threadIdx.x + blockIdx.x * blockDim.x;
    uint64_t w[8];
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        w[k] = (uint64_t)(t * 2654435761u + k);
        a[k] = t ^ (seed + 97u * k);
    }
    const uint32_t b = seed | 1u, p = 0x7fffffffu;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (KIND == 0 || KIND == 2) {
                asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(w[k]) : "r"(a[k]), "r"(b));
            }
            if (KIND == 1 || KIND == 2) {
                uint32_t s;
                asm volatile("add.u32 %0, %1, %2;" : "=r"(s) : "r"(a[k]), "r"(b));
                asm volatile("min.u32 %0, %1, %2;" : "=r"(a[k]) : "r"(s), "r"(s - p));
            }
            if (KIND == 3) {
                asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(b), "r"(p));
            }
        }
        if (KIND == 4) {
            const uint32_t v = b + (uint32_t)i * 0x9e3779b9u;
#pragma unroll
            for (int k = 0; k < 8; ++k) asm volatile("min.u32 %0, %0, %1;" : "+r"(a[k]) : "r"(v));
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc ^= (uint32_t)w[k] ^ (uint32_t)(w[k] >> 32) ^ a[k];
    if (acc == 0x12345678u) out[0] = acc;  // keep the work observable
}

}  // namespace dr

extern "C" int dr_bench_int_peak(int32_t kind, double* lane_ops_per_s) {
    using namespace dr;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DR_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (kind < 0 || kind > 4) {
        set_error("dr_bench_int_peak: kind must be 0..4");
        return DR_ERR_ARG;
    }
    uint32_t* out = nullptr;
    if (cudaMalloc(&out, 16) != cudaSuccess) return DR_ERR_NOMEM;
    const int iters = 4096, threads = 256, blocks = sms * 8;
    auto launch = [&](int it) {
        if (kind == 0) k_int_peak<0><<<blocks, threads>>>(out, it, 12345u);
        else if (kind == 1) k_int_peak<1><<<blocks, threads>>>(out, it, 12345u);
        else if (kind == 2) k_int_peak<2><<<blocks, threads>>>(out, it, 12345u);
        else if (kind == 3) k_int_peak<3><<<blocks, threads>>>(out, it, 12345u);
        else k_int_peak<4><<<blocks, threads>>>(out, it, 12345u);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch(iters);
    cudaEventRecord(e0);
    launch(iters);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) {
        set_error(cudaGetErrorString(err));
        return DR_ERR_CUDA;
    }
    const double per_iter = kind == 1 ? 16.0 : kind == 2 ? 24.0 : 8.0;
    *lane_ops_per_s = per_iter * iters * (double)threads * blocks / (ms * 1e-3);
    return DR_OK;
}
