// Launch entry points of the kernel translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dr {

struct WalkArgs;
struct ShadowArgs;

// Garner CRT tables of one moduli set (crt.cu).
struct CrtTables {
    const uint32_t* moduli;   // [K]
    const uint32_t* pinv;     // [K]
    const uint32_t* r2;       // [K]
    const uint32_t* ginv;     // [K]  inv(M_i mod p_i), Montgomery form mod p_i
    const uint32_t* Mlimbs;   // [K][L]  M_i (M_0 = 1), little-endian limbs
    const uint32_t* Mtotal;   // [L]  product of all moduli
    int K, L;
    // [K][K] p_i^-1 mod p_j for i < j, Montgomery form mod p_j (null: not
    // built).  Built for the standard prime table only -- distinct primes
    // above 2^30 -- where it lets one lane run a value's whole Garner chain.
    const uint32_t* garner = nullptr;
};

// Largest K the lane-per-value CRT kernel takes (its per-warp shared memory
// grows with K); larger K use the warp-per-value kernel.
constexpr int kCrtLanesMaxK = 256;

// Delta kernel arguments (delta_topk.cu).  Item i reads p at p + i*istride,
// q at q + i*istride (nl limbs each), signs at ps/qs + i*sstride, and target
// t = per_item ? i : 0 as ln/ld + t*listride (lnl limbs), sign lns[t*lsstride]
// times (lds ? lds[t*lsstride] : 1); the target denominator's magnitude is used.
struct DeltaArgs {
    const uint32_t* p; const uint32_t* q;
    const int32_t* ps; const int32_t* qs;
    int n, nl;
    size_t istride, sstride;
    const uint32_t* ln; const uint32_t* ld;
    const int32_t* lns; const int32_t* lds;
    int lnl, per_item;
    size_t listride, lsstride;
    double* out;
    int maxlen;                              // product length bound (limbs)
    // bank mode (bank_n > 0): item i scores row rows[i / bank_n] (row i / bank_n
    // when rows is null) of p, q against target i % bank_n (hits or every walk
    // against a constant bank)
    const uint32_t* rows;
    int bank_n;
};

cudaError_t launch_crt_setup(const uint32_t* moduli, int K, int L, uint32_t* pinv, uint32_t* r2,
                             uint32_t* ginv, uint32_t* Mlimbs, uint32_t* Mtotal, uint32_t* garner,
                             cudaStream_t st);
// in_off[j]: offset of value j's K residues (null: j*K); out_idx[j]: output
// row of value j in limbs/sign/nl (null: j).
cudaError_t launch_crt(const uint32_t* res, int n, const CrtTables& T, uint32_t* limbs, int stride,
                       int32_t* sign, int32_t* nl, uint32_t* ul, int sms, cudaStream_t st,
                       const uint64_t* in_off = nullptr, const uint32_t* out_idx = nullptr);
cudaError_t launch_delta(const DeltaArgs& D, int sms, cudaStream_t st);
struct DevWalk;
// Per-walk CRT overflow flags from the pipeline's limbs and the FP64 shadow.
cudaError_t launch_crt_check(const uint32_t* limbs, const int32_t* signs, int L, int n,
                             const DevWalk* walks, const double* shadow, uint32_t* status,
                             cudaStream_t st);
cudaError_t launch_topk_tile(const double* vals, const uint64_t* in_keys, const uint32_t* in_idx,
                             int n, int k, uint64_t* out_keys, uint32_t* out_idx, cudaStream_t st);
int topk_tile_size();
// the tile of a launch_topk_tile pass over n values keeping k per tile
int topk_tile_for(int n, int k);
// threshold-filter top-k of large arrays (delta_topk.cu)
cudaError_t launch_topk_sample(const double* vals, int64_t stride, int s, uint64_t* keys, uint32_t* idx,
                               cudaStream_t st);
cudaError_t launch_topk_filter(const double* vals, int n, const uint64_t* thr, uint64_t* cand_keys,
                               uint32_t* cand_idx, int cap, unsigned int* count, int sms, cudaStream_t st);
cudaError_t launch_topk_gather(const double* vals, const uint32_t* idx, int k, double* vals_out,
                               int32_t* idx_out, cudaStream_t st);

// occ != nullptr: only report resident blocks per SM for (block, smem).
cudaError_t walk_dispatch(uint32_t cls, uint32_t m, uint32_t D, int grid, int block, size_t smem,
                          cudaStream_t st, const WalkArgs& a, int* occ);
// interpreted shadow: evaluation (U sub-blocks per pass) and chain kernels
cudaError_t shadow_eval_dispatch(uint32_t U, int grid, int block, size_t smem, cudaStream_t st,
                                 const ShadowArgs& a, int* occ);
// flags: bit 0 companion-shaped step matrices, bit 1 state-vector walks
cudaError_t shadow_chain_dispatch(uint32_t m, uint32_t flags, int grid, int block, size_t smem,
                                  cudaStream_t st, const ShadowArgs& a, int* occ);
size_t shadow_chain_smem(uint32_t m, bool comp);
// Split shadow (integer-difference head, then the interpreted chain's tail):
// the (class, m, D) it is built for, and its launch.
bool shadow_split_supported(uint32_t cls, uint32_t m, uint32_t D);
cudaError_t shadow_split_dispatch(uint32_t cls, uint32_t m, uint32_t D, int grid, int block, size_t smem,
                                  cudaStream_t st, const ShadowArgs& a, int* occ);
cudaError_t shadow_fd_dispatch(uint32_t cls, uint32_t m, uint32_t D, int grid, int block,
                               size_t smem, cudaStream_t st, const ShadowArgs& a, int* occ);

// per-class dispatchers (one translation unit each, compiled in parallel)
cudaError_t walk_dispatch_companion(uint32_t m, uint32_t D, int grid, int block, size_t smem,
                                    cudaStream_t st, const WalkArgs& a, int* occ);
cudaError_t walk_dispatch_rational(uint32_t m, uint32_t D, int grid, int block, size_t smem,
                                   cudaStream_t st, const WalkArgs& a, int* occ);
cudaError_t walk_dispatch_dense(uint32_t m, uint32_t D, int grid, int block, size_t smem,
                                cudaStream_t st, const WalkArgs& a, int* occ);
cudaError_t walk_dispatch_interp(uint32_t m, int grid, int block, size_t smem, cudaStream_t st,
                                 const WalkArgs& a, int* occ);

// Launches carry their stream's priority as a launch attribute, so the
// priority also holds for the kernel nodes of a captured CUDA graph.  With
// early_start the launch is a programmatic dependent of the previous kernel
// in the stream: its blocks may become resident while that kernel still
// runs (once it has executed griddepcontrol.launch_dependents) and must
// execute griddepcontrol.wait before reading what it wrote.
// A launch made while a StartedEvent is in scope on the calling thread also
// records that event once all its blocks have begun execution (the launch
// completion event), so other streams can wait for the kernel to be placed
// without waiting for it to finish.
inline thread_local cudaEvent_t tl_started_event = nullptr;
struct StartedEvent {
    explicit StartedEvent(cudaEvent_t e) { tl_started_event = e; }
    ~StartedEvent() { tl_started_event = nullptr; }
    StartedEvent(const StartedEvent&) = delete;
    StartedEvent& operator=(const StartedEvent&) = delete;
};

template <typename KernelT, typename ArgT>
inline cudaError_t run_kernel(KernelT k, int grid, int block, size_t smem, cudaStream_t st,
                              const ArgT& a, int* occ, bool early_start = false) {
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, block, smem);
    int prio = 0;
    const bool has_prio = st && cudaStreamGetPriority(st, &prio) == cudaSuccess && prio != 0;
    const cudaEvent_t started = tl_started_event;
    if (has_prio || early_start || started) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3((unsigned)block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[3];
        unsigned n = 0;
        if (has_prio) {
            attr[n].id = cudaLaunchAttributePriority;
            attr[n].val.priority = prio;
            ++n;
        }
        if (early_start) {
            attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[n].val.programmaticStreamSerializationAllowed = 1;
            ++n;
        }
        if (started) {
            attr[n].id = cudaLaunchAttributeLaunchCompletionEvent;
            attr[n].val.launchCompletionEvent.event = started;
            attr[n].val.launchCompletionEvent.flags = 0;
            ++n;
        }
        cfg.attrs = attr;
        cfg.numAttrs = n;
        return cudaLaunchKernelEx(&cfg, k, a);
    }
    k<<<grid, block, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace dr
