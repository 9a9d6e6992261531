// Host engine: device context, prepared walk batches, CRT/delta/top-k helpers.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/dreams_b200.h"
#include "dr_types.h"
#include "program.h"

namespace dr {

// Device block cache of the context: prepared batches take their buffers
// from it and give them back when destroyed (after the device is idle), so
// building and dropping a batch per call costs no cudaMalloc / cudaFree (the
// latter synchronises the whole device).  Bounded; larger surpluses are freed.
void* devcache_take(size_t n, size_t* got);
void devcache_put(void* p, size_t bytes);

// Owning device allocation.  A pooled buffer comes from and returns to the
// context's block cache; its owner guarantees no work still uses it when it
// is released.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool pooled = false;
    bool view = false;   // p points into another buffer, which owns the memory
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p && !view) {
            if (pooled) devcache_put(p, bytes);
            else cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
        view = false;
    }
    void set_view(void* q, size_t n) {
        release();
        p = q;
        bytes = n;
        view = true;
    }
    cudaError_t alloc(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        if (n == 0) n = 16;
        if (pooled) {
            p = devcache_take(n, &bytes);
            if (p) return cudaSuccess;
        }
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Host worker threads for batch construction.  run(parts, n, fn) splits
// [0, n) into `parts` contiguous ranges in order and calls fn(part, lo, hi)
// once for each, on the workers and the calling thread; it returns when all
// are done.  One job at a time.
class HostPool {
  public:
    explicit HostPool(int workers);
    ~HostPool();
    HostPool(const HostPool&) = delete;
    HostPool& operator=(const HostPool&) = delete;
    void run(int parts, size_t n, const std::function<void(int, size_t, size_t)>& fn);
    int threads() const { return (int)threads_.size() + 1; }

  private:
    void worker();
    void take_parts(const std::function<void(int, size_t, size_t)>* fn, int parts, size_t n);
    std::vector<std::thread> threads_;
    std::mutex run_mu_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int, size_t, size_t)>* fn_ = nullptr;
    int parts_ = 0;
    size_t n_ = 0;
    std::atomic<int> next_{0};
    int done_ = 0, active_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// The context's pool (created on first use).
HostPool& host_pool();

// Hash of a program blob for the plan cache: eight bytes per round
// (multiply, xor-shift), then the tail; several times faster than a
// byte-wise string hash on the kilobyte-sized blobs a batch looks up.
struct BlobHash {
    size_t operator()(std::string_view s) const noexcept {
        const uint64_t kMul = 0x9E3779B97F4A7C15ull;
        uint64_t h = 0x243F6A8885A308D3ull ^ (uint64_t)s.size();
        const unsigned char* p = reinterpret_cast<const unsigned char*>(s.data());
        size_t n = s.size();
        while (n >= 8) {
            uint64_t w;
            std::memcpy(&w, p, 8);
            h = (h ^ w) * kMul;
            h ^= h >> 29;
            p += 8;
            n -= 8;
        }
        uint64_t w = 0;
        std::memcpy(&w, p, n);
        h = (h ^ w) * kMul;
        return (size_t)(h ^ (h >> 32));
    }
};

struct CrtSet {
    int K = 0, L = 0;
    DevBuf moduli, pinv, r2, ginv, Mlimbs, Mtotal;
    DevBuf garner;     // standard primes only: the lane kernel's Garner constants
};

struct Context {
    int device = -1;
    int sms = 0;
    cudaStream_t stream = nullptr, side = nullptr;
    std::vector<cudaStream_t> pool;   // launch groups of a batch run concurrently on these
    std::vector<cudaStream_t> hpool;  // high-priority streams for the FP64 shadow launches
    DevBuf primes, pinv, r2;   // DR_MAX_K-entry prime table
    std::mutex mu;
    // plan cache keyed by program bytes (views into each Plan's own copy);
    // plan_mu guards it and code_ids (lookups shared, inserts exclusive)
    std::shared_mutex plan_mu;
    std::unordered_map<std::string_view, std::shared_ptr<Plan>, BlobHash> plan_cache;
    // interned instruction streams: programs that differ only in their
    // constants share one copy of device code in a batch
    std::unordered_map<std::string, uint32_t> code_ids;
    uint32_t next_code_id = 1;   // never reused, so a cleared table cannot alias
    std::map<int, std::shared_ptr<CrtSet>> crt_std;  // CRT tables of the standard primes
    struct TunedShape { uint32_t chunk, wpb, pack; };   // chunk steps, warps/block, chain pack depth
    std::map<std::string, TunedShape> tuned;              // by workload signature
    std::mutex cache_mu;
    std::multimap<size_t, void*> cache;   // free device blocks by size
    size_t cached_bytes = 0;
    // pinned staging of a batch's tables: one host-to-device copy per build.
    // stage_mu is held from filling it until the build's stream sync.
    std::mutex stage_mu;
    void* stage_host = nullptr;
    size_t stage_bytes = 0;
};

Context* ctx();           // nullptr before dr_init
int ensure_ctx();         // DR_OK or DR_ERR_NOT_INIT

// Get (and cache) the plan of a program blob.
int get_plan(const uint8_t* blob, uint64_t size, std::shared_ptr<Plan>* out, std::string* err);

// Standard-prime CRT tables for K (cached).
int crt_tables_std(int K, std::shared_ptr<CrtSet>* out);
int crt_limbs_for(int K);  // L: limbs of prod(moduli) + 1

struct LaunchSpec {
    int kind;                  // 0 walk, 1 shadow (interpreted), 2 shadow (integer differences)
    uint32_t cls, m, D;        // kind 1: cls bit 0 companion-shaped float matrix, bit 1 state vectors
    uint32_t off, count;       // tiles / list entries of this launch
    uint32_t items;            // work items (tiles, evaluation items or 32-walk groups)
    uint32_t queue;            // queue counter index
    uint32_t rows_regs, rows_consts, rows_stage, rows_per_warp;
    size_t smem;
    int grid, block;
    // kind 1: the evaluation launch above is followed by the chain launch.
    // rows_axes: axis rows per sub-block (kind 1) or, for a walk launch, the
    // rows each of axis start values, steps and current values per warp
    uint32_t U = 1, rows_axes = 0, eoff = 0;   // sub-blocks, axis rows, first evaluation item
    uint32_t items2 = 0, queue2 = 0;
    size_t smem2 = 0;
    int grid2 = 0, block2 = 0;
    bool follow = false;       // runs on the stream of the previous launch (shadow rounds)
    bool lean = false;         // shadow chains co-located with the walks: exact steps, which
                               // skip the rescale work on the steps without one (fewest
                               // instructions, as they share issue slots with the walks)
    // kind 1 with split_D > 0: a split shadow, whose chain launch is
    // k_shadow_split (integer-difference head of class split_cls and depth
    // split_D, then the interpreted tail); the head's rows per warp
    uint32_t split_cls = 0, split_D = 0, split_rows_regs = 0, split_rows_per_warp = 0;
};

// Interpreted-shadow launch geometry shared by batches and serving waves:
// picks U and the per-warp rows of the evaluation kernel, the chain kernel's
// shared memory, and both grids.  Returns DR_OK or an error status.
// whole_sm: the chain blocks claim a whole SM's shared memory (batches,
// whose walks run beside them); serving waves request only what they use.
int shadow_interp_geometry(LaunchSpec& L, uint32_t max_dim, int sms, const DevShadowSeg* segs,
                           bool whole_sm = true, double walk_ns = 0.0);
// The chain launch geometry of a split shadow group (LaunchSpec::split_D).
int shadow_split_geometry(LaunchSpec& L, int sms);

// FP64 chain kernels (interpreted chain, integer-difference shadow) run as
// blocks of kChainWarps warps that claim a whole SM's shared memory, so no
// walk block shares their SM's issue slots; the grid is sized so the chains
// finish with the longest one.
constexpr int kChainWarps = 4;
// walk_ns: expected duration of the walk kernels running beside the chains
// (0: unknown); the chains get enough SMs to finish within the longer of it
// and their own longest chain, and no more.
// wpb: warps per chain block.
int chain_blocks(const DevShadowSeg* segs, uint32_t count, uint32_t m, double walk_ns = 0.0,
                 int wpb = kChainWarps);
// Whether chains this short next to the walks run best spread over all SMs
// beside the walk warps (one warp per block, no whole-SM claim): their
// longest chain, even slowed by sharing issue slots, ends well before the walks.
bool chain_colocate(const DevShadowSeg* segs, uint32_t count, uint32_t m, double walk_ns);
// FP64 chain step time (ns) of an m x m shadow, rescaling every step.
inline double chain_step_ns(uint32_t m) { return 75.0 * m * m; }
size_t chain_hog_smem();

// Builds the interpreted-shadow launches of one (m, shape) group (shape bit 0:
// companion-shaped float matrix, bit 1: state-vector walks):
// segs (sorted longest first) become one launch, or several rounds of at most
// `round_steps` steps with resident state slots from slot_base (round_steps =
// UINT64_MAX: one launch, the segments' own state slots).  Appends to list and
// eval_items and returns the doubles of step-matrix buffer the group needs
// (its segments' mf_off start at mf_base).
uint64_t shadow_interp_plan(std::vector<LaunchSpec>& launches, std::vector<DevShadowSeg>& list,
                            std::vector<uint32_t>& eval_items, const std::vector<DevShadowSeg>& segs,
                            uint32_t m, uint32_t shape, uint32_t rows_regs, uint64_t mf_base,
                            uint64_t round_steps, uint32_t slot_base);

struct Batch {
    int32_t id = 0;
    uint32_t n_walks = 0;
    uint64_t n_res = 0;
    uint64_t prime_steps = 0;
    std::vector<LaunchSpec> launches;
    uint32_t n_tiles = 0, n_groups = 0, n_queues = 0;
    uint32_t n_progs = 0, n_slots = 0;            // table sizes (DR_DEBUG bounds checks)
    uint64_t n_code = 0, n_consts = 0, n_axis = 0;
    DevBuf dbg;                                   // DR_DEBUG builds: first failed device check
    uint32_t chunk_stride = 0;   // words per chunk-product slot
    DevBuf tables;   // one copy of progs, code, consts, walks, axis, tiles, groups, shadow_list, eval_items
    DevBuf progs, code, consts, walks, axis, tiles, groups, group_done, chunkP, chunkSig;
    DevBuf shadow_list, queues, res, shadow, status;   // res: p residues then q residues
    DevBuf mf, eval_items, shadow_state;               // interpreted shadow
    // device pipeline (CRT -> delta -> top-k)
    dr_pipeline pipe{};
    bool pipe_on = false;
    int Lmax = 0;                       // limbs per reconstructed value
    struct CrtGroup { int K; uint32_t off, count; };
    std::vector<CrtGroup> crt_groups;
    DevBuf crt_in, crt_out, limbs, signs, delta, tgt_num, tgt_den, tgt_sign;
    DevBuf tk_keys[2], tk_idx[2];
    int bank_n = 0, bank_l = 0;          // constant bank scored after top-k
    DevBuf bank_num, bank_den, bank_sign, bank_out;
    std::vector<int> tk_counts;         // values entering each top-k pass
    int tk_final = 0;                   // buffer holding the final top-k
    std::vector<uint32_t> h_walk_K;
    std::vector<uint64_t> h_res_off, h_cp_off;
    cudaGraphExec_t graph = nullptr;
    uint32_t runs = 0;             // dr_batch_run calls so far (the first launches directly)
    uint32_t runs_read = 0;        // value of runs when a read last counted the device time
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr, join = nullptr;
    std::vector<cudaEvent_t> joins;
    std::vector<cudaEvent_t> evals;     // per launch: its step-matrix evaluation is done
    DevBuf tstamps;                     // diagnostics: 4 timestamps per launch
    bool stamping = false;
    DevBuf item_log;                    // diagnostics: per chain item of kind-2 launches
    std::vector<uint32_t> item_log_off; // first item of each launch in item_log
    std::vector<float> item_rows;       // last timeline's items (see dr_debug_chain_items)
    float last_ms = 0.f;
    bool has_shadow = false;
    std::string signature;              // autotuner cache key (workload shape)
    uint32_t chunk_used = 0, wpb_used = 0;
    Batch();
    ~Batch();
};

// Build a batch (validation, planning, upload).  engine_override forces an engine.
int batch_build(const dr_walk_desc* walks, int32_t n_walks, const uint8_t* blobs,
                const uint64_t* blob_offsets, int32_t n_programs, const int64_t* axis_params,
                uint64_t n_axis_params, const dr_tune* tune, uint64_t n_res,
                std::unique_ptr<Batch>* out);
int batch_run(Batch& B, cudaStream_t st);
int batch_read(Batch& B, uint32_t* p_res, uint32_t* q_res, uint64_t n_res, double* shadow,
               uint32_t* status);

int cuda_fail(cudaError_t e, const char* where);

struct ShadowArgs;
// Evaluation then chain launch of one interpreted-shadow launch group on s;
// sa carries the batch-wide pointers and this launch's segs / rows.
// evaluated: recorded on s between the two kernels when not null.
cudaError_t launch_shadow_interp(const LaunchSpec& L, ShadowArgs sa, uint32_t* queues,
                                 const uint32_t* eval_items, cudaStream_t s,
                                 cudaEvent_t evaluated = nullptr);

}  // namespace dr
