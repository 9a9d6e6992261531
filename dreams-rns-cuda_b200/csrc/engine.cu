// Host engine and the device-facing C ABI: context, prepared walk batches,
// CRT, delta and top-k entry points.
#include "engine.h"

#include <chrono>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "../../include/dreams_b200.h"
#include "../../include/dreams_b200_debug.h"
#include "debug_check.cuh"
#include "host_common.h"
#include "launch.h"
#include "shadow_impl.cuh"
#include "walk_impl.cuh"

namespace dr {


namespace {
Context* g_ctx = nullptr;
std::mutex g_init_mu;
std::mutex g_batch_mu;
std::map<int32_t, std::unique_ptr<Batch>> g_batches;
int32_t g_next_batch = 1;
}  // namespace

Context* ctx() { return g_ctx; }

int ensure_ctx() {
    if (!g_ctx) {
        set_error("dr_init has not been called");
        return DR_ERR_NOT_INIT;
    }
    cudaSetDevice(g_ctx->device);
    return DR_OK;
}

int cuda_fail(cudaError_t e, const char* where) {
    set_error(std::string(where) + ": " + cudaGetErrorString(e));
    cudaGetLastError();  // clear sticky-free errors so later calls can proceed
    return e == cudaErrorMemoryAllocation ? DR_ERR_NOMEM : DR_ERR_CUDA;
}

#define DR_CUDA(call)                                   \
    do {                                                \
        cudaError_t e__ = (call);                       \
        if (e__ != cudaSuccess) return cuda_fail(e__, #call); \
    } while (0)

int get_plan(const uint8_t* blob, uint64_t size, std::shared_ptr<Plan>* out, std::string* err) {
    // the cache is keyed by the blob's bytes; lookups hash them in place
    const std::string_view key(reinterpret_cast<const char*>(blob), (size_t)size);
    {
        std::shared_lock<std::shared_mutex> lk(g_ctx->plan_mu);
        auto it = g_ctx->plan_cache.find(key);
        if (it != g_ctx->plan_cache.end()) {
            *out = it->second;
            return DR_OK;
        }
    }
    RawProgram raw;
    auto plan = std::make_shared<Plan>();
    int rc = parse_blob(blob, size, &raw, err);
    if (rc == DR_OK) rc = plan_program(raw, plan.get(), err);
    if (rc != DR_OK) return rc;
    plan->fcomp = float_companion_shape(*plan);
    plan->blob.assign(key.data(), key.size());
    std::string code_key(sizeof(uint32_t) + sizeof(Insn) * (plan->ops.size() + plan->dops.size()), '\0');
    {
        const uint32_t n_ops = (uint32_t)plan->ops.size();
        char* q = &code_key[0];
        std::memcpy(q, &n_ops, sizeof n_ops);
        if (n_ops) std::memcpy(q + sizeof n_ops, plan->ops.data(), sizeof(Insn) * n_ops);
        if (!plan->dops.empty())
            std::memcpy(q + sizeof n_ops + sizeof(Insn) * n_ops, plan->dops.data(), sizeof(Insn) * plan->dops.size());
    }
    std::unique_lock<std::shared_mutex> lk(g_ctx->plan_mu);
    if (g_ctx->code_ids.size() > 100000) g_ctx->code_ids.clear();
    auto ci = g_ctx->code_ids.find(code_key);
    if (ci == g_ctx->code_ids.end()) ci = g_ctx->code_ids.emplace(std::move(code_key), g_ctx->next_code_id++).first;
    plan->code_id = ci->second;
    if (g_ctx->plan_cache.size() > 200000) g_ctx->plan_cache.clear();
    g_ctx->plan_cache.emplace(std::string_view(plan->blob), plan);
    *out = plan;
    return DR_OK;
}

HostPool::HostPool(int workers) {
    for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { worker(); });
}

HostPool::~HostPool() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
}

void HostPool::take_parts(const std::function<void(int, size_t, size_t)>* fn, int parts, size_t n) {
    for (;;) {
        const int p = next_.fetch_add(1);
        if (p >= parts) return;
        (*fn)(p, n * (size_t)p / (size_t)parts, n * (size_t)(p + 1) / (size_t)parts);
        std::lock_guard<std::mutex> lk(mu_);
        if (++done_ == parts) done_cv_.notify_all();
    }
}

void HostPool::worker() {
    uint64_t seen = 0;
    for (;;) {
        const std::function<void(int, size_t, size_t)>* fn;
        int parts;
        size_t n;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            // the job's fields stay as read here until active_ returns to 0
            fn = fn_;
            parts = fn ? parts_ : 0;
            n = n_;
            ++active_;
        }
        // a worker that woke after the job ended holds no job: it must not
        // touch the part counter, which the next job may already use
        if (fn) take_parts(fn, parts, n);
        std::lock_guard<std::mutex> lk(mu_);
        if (--active_ == 0) done_cv_.notify_all();
    }
}

void HostPool::run(int parts, size_t n, const std::function<void(int, size_t, size_t)>& fn) {
    std::lock_guard<std::mutex> one(run_mu_);
    {
        std::lock_guard<std::mutex> lk(mu_);
        fn_ = &fn;
        parts_ = parts;
        n_ = n;
        next_.store(0);
        done_ = 0;
        ++gen_;
    }
    cv_.notify_all();
    take_parts(&fn, parts, n);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return done_ == parts && active_ == 0; });
    fn_ = nullptr;
}

HostPool& host_pool() {
    static HostPool pool(std::max(1, std::min(7, (int)std::thread::hardware_concurrency() / 2 - 1)));
    return pool;
}

int crt_limbs_for(int K) { return (31 * K + 31) / 32 + 2; }

// standard: the moduli are the prime table's (distinct primes above 2^30),
// which the lane-per-value CRT kernel needs
static int build_crt_set(const uint32_t* moduli_host, int K, CrtSet& S, cudaStream_t st, bool standard) {
    S.K = K;
    S.L = crt_limbs_for(K);
    DR_CUDA(S.moduli.alloc(4ull * K));
    DR_CUDA(S.pinv.alloc(4ull * K));
    DR_CUDA(S.r2.alloc(4ull * K));
    DR_CUDA(S.ginv.alloc(4ull * K));
    DR_CUDA(S.Mlimbs.alloc(4ull * K * S.L));
    DR_CUDA(S.Mtotal.alloc(4ull * S.L));
    const bool lanes = standard && K <= kCrtLanesMaxK;
    if (lanes) DR_CUDA(S.garner.alloc(4ull * K * K));
    DR_CUDA(cudaMemcpyAsync(S.moduli.p, moduli_host, 4ull * K, cudaMemcpyHostToDevice, st));
    DR_CUDA(launch_crt_setup(S.moduli.as<uint32_t>(), K, S.L, S.pinv.as<uint32_t>(), S.r2.as<uint32_t>(),
                             S.ginv.as<uint32_t>(), S.Mlimbs.as<uint32_t>(), S.Mtotal.as<uint32_t>(),
                             lanes ? S.garner.as<uint32_t>() : nullptr, st));
    DR_CUDA(cudaStreamSynchronize(st));
    return DR_OK;
}

int crt_tables_std(int K, std::shared_ptr<CrtSet>* out) {
    {
        std::lock_guard<std::mutex> lk(g_ctx->mu);
        auto it = g_ctx->crt_std.find(K);
        if (it != g_ctx->crt_std.end()) {
            *out = it->second;
            return DR_OK;
        }
    }
    auto S = std::make_shared<CrtSet>();
    const auto& tab = prime_table(K);
    int rc = build_crt_set(tab.data(), K, *S, g_ctx->stream, true);
    if (rc != DR_OK) return rc;
    std::lock_guard<std::mutex> lk(g_ctx->mu);
    g_ctx->crt_std[K] = S;
    *out = S;
    return DR_OK;
}

void* devcache_take(size_t n, size_t* got) {
    Context* c = g_ctx;
    if (!c) return nullptr;
    std::lock_guard<std::mutex> lk(c->cache_mu);
    // smallest cached block that fits without wasting more than half of it
    auto it = c->cache.lower_bound(n);
    if (it == c->cache.end() || it->first > 2 * n + (1u << 20)) return nullptr;
    void* p = it->second;
    *got = it->first;
    c->cached_bytes -= it->first;
    c->cache.erase(it);
    return p;
}

void devcache_put(void* p, size_t bytes) {
    Context* c = g_ctx;
    constexpr size_t kCap = 8ull << 30;
    if (c) {
        std::lock_guard<std::mutex> lk(c->cache_mu);
        if (c->cached_bytes + bytes <= kCap) {
            c->cache.emplace(bytes, p);
            c->cached_bytes += bytes;
            return;
        }
    }
    cudaFree(p);
}

Batch::Batch() {
    for (DevBuf* b : {&tables, &progs, &code, &consts, &walks, &axis, &tiles, &groups, &group_done, &chunkP,
                      &chunkSig, &shadow_list, &queues, &res, &shadow, &status, &mf, &eval_items,
                      &shadow_state, &tstamps, &crt_in, &crt_out, &limbs, &signs, &delta, &tgt_num,
                      &tgt_den, &tgt_sign, &tk_keys[0], &tk_keys[1], &tk_idx[0], &tk_idx[1],
                      &bank_num, &bank_den, &bank_sign, &bank_out})
        b->pooled = true;
}

Batch::~Batch() {
    // pooled buffers go back to the cache: no work of this batch may remain
    if (g_ctx) cudaStreamSynchronize(g_ctx->stream);
    if (graph) cudaGraphExecDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    for (cudaEvent_t e : joins) cudaEventDestroy(e);
}

// ---- batch construction ---------------------------------------------------------

namespace {

struct LaunchKey {
    int kind;
    uint32_t cls, m, D;
    bool operator<(const LaunchKey& o) const {
        return std::tie(kind, cls, m, D) < std::tie(o.kind, o.cls, o.m, o.D);
    }
};

// Appends v to out longest first, keeping the input order among equal lengths
// (a stable sort).  Tile lengths usually take a handful of values, which a
// counting sort places in two passes over v; more than 64 distinct lengths
// fall back to std::stable_sort.  Lengths within 1/64 of each other (equal
// splits of equal depths) are appended as they are: the order only balances
// the queue's tail, and there it changes nothing.  (Skipping the sort for
// lengths within a factor of two, a checkpoint's shorter chunks among the
// others, made the benchmark's walk kernels 2% slower.)
template <class T, class Len>
static void append_longest_first(std::vector<T>& out, std::vector<T>& v, Len len) {
    constexpr uint32_t kMaxKeys = 64;
    uint64_t lo = UINT64_MAX, hi = 0;
    for (const T& t : v) {
        const uint64_t l = len(t);
        lo = std::min(lo, l);
        hi = std::max(hi, l);
    }
    if (v.empty() || hi - lo <= hi / 64) {
        out.insert(out.end(), v.begin(), v.end());
        return;
    }
    uint64_t keys[kMaxKeys];
    uint32_t nk = 0, last = 0;
    for (const T& t : v) {
        const uint64_t l = len(t);
        if (nk && keys[last] == l) continue;
        uint32_t k = 0;
        while (k < nk && keys[k] != l) ++k;
        if (k == nk) {
            if (nk == kMaxKeys) {
                std::stable_sort(v.begin(), v.end(), [&](const T& x, const T& y) { return len(x) > len(y); });
                out.insert(out.end(), v.begin(), v.end());
                return;
            }
            keys[nk++] = l;
        }
        last = k;
    }
    if (nk <= 1) {
        out.insert(out.end(), v.begin(), v.end());
        return;
    }
    std::sort(keys, keys + nk, [](uint64_t x, uint64_t y) { return x > y; });
    std::vector<uint8_t> kidx(v.size());
    size_t count[kMaxKeys] = {0};
    last = 0;
    for (size_t i = 0; i < v.size(); ++i) {
        const uint64_t l = len(v[i]);
        if (keys[last] != l) {
            last = 0;
            while (keys[last] != l) ++last;
        }
        kidx[i] = (uint8_t)last;
        ++count[last];
    }
    size_t pos[kMaxKeys];
    size_t acc = out.size();
    for (uint32_t k = 0; k < nk; ++k) { pos[k] = acc; acc += count[k]; }
    out.resize(acc);
    for (size_t i = 0; i < v.size(); ++i) out[pos[kidx[i]]++] = v[i];
}

template <class T>
int upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
    DR_CUDA(b.alloc(sizeof(T) * std::max<size_t>(v.size(), 1)));
    if (!v.empty()) DR_CUDA(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
    return DR_OK;
}

uint32_t chunk_policy(uint64_t total_group_steps, uint64_t n_groups, int sms, const dr_tune* tune) {
    if (tune && tune->chunk_steps) return tune->chunk_steps;
    // aim for ~6 tiles per resident warp slot (24 per SM) so the longest-first
    // queue balances, with chunks no shorter than 256 steps
    const double target_tiles = (double)sms * 24.0 * 6.0;
    double c = (double)total_group_steps / target_tiles;
    if (n_groups > target_tiles) c = 1e18;  // enough groups already: one chunk each
    c = std::max(c, 256.0);
    c = std::min(c, 4194304.0);
    return (uint32_t)c;
}

}  // namespace

// host time of the phases of the last batch_build (diagnostics): plan
// lookup, descriptors, code copy, walks, workload shape, tile count, tile
// fill, tile order, shadow lists, geometry, table copy, buffers and
// events, final sync
constexpr int kBuildPhases = 13;
// (per thread: batches may be built on several threads at once)
static thread_local double g_build_ms[kBuildPhases];
static thread_local std::chrono::steady_clock::time_point g_build_t0;
static void build_mark(int i) {
    const auto t = std::chrono::steady_clock::now();
    if (i == 0) g_build_t0 = t;
    else g_build_ms[i - 1] = std::chrono::duration<double, std::milli>(t - g_build_t0).count();
}

// Split shadows: walks with at least this many integer-exact head steps (and
// twice as many in all) run the head on integer differences.
// DREAMS_B200_SPLIT_SHADOW=0 turns it off (every such walk then takes the
// interpreted shadow).
constexpr uint64_t kSplitMin = 256;
static bool split_shadow_on() {
    static const bool on = [] {
        const char* v = std::getenv("DREAMS_B200_SPLIT_SHADOW");
        return !(v && v[0] == '0');
    }();
    return on;
}

// Host-pool use in batch construction: parts for n items (one part below
// kPoolMin items; about kPoolGrain items per part otherwise).
constexpr size_t kPoolMin = 1024, kPoolGrain = 512;
static int build_parts(size_t n) {
    if (n < kPoolMin) return 1;
    return (int)std::min<size_t>((size_t)host_pool().threads() * 2, (n + kPoolGrain - 1) / kPoolGrain);
}
// First error of a part (item index, status, message); the lowest index wins.
struct BuildErr {
    int64_t at = -1;
    int rc = DR_OK;
    std::string msg;
};
static int first_error(const std::vector<BuildErr>& e) {
    const BuildErr* best = nullptr;
    for (const BuildErr& x : e)
        if (x.at >= 0 && (!best || x.at < best->at)) best = &x;
    if (!best) return DR_OK;
    set_error(best->msg);
    return best->rc;
}

int batch_build(const dr_walk_desc* walks, int32_t n_walks, const uint8_t* blobs,
                const uint64_t* blob_offsets, int32_t n_programs, const int64_t* axis,
                uint64_t n_axis, const dr_tune* tune, uint64_t n_res, std::unique_ptr<Batch>* out) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Context& C = *g_ctx;
    if (n_walks < 0 || n_programs < 0 || (n_walks > 0 && (!walks || !blob_offsets || !blobs))) {
        set_error("null walk or program arrays");
        return DR_ERR_ARG;
    }
    const uint32_t engine = tune ? tune->engine : DR_ENGINE_AUTO;
    auto B = std::make_unique<Batch>();
    B->n_walks = (uint32_t)n_walks;
    B->n_res = n_res;
    build_mark(0);
    NvtxRange nvtx_build("dr.build");
    const auto t_build0 = std::chrono::steady_clock::now();

    // ---- programs
    std::vector<std::shared_ptr<Plan>> plans(n_programs);
    std::vector<DevProgram> dprogs(n_programs);
    std::vector<uint4> code;
    std::vector<int64_t> consts;

    std::unordered_map<uint32_t, std::pair<uint32_t, uint32_t>> code_at;   // code_id -> (op_off, dop_off)
    uint32_t last_code_id = 0;
    std::pair<uint32_t, uint32_t> last_code_at{0, 0};
    // plans on the host pool (parts in program order; the first failing
    // program is reported, as a serial pass would)
    {
        const int parts = build_parts(n_programs);
        std::vector<BuildErr> perr(parts);
        auto plan_range = [&](int part, size_t lo, size_t hi) {
            for (size_t i = lo; i < hi; ++i)
                if (blob_offsets[i + 1] < blob_offsets[i]) {
                    perr[part] = {(int64_t)i, DR_ERR_ARG, "blob_offsets not increasing"};
                    hi = i;
                    break;
                }
            {
                // cached plans under one shared lock per part
                std::shared_lock<std::shared_mutex> lk(C.plan_mu);
                for (size_t i = lo; i < hi; ++i) {
                    const std::string_view key(reinterpret_cast<const char*>(blobs + blob_offsets[i]),
                                               (size_t)(blob_offsets[i + 1] - blob_offsets[i]));
                    auto it = C.plan_cache.find(key);
                    if (it != C.plan_cache.end()) plans[i] = it->second;
                }
            }
            for (size_t i = lo; i < hi; ++i) {
                if (plans[i]) continue;
                std::string err;
                const int r = get_plan(blobs + blob_offsets[i], blob_offsets[i + 1] - blob_offsets[i],
                                       &plans[i], &err);
                if (r) {
                    if (perr[part].at < 0 || (int64_t)i < perr[part].at)
                        perr[part] = {(int64_t)i, r, "program " + std::to_string(i) + ": " + err};
                    return;
                }
            }
        };
        if (parts > 1) host_pool().run(parts, (size_t)n_programs, plan_range);
        else plan_range(0, 0, (size_t)n_programs);
        if ((rc = first_error(perr))) return rc;
    }
    build_mark(1);
    // descriptors and offsets (serial, cheap); programs with the same
    // instruction streams share one copy of them
    std::vector<uint8_t> copy_code(n_programs, 0);     // first program of its code_id
    size_t code_total = 0, consts_total = 0;
    for (int32_t i = 0; i < n_programs; ++i) {
        const Plan& P = *plans[i];
        DevProgram d{};
        d.m = P.m;
        d.dim = P.dim;
        // AUTO and PLAIN run the planned class; INTERP forces the interpreter
        d.cls = (engine == DR_ENGINE_INTERP) ? (uint32_t)CLS_INTERP : (uint32_t)P.cls;
        d.degree = P.degree;
        if (P.code_id != last_code_id) {
            auto at = code_at.find(P.code_id);
            if (at == code_at.end()) {
                std::pair<uint32_t, uint32_t> off((uint32_t)code_total, (uint32_t)(code_total + P.ops.size()));
                code_total += P.ops.size() + P.dops.size();
                copy_code[i] = 1;
                at = code_at.emplace(P.code_id, off).first;
            }
            last_code_id = P.code_id;
            last_code_at = at->second;
        }
        d.op_off = last_code_at.first;
        d.n_ops = (uint32_t)P.ops.size();
        d.n_regs = P.n_regs;
        d.dop_off = last_code_at.second;
        d.dn_ops = (uint32_t)P.dops.size();
        d.dn_regs = P.dn_regs;
        d.c_off = (uint32_t)consts_total;
        d.n_consts = (uint32_t)P.consts.size();
        consts_total += P.consts.size();
        d.n_streams = P.n_streams;
        d.zero_reg = P.zero_reg;
        d.shadow_fd = (!P.has_inv && (P.cls == CLS_COMPANION || P.cls == CLS_DENSE)) ? 1u : 0u;
        d.fcomp = P.fcomp ? 1u : 0u;
        dprogs[i] = d;
    }
    if (code_total > UINT32_MAX || consts_total > UINT32_MAX) {
        set_error("programs too large: more than 2^32 instructions or constants");
        return DR_ERR_UNSUPPORTED;
    }
    build_mark(2);
    // the instruction streams (Insn and uint4 are both four 32-bit words) and
    // constants, copied on the host pool
    static_assert(sizeof(Insn) == sizeof(uint4), "instruction layout");
    code.resize(std::max<size_t>(code_total, 1));
    consts.resize(std::max<size_t>(consts_total, 1));
    {
        auto copy_range = [&](int, size_t lo, size_t hi) {
            for (size_t i = lo; i < hi; ++i) {
                const Plan& P = *plans[i];
                const DevProgram& d = dprogs[i];
                if (copy_code[i]) {
                    if (!P.ops.empty()) std::memcpy(&code[d.op_off], P.ops.data(), sizeof(Insn) * P.ops.size());
                    if (!P.dops.empty()) std::memcpy(&code[d.dop_off], P.dops.data(), sizeof(Insn) * P.dops.size());
                }
                if (!P.consts.empty())
                    std::memcpy(&consts[d.c_off], P.consts.data(), sizeof(int64_t) * P.consts.size());
            }
        };
        const int parts = build_parts(n_programs);
        if (parts > 1) host_pool().run(parts, (size_t)n_programs, copy_range);
        else copy_range(0, 0, (size_t)n_programs);
    }

    build_mark(3);
    // ---- walks
    std::vector<DevWalk> dwalks(n_walks);
    // split shadow: the head length of walks whose float intermediates are
    // integer-exact only over their first steps (0: not split)
    std::vector<uint64_t> split_at(n_walks, 0);
    const bool split_shadow = split_shadow_on();
    uint64_t total_group_steps = 0, n_groups = 0;
    std::map<LaunchKey, std::pair<uint64_t, uint64_t>> shape;   // workload shape, merged from the parts
    uint64_t longest = 0;
    {
        // validation and device descriptors on the host pool; per-part sums
        struct WalkAcc {
            uint64_t group_steps = 0, groups = 0, prime_steps = 0;
            bool shadow = false;
            // workload shape (see below): per launch key, (walk, prime block)
            // count and their steps, and the longest walk
            std::map<LaunchKey, std::pair<uint64_t, uint64_t>> shape;
            uint64_t longest = 0;
        };
        const int parts = build_parts((size_t)n_walks);
        std::vector<BuildErr> perr(parts);
        std::vector<WalkAcc> accs(parts);
        auto walk_range = [&](int part, size_t w_lo, size_t w_hi) {
            WalkAcc& acc = accs[part];
            LaunchKey shape_prev{-1, 0, 0, 0};
            std::pair<uint64_t, uint64_t>* shape_cur = nullptr;
            for (size_t wi = w_lo; wi < w_hi; ++wi) {
                const int32_t w = (int32_t)wi;
                auto fail = [&](int code, const char* msg) { perr[part] = {(int64_t)w, code, msg}; };
                const dr_walk_desc& W = walks[w];
                if (W.program >= (uint32_t)n_programs) { fail(DR_ERR_ARG, "walk program index out of range"); return; }
                const DevProgram& G = dprogs[W.program];
                if (W.K < 1 || W.K > DR_MAX_K) { fail(DR_ERR_UNSUPPORTED, "K outside 1..DR_MAX_K"); return; }
                if (W.q_row >= G.m || W.p_row >= G.m) { fail(DR_ERR_ARG, "p_row or q_row >= m"); return; }
                if (W.flags & DR_WALK_VEC) {
                    if (W.flags & DR_WALK_INIT_PCF) {
                        fail(DR_ERR_ARG, "a state-vector walk starts from v(0), not the PCF initial matrix"); return;
                    }
                    if (W.checkpoint) { fail(DR_ERR_UNSUPPORTED, "state-vector walks have no checkpoint"); return; }
                    if (W.vec_offset + (uint64_t)G.m * W.K + G.m > n_axis) {
                        fail(DR_ERR_ARG, "state-vector initial values out of range of the axis parameters"); return;
                    }
                }
                if (W.checkpoint && W.checkpoint >= W.depth) { fail(DR_ERR_ARG, "checkpoint must be < depth"); return; }
                if ((W.flags & DR_WALK_INIT_PCF) && G.m < 2) {
                    fail(DR_ERR_ARG, "PCF initial matrix needs m >= 2");
                    return;
                }
                if (W.res_offset + W.K > n_res || (W.checkpoint && W.cp_res_offset + W.K > n_res)) {
                    fail(DR_ERR_ARG, "residue output offset out of range"); return;
                }
                if (W.axis_offset + 4ull * G.dim > n_axis) { fail(DR_ERR_ARG, "axis parameters out of range"); return; }
                if (W.depth > (1ull << 40)) { fail(DR_ERR_UNSUPPORTED, "depth above 2^40"); return; }
                for (uint32_t a = 0; a < G.dim; ++a) {
                    const int64_t* ax = axis + W.axis_offset + 4 * a;
                    if (ax[1] == 0 || ax[3] == 0) {
                        // the reference divides by float(sd*td) (cmf_walk.py:281): ZeroDivisionError
                        fail(DR_ERR_ARG, "zero shift or trajectory denominator"); return;
                    }
                    const __int128 hi = (__int128)ax[0] * ax[3];
                    const __int128 st = (__int128)ax[2] * ax[1];
                    const __int128 lim = (__int128)1 << 62;
                    const __int128 span = st * (__int128)(W.depth + 64);
                    if (hi > lim || hi < -lim || span > lim || span < -lim || (__int128)ax[1] * ax[3] > lim ||
                        (__int128)ax[1] * ax[3] < -lim) {
                        fail(DR_ERR_UNSUPPORTED, "axis numerators exceed 2^62 over the walk"); return;
                    }
                }
                DevWalk d{};
                d.prog = W.program;
                d.K = W.K;
                d.flags = W.flags;
                d.q_row = W.q_row;
                d.a0 = W.a0;
                d.depth = W.depth;
                d.checkpoint = W.checkpoint;
                d.axis_off = W.axis_offset;
                d.res_off = W.res_offset;
                d.cp_res_off = W.cp_res_offset;
                d.p_row = W.p_row;
                d.vec_off = W.vec_offset;
                d.shadow_mode = SHADOW_NONE;
                if (W.flags & DR_WALK_SHADOW) {
                    d.shadow_mode = SHADOW_INTERP;
                    const Plan& P = *plans[W.program];
                    const int Dt = template_degree(P.cls, P.m, P.degree);
                    if (G.shadow_fd && G.cls != CLS_INTERP && Dt > 0 && !(W.flags & DR_WALK_VEC)) {
                        const int64_t* ax = axis + W.axis_offset;
                        auto exact_to = [&](uint64_t steps) {   // integer-exact float intermediates over [0, steps)
                            const double b = float_bound_log2(P, ax, steps + 1);
                            return b < 53.0 && b + Dt < 61.0;
                        };
                        if (exact_to(W.depth)) {
                            d.shadow_mode = SHADOW_INTFD;
                        } else if (split_shadow && G.fcomp && shadow_split_supported(G.cls, G.m, (uint32_t)Dt) &&
                                   W.depth >= 2 * kSplitMin && exact_to(kSplitMin)) {
                            // exact over a head of the walk: the split shadow
                            // runs the head on integer differences (the bound
                            // is monotone in the step count; 8 halvings place
                            // the head within depth/256 of the largest)
                            uint64_t lo = kSplitMin, hi = W.depth;
                            for (int it = 0; it < 8 && hi - lo > 32; ++it) {
                                const uint64_t mid = lo + (hi - lo) / 2;
                                if (exact_to(mid)) lo = mid;
                                else hi = mid;
                            }
                            split_at[w] = lo;
                        }
                    }
                    acc.shadow = true;
                }
                dwalks[w] = d;
                const uint64_t nb = (W.K + 31) / 32;
                acc.group_steps += nb * std::max<uint64_t>(W.depth, 1);
                acc.groups += nb;
                acc.prime_steps += (uint64_t)W.K * W.depth;
                {
                    const Plan& P = *plans[W.program];
                    LaunchKey key{0, G.cls, G.m, 0};
                    if (G.cls != CLS_INTERP) key.D = (uint32_t)template_degree(P.cls, P.m, P.degree);
                    if (!shape_cur || key < shape_prev || shape_prev < key) {
                        shape_cur = &acc.shape[key];
                        shape_prev = key;
                    }
                    shape_cur->first += nb;
                    shape_cur->second += nb * W.depth;
                    acc.longest = std::max<uint64_t>(acc.longest, W.depth);
                }
            }
        };
        if (parts > 1) host_pool().run(parts, (size_t)n_walks, walk_range);
        else walk_range(0, 0, (size_t)n_walks);
        if ((rc = first_error(perr))) return rc;
        for (const WalkAcc& a : accs) {
            total_group_steps += a.group_steps;
            n_groups += a.groups;
            B->prime_steps += a.prime_steps;
            B->has_shadow |= a.shadow;
            for (const auto& kv : a.shape) {
                auto& e = shape[kv.first];
                e.first += kv.second.first;
                e.second += kv.second.second;
            }
            longest = std::max(longest, a.longest);
        }
    }

    build_mark(4);
    // ---- tiles and groups
    const bool plain = engine == DR_ENGINE_PLAIN;
    // workload shape for the autotuner: per launch key, log2 buckets of the
    // (walk, prime block) count and of their steps, plus the longest walk
    // (summed per part in the walk pass above)
    {
        auto lg = [](uint64_t v) { int b = 0; while (v > 1) { v >>= 1; ++b; } return b; };
        std::string sig = std::to_string(lg(longest)) + (B->has_shadow ? "s" : "n");
        for (auto& kv : shape)
            sig += "|" + std::to_string(kv.first.cls) + "," + std::to_string(kv.first.m) + "," +
                   std::to_string(kv.first.D) + ":" + std::to_string(lg(kv.second.first)) + "," +
                   std::to_string(lg(kv.second.second));
        B->signature = sig;
    }
    build_mark(5);
    // an autotuned choice for this shape applies unless the caller fixed one
    uint32_t tuned_chunk = 0, tuned_wpb = 0, tuned_pack = 0;
    if (!plain && !(tune && (tune->chunk_steps || tune->warps_per_block))) {
        std::lock_guard<std::mutex> lk(C.cache_mu);
        auto it = C.tuned.find(B->signature);
        if (it != C.tuned.end()) {
            tuned_chunk = it->second.chunk;
            tuned_wpb = it->second.wpb;
            tuned_pack = it->second.pack;
        }
    }
    const uint32_t chain_pack = (tune && tune->chain_pack_depth) ? tune->chain_pack_depth : tuned_pack;
    const uint32_t chunk = plain ? 0xffffffffu
                         : tuned_chunk ? tuned_chunk
                         : chunk_policy(total_group_steps, n_groups, C.sms, tune);
    B->chunk_used = chunk;
    // Tiles and combine groups in walk order, on the host pool: a counting
    // pass gives every part its offsets in the tile set of each launch class,
    // in the group array and in the chunk slots, so each part writes its
    // tiles in place with their final indices (the arrays one pass over the
    // walks would give).
    auto walk_key = [&](const DevWalk& W) {
        const DevProgram& G = dprogs[W.prog];
        const Plan& P = *plans[W.prog];
        LaunchKey key{0, G.cls, G.m, 0};
        if (G.cls != CLS_INTERP) key.D = (uint32_t)template_degree(P.cls, P.m, P.degree);
        return key;
    };
    auto n_chunks_of = [&](const DevWalk& W) -> uint64_t {   // the ranges split() makes
        auto nc = [&](uint64_t len) { return std::max<uint64_t>(1, (len + chunk - 1) / chunk); };
        if (W.depth == 0) return 1;
        if (W.checkpoint) return nc(W.checkpoint) + nc(W.depth - W.checkpoint);
        return nc(W.depth);
    };
    // per launch: the most registers, constants and axes of its programs
    // (the rows of its per-warp shared memory)
    struct Rows {
        uint32_t regs = 1, consts = 1, axes = 1;
        void merge(const Rows& o) {
            regs = std::max(regs, o.regs);
            consts = std::max(consts, o.consts);
            axes = std::max(axes, o.axes);
        }
    };
    struct TileCount {
        std::map<LaunchKey, size_t> tiles;   // count, then this part's first index in the set
        std::map<LaunchKey, Rows> rows;
        uint64_t groups = 0, slots = 0;      // count, then this part's first group / slot
    };
    const int tparts = build_parts((size_t)n_walks);
    std::vector<TileCount> tcount(tparts);
    auto count_range = [&](int part, size_t w_lo, size_t w_hi) {
        TileCount& T = tcount[part];
        LaunchKey prev{-1, 0, 0, 0};
        size_t* cur = nullptr;
        Rows* rows = nullptr;
        for (size_t w = w_lo; w < w_hi; ++w) {
            const DevWalk& W = dwalks[w];
            const LaunchKey key = walk_key(W);
            if (!cur || key < prev || prev < key) {
                cur = &T.tiles[key];
                rows = &T.rows[key];
                prev = key;
            }
            const DevProgram& G = dprogs[W.prog];
            rows->merge(Rows{std::max(G.n_regs, G.dn_regs), G.n_consts, G.dim});
            const uint64_t nb = (W.K + 31) / 32, nc = n_chunks_of(W);
            *cur += nb * nc;
            T.groups += nb;
            if (nc > 1) T.slots += nb * nc;
        }
    };
    if (tparts > 1) host_pool().run(tparts, (size_t)n_walks, count_range);
    else count_range(0, 0, (size_t)n_walks);
    build_mark(6);
    std::map<LaunchKey, std::vector<DevTile>> tile_sets;
    std::map<LaunchKey, Rows> key_rows;
    uint64_t n_group_total = 0, slots64 = 0;
    {
        std::map<LaunchKey, size_t> total;
        for (const TileCount& T : tcount)
            for (const auto& kv : T.rows) key_rows[kv.first].merge(kv.second);
        for (TileCount& T : tcount) {
            for (auto& kv : T.tiles) {
                const size_t c = kv.second;
                kv.second = total[kv.first];
                total[kv.first] += c;
            }
            const uint64_t g = T.groups, sl = T.slots;
            T.groups = n_group_total;
            T.slots = slots64;
            n_group_total += g;
            slots64 += sl;
        }
        for (const auto& kv : total) tile_sets[kv.first].resize(kv.second);
    }
    if (slots64 > UINT32_MAX || n_group_total > UINT32_MAX) {
        set_error("batch too large: more than 2^32 chunk slots or groups");
        return DR_ERR_UNSUPPORTED;
    }
    std::vector<DevGroup> groups(n_group_total);
    const uint32_t slots = (uint32_t)slots64;
    auto fill_range = [&](int part, size_t w_lo, size_t w_hi) {
        TileCount& T = tcount[part];
        std::vector<std::pair<uint64_t, uint64_t>> ranges;
        LaunchKey prev{-1, 0, 0, 0};
        DevTile* out = nullptr;      // next tile of prev's set
        size_t* cursor = nullptr;
        uint32_t gi = (uint32_t)T.groups, slot = (uint32_t)T.slots;
        for (size_t w = w_lo; w < w_hi; ++w) {
            const DevWalk& W = dwalks[w];
            const LaunchKey key = walk_key(W);
            if (!cursor || key < prev || prev < key) {
                // find (not operator[]) on the shared map: safe beside the other parts
                if (cursor) *cursor = (size_t)(out - tile_sets.find(prev)->second.data());
                cursor = &T.tiles.find(key)->second;
                out = tile_sets.find(key)->second.data() + *cursor;
                prev = key;
            }
            // chunk boundaries; a checkpoint always ends a chunk
            ranges.clear();
            auto split = [&](uint64_t a, uint64_t b) {
                const uint64_t len = b - a;
                const uint64_t nc = std::max<uint64_t>(1, (len + chunk - 1) / chunk);
                for (uint64_t c = 0; c < nc; ++c)
                    ranges.emplace_back(a + len * c / nc, a + len * (c + 1) / nc);
            };
            if (W.depth == 0) ranges.emplace_back(0, 0);
            else if (W.checkpoint) { split(0, W.checkpoint); split(W.checkpoint, W.depth); }
            else split(0, W.depth);
            uint32_t cp_chunks = 0;
            if (W.checkpoint)
                for (auto& r : ranges) cp_chunks += r.second <= W.checkpoint;
            for (uint32_t p0 = 0; p0 < W.K; p0 += 32) {
                DevGroup g{};
                g.walk = (uint32_t)w;
                g.prime0 = p0;
                g.nprimes = std::min<uint32_t>(32, W.K - p0);
                g.n_chunks = (uint32_t)ranges.size();
                g.cp_chunks = cp_chunks;
                g.slot0 = g.n_chunks > 1 ? slot : 0;
                g.state = kNoState;
                g.flags = 0;
                if (g.n_chunks > 1) slot += g.n_chunks;
                groups[gi] = g;
                for (uint32_t c = 0; c < g.n_chunks; ++c) {
                    DevTile& t = *out++;
                    t = DevTile{};
                    t.walk = (uint32_t)w;
                    t.group = gi;
                    t.prime0 = p0;
                    t.nprimes = g.nprimes;
                    t.chunk = c;
                    t.slot = g.slot0 + c;
                    t.s0 = ranges[c].first;
                    t.s1 = ranges[c].second;
                }
                ++gi;
            }
        }
    };
    if (tparts > 1) host_pool().run(tparts, (size_t)n_walks, fill_range);
    else fill_range(0, 0, (size_t)n_walks);
    build_mark(7);
    size_t n_tiles_est = 0;
    for (auto& kv : tile_sets) n_tiles_est += kv.second.size();
    std::vector<DevTile> tiles;
    tiles.reserve(n_tiles_est);
    for (auto& kv : tile_sets) {
        auto& v = kv.second;
        LaunchSpec L{};
        L.kind = 0;
        L.cls = kv.first.cls;
        L.m = kv.first.m;
        L.D = kv.first.D;
        L.off = (uint32_t)tiles.size();
        L.count = (uint32_t)v.size();
        L.items = L.count;
        const Rows& kr = key_rows[kv.first];
        const uint32_t ns = (uint32_t)std::max(streams_for(L.cls, L.m), 0);
        L.rows_regs = kr.regs;
        L.rows_consts = kr.consts;
        L.rows_axes = std::min<uint32_t>(std::max<uint32_t>(kr.axes, 1), kMaxAxes);
        L.rows_stage = std::max(L.m * L.m, (L.D + 1) * ns);
        L.rows_per_warp = L.rows_regs + L.rows_consts + 3 * L.rows_axes + L.rows_stage;
        append_longest_first(tiles, v, [](const DevTile& t) { return t.s1 - t.s0; });
        B->launches.push_back(L);
    }
    B->n_tiles = (uint32_t)tiles.size();
    B->n_groups = (uint32_t)groups.size();

    build_mark(8);
    // ---- shadow work lists
    std::map<LaunchKey, std::vector<uint32_t>> shadow_sets;
    {
        LaunchKey prev{-1, 0, 0, 0};
        std::vector<uint32_t>* set = nullptr;   // shadow set of prev
        for (int32_t w = 0; w < n_walks; ++w) {
            const DevWalk& W = dwalks[w];
            if (W.shadow_mode == SHADOW_NONE) continue;
            const DevProgram& G = dprogs[W.prog];
            const Plan& P = *plans[W.prog];
            // kind 0 here: split shadows (integer-difference head, interpreted tail)
            const LaunchKey key = W.shadow_mode == SHADOW_INTFD
                ? LaunchKey{2, P.cls, P.m, (uint32_t)template_degree(P.cls, P.m, P.degree)}
                : split_at[w] ? LaunchKey{0, P.cls, P.m, (uint32_t)template_degree(P.cls, P.m, P.degree)}
                : LaunchKey{1, G.fcomp | ((W.flags & DR_WALK_VEC) ? 2u : 0u), G.m, 0};
            if (!set || key < prev || prev < key) {
                set = &shadow_sets[key];
                prev = key;
            }
            set->push_back((uint32_t)w);
        }
    }
    std::vector<DevShadowSeg> shadow_list;
    std::vector<uint32_t> eval_items;
    uint64_t mf_doubles = 0;
    uint32_t state_slots = 0;
    const uint64_t cap_doubles =
        (uint64_t)((tune && tune->shadow_buffer_mb) ? tune->shadow_buffer_mb : 2048) << 17;
    uint32_t max_dim = 1;
    for (auto& d : dprogs) max_dim = std::max(max_dim, d.dim);
    for (auto& kv : shadow_sets) {
        auto& v = kv.second;
        if (kv.first.kind == 0) {
            // split shadows: walks by head length, shortest first (the longest
            // items first); an item switches at its shortest head
            std::stable_sort(v.begin(), v.end(), [&](uint32_t a, uint32_t b) { return split_at[a] < split_at[b]; });
            uint32_t rr_eval = 1, rr_head = 1;
            uint64_t need = 0;
            std::vector<DevShadowSeg> segs;
            segs.reserve(v.size());
            for (size_t k = 0; k < v.size(); ++k) {
                const uint32_t w = v[k];
                const DevProgram& G = dprogs[dwalks[w].prog];
                rr_eval = std::max(rr_eval, G.n_regs);
                rr_head = std::max(rr_head, G.dn_regs);
                const uint64_t sw = split_at[v[k / 32 * 32]];
                segs.push_back(DevShadowSeg{w, kNoState, sw, dwalks[w].depth, 0, 0, 0});
                need += (dwalks[w].depth - sw) * shadow_entries(kv.first.m, true);
            }
            if (need > cap_doubles) {
                // the tails' step matrices would not fit: interpreted shadows
                const DevProgram& G0 = dprogs[dwalks[v[0]].prog];
                auto& interp = shadow_sets[LaunchKey{1, G0.fcomp, kv.first.m, 0}];
                interp.insert(interp.end(), v.begin(), v.end());
                continue;
            }
            const size_t l0 = B->launches.size();
            mf_doubles += shadow_interp_plan(B->launches, shadow_list, eval_items, segs, kv.first.m, 1u, rr_eval,
                                             mf_doubles, UINT64_MAX, state_slots);
            for (size_t i = l0; i < B->launches.size(); ++i) {
                B->launches[i].split_cls = kv.first.cls;
                B->launches[i].split_D = kv.first.D;
                B->launches[i].split_rows_regs = rr_head;
            }
            continue;
        }
        auto deeper = [&](uint32_t a, uint32_t b) { return dwalks[a].depth > dwalks[b].depth; };
        if (!std::is_sorted(v.begin(), v.end(), deeper)) std::stable_sort(v.begin(), v.end(), deeper);
        uint32_t rr = 1;
        for (uint32_t w : v) {
            const DevProgram& G = dprogs[dwalks[w].prog];
            rr = std::max(rr, kv.first.kind == 1 ? G.n_regs : G.dn_regs);
        }
        if (kv.first.kind == 1) {
            // interpreted: the step-matrix buffer holds every step of every
            // walk when it fits under the cap, else the walks run in rounds
            const uint32_t ne = shadow_entries(kv.first.m, (kv.first.cls & 1u) != 0);
            uint64_t need = 0;
            for (uint32_t w : v) need += dwalks[w].depth * ne;
            uint64_t round = UINT64_MAX;
            if (need > cap_doubles) {
                round = cap_doubles / ((uint64_t)v.size() * ne);
                round = std::max<uint64_t>(kEvalSteps, round / kEvalSteps * kEvalSteps);
            }
            std::vector<DevShadowSeg> segs;
            for (uint32_t w : v) segs.push_back(DevShadowSeg{w, kNoState, 0, dwalks[w].depth, 0, 0, 0});
            mf_doubles += shadow_interp_plan(B->launches, shadow_list, eval_items, segs, kv.first.m,
                                             kv.first.cls, rr, mf_doubles, round, state_slots);
            if (round != UINT64_MAX) state_slots += (uint32_t)v.size();
            continue;
        }
        LaunchSpec L{};
        L.kind = 2;
        L.cls = kv.first.cls;
        L.m = kv.first.m;
        L.D = kv.first.D;
        L.off = (uint32_t)shadow_list.size();
        L.count = (uint32_t)v.size();
        L.items = (L.count + 31) / 32;
        L.rows_regs = rr;
        const uint32_t ns = (uint32_t)streams_for(L.cls, L.m);
        L.rows_per_warp = rr + kMaxAxes + (L.D + 1) * ns + ns;
        for (uint32_t w : v) shadow_list.push_back(DevShadowSeg{w, kNoState, 0, dwalks[w].depth, 0, 0, 0});
        B->launches.push_back(L);
    }

    build_mark(9);
    // ---- launch geometry
    // expected duration of the walk kernels: algorithmic lane-ops per
    // prime-step (difference-table streams, product, reduction; the bytecode
    // interpreter ~10x that) at the ~1.7e13 lane-ops/s the walk kernels reach;
    // the FP64 shadow chains beside them are sized against it
    double walk_ops = 0.0;
    for (int32_t w = 0; w < n_walks; ++w) {
        const DevWalk& W = dwalks[w];
        const DevProgram& G = dprogs[W.prog];
        const double m = G.m, D = std::max<uint32_t>(G.degree, 1);
        double per = 2.0 * m * D + m * (m + 4.0 + 2.0 * std::max(0.0, m - 2.0));
        if (G.cls == CLS_DENSE) per *= m;
        if (G.cls == CLS_INTERP) per *= 10.0;
        walk_ops += per * (double)W.K * (double)W.depth;
    }
    const double walk_ns = walk_ops / 1.7e13 * 1e9;
    // the plain engine launches one single-warp block per tile: a warp per
    // (walk, prime block) over the whole depth, no queue
    const int wpb = plain ? 1
                  : (tune && tune->warps_per_block) ? (int)tune->warps_per_block
                  : tuned_wpb ? (int)tuned_wpb : 4;
    B->wpb_used = (uint32_t)wpb;
    uint32_t q = 0;
    for (LaunchSpec& L : B->launches) {
        L.queue = q++;
        if (L.kind == 1) {
            L.queue2 = q++;
            if ((rc = shadow_interp_geometry(L, max_dim, C.sms, shadow_list.data() + L.off, true, walk_ns)))
                return rc;
            if (L.split_D && (rc = shadow_split_geometry(L, C.sms))) return rc;
            continue;
        }
        if (L.kind == 2) {
            const size_t per_warp = (size_t)L.rows_per_warp * 32 * 8;
            const bool coloc = chain_colocate(shadow_list.data() + L.off, L.count, L.m, walk_ns);
            L.lean = coloc;
            // two chain warps per scheduler for the packed depths (the tuner's
            // choice: each chain is slower, the walks get the SMs)
            int cw = (chain_pack && L.D <= chain_pack) ? 2 * kChainWarps : kChainWarps;
            if (per_warp * cw > 227 * 1024) cw = kChainWarps;   // no room for the packed block
            L.block = coloc ? 32 : 32 * cw;
            L.smem = coloc ? per_warp : std::max(per_warp * cw, chain_hog_smem());
            if (per_warp * (L.block / 32) > L.smem || L.smem > 227 * 1024) {
                set_error("program needs more shared memory per warp than a block offers");
                return DR_ERR_UNSUPPORTED;
            }
            int occ = 0;
            ShadowArgs sa{};
            cudaError_t e = shadow_fd_dispatch(L.cls, L.m, L.D, 0, L.block, L.smem, nullptr, sa, &occ);
            if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
            if (occ < 1) {
                set_error("kernel cannot be resident with this shared memory size");
                return DR_ERR_UNSUPPORTED;
            }
            L.grid = coloc ? std::min((int)L.items, occ * C.sms)
                           : std::min(chain_blocks(shadow_list.data() + L.off, L.count, L.m, walk_ns, cw),
                                      occ * C.sms);
            continue;
        }
        L.block = 32 * wpb;
        const size_t word = L.kind == 0 ? 4 : 8;
        L.smem = (size_t)L.rows_per_warp * 32 * word * wpb;
        if (L.smem > 227 * 1024) {
            set_error("program needs more shared memory per warp than a block offers");
            return DR_ERR_UNSUPPORTED;
        }
        int occ = 0;
        cudaError_t e;
        WalkArgs wa{};
        ShadowArgs sa{};
        if (L.kind == 0) e = walk_dispatch(L.cls, L.m, L.D, 0, L.block, L.smem, nullptr, wa, &occ);
        else e = shadow_fd_dispatch(L.cls, L.m, L.D, 0, L.block, L.smem, nullptr, sa, &occ);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
        if (occ < 1) {
            set_error("kernel cannot be resident with this shared memory size");
            return DR_ERR_UNSUPPORTED;
        }
        const int want = (int)((L.items + wpb - 1) / wpb);
        L.grid = plain ? std::max(1, want) : std::max(1, std::min(want, occ * C.sms));
    }
    B->n_queues = q;

    build_mark(10);
    nvtx_build.end();
    NvtxRange nvtx_upload("dr.upload");
    const auto t_upload0 = std::chrono::steady_clock::now();
    // ---- upload
    cudaStream_t st = C.stream;
    // The tables go up as one copy from the context's pinned staging buffer
    // (pageable copies cost a staging pass and a call each); the batch's
    // buffers are views into one device allocation.  stage_mu stays held
    // until the stream sync below, which the copy must pass before the
    // buffer is refilled.
    std::unique_lock<std::mutex> stage_lk(C.stage_mu);
    {
        struct Part { DevBuf* b; const void* src; size_t n; };
        const Part parts[] = {
            {&B->progs, dprogs.data(), sizeof(DevProgram) * dprogs.size()},
            {&B->code, code.data(), sizeof(uint4) * code.size()},
            {&B->consts, consts.data(), sizeof(int64_t) * consts.size()},
            {&B->walks, dwalks.data(), sizeof(DevWalk) * dwalks.size()},
            {&B->axis, axis, sizeof(int64_t) * n_axis},
            {&B->tiles, tiles.data(), sizeof(DevTile) * tiles.size()},
            {&B->groups, groups.data(), sizeof(DevGroup) * groups.size()},
            {&B->shadow_list, shadow_list.data(), sizeof(DevShadowSeg) * shadow_list.size()},
            {&B->eval_items, eval_items.data(), sizeof(uint32_t) * eval_items.size()},
        };
        constexpr size_t kParts = sizeof(parts) / sizeof(parts[0]);
        constexpr size_t kAlign = 256;
        size_t offs[kParts], total = 0;
        for (size_t i = 0; i < kParts; ++i) {
            offs[i] = total;
            total += (std::max<size_t>(parts[i].n, 16) + kAlign - 1) / kAlign * kAlign;
        }
        DR_CUDA(B->tables.alloc(total));
        if (C.stage_bytes < total) {
            if (C.stage_host) DR_CUDA(cudaFreeHost(C.stage_host));
            C.stage_host = nullptr;
            C.stage_bytes = 0;
            const size_t cap = std::max<size_t>(total + total / 4, 1u << 20);
            DR_CUDA(cudaMallocHost(&C.stage_host, cap));
            C.stage_bytes = cap;
        }
        uint8_t* h = static_cast<uint8_t*>(C.stage_host);
        // into the staging buffer in 256 KB pieces, on the host pool when large
        constexpr size_t kPiece = 256u << 10;
        std::vector<std::pair<size_t, size_t>> pieces;   // (part, byte offset)
        for (size_t i = 0; i < kParts; ++i)
            for (size_t o = 0; o < parts[i].n; o += kPiece) pieces.emplace_back(i, o);
        auto copy_pieces = [&](int, size_t lo, size_t hi) {
            for (size_t k = lo; k < hi; ++k) {
                const Part& P = parts[pieces[k].first];
                const size_t o = pieces[k].second;
                std::memcpy(h + offs[pieces[k].first] + o, static_cast<const uint8_t*>(P.src) + o,
                            std::min(kPiece, P.n - o));
            }
        };
        const int cparts = std::min<int>(host_pool().threads(), (int)pieces.size());
        if (cparts > 2) host_pool().run(cparts, pieces.size(), copy_pieces);
        else copy_pieces(0, 0, pieces.size());
        DR_CUDA(cudaMemcpyAsync(B->tables.p, h, total, cudaMemcpyHostToDevice, st));
        uint8_t* d = static_cast<uint8_t*>(B->tables.p);
        for (size_t i = 0; i < kParts; ++i) parts[i].b->set_view(d + offs[i], std::max<size_t>(parts[i].n, 16));
    }
    build_mark(11);
    DR_CUDA(B->mf.alloc(8ull * std::max<uint64_t>(mf_doubles, 1)));
    DR_CUDA(B->shadow_state.alloc(8ull * kShadowStateStride * std::max<uint32_t>(state_slots, 1)));
    DR_CUDA(B->group_done.alloc(4ull * std::max<uint32_t>(B->n_groups, 1)));
    DR_CUDA(cudaMemsetAsync(B->group_done.p, 0, B->group_done.bytes, st));
    uint32_t max_m = 1;
    for (auto& d : dprogs) max_m = std::max(max_m, d.m);
    B->chunk_stride = max_m * max_m * 32;
    DR_CUDA(B->chunkP.alloc(4ull * std::max<uint32_t>(slots, 1) * B->chunk_stride));
    B->n_progs = (uint32_t)n_programs;
    B->n_slots = slots;
    B->n_code = code.size();
    B->n_consts = consts.size();
    B->n_axis = n_axis;
    if (kDebugChecks) {
        DR_CUDA(B->dbg.alloc(16));
        DR_CUDA(cudaMemsetAsync(B->dbg.p, 0, 16, st));
    }
    DR_CUDA(B->chunkSig.alloc(4ull * std::max<uint32_t>(slots, 1) * 32));
    DR_CUDA(B->queues.alloc(4ull * std::max<uint32_t>(B->n_queues, 1)));
    DR_CUDA(B->res.alloc(8ull * std::max<uint64_t>(n_res, 1)));
    DR_CUDA(cudaMemsetAsync(B->res.p, 0, B->res.bytes, st));
    B->h_walk_K.resize(n_walks);
    B->h_res_off.resize(n_walks);
    B->h_cp_off.resize(n_walks);
    for (int32_t w = 0; w < n_walks; ++w) {
        B->h_walk_K[w] = walks[w].K;
        B->h_res_off[w] = walks[w].res_offset;
        B->h_cp_off[w] = walks[w].checkpoint ? walks[w].cp_res_offset : UINT64_MAX;
    }
    DR_CUDA(B->shadow.alloc(8ull * 6 * std::max<int32_t>(n_walks, 1)));
    DR_CUDA(cudaMemsetAsync(B->shadow.p, 0, B->shadow.bytes, st));
    DR_CUDA(B->status.alloc(4ull * std::max<int32_t>(n_walks, 1)));
    DR_CUDA(cudaEventCreate(&B->ev0));
    DR_CUDA(cudaEventCreate(&B->ev1));
    DR_CUDA(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
    DR_CUDA(cudaEventCreateWithFlags(&B->join, cudaEventDisableTiming));
    B->joins.resize(C.pool.size() + C.hpool.size());
    B->evals.assign(B->launches.size(), nullptr);
    for (size_t i = 0; i < B->launches.size(); ++i)
        if (B->launches[i].kind == 1 || (B->launches[i].kind == 2 && !B->launches[i].lean))
            DR_CUDA(cudaEventCreateWithFlags(&B->evals[i], cudaEventDisableTiming));
    for (auto& e : B->joins) DR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    build_mark(12);
    DR_CUDA(cudaStreamSynchronize(st));
    build_mark(13);
    {
        using ms = std::chrono::duration<double, std::milli>;
        const auto t_end = std::chrono::steady_clock::now();
        stage_add(STAGE_BUILD, ms(t_upload0 - t_build0).count());
        stage_add(STAGE_UPLOAD, ms(t_end - t_upload0).count());
    }
    *out = std::move(B);
    return DR_OK;
}

uint64_t shadow_interp_plan(std::vector<LaunchSpec>& launches, std::vector<DevShadowSeg>& list,
                            std::vector<uint32_t>& eval_items, const std::vector<DevShadowSeg>& segs,
                            uint32_t m, uint32_t shape, uint32_t rows_regs, uint64_t mf_base,
                            uint64_t round_steps, uint32_t slot_base) {
    const uint32_t ne = shadow_entries(m, (shape & 1u) != 0);
    const bool rounds = round_steps != UINT64_MAX;
    uint64_t region = 0;
    for (uint64_t r = 0;; ++r) {
        LaunchSpec L{};
        L.kind = 1;
        L.cls = shape;
        L.m = m;
        L.follow = r > 0;
        L.off = (uint32_t)list.size();
        L.eoff = (uint32_t)eval_items.size();
        L.rows_regs = rows_regs;
        uint64_t off = mf_base;
        uint32_t idx = 0;
        for (size_t i = 0; i < segs.size(); ++i) {
            const DevShadowSeg& g = segs[i];
            const uint64_t a = rounds ? g.s0 + r * round_steps : g.s0;
            if (a >= g.s1 && !(r == 0 && g.s0 == g.s1)) continue;
            const uint64_t b = rounds ? std::min(g.s1, a + round_steps) : g.s1;
            DevShadowSeg n = g;
            n.s0 = a;
            n.s1 = b;
            n.mf_off = off;
            n.item0 = (uint32_t)(eval_items.size() - L.eoff);
            if (rounds) n.state = slot_base + (uint32_t)i;
            const uint64_t nit = (b - a + kEvalSteps - 1) / kEvalSteps;
            for (uint64_t k = 0; k < nit; ++k) eval_items.push_back(idx);
            list.push_back(n);
            ++idx;
            off += (b - a) * ne;
        }
        if (idx == 0) break;
        L.count = idx;
        L.items = (uint32_t)(eval_items.size() - L.eoff);
        L.items2 = (idx + 31) / 32;
        launches.push_back(L);
        region = std::max(region, off - mf_base);
        if (!rounds) break;
    }
    return region;
}

size_t chain_hog_smem() {
    static size_t bytes = 0;
    if (!bytes) {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0)
            v = 96 * 1024;
        bytes = (size_t)v;
    }
    return bytes;
}

bool chain_colocate(const DevShadowSeg* segs, uint32_t count, uint32_t m, double walk_ns) {
    uint64_t longest = 0;
    if (count) longest = segs[0].s1 - segs[0].s0;   // sorted longest first
    for (uint32_t k = 0; k < count && k < 64; ++k) longest = std::max<uint64_t>(longest, segs[k].s1 - segs[k].s0);
    // shared issue slots slow a chain by ~1.6x; keep a margin on top
    return walk_ns > 0 && 3.0 * (double)longest * chain_step_ns(m) < walk_ns;
}

int chain_blocks(const DevShadowSeg* segs, uint32_t count, uint32_t m, double walk_ns, int wpb) {
    // segments are sorted longest first; a warp takes 32 of them, so item k
    // lasts as long as segment 32k.  Enough warps that the total chain work
    // spread over them ends with the longest chain, or with the walk kernels
    // when those take longer (a chain step is ~300 ns), plus one block of slack.
    const double kStepNs = chain_step_ns(m);
    uint64_t total = 0, longest = 0;
    for (uint32_t k = 0; k < count; k += 32) {
        const uint64_t len = segs[k].s1 - segs[k].s0;
        total += std::max<uint64_t>(len, 1);
        longest = std::max<uint64_t>(longest, std::max<uint64_t>(len, 1));
    }
    const uint32_t items = (count + 31) / 32;
    const double span = std::max((double)longest * kStepNs, walk_ns);
    const uint64_t warps = span > 0 ? (uint64_t)std::ceil((double)total * kStepNs / span) : 1;
    const uint64_t blocks = (warps + wpb - 1) / wpb + 1;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (items + wpb - 1) / wpb));
}

int shadow_interp_geometry(LaunchSpec& L, uint32_t max_dim, int sms, const DevShadowSeg* segs,
                           bool whole_sm, double walk_ns) {
    const uint32_t base = L.rows_regs + max_dim + L.m * L.m;
    uint32_t U = 1;
    for (uint32_t u : {4u, 2u})
        if ((size_t)u * base * 32 * 8 <= 16 * 1024) { U = u; break; }
    L.U = U;
    L.rows_axes = max_dim;
    L.rows_per_warp = U * base;
    const size_t per_warp = (size_t)L.rows_per_warp * 32 * 8;
    int wpb = 4;
    while (wpb > 1 && per_warp * wpb > 227 * 1024) wpb /= 2;
    if (per_warp * wpb > 227 * 1024) {
        set_error("program needs more shared memory per warp than a block offers");
        return DR_ERR_UNSUPPORTED;
    }
    L.block = 32 * wpb;
    L.smem = per_warp * wpb;
    ShadowArgs sa{};
    int occ = 0;
    cudaError_t e = shadow_eval_dispatch(U, 0, L.block, L.smem, nullptr, sa, &occ);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
    if (occ < 1) {
        set_error("kernel cannot be resident with this shared memory size");
        return DR_ERR_UNSUPPORTED;
    }
    L.grid = std::max(1, std::min((int)((L.items + wpb - 1) / wpb), occ * sms));
    const bool coloc = whole_sm && chain_colocate(segs, L.count, L.m, walk_ns);
    L.lean = coloc;
    // chain warps per block: fewer when their staging buffers would not fit
    const size_t chain_warp_smem = shadow_chain_smem(L.m, (L.cls & 1u) != 0);
    int cw = kChainWarps;
    while (cw > 1 && chain_warp_smem * cw > 227 * 1024) cw /= 2;
    L.block2 = coloc ? 32 : 32 * cw;
    L.smem2 = chain_warp_smem * (L.block2 / 32);
    if (whole_sm && !coloc) L.smem2 = std::max(L.smem2, chain_hog_smem());
    e = shadow_chain_dispatch(L.m, L.cls, 0, L.block2, L.smem2, nullptr, sa, &occ);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
    if (occ < 1) {
        set_error("kernel cannot be resident with this shared memory size");
        return DR_ERR_UNSUPPORTED;
    }
    L.grid2 = coloc ? std::min((int)L.items2, occ * sms)
                    : std::min(chain_blocks(segs, L.count, L.m, walk_ns, cw), occ * sms);
    return DR_OK;
}

// The chain launch of a split shadow: one item per warp (items are 32 walks
// of about equal length, and the longest go first), kChainWarps warps per
// block claiming a whole SM; per warp the head's rows or the tail's staging
// buffers, whichever is larger.
int shadow_split_geometry(LaunchSpec& L, int sms) {
    const uint32_t ns = (uint32_t)std::max(streams_for(L.split_cls, L.m), 1);
    const uint32_t head_rows = L.split_rows_regs + kMaxAxes + (L.split_D + 1) * ns + ns;
    const uint32_t tail_rows = (uint32_t)(shadow_chain_smem(L.m, true) / (32 * sizeof(double)));
    L.split_rows_per_warp = std::max(head_rows, tail_rows);
    const size_t per_warp = (size_t)L.split_rows_per_warp * 32 * sizeof(double);
    int cw = kChainWarps;
    while (cw > 1 && per_warp * cw > 227 * 1024) cw /= 2;
    if (per_warp * cw > 227 * 1024) {
        set_error("program needs more shared memory per warp than a block offers");
        return DR_ERR_UNSUPPORTED;
    }
    L.lean = false;
    L.block2 = 32 * cw;
    L.smem2 = std::max(per_warp * cw, chain_hog_smem());
    ShadowArgs sa{};
    int occ = 0;
    cudaError_t e = shadow_split_dispatch(L.split_cls, L.m, L.split_D, 0, L.block2, L.smem2, nullptr, sa, &occ);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
    if (occ < 1) {
        set_error("kernel cannot be resident with this shared memory size");
        return DR_ERR_UNSUPPORTED;
    }
    L.grid2 = std::max(1, std::min((int)((L.items2 + cw - 1) / cw), occ * sms));
    return DR_OK;
}

// The chain launch of an interpreted (or split) shadow group.
static cudaError_t interp_chain_dispatch(const LaunchSpec& L, ShadowArgs sa, cudaStream_t s) {
    if (L.split_D) {
        sa.rows_regs = L.split_rows_regs;
        sa.rows_per_warp = L.split_rows_per_warp;
        return shadow_split_dispatch(L.split_cls, L.m, L.split_D, L.grid2, L.block2, L.smem2, s, sa, nullptr);
    }
    return shadow_chain_dispatch(L.m, L.cls, L.grid2, L.block2, L.smem2, s, sa, nullptr);
}

cudaError_t launch_shadow_interp(const LaunchSpec& L, ShadowArgs sa, uint32_t* queues,
                                 const uint32_t* eval_items, cudaStream_t s, cudaEvent_t evaluated) {
    sa.eval_items = eval_items + L.eoff;
    sa.n_items = L.items;
    sa.queue = queues + L.queue;
    sa.rows_axes = L.rows_axes;
    if (L.items) {
        cudaError_t e = shadow_eval_dispatch(L.U, L.grid, L.block, L.smem, s, sa, nullptr);
        if (e != cudaSuccess) return e;
    }
    if (evaluated) {
        cudaError_t e = cudaEventRecord(evaluated, s);
        if (e != cudaSuccess) return e;
    }
    sa.n_items = L.items2;
    sa.queue = queues + L.queue2;
    if (sa.tstamp) sa.tstamp += 2;
    return interp_chain_dispatch(L, sa, s);
}

static CrtTables tables_of(const CrtSet& S);

// CRT (one launch per K), delta and top-k passes on st after the walk.
static int enqueue_pipeline(Batch& B, cudaStream_t st) {
    Context& C = *g_ctx;
    const uint64_t qoff = std::max<uint64_t>(B.n_res, 1);
    (void)qoff;
    for (const Batch::CrtGroup& g : B.crt_groups) {
        std::shared_ptr<CrtSet> S;
        int rc = crt_tables_std(g.K, &S);
        if (rc) return rc;
        cudaError_t e = launch_crt(B.res.as<uint32_t>(), (int)g.count, tables_of(*S), B.limbs.as<uint32_t>(),
                                   B.Lmax, B.signs.as<int32_t>(), nullptr, nullptr, C.sms, st,
                                   B.crt_in.as<uint64_t>() + g.off, B.crt_out.as<uint32_t>() + g.off);
        if (e != cudaSuccess) return cuda_fail(e, "pipeline crt");
    }
    if (B.pipe.delta_mode != DR_DELTA_NONE) {
        DeltaArgs D{};
        const bool self = B.pipe.delta_mode == DR_DELTA_SELF;
        const size_t L = (size_t)B.Lmax;
        const uint32_t* lim = B.limbs.as<uint32_t>();
        const int32_t* sg = B.signs.as<int32_t>();
        D.p = lim + (self ? 2 : 0) * L;
        D.q = lim + (self ? 3 : 1) * L;
        D.ps = sg + (self ? 2 : 0);
        D.qs = sg + (self ? 3 : 1);
        D.n = (int)B.n_walks;
        D.nl = B.Lmax;
        D.istride = 4 * L;
        D.sstride = 4;
        if (self) {
            D.ln = lim;
            D.ld = lim + L;
            D.lns = sg;
            D.lds = sg + 1;
            D.lnl = B.Lmax;
            D.per_item = 1;
            D.listride = 4 * L;
            D.lsstride = 4;
        } else {
            D.ln = B.tgt_num.as<uint32_t>();
            D.ld = B.tgt_den.as<uint32_t>();
            D.lns = B.tgt_sign.as<int32_t>();
            D.lds = nullptr;
            D.lnl = B.pipe.l_limbs;
            D.per_item = 0;
            D.listride = 0;
            D.lsstride = 0;
        }
        D.out = B.delta.as<double>();
        D.maxlen = ((B.Lmax + std::max(B.Lmax, B.pipe.l_limbs) + 4) + 1) & ~1;
        cudaError_t e = launch_delta(D, C.sms, st);
        if (e != cudaSuccess) return cuda_fail(e, "pipeline delta");
        for (size_t pass = 0; pass < B.tk_counts.size(); ++pass) {
            const int src = (int)(pass & 1) ^ 1, dst = (int)(pass & 1);
            e = launch_topk_tile(pass == 0 ? B.delta.as<double>() : nullptr,
                                 pass == 0 ? nullptr : B.tk_keys[src].as<uint64_t>(),
                                 pass == 0 ? nullptr : B.tk_idx[src].as<uint32_t>(),
                                 B.tk_counts[pass], B.pipe.topk, B.tk_keys[dst].as<uint64_t>(),
                                 B.tk_idx[dst].as<uint32_t>(), st);
            if (e != cudaSuccess) return cuda_fail(e, "pipeline topk");
        }
    }
    if (B.bank_n > 0) {
        // the top-k hits (or, without a top-k, every walk): final p/q against
        // every bank constant
        const bool hits = !B.tk_counts.empty();
        const size_t L = (size_t)B.Lmax;
        DeltaArgs K{};
        K.p = B.limbs.as<uint32_t>();
        K.q = B.limbs.as<uint32_t>() + L;
        K.ps = B.signs.as<int32_t>();
        K.qs = B.signs.as<int32_t>() + 1;
        K.nl = B.Lmax;
        K.istride = 4 * L;
        K.sstride = 4;
        K.ln = B.bank_num.as<uint32_t>();
        K.ld = B.bank_den.as<uint32_t>();
        K.lns = B.bank_sign.as<int32_t>();
        K.lds = nullptr;
        K.lnl = B.bank_l;
        K.per_item = 1;
        K.listride = (size_t)B.bank_l;
        K.lsstride = 1;
        K.rows = hits ? B.tk_idx[B.tk_final].as<uint32_t>() : nullptr;
        K.bank_n = B.bank_n;
        K.n = (hits ? std::min<int>(B.pipe.topk, (int)B.n_walks) : (int)B.n_walks) * B.bank_n;
        K.out = B.bank_out.as<double>();
        K.maxlen = ((B.Lmax + std::max(B.Lmax, B.bank_l) + 4) + 1) & ~1;
        cudaError_t e = launch_delta(K, C.sms, st);
        if (e != cudaSuccess) return cuda_fail(e, "pipeline bank");
    }
    return DR_OK;
}

// CRT overflow flags: the pipeline's values against the finished FP64 shadow.
static int enqueue_crt_check(Batch& B, cudaStream_t st) {
    if (!B.pipe_on || !B.has_shadow || B.crt_groups.empty()) return DR_OK;
    cudaError_t e = launch_crt_check(B.limbs.as<uint32_t>(), B.signs.as<int32_t>(), B.Lmax,
                                     (int)B.n_walks, B.walks.as<DevWalk>(), B.shadow.as<double>(),
                                     B.status.as<uint32_t>(), st);
    return e == cudaSuccess ? DR_OK : cuda_fail(e, "pipeline crt check");
}

static void batch_args(Batch& B, WalkArgs& wa, ShadowArgs& sa) {
    Context& C = *g_ctx;
    wa = WalkArgs{};
    wa.progs = B.progs.as<DevProgram>();
    wa.code = B.code.as<uint4>();
    wa.consts = B.consts.as<int64_t>();
    wa.walks = B.walks.as<DevWalk>();
    wa.axis = B.axis.as<int64_t>();
    wa.groups = B.groups.as<DevGroup>();
    wa.group_done = B.group_done.as<uint32_t>();
    wa.chunk_P = B.chunkP.as<uint32_t>();
    wa.chunk_stride = B.chunk_stride;
    wa.chunk_sig = B.chunkSig.as<uint32_t>();
    wa.state_P = nullptr;
    wa.state_sig = nullptr;
    wa.primes = C.primes.as<uint32_t>();
    wa.pinv = C.pinv.as<uint32_t>();
    wa.r2 = C.r2.as<uint32_t>();
    wa.p_res = B.res.as<uint32_t>();
    wa.q_res = B.res.as<uint32_t>() + std::max<uint64_t>(B.n_res, 1);
    wa.status = B.status.as<uint32_t>();
    wa.n_progs = B.n_progs;
    wa.n_walks = B.n_walks;
    wa.n_groups = B.n_groups;
    wa.n_slots = B.n_slots;
    wa.n_code = B.n_code;
    wa.n_consts = B.n_consts;
    wa.n_axis = B.n_axis;
    wa.n_res = B.n_res;
    wa.dbg = kDebugChecks ? B.dbg.as<uint32_t>() : nullptr;
    sa = ShadowArgs{};
    sa.progs = wa.progs;
    sa.code = wa.code;
    sa.consts = wa.consts;
    sa.walks = wa.walks;
    sa.axis = wa.axis;
    sa.shadow = B.shadow.as<double>();
    sa.n_walks = B.n_walks;
    sa.status = wa.status;
    sa.state = B.shadow_state.as<double>();
    sa.mf = B.mf.as<double>();
}

// Whether the walk launches wait for the integer-difference shadow chains to
// be placed (launch completion events).  DREAMS_B200_CHAIN_FIRST=0 turns it
// off.
static bool chain_first() {
    static const bool on = [] {
        const char* v = std::getenv("DREAMS_B200_CHAIN_FIRST");
        return !(v && v[0] == '0');
    }();
    return on;
}

static cudaError_t launch_one(Batch& B, const LaunchSpec& L, WalkArgs& wa, ShadowArgs& sa, cudaStream_t s) {
    unsigned long long* ts = B.stamping ? B.tstamps.as<unsigned long long>() + 4 * (&L - B.launches.data()) : nullptr;
    wa.tstamp = ts;
    sa.tstamp = ts;
    sa.item_log = (B.stamping && L.kind != 0)
                      ? B.item_log.as<unsigned long long>() + 4ull * B.item_log_off[&L - B.launches.data()]
                      : nullptr;
    if (L.kind == 0) {
        wa.tiles = B.tiles.as<DevTile>() + L.off;
        wa.n_tiles = L.count;
        wa.queue = B.queues.as<uint32_t>() + L.queue;
        wa.rows_regs = L.rows_regs;
        wa.rows_consts = L.rows_consts;
        wa.rows_stage = L.rows_stage;
        wa.rows_axes = L.rows_axes;
        wa.rows_per_warp = L.rows_per_warp;
        return walk_dispatch(L.cls, L.m, L.D, L.grid, L.block, L.smem, s, wa, nullptr);
    }
    sa.segs = B.shadow_list.as<DevShadowSeg>() + L.off;
    sa.n_list = L.count;
    sa.rows_regs = L.rows_regs;
    sa.rows_per_warp = L.rows_per_warp;
    sa.lean = L.lean ? 1u : 0u;
    if (L.kind == 2) {
        sa.n_items = L.items;
        sa.queue = B.queues.as<uint32_t>() + L.queue;
        // the walk launches wait until these chain blocks are placed (not
        // finished), so the chains get their SMs before the walks fill them
        const cudaEvent_t started = (chain_first() && !L.lean) ? B.evals[&L - B.launches.data()] : nullptr;
        StartedEvent se(started);
        return shadow_fd_dispatch(L.cls, L.m, L.D, L.grid, L.block, L.smem, s, sa, nullptr);
    }
    const size_t i = &L - B.launches.data();
    return launch_shadow_interp(L, sa, B.queues.as<uint32_t>(), B.eval_items.as<uint32_t>(), s,
                                i < B.evals.size() && !L.follow ? B.evals[i] : nullptr);
}

// One run of a batch: zero the work counters and status words, then every
// launch group (shadow kernels first, on high-priority streams: they hold
// the longest serial chains) on its own stream, forked from and joined back
// into st.
static int enqueue_batch(Batch& B, cudaStream_t st, std::vector<cudaEvent_t>* ends = nullptr) {
    Context& C = *g_ctx;
    DR_CUDA(cudaMemsetAsync(B.queues.p, 0, B.queues.bytes, st));
    DR_CUDA(cudaMemsetAsync(B.status.p, 0, B.status.bytes, st));
    WalkArgs wa;
    ShadowArgs sa;
    batch_args(B, wa, sa);
    DR_CUDA(cudaEventRecord(B.fork, st));
    std::vector<cudaStream_t> used;
    auto take = [&](std::vector<cudaStream_t>& pool, size_t& k) -> cudaStream_t {
        cudaStream_t s = pool[k % pool.size()];
        if (k < pool.size()) {
            used.push_back(s);
            if (cudaStreamWaitEvent(s, B.fork, 0) != cudaSuccess) return nullptr;
        }
        ++k;
        return s;
    };
    size_t k_lo = 0, k_hi = 0;
    cudaStream_t prev = nullptr;
    int rc = DR_OK;
    // Launch order: the integer-difference chains first (their blocks claim
    // whole SMs, so they must be placed before the evaluation kernel fills
    // the GPU), then the interpreted shadows, then the walks.
    for (int pass = 0; pass < 3 && rc == DR_OK; ++pass) {
        const int kind = pass == 0 ? 2 : pass == 1 ? 1 : 0;
        for (const LaunchSpec& L : B.launches) {
            if ((L.items == 0 && L.items2 == 0) || L.kind != kind) continue;
            cudaStream_t s = prev;
            if (!L.follow || !prev) {
                s = pass < 2 ? take(C.hpool, k_hi) : take(C.pool, k_lo);
                // walks start once the step matrices are evaluated, so the
                // shadow chains (high priority) are placed before them
                if (s && pass == 2)
                    for (size_t j = 0; j < B.launches.size(); ++j)
                        if ((B.launches[j].kind == 1 ||
                             (B.launches[j].kind == 2 && chain_first() && !B.launches[j].lean)) &&
                            !B.launches[j].follow && B.launches[j].items)
                            if (cudaStreamWaitEvent(s, B.evals[j], 0) != cudaSuccess) s = nullptr;
            }
            if (!s) { rc = cuda_fail(cudaErrorUnknown, "stream fork"); break; }
            prev = s;
            cudaError_t e = launch_one(B, L, wa, sa, s);
            if (e == cudaSuccess && ends) e = cudaEventRecord((*ends)[&L - B.launches.data()], s);
            if (e != cudaSuccess) {
                rc = cuda_fail(e, L.kind == 0 ? "walk launch" : "shadow launch");
                break;
            }
        }
    }
    // rejoin the walk streams first: CRT, delta, top-k and the bank need only
    // the residues and run while the FP64 shadow chains are still going; the
    // shadow streams join before the CRT overflow check, which reads them
    // (every forked stream is rejoined, also on errors, so a capture ends cleanly)
    const size_t n_hi = std::min(k_hi, C.hpool.size());
    for (size_t i = 0; i < used.size(); ++i) {
        cudaEventRecord(B.joins[i], used[i]);
        if (i >= n_hi) cudaStreamWaitEvent(st, B.joins[i], 0);
    }
    if (rc == DR_OK && B.pipe_on) rc = enqueue_pipeline(B, st);
    for (size_t i = 0; i < n_hi && i < used.size(); ++i) cudaStreamWaitEvent(st, B.joins[i], 0);
    if (rc != DR_OK) return rc;
    DR_CUDA(cudaGetLastError());
    return enqueue_crt_check(B, st);
}

// Every launch group alone, one after another on one stream, timed with
// events: where a batch's time goes (used by the autotuner and diagnostics).
int batch_profile(Batch& B, std::vector<float>* ms, std::vector<float>* ms2) {
    Context& C = *g_ctx;
    cudaStream_t st = C.stream;
    WalkArgs wa;
    ShadowArgs sa;
    batch_args(B, wa, sa);
    DR_CUDA(cudaMemsetAsync(B.queues.p, 0, B.queues.bytes, st));
    DR_CUDA(cudaMemsetAsync(B.status.p, 0, B.status.bytes, st));
    const size_t n = B.launches.size();
    std::vector<cudaEvent_t> ev(2 * n + 1);
    for (auto& e : ev) DR_CUDA(cudaEventCreate(&e));
    DR_CUDA(cudaEventRecord(ev[0], st));
    for (size_t i = 0; i < n; ++i) {
        const LaunchSpec& L = B.launches[i];
        cudaError_t e = cudaSuccess;
        if (L.kind == 1) {
            // the evaluation and the chain timed apart
            sa.segs = B.shadow_list.as<DevShadowSeg>() + L.off;
            sa.n_list = L.count;
            sa.rows_regs = L.rows_regs;
            sa.rows_per_warp = L.rows_per_warp;
            sa.rows_axes = L.rows_axes;
            sa.eval_items = B.eval_items.as<uint32_t>() + L.eoff;
            if (L.items) {
                sa.n_items = L.items;
                sa.queue = B.queues.as<uint32_t>() + L.queue;
                e = shadow_eval_dispatch(L.U, L.grid, L.block, L.smem, st, sa, nullptr);
            }
            if (e == cudaSuccess) e = cudaEventRecord(ev[2 * i + 1], st);
            if (e == cudaSuccess) {
                sa.n_items = L.items2;
                sa.queue = B.queues.as<uint32_t>() + L.queue2;
                e = interp_chain_dispatch(L, sa, st);
            }
        } else {
            if (L.items) e = launch_one(B, L, wa, sa, st);
            if (e == cudaSuccess) e = cudaEventRecord(ev[2 * i + 1], st);
        }
        if (e != cudaSuccess) return cuda_fail(e, "profile launch");
        DR_CUDA(cudaEventRecord(ev[2 * i + 2], st));
    }
    DR_CUDA(cudaStreamSynchronize(st));
    ms->assign(n, 0.f);
    ms2->assign(n, 0.f);
    for (size_t i = 0; i < n; ++i) {
        cudaEventElapsedTime(&(*ms)[i], ev[2 * i], ev[2 * i + 1]);
        cudaEventElapsedTime(&(*ms2)[i], ev[2 * i + 1], ev[2 * i + 2]);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return DR_OK;
}

// One eager (uncaptured) run with the launch groups concurrent as in a
// normal run, the kernels stamping when their first block started and their
// last block ended: per launch [start, end, start2, end2] in ms after the
// earliest start (start2/end2: kind 1's chain kernel; -1 = did not run).
int batch_timeline(Batch& B, std::vector<float>* out) {
    Context& C = *g_ctx;
    cudaStream_t st = C.stream;
    const size_t n = B.launches.size();
    std::vector<unsigned long long> h(4 * n);
    for (size_t i = 0; i < n; ++i) {
        h[4 * i] = h[4 * i + 2] = ~0ull;
        h[4 * i + 1] = h[4 * i + 3] = 0;
    }
    DR_CUDA(B.tstamps.alloc(8 * h.size()));
    DR_CUDA(cudaMemcpy(B.tstamps.p, h.data(), 8 * h.size(), cudaMemcpyHostToDevice));
    // per chain item of the integer-difference launches: 4 words each
    B.item_log_off.assign(n, 0);
    uint32_t n_items = 0;
    for (size_t i = 0; i < n; ++i) {
        B.item_log_off[i] = n_items;
        if (B.launches[i].kind == 2) n_items += B.launches[i].items;
        if (B.launches[i].kind == 1) n_items += B.launches[i].items2;
    }
    DR_CUDA(B.item_log.alloc(32ull * std::max<uint32_t>(n_items, 1)));
    DR_CUDA(cudaMemset(B.item_log.p, 0, 32ull * std::max<uint32_t>(n_items, 1)));
    B.stamping = true;
    int rc = enqueue_batch(B, st);
    B.stamping = false;
    if (rc) return rc;
    DR_CUDA(cudaStreamSynchronize(st));
    DR_CUDA(cudaMemcpy(h.data(), B.tstamps.p, 8 * h.size(), cudaMemcpyDeviceToHost));
    std::vector<unsigned long long> il(4ull * n_items);
    if (n_items) DR_CUDA(cudaMemcpy(il.data(), B.item_log.p, 8 * il.size(), cudaMemcpyDeviceToHost));
    unsigned long long t0 = ~0ull;
    for (size_t i = 0; i < 2 * n; ++i) t0 = std::min(t0, h[2 * i]);
    // items: launch, start, tables built, end (ms after t0), re-run chunks, exact steps
    B.item_rows.clear();
    for (size_t i = 0; i < n; ++i) {
        if (B.launches[i].kind == 0) continue;
        const uint32_t items = B.launches[i].kind == 2 ? B.launches[i].items : B.launches[i].items2;
        for (uint32_t k = 0; k < items; ++k) {
            const unsigned long long* r = &il[4ull * (B.item_log_off[i] + k)];
            if (!r[0] || r[0] < t0) continue;
            B.item_rows.insert(B.item_rows.end(),
                               {(float)i, (float)((r[0] - t0) * 1e-6), (float)((r[1] - t0) * 1e-6),
                                (float)((r[2] - t0) * 1e-6), (float)(r[3] >> 32), (float)(r[3] & 0xffffffffu)});
        }
    }
    out->assign(4 * n, -1.f);
    for (size_t i = 0; i < 2 * n; ++i)
        if (h[2 * i] != ~0ull) {
            (*out)[2 * i] = (float)((h[2 * i] - t0) * 1e-6);
            (*out)[2 * i + 1] = (float)((h[2 * i + 1] - t0) * 1e-6);
        }
    return DR_OK;
}

int batch_run(Batch& B, cudaStream_t st) {
    Context& C = *g_ctx;
    if (!st) st = C.stream;
    if (B.runs++ == 0) {
        // a batch run once (a sweep) launches directly: capturing and
        // instantiating the graph would cost more host time than it saves
        DR_CUDA(cudaEventRecord(B.ev0, st));
        int rc = enqueue_batch(B, st);
        if (rc) return rc;
        DR_CUDA(cudaEventRecord(B.ev1, st));
        return DR_OK;
    }
    if (!B.graph) {
        cudaStream_t cap;
        DR_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        int rc = DR_OK;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess) { cudaStreamDestroy(cap); return cuda_fail(e, "begin capture"); }
        rc = enqueue_batch(B, cap);
        e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(e, "end capture");
        // node priorities: the shadow chains are placed before the walk blocks
        e = cudaGraphInstantiateWithFlags(&B.graph, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { B.graph = nullptr; return cuda_fail(e, "graph instantiate"); }
    }
    DR_CUDA(cudaEventRecord(B.ev0, st));
    DR_CUDA(cudaGraphLaunch(B.graph, st));
    DR_CUDA(cudaEventRecord(B.ev1, st));
    return DR_OK;
}

// Waits until no work of this batch is in flight: its last run (on whatever
// stream it was enqueued) and the engine stream, which carries its uploads.
// Other work on the device (other batches, a server's waves) goes on.
cudaError_t batch_idle(Batch& B) {
    cudaError_t e = B.ev1 ? cudaEventSynchronize(B.ev1) : cudaSuccess;
    if (e == cudaSuccess && g_ctx) e = cudaStreamSynchronize(g_ctx->stream);
    return e;
}

// DR_DEBUG builds: a failed device bounds check of the batch's runs becomes
// DR_ERR_INDEX with the site, index and bound (the batch must be idle).
static int debug_report(Batch& B) {
    if (!kDebugChecks || !B.dbg.p) return DR_OK;
    uint32_t rec[4] = {0, 0, 0, 0};
    DR_CUDA(cudaMemcpy(rec, B.dbg.p, sizeof(rec), cudaMemcpyDeviceToHost));
    if (!rec[0]) return DR_OK;
    set_error("device bounds check failed (DR_DEBUG build): site " + std::to_string(rec[0]) + ", index " +
              std::to_string(rec[1]) + " not below " + std::to_string(rec[2]) + " (" +
              std::to_string(rec[3]) + " failed checks)");
    return DR_ERR_INDEX;
}

int batch_read(Batch& B, uint32_t* p_res, uint32_t* q_res, uint64_t n_res, double* shadow,
               uint32_t* status) {
    Context& C = *g_ctx;
    DR_CUDA(cudaStreamSynchronize(C.stream));
    DR_CUDA(cudaEventSynchronize(B.ev1));
    cudaEventElapsedTime(&B.last_ms, B.ev0, B.ev1);
    if (B.runs != B.runs_read) {      // each run's device time is counted once
        stage_add(STAGE_DEVICE, B.last_ms);
        B.runs_read = B.runs;
    }
    int rc = debug_report(B);
    if (rc) return rc;
    const uint64_t n = std::min(n_res, B.n_res);
    if (p_res) DR_CUDA(cudaMemcpy(p_res, B.res.p, 4 * n, cudaMemcpyDeviceToHost));
    if (q_res)
        DR_CUDA(cudaMemcpy(q_res, B.res.as<uint32_t>() + std::max<uint64_t>(B.n_res, 1), 4 * n,
                           cudaMemcpyDeviceToHost));
    if (shadow) DR_CUDA(cudaMemcpy(shadow, B.shadow.p, 8ull * 6 * B.n_walks, cudaMemcpyDeviceToHost));
    if (status) DR_CUDA(cudaMemcpy(status, B.status.p, 4ull * B.n_walks, cudaMemcpyDeviceToHost));
    return DR_OK;
}

}  // namespace dr

// =============================================================================
// C ABI
// =============================================================================
using namespace dr;

namespace dr {

static CrtTables tables_of(const CrtSet& S) {
    CrtTables T;
    T.moduli = S.moduli.as<uint32_t>();
    T.pinv = S.pinv.as<uint32_t>();
    T.r2 = S.r2.as<uint32_t>();
    T.ginv = S.ginv.as<uint32_t>();
    T.Mlimbs = S.Mlimbs.as<uint32_t>();
    T.Mtotal = S.Mtotal.as<uint32_t>();
    T.K = S.K;
    T.L = S.L;
    T.garner = S.garner.p ? S.garner.as<uint32_t>() : nullptr;
    return T;
}

static int moduli_ok(const uint32_t* m, int K) {
    for (int k = 0; k < K; ++k)
        if (m[k] < 3u || m[k] >= (1u << 31) || !(m[k] & 1u)) {
            set_error("CRT modulus " + std::to_string(m[k]) + " outside odd [3, 2^31)");
            return DR_ERR_MODULUS;
        }
    return DR_OK;
}

// CRT on device pointers; custom moduli are copied to the host for validation.
static int crt_device(const uint32_t* res_d, int32_t K, int32_t n, const uint32_t* moduli_host,
                      uint32_t* limbs_d, int32_t stride, int32_t* sign_d, int32_t* nl_d,
                      uint32_t* ul_d, cudaStream_t st) {
    if (K < 1 || K > 1024 || n < 0) { set_error("CRT supports 1 <= K <= 1024"); return K > 1024 ? DR_ERR_UNSUPPORTED : DR_ERR_ARG; }
    std::shared_ptr<CrtSet> S;
    CrtSet custom;
    if (moduli_host) {
        int rc = moduli_ok(moduli_host, K);
        if (rc) return rc;
        rc = build_crt_set(moduli_host, K, custom, g_ctx->stream, false);
        if (rc) return rc;
    } else {
        int rc = crt_tables_std(K, &S);
        if (rc) return rc;
    }
    const CrtSet& set = moduli_host ? custom : *S;
    if (stride < set.L) { set_error("limb_stride below ceil(31K/32)+2"); return DR_ERR_ARG; }
    cudaError_t e = launch_crt(res_d, n, tables_of(set), limbs_d, stride, sign_d, nl_d, ul_d, g_ctx->sms, st);
    if (e != cudaSuccess) return cuda_fail(e, "crt launch");
    if (moduli_host) DR_CUDA(cudaStreamSynchronize(st));  // custom tables die with this call
    return DR_OK;
}

}  // namespace dr

extern "C" {

int dr_init(int device) {
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (g_ctx) {
        if (g_ctx->device == device) return DR_OK;
        set_error("dr_init: already initialised on another device");
        return DR_ERR_ARG;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return cuda_fail(e == cudaSuccess ? cudaErrorNoDevice : e, "dr_init");
    if (device < 0 || device >= n) { set_error("dr_init: no such device"); return DR_ERR_ARG; }
    DR_CUDA(cudaSetDevice(device));
    auto* c = new Context();
    c->device = device;
    DR_CUDA(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    DR_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    DR_CUDA(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    c->pool.resize(24);   // more than the launch groups of any batch, so none queue behind another
    for (auto& s : c->pool) DR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int prio_lo = 0, prio_hi = 0;
    DR_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    c->hpool.resize(8);
    for (auto& s : c->hpool) DR_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio_hi));
    const auto& tab = prime_table(DR_MAX_K);
    std::vector<uint32_t> pinv(DR_MAX_K), r2(DR_MAX_K);
    for (int k = 0; k < DR_MAX_K; ++k) {
        PrimeMeta m = prime_meta(tab[k]);
        pinv[k] = m.pinv;
        r2[k] = m.r2;
    }
    DR_CUDA(c->primes.alloc(4ull * DR_MAX_K));
    DR_CUDA(c->pinv.alloc(4ull * DR_MAX_K));
    DR_CUDA(c->r2.alloc(4ull * DR_MAX_K));
    DR_CUDA(cudaMemcpy(c->primes.p, tab.data(), 4ull * DR_MAX_K, cudaMemcpyHostToDevice));
    DR_CUDA(cudaMemcpy(c->pinv.p, pinv.data(), 4ull * DR_MAX_K, cudaMemcpyHostToDevice));
    DR_CUDA(cudaMemcpy(c->r2.p, r2.data(), 4ull * DR_MAX_K, cudaMemcpyHostToDevice));
    g_ctx = c;
    return DR_OK;
}

int dr_walk_batch(const dr_walk_desc* walks, int32_t n_walks, const uint8_t* blobs,
                  const uint64_t* blob_offsets, int32_t n_programs, const int64_t* axis_params,
                  uint64_t n_axis_params, const dr_tune* tune, uint32_t* p_res, uint32_t* q_res,
                  uint64_t n_res, double* shadow, uint32_t* status) {
    std::unique_ptr<Batch> B;
    int rc = batch_build(walks, n_walks, blobs, blob_offsets, n_programs, axis_params,
                         n_axis_params, tune, n_res, &B);
    if (rc) return rc;
    if (n_walks == 0) return DR_OK;
    {
        StageScope sc(STAGE_RUN, "dr.run");
        rc = batch_run(*B, ctx()->stream);
        if (rc == DR_OK) {
            const cudaError_t e = cudaEventSynchronize(B->ev1);
            if (e != cudaSuccess) rc = cuda_fail(e, "dr_walk_batch");
        }
    }
    if (rc) return rc;
    StageScope sc(STAGE_READ, "dr.read");
    return batch_read(*B, p_res, q_res, n_res, shadow, status);
}

int dr_batch_create(const dr_walk_desc* walks, int32_t n_walks, const uint8_t* blobs,
                    const uint64_t* blob_offsets, int32_t n_programs, const int64_t* axis_params,
                    uint64_t n_axis_params, const dr_tune* tune, int32_t* batch_out) {
    if (!batch_out) return DR_ERR_ARG;
    uint64_t n_res = 0;
    for (int32_t w = 0; w < n_walks; ++w) {
        n_res = std::max<uint64_t>(n_res, walks[w].res_offset + walks[w].K);
        if (walks[w].checkpoint) n_res = std::max<uint64_t>(n_res, walks[w].cp_res_offset + walks[w].K);
    }
    std::unique_ptr<Batch> B;
    int rc = batch_build(walks, n_walks, blobs, blob_offsets, n_programs, axis_params,
                         n_axis_params, tune, n_res, &B);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_batch_mu);
    const int32_t id = g_next_batch++;
    B->id = id;
    g_batches[id] = std::move(B);
    *batch_out = id;
    return DR_OK;
}

static Batch* find_batch(int32_t id) {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    auto it = g_batches.find(id);
    return it == g_batches.end() ? nullptr : it->second.get();
}

int dr_batch_run(int32_t batch, void* stream) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    if (B->n_walks == 0) return DR_OK;
    StageScope sc(STAGE_RUN, "dr.run");
    return batch_run(*B, static_cast<cudaStream_t>(stream));
}

int dr_stream_create(void** stream_out) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (!stream_out) return DR_ERR_ARG;
    cudaStream_t s = nullptr;
    DR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream_out = s;
    return DR_OK;
}

int dr_stream_destroy(void* stream) {
    if (!stream) return DR_ERR_ARG;
    DR_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    DR_CUDA(cudaStreamDestroy(static_cast<cudaStream_t>(stream)));
    return DR_OK;
}

int dr_batch_read(int32_t batch, uint32_t* p_res, uint32_t* q_res, uint64_t n_res, double* shadow,
                  uint32_t* status) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    // batch_read waits for this batch's end event (recorded on the stream it
    // ran on); other work on the device, a server's waves included, goes on
    StageScope sc(STAGE_READ, "dr.read");
    return batch_read(*B, p_res, q_res, n_res, shadow, status);
}

int dr_batch_stats(int32_t batch, uint64_t* prime_steps, uint32_t* n_tiles, uint32_t* n_launches,
                   float* last_ms) {
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    if (prime_steps) *prime_steps = B->prime_steps;
    if (n_tiles) *n_tiles = B->n_tiles;
    if (n_launches) {
        uint32_t k = 0;
        for (auto& L : B->launches) k += (L.items > 0) + (L.kind == 1 && L.items2 > 0);
        *n_launches = k;
    }
    if (last_ms) {
        if (B->ev1 && cudaEventQuery(B->ev1) == cudaSuccess) cudaEventElapsedTime(&B->last_ms, B->ev0, B->ev1);
        *last_ms = B->last_ms;
    }
    return DR_OK;
}

int dr_batch_set_pipeline(int32_t batch, const dr_pipeline* pl) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    if (!pl) return DR_ERR_ARG;
    if (pl->delta_mode < DR_DELTA_NONE || pl->delta_mode > DR_DELTA_SELF || pl->topk < 0 ||
        (pl->delta_mode != DR_DELTA_NONE && !pl->crt) || (pl->topk && pl->delta_mode == DR_DELTA_NONE)) {
        set_error("inconsistent pipeline (delta needs crt, top-k needs delta)");
        return DR_ERR_ARG;
    }
    if (pl->topk > topk_tile_size() / 2) { set_error("top-k above 2048"); return DR_ERR_UNSUPPORTED; }
    const uint32_t n = B->n_walks;
    int Kmax = 1;
    for (uint32_t w = 0; w < n; ++w) {
        Kmax = std::max<int>(Kmax, (int)B->h_walk_K[w]);
        if (pl->delta_mode == DR_DELTA_SELF && B->h_cp_off[w] == UINT64_MAX) {
            set_error("DR_DELTA_SELF needs a checkpoint on every walk");
            return DR_ERR_ARG;
        }
    }
    if (pl->crt && Kmax > 1024) { set_error("device CRT supports K <= 1024"); return DR_ERR_UNSUPPORTED; }
    if (pl->delta_mode == DR_DELTA_FIXED && (!pl->lnum || !pl->lden || pl->l_limbs < 1)) return DR_ERR_ARG;
    cudaStream_t st = g_ctx->stream;
    DR_CUDA(batch_idle(*B));
    if (B->graph) { cudaGraphExecDestroy(B->graph); B->graph = nullptr; }
    B->pipe = *pl;
    B->pipe.lnum = nullptr;
    B->pipe.lden = nullptr;
    B->pipe_on = pl->crt != 0;
    if (!B->pipe_on) return DR_OK;
    B->Lmax = crt_limbs_for(Kmax);
    // CRT values grouped by K: rows 4w + {p, q, checkpoint p, checkpoint q}
    const uint64_t qoff = std::max<uint64_t>(B->n_res, 1);
    std::map<int, std::vector<std::pair<uint64_t, uint32_t>>> byK;
    for (uint32_t w = 0; w < n; ++w) {
        auto& v = byK[(int)B->h_walk_K[w]];
        v.emplace_back(B->h_res_off[w], 4 * w);
        v.emplace_back(qoff + B->h_res_off[w], 4 * w + 1);
        if (B->h_cp_off[w] != UINT64_MAX) {
            v.emplace_back(B->h_cp_off[w], 4 * w + 2);
            v.emplace_back(qoff + B->h_cp_off[w], 4 * w + 3);
        }
    }
    std::vector<uint64_t> in;
    std::vector<uint32_t> out;
    B->crt_groups.clear();
    for (auto& kv : byK) {
        std::shared_ptr<CrtSet> S;
        rc = crt_tables_std(kv.first, &S);   // build tables now, outside any capture
        if (rc) return rc;
        B->crt_groups.push_back({kv.first, (uint32_t)in.size(), (uint32_t)kv.second.size()});
        for (auto& e : kv.second) { in.push_back(e.first); out.push_back(e.second); }
    }
    if ((rc = upload(B->crt_in, in, st))) return rc;
    if ((rc = upload(B->crt_out, out, st))) return rc;
    DR_CUDA(B->limbs.alloc(4ull * 4 * std::max<uint32_t>(n, 1) * B->Lmax));
    DR_CUDA(cudaMemsetAsync(B->limbs.p, 0, B->limbs.bytes, st));
    DR_CUDA(B->signs.alloc(4ull * 4 * std::max<uint32_t>(n, 1)));
    DR_CUDA(cudaMemsetAsync(B->signs.p, 0, B->signs.bytes, st));
    DR_CUDA(B->delta.alloc(8ull * std::max<uint32_t>(n, 1)));
    if (pl->delta_mode == DR_DELTA_FIXED) {
        std::vector<uint32_t> ln(pl->lnum, pl->lnum + pl->l_limbs), ld(pl->lden, pl->lden + pl->l_limbs);
        std::vector<int32_t> sg{pl->lnum_sign};
        if ((rc = upload(B->tgt_num, ln, st))) return rc;
        if ((rc = upload(B->tgt_den, ld, st))) return rc;
        if ((rc = upload(B->tgt_sign, sg, st))) return rc;
    }
    B->tk_counts.clear();
    if (pl->topk > 0 && n > 0) {
        int cnt = (int)n;
        size_t cap = 16;
        do {
            B->tk_counts.push_back(cnt);
            const int tile = topk_tile_for(cnt, pl->topk);
            cnt = ((cnt + tile - 1) / tile) * std::min(pl->topk, tile);
            cap = std::max(cap, (size_t)cnt);
        } while (cnt > pl->topk);
        for (int i = 0; i < 2; ++i) {
            DR_CUDA(B->tk_keys[i].alloc(8 * cap));
            DR_CUDA(B->tk_idx[i].alloc(4 * cap));
        }
        B->tk_final = (int)((B->tk_counts.size() - 1) & 1);
    }
    DR_CUDA(cudaStreamSynchronize(st));
    return DR_OK;
}

int dr_batch_set_bank(int32_t batch, int32_t n_consts, int32_t l_limbs, const uint32_t* num,
                      const int32_t* num_sign, const uint32_t* den) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    if (n_consts < 0 || (n_consts > 0 && (l_limbs < 1 || !num || !num_sign || !den))) return DR_ERR_ARG;
    if (n_consts > 4096 || l_limbs > 1024) { set_error("bank above 4096 constants or 1024 limbs"); return DR_ERR_UNSUPPORTED; }
    DR_CUDA(batch_idle(*B));
    if (B->graph) { cudaGraphExecDestroy(B->graph); B->graph = nullptr; }
    B->bank_n = n_consts;
    B->bank_l = l_limbs;
    if (!n_consts) return DR_OK;
    cudaStream_t st = g_ctx->stream;
    std::vector<uint32_t> nv(num, num + (size_t)n_consts * l_limbs), dv(den, den + (size_t)n_consts * l_limbs);
    std::vector<int32_t> sv(num_sign, num_sign + n_consts);
    if ((rc = upload(B->bank_num, nv, st))) return rc;
    if ((rc = upload(B->bank_den, dv, st))) return rc;
    if ((rc = upload(B->bank_sign, sv, st))) return rc;
    DR_CUDA(B->bank_out.alloc(8ull * std::max<uint32_t>(B->n_walks, 1) * n_consts));
    DR_CUDA(cudaStreamSynchronize(st));
    return DR_OK;
}

int dr_batch_read_bank(int32_t batch, double* delta, int32_t max_values) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    if (!B->pipe_on || B->bank_n <= 0) {
        set_error("no constant bank on this batch");
        return DR_ERR_ARG;
    }
    DR_CUDA(batch_idle(*B));
    const int64_t n = (int64_t)(B->tk_counts.empty() ? (int)B->n_walks
                                                     : std::min<int>(B->pipe.topk, (int)B->n_walks)) * B->bank_n;
    DR_CUDA(cudaMemcpy(delta, B->bank_out.p, 8ull * std::min<int64_t>(n, max_values), cudaMemcpyDeviceToHost));
    return DR_OK;
}

int dr_batch_read_pipeline(int32_t batch, double* delta, int32_t* topk_idx, double* topk_val,
                           uint32_t* limbs, int32_t* signs, int32_t limb_stride) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    if (!B->pipe_on) { set_error("no pipeline set on this batch"); return DR_ERR_ARG; }
    StageScope sc(STAGE_READ, "dr.read");
    DR_CUDA(batch_idle(*B));
    if ((rc = debug_report(*B))) return rc;
    const uint32_t n = B->n_walks;
    std::vector<double> dl;
    if ((delta || topk_val) && B->pipe.delta_mode != DR_DELTA_NONE) {
        dl.resize(n);
        DR_CUDA(cudaMemcpy(dl.data(), B->delta.p, 8ull * n, cudaMemcpyDeviceToHost));
        if (delta) std::memcpy(delta, dl.data(), 8ull * n);
    }
    if ((topk_idx || topk_val) && !B->tk_counts.empty()) {
        const int keep = std::min<int>(B->pipe.topk, (int)n);
        std::vector<uint32_t> idx(keep);
        DR_CUDA(cudaMemcpy(idx.data(), B->tk_idx[B->tk_final].p, 4ull * keep, cudaMemcpyDeviceToHost));
        for (int i = 0; i < keep; ++i) {
            if (topk_idx) topk_idx[i] = (int32_t)idx[i];
            if (topk_val) topk_val[i] = dl[idx[i]];
        }
    }
    if (limbs) {
        if (limb_stride < B->Lmax) { set_error("limb_stride below the batch's limb count"); return DR_ERR_ARG; }
        std::vector<uint32_t> tmp(4ull * n * B->Lmax);
        DR_CUDA(cudaMemcpy(tmp.data(), B->limbs.p, 4ull * tmp.size(), cudaMemcpyDeviceToHost));
        for (size_t r = 0; r < 4ull * n; ++r) {
            std::memcpy(limbs + r * limb_stride, tmp.data() + r * B->Lmax, 4ull * B->Lmax);
            std::memset(limbs + r * limb_stride + B->Lmax, 0, 4ull * (limb_stride - B->Lmax));
        }
    }
    if (signs) DR_CUDA(cudaMemcpy(signs, B->signs.p, 4ull * 4 * n, cudaMemcpyDeviceToHost));
    return DR_OK;
}

// Autotuner: time candidate depth-chunk lengths and warps per block on the
// batch itself (graph replays, CUDA events, best of three after a capture
// run) and remember the fastest for batches of the same shape.
int dr_autotune(const dr_walk_desc* walks, int32_t n_walks, const uint8_t* blobs,
                const uint64_t* blob_offsets, int32_t n_programs, const int64_t* axis_params,
                uint64_t n_axis_params, dr_tune* best, float* best_ms) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (!best) return DR_ERR_ARG;
    Context& C = *g_ctx;
    uint64_t n_res = 0;
    for (int32_t w = 0; w < n_walks; ++w) {
        n_res = std::max<uint64_t>(n_res, walks[w].res_offset + walks[w].K);
        if (walks[w].checkpoint) n_res = std::max<uint64_t>(n_res, walks[w].cp_res_offset + walks[w].K);
    }
    auto time_one = [&](const dr_tune& t, float* ms, uint32_t* chunk_used, std::string* sig) -> int {
        std::unique_ptr<Batch> B;
        int r = batch_build(walks, n_walks, blobs, blob_offsets, n_programs, axis_params, n_axis_params,
                            &t, n_res, &B);
        if (r) return r;
        if (chunk_used) *chunk_used = B->chunk_used;
        if (sig) *sig = B->signature;
        if ((r = batch_run(*B, C.stream))) return r;
        float m = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            if ((r = batch_run(*B, C.stream))) return r;
            DR_CUDA(cudaEventSynchronize(B->ev1));
            float x = 0.f;
            cudaEventElapsedTime(&x, B->ev0, B->ev1);
            m = std::min(m, x);
        }
        *ms = m;
        return DR_OK;
    };
    // the default policy's chunk anchors the candidates
    dr_tune t{};
    t.engine = best->engine;
    t.shadow_buffer_mb = best->shadow_buffer_mb;
    t.warps_per_block = 4;
    uint32_t c0 = 0;
    std::string sig;
    float ms0 = 0.f;
    if ((rc = time_one(t, &ms0, &c0, &sig))) return rc;
    dr_tune bt = t;
    bt.chunk_steps = c0;
    float bms = ms0;
    for (uint32_t f : {1u, 2u, 4u}) {
        for (uint32_t wpb : {1u, 2u, 4u}) {   // k_walk is compiled for at most 128 threads
            for (int dir = 0; dir < 2; ++dir) {
                if (f == 1 && dir == 1) continue;
                const uint64_t c = dir == 0 ? (uint64_t)c0 * f : (uint64_t)c0 / f;
                if (c < 256 || c > 4194304 || (f == 1 && wpb == 4)) continue;
                dr_tune cand = t;
                cand.chunk_steps = (uint32_t)c;
                cand.warps_per_block = wpb;
                float ms = 0.f;
                rc = time_one(cand, &ms, nullptr, nullptr);
                if (rc == DR_ERR_UNSUPPORTED) continue;   // e.g. shared memory of a wider block
                if (rc) return rc;
                // a shape must beat the default policy by 2% (replay times
                // spread by ~1%): shorter chunks mean more tiles, which every
                // build pays for on the host, for a gain below the noise
                if (ms < bms && ms < 0.98f * ms0) { bms = ms; bt = cand; }
            }
        }
    }
    // then two chain warps per scheduler for the integer-difference shadows of
    // depth up to d: worth it when those chains end before the walks do.
    // Every depth is timed and the fastest kept if it beats no packing by 1%
    // (above the replays' spread of ~0.5% for a best of 3; packing costs the
    // host nothing)
    dr_tune pt = bt;
    float pms = bms;
    for (uint32_t d : {1u, 2u, 3u, 4u, 16u}) {
        dr_tune cand = bt;
        cand.chain_pack_depth = d;
        float ms = 0.f;
        rc = time_one(cand, &ms, nullptr, nullptr);
        if (rc == DR_ERR_UNSUPPORTED) continue;
        if (rc) return rc;
        if (ms < pms) { pms = ms; pt = cand; }
    }
    if (pms < 0.99f * bms) { bms = pms; bt = pt; }
    {
        std::lock_guard<std::mutex> lk(C.cache_mu);
        C.tuned[sig] = {bt.chunk_steps, bt.warps_per_block, bt.chain_pack_depth};
    }
    best->chunk_steps = bt.chunk_steps;
    best->warps_per_block = bt.warps_per_block;
    best->chain_pack_depth = bt.chain_pack_depth;
    if (best_ms) *best_ms = bms;
    return DR_OK;
}

int dr_debug_host_pool(int32_t parts, uint64_t n, int32_t repeats, uint64_t* index_sum, uint64_t* visits) {
    if (parts < 1 || repeats < 0 || !index_sum || !visits || n > (1ull << 32)) return DR_ERR_ARG;
    uint64_t sum = 0, count = 0;
    for (int32_t r = 0; r < repeats; ++r) {
        const int p = 1 + (int)((parts + r) % parts);          // vary the part count per job
        std::vector<uint64_t> psum(p, 0), pcount(p, 0);
        std::vector<uint8_t> seen(n, 0);
        host_pool().run(p, (size_t)n, [&](int part, size_t lo, size_t hi) {
            for (size_t i = lo; i < hi; ++i) {
                psum[part] += i;
                ++pcount[part];
                seen[i] = (uint8_t)(seen[i] + 1);
            }
        });
        for (int k = 0; k < p; ++k) {
            sum += psum[k];
            count += pcount[k];
        }
        for (uint64_t i = 0; i < n; ++i)
            if (seen[i] != 1) return DR_ERR_INDEX;
    }
    *index_sum = sum;
    *visits = count;
    return DR_OK;
}

int dr_debug_build_phases(double* ms, int32_t n) {
    for (int i = 0; i < n && i < kBuildPhases; ++i) ms[i] = g_build_ms[i];
    return DR_OK;
}

int dr_debug_build_info(int32_t* debug_checks) {
    if (!debug_checks) return DR_ERR_ARG;
    *debug_checks = kDebugChecks ? 1 : 0;
    return DR_OK;
}

int dr_debug_batch_timeline(int32_t batch, int32_t max_launches, int32_t* n_launches, float* spans) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    std::vector<float> t;
    rc = batch_timeline(*B, &t);
    if (rc) return rc;
    if (n_launches) *n_launches = (int32_t)(t.size() / 4);
    for (int i = 0; i < (int)t.size() && i < 4 * max_launches; ++i)
        if (spans) spans[i] = t[i];
    return DR_OK;
}

int dr_debug_chain_items(int32_t batch, int32_t max_items, int32_t* n_items, float* rows) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    if (n_items) *n_items = (int32_t)(B->item_rows.size() / 6);
    for (size_t i = 0; i < B->item_rows.size() && i < 6ull * std::max(max_items, 0); ++i)
        if (rows) rows[i] = B->item_rows[i];
    return DR_OK;
}

int dr_batch_profile(int32_t batch, int32_t max_launches, int32_t* n_launches, int32_t* kind,
                     int32_t* cls, int32_t* m, int32_t* degree, uint32_t* items, float* ms,
                     float* ms2) {
    int rc = ensure_ctx();
    if (rc) return rc;
    Batch* B = find_batch(batch);
    if (!B) return DR_ERR_HANDLE;
    std::vector<float> t, t2;
    rc = batch_profile(*B, &t, &t2);
    if (rc) return rc;
    const int n = (int)B->launches.size();
    if (n_launches) *n_launches = n;
    for (int i = 0; i < n && i < max_launches; ++i) {
        const LaunchSpec& L = B->launches[i];
        if (kind) kind[i] = L.kind;
        if (cls) cls[i] = (int32_t)L.cls;
        if (m) m[i] = (int32_t)L.m;
        if (degree) degree[i] = (int32_t)(L.kind == 1 ? L.split_D : L.D);
        if (items) items[i] = L.items;
        if (ms) ms[i] = t[i];
        if (ms2) ms2[i] = t2[i];
    }
    return DR_OK;
}

int dr_batch_destroy(int32_t batch) {
    std::unique_ptr<Batch> B;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        auto it = g_batches.find(batch);
        if (it == g_batches.end()) return DR_ERR_HANDLE;
        B = std::move(it->second);
        g_batches.erase(it);
    }
    if (g_ctx) batch_idle(*B);
    return DR_OK;
}

int dr_crt_batch(const uint32_t* residues, int32_t K, int32_t n, const uint32_t* moduli, uint32_t* limbs,
                 int32_t limb_stride, int32_t* sign_out, int32_t* nlimbs_out, uint32_t* unsigned_limbs) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (n == 0) return DR_OK;
    if (!residues || !limbs || !sign_out || !nlimbs_out || n < 0) return DR_ERR_ARG;
    if (K < 1 || K > 1024) { set_error("CRT supports 1 <= K <= 1024"); return K > 1024 ? DR_ERR_UNSUPPORTED : DR_ERR_ARG; }
    if (limb_stride < crt_limbs_for(K)) { set_error("limb_stride below ceil(31K/32)+2"); return DR_ERR_ARG; }
    cudaStream_t st = g_ctx->stream;
    DevBuf r, l, s, nl, ul;
    DR_CUDA(r.alloc(4ull * K * n));
    DR_CUDA(l.alloc(4ull * limb_stride * n));
    DR_CUDA(s.alloc(4ull * n));
    DR_CUDA(nl.alloc(4ull * n));
    if (unsigned_limbs) DR_CUDA(ul.alloc(4ull * limb_stride * n));
    DR_CUDA(cudaMemcpyAsync(r.p, residues, 4ull * K * n, cudaMemcpyHostToDevice, st));
    rc = crt_device(r.as<uint32_t>(), K, n, moduli, l.as<uint32_t>(), limb_stride, s.as<int32_t>(),
                    nl.as<int32_t>(), unsigned_limbs ? ul.as<uint32_t>() : nullptr, st);
    if (rc) return rc;
    DR_CUDA(cudaMemcpyAsync(limbs, l.p, 4ull * limb_stride * n, cudaMemcpyDeviceToHost, st));
    DR_CUDA(cudaMemcpyAsync(sign_out, s.p, 4ull * n, cudaMemcpyDeviceToHost, st));
    DR_CUDA(cudaMemcpyAsync(nlimbs_out, nl.p, 4ull * n, cudaMemcpyDeviceToHost, st));
    if (unsigned_limbs) DR_CUDA(cudaMemcpyAsync(unsigned_limbs, ul.p, 4ull * limb_stride * n, cudaMemcpyDeviceToHost, st));
    DR_CUDA(cudaStreamSynchronize(st));
    return DR_OK;
}

int dr_crt_batch_device(const uint32_t* residues_d, int32_t K, int32_t n, const uint32_t* moduli_d,
                        uint32_t* limbs_d, int32_t limb_stride, int32_t* sign_d, int32_t* nlimbs_d,
                        void* stream) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (n == 0) return DR_OK;
    std::vector<uint32_t> mh;
    if (moduli_d) {
        if (K < 1 || K > 1024) return DR_ERR_UNSUPPORTED;
        mh.resize(K);
        DR_CUDA(cudaMemcpy(mh.data(), moduli_d, 4ull * K, cudaMemcpyDeviceToHost));
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g_ctx->stream;
    return crt_device(residues_d, K, n, moduli_d ? mh.data() : nullptr, limbs_d, limb_stride, sign_d,
                      nlimbs_d, nullptr, st);
}

int dr_delta_batch(const uint32_t* p_limbs, const int32_t* p_sign, const uint32_t* q_limbs,
                   const int32_t* q_sign, int32_t n, int32_t limb_stride, const uint32_t* lnum_limbs,
                   const int32_t* lnum_sign, const uint32_t* lden_limbs, int32_t l_stride,
                   int32_t per_item_target, double* delta_out) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (n == 0) return DR_OK;
    if (n < 0 || !p_limbs || !q_limbs || !p_sign || !q_sign || !lnum_limbs || !lnum_sign ||
        !lden_limbs || !delta_out || limb_stride < 1 || l_stride < 1)
        return DR_ERR_ARG;
    if (limb_stride + l_stride > 4096) { set_error("delta limbs above 4096"); return DR_ERR_UNSUPPORTED; }
    const int nt = per_item_target ? n : 1;
    cudaStream_t st = g_ctx->stream;
    DevBuf p, ps, q, qs, ln, lns, ld, out;
    DR_CUDA(p.alloc(4ull * limb_stride * n));
    DR_CUDA(q.alloc(4ull * limb_stride * n));
    DR_CUDA(ps.alloc(4ull * n));
    DR_CUDA(qs.alloc(4ull * n));
    DR_CUDA(ln.alloc(4ull * l_stride * nt));
    DR_CUDA(lns.alloc(4ull * nt));
    DR_CUDA(ld.alloc(4ull * l_stride * nt));
    DR_CUDA(out.alloc(8ull * n));
    DR_CUDA(cudaMemcpyAsync(p.p, p_limbs, 4ull * limb_stride * n, cudaMemcpyHostToDevice, st));
    DR_CUDA(cudaMemcpyAsync(q.p, q_limbs, 4ull * limb_stride * n, cudaMemcpyHostToDevice, st));
    DR_CUDA(cudaMemcpyAsync(ps.p, p_sign, 4ull * n, cudaMemcpyHostToDevice, st));
    DR_CUDA(cudaMemcpyAsync(qs.p, q_sign, 4ull * n, cudaMemcpyHostToDevice, st));
    DR_CUDA(cudaMemcpyAsync(ln.p, lnum_limbs, 4ull * l_stride * nt, cudaMemcpyHostToDevice, st));
    DR_CUDA(cudaMemcpyAsync(lns.p, lnum_sign, 4ull * nt, cudaMemcpyHostToDevice, st));
    DR_CUDA(cudaMemcpyAsync(ld.p, lden_limbs, 4ull * l_stride * nt, cudaMemcpyHostToDevice, st));
    DeltaArgs D{};
    D.p = p.as<uint32_t>(); D.ps = ps.as<int32_t>();
    D.q = q.as<uint32_t>(); D.qs = qs.as<int32_t>();
    D.n = n; D.nl = limb_stride; D.istride = (size_t)limb_stride; D.sstride = 1;
    D.ln = ln.as<uint32_t>(); D.lns = lns.as<int32_t>(); D.ld = ld.as<uint32_t>(); D.lds = nullptr;
    D.lnl = l_stride; D.listride = (size_t)l_stride; D.lsstride = 1;
    D.per_item = per_item_target ? 1 : 0;
    D.out = out.as<double>();
    D.maxlen = ((limb_stride + l_stride + 4) + 1) & ~1;
    cudaError_t e = launch_delta(D, g_ctx->sms, st);
    if (e != cudaSuccess) return cuda_fail(e, "delta launch");
    DR_CUDA(cudaMemcpyAsync(delta_out, out.p, 8ull * n, cudaMemcpyDeviceToHost, st));
    DR_CUDA(cudaStreamSynchronize(st));
    return DR_OK;
}

}  // extern "C"

namespace dr {

// Tile sort of n (key, index) pairs -- from vals (keys computed) or from
// in_keys/in_idx -- down to the best k, in passes over the two scratch pairs;
// returns the buffer pair holding the sorted best k (at least min(k, n)).
static int topk_tiles(const double* vals, const uint64_t* in_keys, const uint32_t* in_idx, int n, int k,
                      DevBuf (&keys)[2], DevBuf (&idx)[2], cudaStream_t st, int* out_buf) {
    const int tile0 = topk_tile_for(n, k);
    const size_t cap = (size_t)((n + tile0 - 1) / tile0) * k + 16;
    for (int b = 0; b < 2; ++b) {
        keys[b].pooled = idx[b].pooled = true;
        DR_CUDA(keys[b].alloc(8 * cap));
        DR_CUDA(idx[b].alloc(4 * cap));
    }
    int cnt = n, cur = 0;
    cudaError_t e = launch_topk_tile(vals, in_keys, in_idx, cnt, k, keys[0].as<uint64_t>(), idx[0].as<uint32_t>(), st);
    if (e != cudaSuccess) return cuda_fail(e, "topk");
    cnt = ((cnt + tile0 - 1) / tile0) * std::min(k, tile0);
    while (cnt > k) {
        const int tile = topk_tile_for(cnt, k);
        e = launch_topk_tile(nullptr, keys[cur].as<uint64_t>(), idx[cur].as<uint32_t>(), cnt, k,
                             keys[cur ^ 1].as<uint64_t>(), idx[cur ^ 1].as<uint32_t>(), st);
        if (e != cudaSuccess) return cuda_fail(e, "topk");
        cnt = ((cnt + tile - 1) / tile) * std::min(k, tile);
        cur ^= 1;
    }
    *out_buf = cur;
    return DR_OK;
}

// Values below this count use the tile sort directly; above it the
// threshold filter (delta_topk.cu) reads them once.
constexpr int kTopkFilterMin = 1 << 18;
constexpr int kTopkSample = 1 << 16;
constexpr int kTopkCand = 1 << 16;   // largest candidate buffer

// Top-k (k <= 2048) of n device doubles, highest first, NaN last, ties by
// lower index: idx_d[j], val_d[j] (device pointers; either may be null) for
// j < min(k, n).  Ends with a stream synchronisation (the filter's count is
// checked on the host).  *filtered: whether the threshold filter decided.
int topk_device(const double* vals, int n, int k, int32_t* idx_d, double* val_d, cudaStream_t st,
                bool* filtered) {
    const int keep = std::min(k, n);
    if (filtered) *filtered = false;
    if (keep <= 0) return DR_OK;
    DevBuf keys[2], idx[2];
    int out = 0, rc;
    if (n >= kTopkFilterMin) {
        // threshold: the r-th best of a strided sample, r about 4x the k it
        // should hold at the sample's density, plus a margin
        const int64_t stride = n / kTopkSample;
        const int s = kTopkSample;
        const int r = std::min(topk_tile_size() / 2,
                               (int)(4 * (((int64_t)k * s + n - 1) / n)) + 8);
        // candidates: about r * n / s values reach the threshold; the
        // buffer holds twice that (a power of two, 4096 .. kTopkCand), and
        // an overflow falls back to sorting everything
        const int64_t expect = (int64_t)r * ((n + s - 1) / s);
        int cand = 4096;
        while (cand < kTopkCand && cand < 2 * expect) cand <<= 1;
        DevBuf skeys, sidx, ckeys, cidx, count;
        skeys.pooled = sidx.pooled = ckeys.pooled = cidx.pooled = count.pooled = true;
        DR_CUDA(skeys.alloc(8ull * s));
        DR_CUDA(sidx.alloc(4ull * s));
        DR_CUDA(ckeys.alloc(8ull * cand));
        DR_CUDA(cidx.alloc(4ull * cand));
        DR_CUDA(count.alloc(16));
        DR_CUDA(launch_topk_sample(vals, stride, s, skeys.as<uint64_t>(), sidx.as<uint32_t>(), st));
        DevBuf sk[2], si[2];
        int sb = 0;
        if ((rc = topk_tiles(nullptr, skeys.as<uint64_t>(), sidx.as<uint32_t>(), s, r, sk, si, st, &sb))) return rc;
        const uint64_t* thr = sk[sb].as<uint64_t>() + (r - 1);
        DR_CUDA(cudaMemsetAsync(ckeys.p, 0, 8ull * cand, st));      // key 0, index ~0: rank last
        DR_CUDA(cudaMemsetAsync(cidx.p, 0xff, 4ull * cand, st));
        DR_CUDA(cudaMemsetAsync(count.p, 0, 16, st));
        DR_CUDA(launch_topk_filter(vals, n, thr, ckeys.as<uint64_t>(), cidx.as<uint32_t>(), cand,
                                   count.as<unsigned int>(), g_ctx->sms, st));
        if ((rc = topk_tiles(nullptr, ckeys.as<uint64_t>(), cidx.as<uint32_t>(), cand, k, keys, idx, st, &out)))
            return rc;
        DR_CUDA(launch_topk_gather(vals, idx[out].as<uint32_t>(), keep, val_d, idx_d, st));
        unsigned int cnt = 0;
        DR_CUDA(cudaMemcpyAsync(&cnt, count.p, sizeof(cnt), cudaMemcpyDeviceToHost, st));
        DR_CUDA(cudaStreamSynchronize(st));
        if (cnt >= (unsigned)keep && cnt <= (unsigned)cand) {
            if (filtered) *filtered = true;
            return DR_OK;
        }
        // too few or too many candidates (heavy ties, NaNs): sort everything
    }
    if ((rc = topk_tiles(vals, nullptr, nullptr, n, k, keys, idx, st, &out))) return rc;
    DR_CUDA(launch_topk_gather(vals, idx[out].as<uint32_t>(), keep, val_d, idx_d, st));
    DR_CUDA(cudaStreamSynchronize(st));
    return DR_OK;
}

}  // namespace dr

extern "C" {

int dr_topk(const double* delta, int32_t n, int32_t k, int32_t* idx_out, double* val_out) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (n < 0 || k < 0 || (n > 0 && !delta) || (k > 0 && n > 0 && !idx_out)) return DR_ERR_ARG;
    if (k > topk_tile_size() / 2) { set_error("k above 2048"); return DR_ERR_UNSUPPORTED; }
    const int keep = std::min(k, n);
    if (keep == 0) return DR_OK;
    cudaStream_t st = g_ctx->stream;
    DevBuf v, oi;
    v.pooled = oi.pooled = true;
    DR_CUDA(v.alloc(8ull * n));
    DR_CUDA(oi.alloc(4ull * keep));
    DR_CUDA(cudaMemcpyAsync(v.p, delta, 8ull * n, cudaMemcpyHostToDevice, st));
    if ((rc = topk_device(v.as<double>(), n, k, oi.as<int32_t>(), nullptr, st, nullptr))) return rc;
    DR_CUDA(cudaMemcpy(idx_out, oi.p, 4ull * keep, cudaMemcpyDeviceToHost));
    if (val_out)
        for (int i = 0; i < keep; ++i) val_out[i] = delta[idx_out[i]];
    return DR_OK;
}

int dr_topk_device(const double* delta_d, int32_t n, int32_t k, int32_t* idx_d, double* val_d, void* stream,
                   int32_t* filtered) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (n < 0 || k < 0 || (n > 0 && !delta_d)) return DR_ERR_ARG;
    if (k > topk_tile_size() / 2) { set_error("k above 2048"); return DR_ERR_UNSUPPORTED; }
    bool f = false;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g_ctx->stream;
    if ((rc = topk_device(delta_d, n, k, idx_d, val_d, st, &f))) return rc;
    if (filtered) *filtered = f ? 1 : 0;
    return DR_OK;
}

}  // extern "C"
