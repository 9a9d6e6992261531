// Serving: continuous batching of walk requests (dr_serve_*).
//
// A scheduler thread owns the device side.  Submitted requests wait in a FIFO
// until their device state fits under the memory cap (running product and
// denominator per 32-prime block, FP64 shadow state, outputs); admitted
// requests are cut into segments.  Every wave takes the next walk segment and
// the next shadow segment of each admitted request that is not already in
// flight, builds the tiles (depth chunks x prime blocks), and launches the
// same persistent kernels as batches do, with combine groups that resume from
// and write back to resident state slots.  Up to max_inflight waves run at
// once on separate streams, so requests that arrive while others are on the
// GPU join the next wave and their work overlaps with what is running.
// Completion is observed with cudaEventQuery from the host thread; the
// device never waits on anything.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "../../include/dreams_b200.h"
#include "../../include/dreams_b200_debug.h"
#include "engine.h"
#include "host_common.h"
#include "launch.h"
#include "shadow_impl.cuh"
#include "walk_impl.cuh"

namespace dr {
namespace {

using Clock = std::chrono::steady_clock;

constexpr int kServeMaxM = 4;
constexpr uint32_t kServeStride = kServeMaxM * kServeMaxM * 32;   // words per state slot

struct Req {
    int64_t id = 0;
    std::shared_ptr<Plan> plan;
    std::string blob;
    dr_walk_desc d{};
    std::vector<int64_t> axis;
    uint32_t shadow_mode = SHADOW_NONE;
    int tdeg = 0;                 // kernel difference depth
    uint64_t walk_next = 0, shadow_next = 0;
    bool walk_done = false, shadow_done = false;
    bool inflight = false, admitted = false, done = false, cancelled = false;
    std::vector<uint32_t> slots;  // resident product slots, one per prime block
    int shadow_slot = -1;
    uint64_t need = 0;
    Clock::time_point t_submit, t_done;
    std::vector<uint32_t> p, q;
    double sh[3] = {0, 0, 0};
    uint32_t status = 0;
    int error = DR_OK;            // the request failed (done with no results): poll returns it
    std::string error_msg;
};

struct Wave {
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev = nullptr;
    bool busy = false;
    bool has_long = false;                // carries requests that need more waves
    size_t log = 0;                       // index of this launch in Server::wlog
    std::vector<int64_t> reqs;            // requests with a segment in this wave
    std::vector<uint8_t> walk_final;      // per request: walk part finishes here
    std::vector<uint8_t> shadow_final;    // per request: shadow finishes here
    std::vector<uint64_t> walk_end, shadow_end;
    std::vector<uint64_t> res_off;        // output offsets of finishing walks
    std::vector<uint32_t> widx;           // walk-table index per request
    // one upload (programs, code, constants, walks, axes, tiles, groups,
    // shadow segments, eval items) and one zero-filled block (combine
    // counters, queues, status); buffers only grow, from the engine's pool,
    // so a wave never frees device memory while other waves run
    DevBuf up, zero, chunkP, chunkSig, res, shadow, mf;
    uint8_t* h_up = nullptr;              // pinned staging of the upload
    uint32_t* h_res = nullptr;            // pinned outputs
    double* h_sh = nullptr;
    uint32_t* h_st = nullptr;
    size_t h_up_cap = 0, h_res_cap = 0, h_sh_cap = 0, h_st_cap = 0;
    uint64_t n_res = 0;
    uint32_t n_walks = 0;
    uint64_t prime_steps = 0;
    uint64_t n_tiles = 0, max_span = 0;   // walk tiles and longest shadow segment of the launch
    double t_geom = 0, t_alloc = 0, t_launch = 0;   // host ms at the end of each launch_wave phase
    Wave() {
        for (DevBuf* b : {&up, &zero, &chunkP, &chunkSig, &res, &shadow, &mf}) b->pooled = true;
    }
};

// Per-launch record of the scheduler (dr_debug_serve_waves).
struct WaveLog {
    double t_sel = 0, t_launched = 0, t_harvest = 0;   // ms since dr_serve_open
    float gpu_ms = 0;
    uint32_t n_req = 0, has_long = 0, wave = 0;
    uint64_t walk_tiles = 0, shadow_span = 0;
    double t_geom = 0, t_alloc = 0, t_launch = 0;      // ms since dr_serve_open: launch_wave phases
};

struct Server {
    dr_serve_config cfg{};
    uint64_t cap = 0, admitted = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::thread thr;
    bool stop = false;
    std::deque<int64_t> pending;
    std::vector<int64_t> active;
    std::unordered_map<int64_t, std::unique_ptr<Req>> reqs;
    int64_t next_id = 1;
    DevBuf stP, stSig, stShadow;
    std::vector<uint32_t> free_slots, free_shadow;
    std::deque<Wave> waves;               // deque: elements never move
    uint64_t completed = 0, prime_steps = 0;
    Clock::time_point t_open;
    std::vector<WaveLog> wlog;            // capped at kMaxWaveLog entries
    std::map<std::tuple<int, uint32_t, uint32_t, uint32_t, size_t>, int> occ_cache;
    std::vector<void*> retired_pinned;    // outgrown pinned buffers, freed at close
    int error = DR_OK;
    std::string error_msg;
    uint64_t failed = 0;                  // requests ended with an error of their own
    // host-side fault injection (dr_debug_serve_inject): the next admissions
    // fail as if allocating their resident state had failed, and the next
    // wave launches fail as if growing their device buffers had failed
    uint32_t inject_admit = 0, inject_wave = 0;
};

std::mutex g_srv_mu;
std::map<int32_t, std::unique_ptr<Server>> g_servers;
int32_t g_next_srv = 1;

Server* find_server(int32_t h) {
    std::lock_guard<std::mutex> lk(g_srv_mu);
    auto it = g_servers.find(h);
    return it == g_servers.end() ? nullptr : it->second.get();
}

constexpr size_t kMaxWaveLog = 1u << 16;

double ms_since(const Server& S, Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(t - S.t_open).count();
}

uint64_t request_bytes(const Req& r) {
    const uint64_t nb = (r.d.K + 31) / 32;
    return nb * (kServeStride + 32) * 4 + (r.shadow_mode ? kShadowStateStride * 8 : 0) + 8ull * r.d.K;
}

// Grow-only device buffer with headroom, so steady-state waves allocate nothing.
cudaError_t grow(DevBuf& b, size_t n) {
    if (b.p && n <= b.bytes) return cudaSuccess;
    return b.alloc(std::max<size_t>(n + n / 2, 1u << 16));
}

// Grow-only pinned host buffer.  cudaFreeHost waits for the whole device
// (every wave in flight), so an outgrown buffer is not freed here but kept in
// `retired` until the server closes; growth doubles, so that costs at most
// the final size again.
template <class T>
cudaError_t grow_host(T*& p, size_t& cap, size_t n, std::vector<void*>& retired) {
    if (p && n <= cap) return cudaSuccess;
    if (p) retired.push_back(p);
    p = nullptr;
    cap = std::max<size_t>(2 * n, (1u << 18) / sizeof(T));
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&p), sizeof(T) * cap);
    if (e != cudaSuccess) { p = nullptr; cap = 0; }
    return e;
}

// Layout of the packed upload: byte offset of each array, 16-byte aligned.
struct Packer {
    size_t total = 0;
    template <class T> size_t add(const std::vector<T>& v) {
        const size_t off = total;
        total += (sizeof(T) * v.size() + 15) & ~size_t(15);
        return off;
    }
};

int occupancy(Server& S, int kind, uint32_t cls, uint32_t m, uint32_t D, int block, size_t smem) {
    auto key = std::make_tuple(kind, cls, m, D, smem);
    auto it = S.occ_cache.find(key);
    if (it != S.occ_cache.end()) return it->second;
    int occ = 0;
    WalkArgs wa{};
    ShadowArgs sa{};
    cudaError_t e;
    if (kind == 0) e = walk_dispatch(cls, m, D, 0, block, smem, nullptr, wa, &occ);
    else e = shadow_fd_dispatch(cls, m, D, 0, block, smem, nullptr, sa, &occ);
    if (e != cudaSuccess) occ = 0;
    S.occ_cache[key] = occ;
    return occ;
}

// Build and launch one wave from the admitted requests (called with S.mu held
// only for the selection; the device work is issued without the lock).
int launch_wave(Server& S, Wave& W, const std::vector<Req*>& sel) {
    Context& C = *ctx();
    const uint32_t chunk = S.cfg.chunk_steps ? S.cfg.chunk_steps : 4096;
    const uint64_t seg_walk = (uint64_t)chunk * 16;
    // interpreted shadow segments: at most 8192 steps, fewer when the wave's
    // step-matrix buffer would pass 1 GiB
    uint64_t n_interp = 0, ne_max = 1;
    for (Req* r : sel)
        if (r->shadow_mode == SHADOW_INTERP && !r->shadow_done) {
            ++n_interp;
            ne_max = std::max<uint64_t>(ne_max, shadow_entries(r->plan->m, r->plan->fcomp));
        }
    uint64_t seg_shadow = 8192;
    if (n_interp) {
        const uint64_t cap = (1ull << 30) / 8;
        seg_shadow = std::min<uint64_t>(
            8192, std::max<uint64_t>(kEvalSteps, cap / (n_interp * ne_max) / kEvalSteps * kEvalSteps));
    }
    std::map<std::string, int> pidx;
    std::vector<DevProgram> progs;
    std::vector<uint4> code;
    std::vector<int64_t> consts, axis;
    std::vector<DevWalk> walks;
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, std::vector<DevTile>> tsets;
    std::vector<DevGroup> groups;
    std::map<std::tuple<int, uint32_t, uint32_t, uint32_t>, std::vector<DevShadowSeg>> ssets;
    uint32_t slots = 0;
    uint64_t nres = 0, ps = 0;
    W.max_span = 0;
    W.reqs.clear();
    W.walk_final.clear();
    W.shadow_final.clear();
    W.walk_end.clear();
    W.shadow_end.clear();
    W.res_off.clear();
    W.widx.clear();
    for (Req* r : sel) {
        const Plan& P = *r->plan;
        auto it = pidx.find(r->blob);
        int pi;
        if (it == pidx.end()) {
            DevProgram d{};
            d.m = P.m; d.dim = P.dim; d.cls = P.cls; d.degree = P.degree;
            d.op_off = (uint32_t)code.size(); d.n_ops = (uint32_t)P.ops.size();
            for (const Insn& in : P.ops) code.push_back(make_uint4(in.op, in.a, in.b, in.c));
            d.n_regs = P.n_regs;
            d.dop_off = (uint32_t)code.size(); d.dn_ops = (uint32_t)P.dops.size();
            for (const Insn& in : P.dops) code.push_back(make_uint4(in.op, in.a, in.b, in.c));
            d.dn_regs = P.dn_regs;
            d.c_off = (uint32_t)consts.size(); d.n_consts = (uint32_t)P.consts.size();
            consts.insert(consts.end(), P.consts.begin(), P.consts.end());
            d.n_streams = P.n_streams; d.zero_reg = P.zero_reg;
            d.fcomp = P.fcomp ? 1u : 0u;
            pi = (int)progs.size();
            progs.push_back(d);
            pidx.emplace(r->blob, pi);
        } else {
            pi = it->second;
        }
        const uint32_t wi = (uint32_t)walks.size();
        DevWalk w{};
        w.prog = (uint32_t)pi; w.K = r->d.K; w.flags = r->d.flags; w.q_row = r->d.q_row;
        w.p_row = r->d.p_row;
        w.a0 = r->d.a0; w.depth = r->d.depth; w.checkpoint = 0;
        w.axis_off = axis.size();
        axis.insert(axis.end(), r->axis.begin(), r->axis.end());
        w.shadow_mode = r->shadow_mode;
        const uint64_t we = std::min<uint64_t>(r->d.depth, r->walk_next + seg_walk);
        const bool wfinal = !r->walk_done && we >= r->d.depth;
        w.res_off = wfinal ? nres : 0;
        if (wfinal) nres += r->d.K;
        walks.push_back(w);
        W.reqs.push_back(r->id);
        W.widx.push_back(wi);
        W.walk_final.push_back(wfinal);
        W.walk_end.push_back(we);
        W.res_off.push_back(w.res_off);
        // walk tiles for [walk_next, we)
        if (!r->walk_done) {
            const uint64_t a = r->walk_next, b = we;
            std::vector<std::pair<uint64_t, uint64_t>> ranges;
            if (b == a) ranges.emplace_back(a, a);
            for (uint64_t s0 = a; s0 < b; s0 += chunk) ranges.emplace_back(s0, std::min<uint64_t>(b, s0 + chunk));
            const uint32_t cls = P.cls;
            const uint32_t D = cls == CLS_INTERP ? 0u : (uint32_t)r->tdeg;
            auto& tv = tsets[std::make_tuple(cls, P.m, D)];
            for (uint32_t blk = 0, p0 = 0; p0 < r->d.K; p0 += 32, ++blk) {
                DevGroup g{};
                g.walk = wi; g.prime0 = p0; g.nprimes = std::min<uint32_t>(32, r->d.K - p0);
                g.n_chunks = (uint32_t)ranges.size(); g.slot0 = slots; slots += g.n_chunks;
                g.cp_chunks = 0; g.state = r->slots[blk];
                g.flags = (a == 0 ? GROUP_FIRST : 0u) | (wfinal ? GROUP_FINAL : 0u);
                const uint32_t gi = (uint32_t)groups.size();
                groups.push_back(g);
                for (uint32_t c = 0; c < g.n_chunks; ++c) {
                    DevTile t{};
                    t.walk = wi; t.group = gi; t.prime0 = p0; t.nprimes = g.nprimes; t.chunk = c;
                    t.slot = g.slot0 + c; t.s0 = ranges[c].first; t.s1 = ranges[c].second;
                    tv.push_back(t);
                }
            }
            ps += (uint64_t)r->d.K * (b - a);
        }
        // shadow segment
        uint64_t se = r->shadow_next;
        bool sfinal = false;
        if (r->shadow_mode != SHADOW_NONE && !r->shadow_done) {
            se = std::min<uint64_t>(r->d.depth, r->shadow_next + seg_shadow);
            sfinal = se >= r->d.depth;
            W.max_span = std::max<uint64_t>(W.max_span, se - r->shadow_next);
            DevShadowSeg g{wi, (uint32_t)r->shadow_slot, r->shadow_next, se, 0, 0, 0};
            if (r->shadow_mode == SHADOW_INTFD)
                ssets[std::make_tuple(2, (uint32_t)P.cls, P.m, (uint32_t)r->tdeg)].push_back(g);
            else
                ssets[std::make_tuple(1, progs[pi].fcomp, P.m, 0u)].push_back(g);
        }
        W.shadow_end.push_back(se);
        W.shadow_final.push_back(sfinal);
    }
    W.n_res = std::max<uint64_t>(nres, 1);
    W.n_walks = (uint32_t)walks.size();
    W.prime_steps = ps;

    // launches
    std::vector<LaunchSpec> L;
    std::vector<DevTile> tiles;
    std::vector<DevShadowSeg> segs;
    const int wpb = 4;
    for (auto& kv : tsets) {
        auto& v = kv.second;
        std::stable_sort(v.begin(), v.end(), [](const DevTile& x, const DevTile& y) { return (x.s1 - x.s0) > (y.s1 - y.s0); });
        LaunchSpec s{};
        s.kind = 0;
        std::tie(s.cls, s.m, s.D) = kv.first;
        s.off = (uint32_t)tiles.size(); s.count = (uint32_t)v.size(); s.items = s.count;
        uint32_t rr = 1, rc = 1;
        for (auto& t : v) {
            const DevProgram& G = progs[walks[t.walk].prog];
            rr = std::max(rr, std::max(G.n_regs, G.dn_regs));
            rc = std::max(rc, G.n_consts);
        }
        const uint32_t ns = (uint32_t)std::max(streams_for(s.cls, s.m), 0);
        s.rows_regs = rr; s.rows_consts = rc; s.rows_stage = std::max(s.m * s.m, (s.D + 1) * ns);
        s.rows_per_warp = s.rows_regs + s.rows_consts + 3 * kMaxAxes + s.rows_stage;
        tiles.insert(tiles.end(), v.begin(), v.end());
        L.push_back(s);
    }
    std::vector<uint32_t> eval_items;
    uint64_t mf_doubles = 0;
    uint32_t max_dim = 1;
    for (auto& d : progs) max_dim = std::max(max_dim, d.dim);
    for (auto& kv : ssets) {
        auto& v = kv.second;
        int kind;
        uint32_t cls, m, D;
        std::tie(kind, cls, m, D) = kv.first;
        uint32_t rr = 1;
        for (auto& g : v) {
            const DevProgram& G = progs[walks[g.walk].prog];
            rr = std::max(rr, kind == 1 ? G.n_regs : G.dn_regs);
        }
        if (kind == 1) {
            std::stable_sort(v.begin(), v.end(), [](const DevShadowSeg& x, const DevShadowSeg& y) {
                return (x.s1 - x.s0) > (y.s1 - y.s0);
            });
            mf_doubles += shadow_interp_plan(L, segs, eval_items, v, m, cls, rr, mf_doubles,
                                             UINT64_MAX, 0);
            continue;
        }
        LaunchSpec s{};
        s.kind = kind;
        s.cls = cls; s.m = m; s.D = D;
        s.off = (uint32_t)segs.size(); s.count = (uint32_t)v.size();
        s.items = (s.count + 31) / 32;
        const uint32_t ns = (uint32_t)streams_for(s.cls, s.m);
        s.rows_regs = rr;
        s.rows_per_warp = rr + kMaxAxes + (s.D + 1) * ns + ns;
        segs.insert(segs.end(), v.begin(), v.end());
        L.push_back(s);
    }
    uint32_t q = 0;
    for (auto& s : L) {
        s.queue = q++;
        if (s.kind == 1) {
            s.queue2 = q++;
            const int rc = shadow_interp_geometry(s, max_dim, C.sms, segs.data() + s.off, false);
            if (rc) return rc;
            continue;
        }
        s.block = 32 * wpb;
        s.smem = (size_t)s.rows_per_warp * 32 * (s.kind == 0 ? 4 : 8) * wpb;
        const int occ = occupancy(S, s.kind, s.cls, s.m, s.D, s.block, s.smem);
        if (occ < 1) { set_error("serving: kernel cannot be resident"); return DR_ERR_UNSUPPORTED; }
        s.grid = std::max(1, std::min((int)((s.items + wpb - 1) / wpb), occ * C.sms));
    }
    cudaStream_t st = W.st;
    cudaError_t e = cudaSuccess;
#define SV(x) do { e = (x); if (e != cudaSuccess) return cuda_fail(e, #x); } while (0)
    W.t_geom = ms_since(S, Clock::now());
    W.n_tiles = tiles.size();
    Packer pk;
    const size_t o_progs = pk.add(progs), o_code = pk.add(code), o_consts = pk.add(consts),
                 o_walks = pk.add(walks), o_axis = pk.add(axis), o_tiles = pk.add(tiles),
                 o_groups = pk.add(groups), o_segs = pk.add(segs), o_eval = pk.add(eval_items);
    // zero-filled: combine counters | queues | status
    const size_t n_done = std::max<size_t>(groups.size(), 1), n_q = std::max<uint32_t>(q, 1),
                 n_st = std::max<uint32_t>(W.n_walks, 1);
    const size_t zbytes = 4ull * (n_done + n_q + n_st);
    // every buffer grows before any work is enqueued, so a failed allocation
    // leaves the wave idle and only this wave's requests fail (DR_ERR_NOMEM)
    if (S.inject_wave) {
        --S.inject_wave;
        set_error("serving: wave buffer allocation failed (injected by dr_debug_serve_inject)");
        return DR_ERR_NOMEM;
    }
    {
        const cudaError_t g[] = {
            grow_host(W.h_up, W.h_up_cap, pk.total + 16, S.retired_pinned), grow(W.up, pk.total + 16),
            grow(W.zero, zbytes), grow(W.mf, 8ull * std::max<uint64_t>(mf_doubles, 1)),
            grow(W.chunkP, 4ull * std::max<uint32_t>(slots, 1) * kServeStride),
            grow(W.chunkSig, 4ull * std::max<uint32_t>(slots, 1) * 32), grow(W.res, 8ull * W.n_res),
            grow(W.shadow, 8ull * 6 * std::max<uint32_t>(W.n_walks, 1))};
        for (cudaError_t ge : g)
            if (ge != cudaSuccess) {
                cudaGetLastError();   // an allocation failure is not sticky: clear it
                set_error(std::string("serving: wave buffer allocation failed: ") + cudaGetErrorString(ge));
                return ge == cudaErrorMemoryAllocation ? DR_ERR_NOMEM : DR_ERR_CUDA;
            }
    }
    SV(cudaEventRecord(W.ev0, st));
    auto stage = [&](size_t off, const auto& v) {
        if (!v.empty()) std::memcpy(W.h_up + off, v.data(), sizeof(v[0]) * v.size());
    };
    stage(o_progs, progs); stage(o_code, code); stage(o_consts, consts); stage(o_walks, walks);
    stage(o_axis, axis); stage(o_tiles, tiles); stage(o_groups, groups); stage(o_segs, segs);
    stage(o_eval, eval_items);
    if (pk.total) SV(cudaMemcpyAsync(W.up.p, W.h_up, pk.total, cudaMemcpyHostToDevice, st));
    auto at = [&](size_t off) { return static_cast<uint8_t*>(W.up.p) + off; };
    SV(cudaMemsetAsync(W.zero.p, 0, zbytes, st));
    uint32_t* z_done = W.zero.as<uint32_t>();
    uint32_t* z_queue = z_done + n_done;
    uint32_t* z_status = z_queue + n_q;
    W.t_alloc = ms_since(S, Clock::now());
    WalkArgs wa{};
    wa.progs = reinterpret_cast<const DevProgram*>(at(o_progs));
    wa.code = reinterpret_cast<const uint4*>(at(o_code));
    wa.consts = reinterpret_cast<const int64_t*>(at(o_consts));
    wa.walks = reinterpret_cast<const DevWalk*>(at(o_walks));
    wa.axis = reinterpret_cast<const int64_t*>(at(o_axis));
    wa.groups = reinterpret_cast<const DevGroup*>(at(o_groups));
    wa.group_done = z_done; wa.chunk_P = W.chunkP.as<uint32_t>();
    wa.chunk_stride = kServeStride; wa.chunk_sig = W.chunkSig.as<uint32_t>();
    wa.state_P = S.stP.as<uint32_t>(); wa.state_sig = S.stSig.as<uint32_t>();
    wa.primes = C.primes.as<uint32_t>(); wa.pinv = C.pinv.as<uint32_t>(); wa.r2 = C.r2.as<uint32_t>();
    wa.p_res = W.res.as<uint32_t>(); wa.q_res = W.res.as<uint32_t>() + W.n_res; wa.status = z_status;
    ShadowArgs sa{};
    sa.progs = wa.progs; sa.code = wa.code; sa.consts = wa.consts; sa.walks = wa.walks; sa.axis = wa.axis;
    sa.shadow = W.shadow.as<double>(); sa.n_walks = W.n_walks; sa.status = wa.status;
    sa.state = S.stShadow.as<double>();
    sa.mf = W.mf.as<double>();
    const DevTile* d_tiles = reinterpret_cast<const DevTile*>(at(o_tiles));
    const DevShadowSeg* d_segs = reinterpret_cast<const DevShadowSeg*>(at(o_segs));
    const uint32_t* d_eval = reinterpret_cast<const uint32_t*>(at(o_eval));
    for (auto& s : L) {
        if (s.items == 0 && s.items2 == 0) continue;
        if (s.kind == 0) {
            wa.tiles = d_tiles + s.off; wa.n_tiles = s.count;
            wa.queue = z_queue + s.queue;
            wa.rows_regs = s.rows_regs; wa.rows_consts = s.rows_consts; wa.rows_stage = s.rows_stage;
            wa.rows_per_warp = s.rows_per_warp;
            wa.rows_axes = kMaxAxes;   // the wave layout keeps rows for every axis
            SV(walk_dispatch(s.cls, s.m, s.D, s.grid, s.block, s.smem, st, wa, nullptr));
        } else {
            sa.segs = d_segs + s.off; sa.n_items = s.items; sa.n_list = s.count;
            sa.queue = z_queue + s.queue; sa.rows_regs = s.rows_regs;
            sa.rows_per_warp = s.rows_per_warp;
            if (s.kind == 1) SV(launch_shadow_interp(s, sa, z_queue, d_eval, st));
            else SV(shadow_fd_dispatch(s.cls, s.m, s.D, s.grid, s.block, s.smem, st, sa, nullptr));
        }
    }
    W.t_launch = ms_since(S, Clock::now());
    // outputs back to pinned host memory
    SV(grow_host(W.h_res, W.h_res_cap, 2 * W.n_res, S.retired_pinned));
    SV(grow_host(W.h_sh, W.h_sh_cap, 3ull * W.n_walks, S.retired_pinned));
    SV(grow_host(W.h_st, W.h_st_cap, (size_t)W.n_walks, S.retired_pinned));
    SV(cudaMemcpyAsync(W.h_res, W.res.p, 8ull * W.n_res, cudaMemcpyDeviceToHost, st));
    SV(cudaMemcpyAsync(W.h_sh, W.shadow.p, 8ull * 3 * W.n_walks, cudaMemcpyDeviceToHost, st));
    SV(cudaMemcpyAsync(W.h_st, z_status, 4ull * W.n_walks, cudaMemcpyDeviceToHost, st));
    SV(cudaEventRecord(W.ev, st));
#undef SV
    W.busy = true;
    return DR_OK;
}

void release(Server& S, Req& r) {
    for (uint32_t s : r.slots) S.free_slots.push_back(s);
    r.slots.clear();
    if (r.shadow_slot >= 0) S.free_shadow.push_back((uint32_t)r.shadow_slot);
    r.shadow_slot = -1;
    if (r.admitted) S.admitted -= r.need;
    r.admitted = false;
}

void harvest(Server& S, Wave& W) {
    if (W.log < S.wlog.size()) {
        WaveLog& g = S.wlog[W.log];
        g.t_harvest = ms_since(S, Clock::now());
        float ms = 0;
        if (cudaEventElapsedTime(&ms, W.ev0, W.ev) == cudaSuccess) g.gpu_ms = ms;
    }
    for (size_t i = 0; i < W.reqs.size(); ++i) {
        auto it = S.reqs.find(W.reqs[i]);
        if (it == S.reqs.end()) continue;
        Req& r = *it->second;
        r.inflight = false;
        if (r.cancelled) {
            release(S, r);
            auto a = std::find(S.active.begin(), S.active.end(), r.id);
            if (a != S.active.end()) S.active.erase(a);
            S.reqs.erase(it);
            continue;
        }
        if (!r.walk_done) {
            S.prime_steps += (uint64_t)r.d.K * (W.walk_end[i] - r.walk_next);
            r.walk_next = W.walk_end[i];
            if (W.walk_final[i]) {
                r.walk_done = true;
                r.p.assign(W.h_res + W.res_off[i], W.h_res + W.res_off[i] + r.d.K);
                r.q.assign(W.h_res + W.n_res + W.res_off[i], W.h_res + W.n_res + W.res_off[i] + r.d.K);
            }
        }
        r.status |= W.h_st[W.widx[i]];
        if (r.shadow_mode != SHADOW_NONE && !r.shadow_done) {
            r.shadow_next = W.shadow_end[i];
            if (W.shadow_final[i]) {
                r.shadow_done = true;
                std::memcpy(r.sh, W.h_sh + 3 * W.widx[i], sizeof(r.sh));
            }
        }
        if (r.walk_done && r.shadow_done && !r.done) {
            r.done = true;
            r.t_done = Clock::now();
            ++S.completed;
            release(S, r);
            S.active.erase(std::find(S.active.begin(), S.active.end(), r.id));
        }
    }
    W.busy = false;
}

// End a request with an error of its own: it keeps no slots and no memory,
// poll returns the error, and the server goes on with the others.
void fail_request(Server& S, Req& r, int rc, const std::string& msg) {
    release(S, r);
    r.inflight = false;
    r.error = rc;
    r.error_msg = msg;
    r.done = true;
    r.t_done = Clock::now();
    ++S.failed;
    auto a = std::find(S.active.begin(), S.active.end(), r.id);
    if (a != S.active.end()) S.active.erase(a);
}

void admit(Server& S) {
    for (auto it = S.pending.begin(); it != S.pending.end();) {
        Req& r = *S.reqs[*it];
        if (r.cancelled) { it = S.pending.erase(it); continue; }
        const uint64_t nb = (r.d.K + 31) / 32;
        const bool fits = S.admitted + r.need <= S.cap && S.free_slots.size() >= nb &&
                          (r.shadow_mode == SHADOW_NONE || !S.free_shadow.empty());
        if (!fits) { ++it; continue; }   // smaller later requests may still fit
        if (S.inject_admit) {
            --S.inject_admit;
            fail_request(S, r, DR_ERR_NOMEM,
                         "serving: admission could not allocate the request's resident state "
                         "(injected by dr_debug_serve_inject)");
            it = S.pending.erase(it);
            continue;
        }
        for (uint64_t b = 0; b < nb; ++b) { r.slots.push_back(S.free_slots.back()); S.free_slots.pop_back(); }
        if (r.shadow_mode != SHADOW_NONE) { r.shadow_slot = (int)S.free_shadow.back(); S.free_shadow.pop_back(); }
        S.admitted += r.need;
        r.admitted = true;
        S.active.push_back(r.id);
        it = S.pending.erase(it);
    }
}

// Load every kernel a wave can launch (lazy module loading would otherwise
// put each kernel's first load, about a millisecond, on the latency of the
// requests in the wave that first needs it) and give each wave its first
// staging buffers.
void prewarm(Server& S) {
    WalkArgs wa{};
    ShadowArgs sa{};
    int occ = 0;
    for (uint32_t cls : {(uint32_t)CLS_COMPANION, (uint32_t)CLS_RATIONAL, (uint32_t)CLS_DENSE, (uint32_t)CLS_INTERP})
        for (uint32_t m = 1; m <= (uint32_t)kServeMaxM; ++m)
            for (uint32_t D = 0; D <= (cls == CLS_INTERP ? 0u : 32u); ++D) {
                walk_dispatch(cls, m, D, 0, 128, 0, nullptr, wa, &occ);
                if (cls == CLS_COMPANION || cls == CLS_DENSE) shadow_fd_dispatch(cls, m, D, 0, 128, 0, nullptr, sa, &occ);
            }
    for (uint32_t U : {1u, 2u, 4u}) shadow_eval_dispatch(U, 0, 128, 0, nullptr, sa, &occ);
    for (uint32_t m = 1; m <= (uint32_t)kServeMaxM; ++m)
        for (uint32_t f = 0; f < 4; ++f) shadow_chain_dispatch(m, f, 0, 32, 0, nullptr, sa, &occ);
    cudaGetLastError();   // the instances that do not exist answered cudaErrorInvalidValue
    for (Wave& W : S.waves) {
        // first sizes for waves of several thousand tiles and a few hundred requests
        grow_host(W.h_up, W.h_up_cap, 1u << 20, S.retired_pinned);
        grow_host(W.h_res, W.h_res_cap, 1u << 17, S.retired_pinned);
        grow_host(W.h_sh, W.h_sh_cap, 1u << 13, S.retired_pinned);
        grow_host(W.h_st, W.h_st_cap, 1u << 13, S.retired_pinned);
        grow(W.up, 1u << 20);
        grow(W.chunkP, 8u << 20);     // ~4000 chunk slots
        grow(W.chunkSig, 1u << 19);
        grow(W.mf, 16u << 20);        // ~128 interpreted shadow segments of 8192 steps
        for (DevBuf* b : {&W.zero, &W.res, &W.shadow}) grow(*b, 1);
    }
}

void loop(Server* Sp) {
    Server& S = *Sp;
    cudaSetDevice(ctx()->device);
    const uint32_t max_tiles = S.cfg.max_wave_tiles ? S.cfg.max_wave_tiles : 65536;
    for (;;) {
        std::vector<Req*> sel;
        Wave* free_wave = nullptr;
        {
            std::unique_lock<std::mutex> lk(S.mu);
            for (Wave& W : S.waves)
                if (W.busy && cudaEventQuery(W.ev) == cudaSuccess) harvest(S, W);
            S.cv.notify_all();
            if (S.stop) break;
            admit(S);
            uint32_t free_idx = 0;
            for (Wave& W : S.waves) {
                if (!W.busy) { free_wave = &W; break; }
                ++free_idx;
            }
            if (free_wave) {
                // requests that need more waves ("long": deep walks, long
                // shadows) never share a wave with ones that finish in this
                // wave, and hold at most all but one wave slot, so short
                // requests always find a wave that is not held up by a long
                // segment
                const uint64_t seg_walk = (uint64_t)(S.cfg.chunk_steps ? S.cfg.chunk_steps : 4096) * 16;
                auto is_long = [&](const Req& r) {
                    return (!r.walk_done && r.d.depth - r.walk_next > seg_walk) ||
                           (r.shadow_mode != SHADOW_NONE && !r.shadow_done && r.d.depth - r.shadow_next > 8192);
                };
                uint32_t long_waves = 0;
                for (const Wave& W : S.waves) long_waves += W.busy && W.has_long;
                bool short_pending = false, long_pending = false;
                for (int64_t id : S.active) {
                    const Req& r = *S.reqs[id];
                    if (r.inflight || r.done || r.cancelled) continue;
                    (is_long(r) ? long_pending : short_pending) = true;
                }
                const bool take_long = long_pending && long_waves + 1 < (uint32_t)S.waves.size();
                const bool want_long = take_long && !short_pending ? true : (take_long && long_waves == 0);
                uint64_t tiles = 0;
                for (int64_t id : S.active) {
                    Req& r = *S.reqs[id];
                    if (r.inflight || r.done) continue;
                    if (r.cancelled) continue;
                    const bool lg = is_long(r);
                    if (short_pending && !want_long ? lg : !lg) continue;
                    if (lg && !take_long) continue;
                    const uint64_t nb = (r.d.K + 31) / 32;
                    const uint64_t span = std::min<uint64_t>(r.d.depth - r.walk_next, seg_walk);
                    const uint64_t t = r.walk_done ? 0 : nb * std::max<uint64_t>(1, (span + 4095) / 4096);
                    if (!sel.empty() && tiles + t > max_tiles) break;
                    tiles += t;
                    r.inflight = true;
                    sel.push_back(&r);
                }
                free_wave->has_long = !sel.empty() && is_long(*sel.front());
            }
            if (sel.empty()) {
                S.cv.wait_for(lk, std::chrono::microseconds(200));
                continue;
            }
            free_wave->log = SIZE_MAX;
            if (S.wlog.size() < kMaxWaveLog) {
                WaveLog g;
                g.t_sel = ms_since(S, Clock::now());
                g.n_req = (uint32_t)sel.size();
                g.has_long = free_wave->has_long;
                g.wave = free_idx;
                free_wave->log = S.wlog.size();
                S.wlog.push_back(g);
            }
        }
        int rc;
        {
            NvtxRange nvtx("dr.serve.wave");
            rc = launch_wave(S, *free_wave, sel);
        }
        {
            std::lock_guard<std::mutex> lk(S.mu);
            if (free_wave->log < S.wlog.size()) {
                WaveLog& g = S.wlog[free_wave->log];
                g.t_launched = ms_since(S, Clock::now());
                g.walk_tiles = free_wave->n_tiles;
                g.shadow_span = free_wave->max_span;
                g.t_geom = free_wave->t_geom;
                g.t_alloc = free_wave->t_alloc;
                g.t_launch = free_wave->t_launch;
            }
        }
        if (rc == DR_ERR_NOMEM) {
            // the wave's buffers could not grow: its requests fail, the
            // server (whose context is intact) serves the rest
            std::lock_guard<std::mutex> lk(S.mu);
            const std::string msg = last_error();
            for (Req* r : sel) fail_request(S, *r, rc, msg);
            S.cv.notify_all();
        } else if (rc != DR_OK) {
            std::lock_guard<std::mutex> lk(S.mu);
            S.error = rc;
            S.error_msg = last_error();
            for (Req* r : sel) r->inflight = false;
        }
        if (rc != DR_OK) std::this_thread::sleep_for(std::chrono::milliseconds(1));
    }
}

}  // namespace
}  // namespace dr

using namespace dr;

extern "C" {

int dr_serve_open(const dr_serve_config* cfg, int32_t* server_out) {
    int rc = ensure_ctx();
    if (rc) return rc;
    if (!server_out) return DR_ERR_ARG;
    auto S = std::make_unique<Server>();
    if (cfg) S->cfg = *cfg;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    S->cap = S->cfg.mem_cap_bytes ? S->cfg.mem_cap_bytes : std::min<uint64_t>(fr / 2, 1ull << 30);
    const uint64_t per = (kServeStride + 32) * 4ull;
    uint64_t n_slots = std::min<uint64_t>(S->cap / per + 1, 1u << 20);
    uint64_t n_shadow = std::min<uint64_t>(S->cap / (kShadowStateStride * 8) + 1, 1u << 18);
    {
        cudaError_t e = S->stP.alloc(4ull * kServeStride * n_slots);
        if (e == cudaSuccess) e = S->stSig.alloc(4ull * 32 * n_slots);
        if (e == cudaSuccess) e = S->stShadow.alloc(8ull * kShadowStateStride * n_shadow);
        if (e != cudaSuccess) return cuda_fail(e, "dr_serve_open");
    }
    for (uint64_t i = n_slots; i-- > 0;) S->free_slots.push_back((uint32_t)i);
    for (uint64_t i = n_shadow; i-- > 0;) S->free_shadow.push_back((uint32_t)i);
    const uint32_t nw = S->cfg.max_inflight ? S->cfg.max_inflight : 2;
    S->waves.resize(nw);
    for (Wave& W : S->waves) {
        cudaError_t e = cudaStreamCreateWithFlags(&W.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&W.ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&W.ev);
        if (e != cudaSuccess) return cuda_fail(e, "dr_serve_open");
    }
    prewarm(*S);
    S->t_open = Clock::now();
    Server* raw = S.get();
    S->thr = std::thread(loop, raw);
    std::lock_guard<std::mutex> lk(g_srv_mu);
    const int32_t h = g_next_srv++;
    g_servers[h] = std::move(S);
    *server_out = h;
    return DR_OK;
}

int dr_serve_submit(int32_t server, const dr_walk_desc* walk, const uint8_t* blob, uint64_t blob_size,
                    const int64_t* axis_params, int64_t* request_out) {
    Server* S = find_server(server);
    if (!S) return DR_ERR_HANDLE;
    if (!walk || !blob || !request_out) return DR_ERR_ARG;
    auto r = std::make_unique<Req>();
    std::string err;
    int rc = get_plan(blob, blob_size, &r->plan, &err);
    if (rc) { set_error(err); return rc; }
    const Plan& P = *r->plan;
    if (P.m > (uint32_t)kServeMaxM) { set_error("serving supports m <= 4"); return DR_ERR_UNSUPPORTED; }
    if (walk->K < 1 || walk->K > DR_MAX_K) return DR_ERR_UNSUPPORTED;
    if (walk->q_row >= P.m || walk->p_row >= P.m) return DR_ERR_ARG;
    if (walk->flags & DR_WALK_VEC) {
        set_error("serving does not take state-vector walks");
        return DR_ERR_UNSUPPORTED;
    }
    if (walk->checkpoint) { set_error("serving walks take no checkpoint"); return DR_ERR_ARG; }
    if ((walk->flags & DR_WALK_INIT_PCF) && P.m < 2) return DR_ERR_ARG;
    if (P.dim && !axis_params) return DR_ERR_ARG;
    r->d = *walk;
    r->blob.assign(reinterpret_cast<const char*>(blob), (size_t)blob_size);
    r->axis.assign(axis_params, axis_params + 4 * P.dim);
    for (uint32_t a = 0; a < P.dim; ++a)
        if (r->axis[4 * a + 1] == 0 || r->axis[4 * a + 3] == 0) { set_error("zero denominator"); return DR_ERR_ARG; }
    r->tdeg = P.cls == CLS_INTERP ? 0 : template_degree(P.cls, P.m, P.degree);
    if (walk->flags & DR_WALK_SHADOW) {
        r->shadow_mode = SHADOW_INTERP;
        if (!P.has_inv && (P.cls == CLS_COMPANION || P.cls == CLS_DENSE) && r->tdeg > 0) {
            const double b = float_bound_log2(P, r->axis.data(), walk->depth + 1);
            if (b < 53.0 && b + r->tdeg < 61.0) r->shadow_mode = SHADOW_INTFD;
        }
    } else {
        r->shadow_done = true;
    }
    r->need = request_bytes(*r);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(S->mu);
    if (r->need > S->cap) { set_error("request larger than the admission cap"); return DR_ERR_NOMEM; }
    r->id = S->next_id++;
    *request_out = r->id;
    S->pending.push_back(r->id);
    S->reqs[r->id] = std::move(r);
    S->cv.notify_all();
    return DR_OK;
}

int dr_serve_poll(int32_t server, int64_t request, uint32_t* p_res, uint32_t* q_res, double* shadow,
                  uint32_t* status, double* latency_s) {
    Server* S = find_server(server);
    if (!S) return DR_ERR_HANDLE;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->error) { set_error(S->error_msg); return S->error; }
    auto it = S->reqs.find(request);
    if (it == S->reqs.end()) return DR_ERR_HANDLE;
    Req& r = *it->second;
    if (r.cancelled) return DR_ERR_HANDLE;
    if (!r.done) return DR_ERR_BUSY;
    if (r.error != DR_OK) {
        const int rc = r.error;
        set_error(r.error_msg);
        S->reqs.erase(it);
        return rc;
    }
    if (p_res) std::memcpy(p_res, r.p.data(), 4ull * r.d.K);
    if (q_res) std::memcpy(q_res, r.q.data(), 4ull * r.d.K);
    if (shadow) std::memcpy(shadow, r.sh, sizeof(r.sh));
    if (status) *status = r.status;
    if (latency_s) *latency_s = std::chrono::duration<double>(r.t_done - r.t_submit).count();
    S->reqs.erase(it);
    return DR_OK;
}

int dr_serve_cancel(int32_t server, int64_t request) {
    Server* S = find_server(server);
    if (!S) return DR_ERR_HANDLE;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(request);
    if (it == S->reqs.end()) return DR_ERR_HANDLE;
    Req& r = *it->second;
    if (r.inflight) { r.cancelled = true; return DR_OK; }   // dropped when its wave retires
    r.cancelled = true;
    if (r.admitted) {
        release(*S, r);
        auto a = std::find(S->active.begin(), S->active.end(), r.id);
        if (a != S->active.end()) S->active.erase(a);
    }
    return DR_OK;
}

int dr_serve_stats(int32_t server, uint64_t* completed, uint64_t* prime_steps, uint64_t* admitted_bytes,
                   uint32_t* queue_depth) {
    Server* S = find_server(server);
    if (!S) return DR_ERR_HANDLE;
    std::lock_guard<std::mutex> lk(S->mu);
    if (completed) *completed = S->completed;
    if (prime_steps) *prime_steps = S->prime_steps;
    if (admitted_bytes) *admitted_bytes = S->admitted;
    if (queue_depth) *queue_depth = (uint32_t)(S->pending.size() + S->active.size());
    return DR_OK;
}

int dr_serve_close(int32_t server) {
    std::unique_ptr<Server> S;
    {
        std::lock_guard<std::mutex> lk(g_srv_mu);
        auto it = g_servers.find(server);
        if (it == g_servers.end()) return DR_ERR_HANDLE;
        S = std::move(it->second);
        g_servers.erase(it);
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    if (S->thr.joinable()) S->thr.join();
    for (Wave& W : S->waves) {
        if (W.st) cudaStreamSynchronize(W.st);
        if (W.ev) cudaEventDestroy(W.ev);
        if (W.ev0) cudaEventDestroy(W.ev0);
        if (W.st) cudaStreamDestroy(W.st);
        if (W.h_up) cudaFreeHost(W.h_up);
        if (W.h_res) cudaFreeHost(W.h_res);
        if (W.h_sh) cudaFreeHost(W.h_sh);
        if (W.h_st) cudaFreeHost(W.h_st);
    }
    for (void* p : S->retired_pinned) cudaFreeHost(p);
    return DR_OK;
}

int dr_debug_serve_waves(int32_t server, int32_t max_waves, int32_t* n_waves, double* rows) {
    Server* S = find_server(server);
    if (!S) return DR_ERR_HANDLE;
    if (!n_waves || (max_waves > 0 && !rows)) return DR_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    *n_waves = (int32_t)S->wlog.size();
    const size_t n = std::min<size_t>(S->wlog.size(), (size_t)std::max(max_waves, 0));
    for (size_t i = 0; i < n; ++i) {
        const WaveLog& g = S->wlog[i];
        double* o = rows + 12 * i;
        o[0] = g.t_sel; o[1] = g.t_launched; o[2] = g.t_harvest; o[3] = g.gpu_ms;
        o[4] = g.n_req; o[5] = g.has_long; o[6] = g.wave; o[7] = (double)g.walk_tiles;
        o[8] = (double)g.shadow_span; o[9] = g.t_geom; o[10] = g.t_alloc; o[11] = g.t_launch;
    }
    return DR_OK;
}

int dr_debug_serve_inject(int32_t server, int32_t kind, int32_t count, uint64_t* failed) {
    Server* S = find_server(server);
    if (!S) return DR_ERR_HANDLE;
    if (count < 0 || (kind != DR_INJECT_ADMIT_NOMEM && kind != DR_INJECT_WAVE_NOMEM && kind != 0)) {
        set_error("dr_debug_serve_inject: unknown kind or negative count");
        return DR_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (kind == DR_INJECT_ADMIT_NOMEM) S->inject_admit = (uint32_t)count;
    if (kind == DR_INJECT_WAVE_NOMEM) S->inject_wave = (uint32_t)count;
    if (failed) *failed = S->failed;
    S->cv.notify_all();
    return DR_OK;
}

}  // extern "C"
