// Host-only ABI entry points: errors, prime table, program inspection, and
// the CPU re-statement hook used by the tests.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dreams_b200.h"
#include "../../include/dreams_b200_debug.h"
#include "host_common.h"
#include "program.h"

namespace dr {

namespace {
thread_local std::string g_last_error;
std::mutex g_prime_mu;
std::vector<uint32_t> g_primes;

bool is_prime_u32(uint32_t n) {
    if (n < 2) return false;
    if (n % 2 == 0) return n == 2;
    for (uint32_t d = 3; (uint64_t)d * d <= n; d += 2)
        if (n % d == 0) return false;
    return true;
}
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

const std::vector<uint32_t>& prime_table(int K) {
    std::lock_guard<std::mutex> lk(g_prime_mu);
    if ((int)g_primes.size() < K) {
        uint32_t c = g_primes.empty() ? 0x7fffffffu : g_primes.back() - 2;
        while ((int)g_primes.size() < K && c >= (1u << 30)) {
            if (is_prime_u32(c)) g_primes.push_back(c);
            c -= 2;
        }
    }
    return g_primes;
}

namespace {
std::atomic<uint64_t> g_stage_ns[STAGE_COUNT];
std::atomic<uint64_t> g_stage_calls[STAGE_COUNT];
}  // namespace

void stage_add(int stage, double ms) {
    if (stage < 0 || stage >= STAGE_COUNT || !(ms >= 0.0)) return;
    g_stage_ns[stage].fetch_add((uint64_t)(ms * 1e6), std::memory_order_relaxed);
    g_stage_calls[stage].fetch_add(1, std::memory_order_relaxed);
}

int prime_table_copy(int K, uint32_t* out) {
    std::lock_guard<std::mutex> lk(g_prime_mu);
    if ((int)g_primes.size() < K) {
        uint32_t c = g_primes.empty() ? 0x7fffffffu : g_primes.back() - 2;
        while ((int)g_primes.size() < K && c >= (1u << 30)) {
            if (is_prime_u32(c)) g_primes.push_back(c);
            c -= 2;
        }
    }
    if ((int)g_primes.size() < K) return DR_ERR_UNSUPPORTED;
    if (K > 0) std::memcpy(out, g_primes.data(), sizeof(uint32_t) * (size_t)K);
    return DR_OK;
}

PrimeMeta prime_meta(uint32_t p) {
    // Newton iteration for p^-1 mod 2^32 (p odd): x <- x * (2 - p * x)
    uint32_t x = p;  // correct to 3 bits
    for (int i = 0; i < 5; ++i) x *= 2u - p * x;
    PrimeMeta m;
    m.p = p;
    m.pinv = 0u - x;
    m.r1 = (uint32_t)((1ull << 32) % p);
    m.r2 = (uint32_t)((unsigned __int128)m.r1 * m.r1 % p);
    return m;
}

int sim_walk_prime(const Plan& pl, uint64_t p, uint64_t depth, uint64_t checkpoint,
                   const int64_t* axis, int pcf_init, int64_t a0, uint32_t q_row,
                   uint64_t chunk_len, uint64_t* out);

}  // namespace dr

extern "C" {

const char* dr_strerror(int status) {
    switch (status) {
        case DR_OK: return "ok";
        case DR_ERR_CUDA: return "CUDA runtime error";
        case DR_ERR_ARG: return "invalid argument";
        case DR_ERR_BLOB: return "malformed program blob";
        case DR_ERR_OPCODE: return "unknown opcode";
        case DR_ERR_INDEX: return "index out of range in program";
        case DR_ERR_UNSUPPORTED: return "outside engine limits";
        case DR_ERR_NOMEM: return "device memory exhausted";
        case DR_ERR_NOT_INIT: return "dr_init has not been called";
        case DR_ERR_HANDLE: return "unknown handle";
        case DR_ERR_TIMEOUT: return "bounded wait expired";
        case DR_ERR_MODULUS: return "modulus outside odd [3, 2^31)";
        case DR_ERR_BUSY: return "not finished";
        default: return "unknown status";
    }
}

const char* dr_last_error(void) { return dr::last_error().c_str(); }

int dr_version(void) { return 10000; }

int dr_stage_times(double* ms_out, uint64_t* calls_out, int32_t n, int32_t reset) {
    if (n < 0 || (n > 0 && !ms_out)) {
        dr::set_error("dr_stage_times: null output or negative count");
        return DR_ERR_ARG;
    }
    for (int s = 0; s < dr::STAGE_COUNT; ++s) {
        const uint64_t ns = reset ? dr::g_stage_ns[s].exchange(0) : dr::g_stage_ns[s].load();
        const uint64_t c = reset ? dr::g_stage_calls[s].exchange(0) : dr::g_stage_calls[s].load();
        if (s < n) {
            ms_out[s] = (double)ns * 1e-6;
            if (calls_out) calls_out[s] = c;
        }
    }
    return DR_OK;
}

int dr_prime_table(int K, uint32_t* out) {
    if (K < 0 || K > DR_MAX_K || (K > 0 && !out)) {
        dr::set_error("dr_prime_table: K outside 0..DR_MAX_K");
        return DR_ERR_ARG;
    }
    return dr::prime_table_copy(K, out);
}

int dr_program_info(const uint8_t* blob, uint64_t size, int32_t* cls_out, int32_t* degree_out,
                    int32_t* n_regs_out) {
    dr::RawProgram raw;
    dr::Plan plan;
    std::string err;
    int rc = dr::parse_blob(blob, size, &raw, &err);
    if (rc == DR_OK) rc = dr::plan_program(raw, &plan, &err);
    if (rc != DR_OK) {
        dr::set_error(err);
        return rc;
    }
    if (cls_out) *cls_out = (int32_t)plan.cls;
    if (degree_out) *degree_out = (int32_t)plan.degree;
    if (n_regs_out) *n_regs_out = (int32_t)plan.n_regs;
    return DR_OK;
}

int dr_debug_sim_walk(const uint8_t* blob, uint64_t size, int32_t K, uint64_t depth,
                      uint64_t checkpoint, const int64_t* axis_params, int32_t pcf_init,
                      int64_t a0, uint32_t q_row, uint64_t chunk_steps, int32_t force_interp,
                      uint32_t* p_out, uint32_t* q_out, uint32_t* cp_p_out, uint32_t* cp_q_out) {
    dr::RawProgram raw;
    dr::Plan plan;
    std::string err;
    int rc = dr::parse_blob(blob, size, &raw, &err);
    if (rc == DR_OK) rc = dr::plan_program(raw, &plan, &err);
    if (rc != DR_OK) {
        dr::set_error(err);
        return rc;
    }
    if (force_interp) plan.cls = dr::CLS_INTERP;
    if (q_row >= plan.m || K < 0 || K > DR_MAX_K || (K > 0 && (!p_out || !q_out))) return DR_ERR_ARG;
    std::vector<uint32_t> primes((size_t)K);
    if ((rc = dr::prime_table_copy(K, primes.data())) != DR_OK) return rc;
    for (int k = 0; k < K; ++k) {
        uint64_t o[4];
        dr::sim_walk_prime(plan, primes[k], depth, checkpoint, axis_params, pcf_init, a0, q_row,
                           chunk_steps, o);
        p_out[k] = (uint32_t)o[0];
        q_out[k] = (uint32_t)o[1];
        if (cp_p_out) cp_p_out[k] = (uint32_t)o[2];
        if (cp_q_out) cp_q_out[k] = (uint32_t)o[3];
    }
    return DR_OK;
}

}  // extern "C"

extern "C" int dr_debug_template_degree(int32_t cls, int32_t m, int32_t degree) {
    return dr::template_degree((uint32_t)cls, (uint32_t)m, (uint32_t)degree);
}
