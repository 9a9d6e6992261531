// Host-side helpers shared by the ABI translation units.
#pragma once
#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

namespace dr {

// Last error message of the calling thread (dr_last_error).
void set_error(const std::string& msg);
const std::string& last_error();

// The first K primes below 2^31, descending (reference runner.py:33-52).
// The table grows under a lock; the returned reference may be read without
// it only once the table holds every prime anyone will ask for (dr_init fills
// all DR_MAX_K), so code that may run before dr_init uses prime_table_copy.
const std::vector<uint32_t>& prime_table(int K);
// Copies the first K primes into out while holding the table's lock.
int prime_table_copy(int K, uint32_t* out);

// Montgomery constants for R = 2^32: pinv = -p^-1 mod 2^32, r1 = R mod p,
// r2 = R^2 mod p.
struct PrimeMeta {
    uint32_t p, pinv, r1, r2;
};
PrimeMeta prime_meta(uint32_t p);

// ---- per-stage timers (dr_stage_times) and NVTX ranges ----------------------
// Host milliseconds spent in each stage of the ABI calls, summed since the
// last reset: batch build, allocation + upload, run (enqueue; the wait too
// for the synchronous calls), read-back; plus the device milliseconds of
// every batch run read back (CUDA events).  The NVTX ranges carry the same
// names, so a profiler's timeline shows the stages (header-only NVTX: no
// cost unless a profiler is attached).
enum Stage : int { STAGE_BUILD = 0, STAGE_UPLOAD = 1, STAGE_RUN = 2, STAGE_READ = 3,
                   STAGE_DEVICE = 4, STAGE_COUNT = 5 };
void stage_add(int stage, double ms);

class NvtxRange {
  public:
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    void end() {
        if (on_) nvtxRangePop();
        on_ = false;
    }
    ~NvtxRange() { end(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;

  private:
    bool on_ = true;
};

// Times its scope into one stage and marks it as an NVTX range.
class StageScope {
  public:
    StageScope(int stage, const char* name)
        : stage_(stage), range_(name), t0_(std::chrono::steady_clock::now()) {}
    ~StageScope() {
        stage_add(stage_, std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now() - t0_).count());
    }

  private:
    int stage_;
    NvtxRange range_;
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace dr
