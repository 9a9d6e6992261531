// Host-side helpers shared by the ABI translation units.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dr {

// Last error message of the calling thread (dr_last_error).
void set_error(const std::string& msg);
const std::string& last_error();

// The first K primes below 2^31, descending (reference runner.py:33-52).
const std::vector<uint32_t>& prime_table(int K);

// Montgomery constants for R = 2^32: pinv = -p^-1 mod 2^32, r1 = R mod p,
// r2 = R^2 mod p.
struct PrimeMeta {
    uint32_t p, pinv, r1, r2;
};
PrimeMeta prime_meta(uint32_t p);

}  // namespace dr
