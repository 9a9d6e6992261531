// Device modular arithmetic for 31-bit primes: Montgomery form with R = 2^32.
//
// Values are kept canonical in [0, p).  A Montgomery product is one 32x32->64
// wide multiply, one low multiply for the quotient and one wide multiply-add:
//     t = a*b;  q = (t mod 2^32) * (-p^-1);  u = (t + q*p) / 2^32  in [0, 2p)
// followed by a conditional subtraction done as an unsigned min.  Bounds:
//     t < p*2^32 is needed; a, b < p gives t < p^2 < p*2^32, and a sum of two
//     products gives t < 2p^2 < p*2^32 because 2p < 2^32.  Sums of three or
//     more products exceed p*2^32 for p near 2^31, so dot products of length
//     >= 3 subtract p*2^32 (p from the high word) once after every extra
//     product, which keeps t < p*2^32 (t < p*2^32 + p^2 < 2p*2^32 before the
//     subtraction).
#pragma once
#include <stdint.h>

namespace dr {

struct Mont {
    uint32_t p;     // odd modulus < 2^31
    uint32_t pinv;  // -p^-1 mod 2^32
    uint32_t r2;    // 2^64 mod p
    uint32_t one;   // 2^32 mod p (Montgomery form of 1)
};

__device__ __forceinline__ uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

// canonical reduction of u in [0, 2p)
__device__ __forceinline__ uint32_t csub(uint32_t u, uint32_t p) { return umin32(u, u - p); }

// REDC of t < p*2^32
__device__ __forceinline__ uint32_t redc(uint64_t t, const Mont& M) {
    const uint32_t q = (uint32_t)t * M.pinv;
    const uint64_t u = t + (uint64_t)q * M.p;
    return csub((uint32_t)(u >> 32), M.p);
}

__device__ __forceinline__ uint32_t mmul(uint32_t a, uint32_t b, const Mont& M) {
    return redc((uint64_t)a * b, M);
}

// a*b + c*d (Montgomery), a..d < p
__device__ __forceinline__ uint32_t mmul2(uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                          const Mont& M) {
    return redc((uint64_t)a * b + (uint64_t)c * d, M);
}

// keep a 64-bit accumulator below p*2^32 after adding one more product
__device__ __forceinline__ uint64_t fold_hi(uint64_t t, uint32_t p) {
    uint32_t lo = (uint32_t)t, hi = (uint32_t)(t >> 32);
    hi = csub(hi, p);
    return ((uint64_t)hi << 32) | lo;
}

// sum_k a[k]*b[k] in Montgomery form, N terms, all operands < p
template <int N>
__device__ __forceinline__ uint32_t mdot(const uint32_t* a, const uint32_t* b, const Mont& M) {
    uint64_t t = (uint64_t)a[0] * b[0];
    if (N > 1) t += (uint64_t)a[1] * b[1];
#pragma unroll
    for (int k = 2; k < N; ++k) t = fold_hi(t + (uint64_t)a[k] * b[k], M.p);
    return redc(t, M);
}

__device__ __forceinline__ uint32_t addm(uint32_t a, uint32_t b, uint32_t p) { return csub(a + b, p); }
__device__ __forceinline__ uint32_t subm(uint32_t a, uint32_t b, uint32_t p) {
    const uint32_t d = a - b;
    return umin32(d, d + p);
}
__device__ __forceinline__ uint32_t negm(uint32_t a, uint32_t p) { return subm(0u, a, p); }

// Montgomery form of a signed 64-bit integer
__device__ __forceinline__ uint32_t to_mont_i64(int64_t v, const Mont& M) {
    const int64_t p = (int64_t)M.p;
    int64_t r;
    if (v >= 0 && v < p) r = v;                 // small constants: no 64-bit division
    else if (v < 0 && v > -p) r = v + p;
    else { r = v % p; if (r < 0) r += p; }
    return mmul((uint32_t)r, M.r2, M);
}

__device__ __forceinline__ uint32_t to_mont_u64(uint64_t v, const Mont& M) {
    return mmul((uint32_t)(v % M.p), M.r2, M);
}

__device__ __forceinline__ uint32_t from_mont(uint32_t a, const Mont& M) { return redc(a, M); }

// a^(p-2) in Montgomery form by a fixed 30-step square-and-multiply chain over
// the exponent's bits 29..0 (bit 30 is always set because p > 2^30 + 2).
// Every lane runs the same instruction sequence; the per-lane exponent bit
// only selects a result.  0 maps to 0, matching pow(0, p-2, p) == 0.
__device__ __forceinline__ uint32_t minv(uint32_t a, const Mont& M) {
    const uint32_t e = M.p - 2u;
    uint32_t r = a;
#pragma unroll 1
    for (int bit = 29; bit >= 0; --bit) {
        r = mmul(r, r, M);
        const uint32_t t = mmul(r, a, M);
        r = ((e >> bit) & 1u) ? t : r;
    }
    return r;
}

// general-modulus variant for moduli that may be below 2^30 (CRT inputs):
// plain left-to-right ladder over all 31 bits of p-2
__device__ __forceinline__ uint32_t minv_any(uint32_t a, const Mont& M) {
    const uint32_t e = M.p - 2u;
    uint32_t r = M.one;
#pragma unroll 1
    for (int bit = 30; bit >= 0; --bit) {
        r = mmul(r, r, M);
        const uint32_t t = mmul(r, a, M);
        r = ((e >> bit) & 1u) ? t : r;
    }
    return r;
}

__device__ __forceinline__ Mont make_mont(uint32_t p, uint32_t pinv, uint32_t r2) {
    Mont M;
    M.p = p;
    M.pinv = pinv;
    M.r2 = r2;
    M.one = 0;
    M.one = mmul(r2, 1u, M);  // r2 * 1 / R = R mod p
    return M;
}

}  // namespace dr
