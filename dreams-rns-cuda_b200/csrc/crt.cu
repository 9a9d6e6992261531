// Garner CRT to exact 32-bit limbs (reference runner.py:57-81).
//
// The reference's iterative CRT adds one mixed-radix digit per modulus:
//     t_i = (a_i - x mod p_i) * inv(M_i mod p_i) mod p_i,  x += M_i t_i,
// with M_i = p_0 ... p_{i-1}, x starting at the raw first residue and
// inv(v) = v^(p-2) mod p (0 when p | M_i).  Two kernels compute it.  For the
// standard prime table and K <= kCrtLanesMaxK, k_crt_lanes runs each value's
// whole reconstruction on one lane (32 values per warp; see there).  For any
// other odd moduli, and larger K, k_crt gives one warp to one value:
//   1. digits: for i = 1..K-1 the lane owning modulus i computes t_i and
//      broadcasts it; every lane folds t_i into the running x mod p_j of its
//      own moduli j > i -- K sequential steps, K/32 mulmods each per lane;
//   2. binary: limb l of x = sum_i t_i * M_i[l] (the M_i limbs are built once
//      per moduli set), lane-parallel over limbs, then one carry pass;
//   3. centring x - M if x > M // 2 (runner.py:79-81) to sign + magnitude.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dreams_b200.h"
#include "host_common.h"
#include "launch.h"
#include "modarith.cuh"

namespace dr {

__device__ __forceinline__ Mont mont_of(uint32_t p, uint32_t pinv, uint32_t r2) {
    Mont M;
    M.p = p;
    M.pinv = pinv;
    M.r2 = r2;
    M.one = 0;
    M.one = mmul(r2, 1u, M);
    return M;
}

// Per moduli set: Montgomery constants, Garner inverses and the M_i limbs.
// Thread j handles modulus j; thread 0 builds the limb table.  Setup work,
// run once per moduli set and cached by the host.
__global__ void k_crt_setup(const uint32_t* moduli, int K, int L, uint32_t* pinv, uint32_t* r2,
                            uint32_t* ginv, uint32_t* Mlimbs, uint32_t* Mtotal, uint32_t* garner) {
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
        const uint32_t p = moduli[j];
        uint32_t x = p;
        for (int it = 0; it < 5; ++it) x *= 2u - p * x;   // Newton: p^-1 mod 2^32
        const uint32_t pi = 0u - x;
        const uint64_t r1 = (1ull << 32) % p;
        const uint32_t rr = (uint32_t)((r1 * r1) % p);
        pinv[j] = pi;
        r2[j] = rr;
        const Mont M = mont_of(p, pi, rr);
        uint32_t acc = M.one;  // prod_{i<j} p_i mod p_j
        for (int i = 0; i < j; ++i) {
            const uint32_t pim = mmul(moduli[i] % p, rr, M);
            acc = mmul(acc, pim, M);
            // Garner constant of the lane kernel: p_i^-1 mod p_j, Montgomery form
            if (garner) garner[(size_t)i * K + j] = minv_any(pim, M);
        }
        ginv[j] = minv_any(acc, M);
    }
    if (threadIdx.x == 0) {
        for (int l = 0; l < L; ++l) Mlimbs[l] = 0u;
        Mlimbs[0] = 1u;
        for (int i = 1; i <= K; ++i) {
            const uint32_t* prev = Mlimbs + (size_t)(i - 1) * L;
            uint32_t* cur = (i < K) ? Mlimbs + (size_t)i * L : Mtotal;
            uint64_t carry = 0;
            for (int l = 0; l < L; ++l) {
                const uint64_t t = (uint64_t)prev[l] * moduli[i - 1] + carry;
                cur[l] = (uint32_t)t;
                carry = t >> 32;
            }
        }
    }
}

// Words of dynamic shared memory: block-wide moduli constants, then per warp
// x[Lp] + dig[Kp] + col[2*Lp] (u64).
__host__ __device__ inline size_t crt_block_words(int K) { return (size_t)4 * ((K + 1) & ~1); }
__host__ __device__ inline size_t crt_warp_words(int K, int L) {
    const size_t Lp = (size_t)((L + 1) & ~1), Kp = (size_t)((K + 1) & ~1);
    return Lp + Kp + 4 * Lp;
}

template <int OWN>
__global__ void __launch_bounds__(128) k_crt(const uint32_t* __restrict__ residues, int n,
                                             CrtTables T, uint32_t* __restrict__ limbs, int stride,
                                             int32_t* __restrict__ sign_out,
                                             int32_t* __restrict__ nlimbs_out,
                                             uint32_t* __restrict__ ulimbs,
                                             const uint64_t* __restrict__ in_off,
                                             const uint32_t* __restrict__ out_idx) {
    extern __shared__ uint32_t csm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int K = T.K, L = T.L;
    const int Kp = (K + 1) & ~1, Lp = (L + 1) & ~1;
    uint32_t* sp = csm;            // moduli
    uint32_t* spi = sp + Kp;       // pinv
    uint32_t* sr2 = spi + Kp;      // r2
    uint32_t* sgi = sr2 + Kp;      // ginv
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
        sp[j] = T.moduli[j];
        spi[j] = T.pinv[j];
        sr2[j] = T.r2[j];
        sgi[j] = T.ginv[j];
    }
    __syncthreads();
    uint32_t* x = csm + crt_block_words(K) + (size_t)warp * crt_warp_words(K, L);
    uint32_t* dig = x + Lp;
    uint64_t* col = reinterpret_cast<uint64_t*>(dig + Kp);

    for (int j = blockIdx.x * wpb + warp; j < n; j += gridDim.x * wpb) {
        const uint32_t* a = residues + (in_off ? in_off[j] : (uint64_t)j * K);
        const size_t v = out_idx ? out_idx[j] : (size_t)j;
        const uint32_t r0 = __ldg(a);
        uint32_t acc[OWN];  // x mod p_j, plain
        uint32_t mi[OWN];   // M_i mod p_j, Montgomery form
#pragma unroll
        for (int o = 0; o < OWN; ++o) {
            const int j = lane + 32 * o;
            acc[o] = 0u;
            mi[o] = 0u;
            if (j < K) {
                const Mont M = mont_of(sp[j], spi[j], sr2[j]);
                acc[o] = r0 % M.p;
                mi[o] = mmul(sp[0] % M.p, M.r2, M);
            }
        }
        if (lane == 0) dig[0] = r0;
        for (int i = 1; i < K; ++i) {
            const int own = i & 31, oi = i >> 5;
            uint32_t t = 0;
#pragma unroll
            for (int o = 0; o < OWN; ++o) {
                if (o == oi && lane == own) {
                    const Mont M = mont_of(sp[i], spi[i], sr2[i]);
                    const uint32_t ai = __ldg(a + i) % M.p;
                    // (a_i - x mod p_i) * inv(M_i mod p_i): plain x Montgomery -> plain
                    t = mmul(subm(ai, acc[o], M.p), sgi[i], M);
                    dig[i] = t;
                }
            }
            t = __shfl_sync(0xffffffffu, t, own);
            const uint32_t pi = sp[i];
#pragma unroll
            for (int o = 0; o < OWN; ++o) {
                const int j = lane + 32 * o;
                if (j > i && j < K) {
                    const Mont M = mont_of(sp[j], spi[j], sr2[j]);
                    acc[o] = addm(acc[o], mmul(t, mi[o], M), M.p);   // t < 2^31: t*mi < p*2^32
                    mi[o] = mmul(mmul(mi[o], pi, M), M.r2, M);
                }
            }
        }
        __syncwarp();
        for (int l = lane; l < L; l += 32) {
            uint64_t lo = 0, hi = 0;
            for (int i = 0; i < K; ++i) {
                const uint64_t pr = (uint64_t)dig[i] * __ldg(T.Mlimbs + (size_t)i * L + l);
                lo += pr;
                hi += (lo < pr);
            }
            col[2 * l] = lo;
            col[2 * l + 1] = hi;
        }
        __syncwarp();
        if (lane == 0) {
            unsigned __int128 carry = 0;
            for (int l = 0; l < L; ++l) {
                const unsigned __int128 t = (((unsigned __int128)col[2 * l + 1]) << 64) + col[2 * l] + carry;
                x[l] = (uint32_t)t;
                carry = t >> 32;
            }
            // x >= M ?  and  2x > M ?  (M odd, so 2x > M <=> x > M // 2)
            int ge = 1;
            for (int l = L - 1; l >= 0; --l) {
                const uint32_t mm = __ldg(T.Mtotal + l);
                if (x[l] != mm) { ge = x[l] > mm; break; }
            }
            int twice_gt = (x[L - 1] >> 31) ? 1 : -1;
            if (twice_gt < 0) {
                twice_gt = 0;
                for (int l = L - 1; l >= 0; --l) {
                    const uint32_t tx = (x[l] << 1) | (l > 0 ? (x[l - 1] >> 31) : 0u);
                    const uint32_t mm = __ldg(T.Mtotal + l);
                    if (tx != mm) { twice_gt = tx > mm; break; }
                }
            }
            if (ulimbs) {
                uint32_t* uo = ulimbs + (size_t)v * stride;
                for (int l = 0; l < stride; ++l) uo[l] = l < L ? x[l] : 0u;
            }
            uint32_t* out = limbs + (size_t)v * stride;
            int sgn = 1;
            int64_t borrow = 0;
            if (!ge && twice_gt) {          // negative: M - x
                sgn = -1;
                for (int l = 0; l < L; ++l) {
                    const int64_t d = (int64_t)__ldg(T.Mtotal + l) - (int64_t)x[l] - borrow;
                    borrow = d < 0;
                    out[l] = (uint32_t)(d + (borrow ? (1ll << 32) : 0));
                }
            } else {                        // x, or x - M when x >= M
                for (int l = 0; l < L; ++l) {
                    const int64_t d = (int64_t)x[l] - (ge ? (int64_t)__ldg(T.Mtotal + l) : 0) - borrow;
                    borrow = d < 0;
                    out[l] = (uint32_t)(d + (borrow ? (1ll << 32) : 0));
                }
            }
            for (int l = L; l < stride; ++l) out[l] = 0u;
            int nl = L;
            while (nl > 0 && out[nl - 1] == 0u) --nl;
            sign_out[v] = nl ? sgn : 0;
            if (nlimbs_out) nlimbs_out[v] = nl;
        }
        __syncwarp();
    }
}

// ---- lane-per-value kernel (standard primes) -------------------------------
// One lane carries one value through the whole reconstruction; a warp takes
// 32 values, so every instruction does 32 values' work (the warp-per-value
// kernel above spends a sequential K-step broadcast chain per value).  For
// distinct primes above 2^30 the reference's digits
//     t_k = (a_k - x mod p_k) * inv(M_k mod p_k)  (runner.py:70-74)
// equal Garner's column recurrence
//     d = a_k;  d = (d - t_i mod p_k) * p_i^-1 mod p_k  for i = 0 .. k-1
// (inverses exist and multiply, so inv(M_k) = prod p_i^-1), with t_0 the raw
// first residue as the reference starts from it.  Then x = t_0 + p_0 (t_1 +
// p_1 (t_2 + ...)) by Horner in 32-bit limbs, and the centring of
// runner.py:79-81.  Per warp, shared memory holds the digits [k][lane] and
// the limbs [l][lane] in rows of 33 words, so both the lane-parallel compute
// (lanes differ in the column) and the coalesced load/store of one value's
// row (lanes differ in the row) are free of bank conflicts.
constexpr int kCrtPitch = 33;
constexpr int kCrtCols = 8;   // digit columns per group (interleaved Montgomery chains; 8: 4% faster than 4 on 2^20 values)

__host__ __device__ inline size_t crt_lanes_warp_words(int K, int L) {
    return (size_t)kCrtPitch * ((K > L ? K : L) + L);
}

__global__ void __launch_bounds__(128) k_crt_lanes(const uint32_t* __restrict__ residues, int n,
                                                   CrtTables T, uint32_t* __restrict__ limbs,
                                                   int stride, int32_t* __restrict__ sign_out,
                                                   int32_t* __restrict__ nlimbs_out,
                                                   uint32_t* __restrict__ ulimbs,
                                                   const uint64_t* __restrict__ in_off,
                                                   const uint32_t* __restrict__ out_idx) {
    extern __shared__ uint32_t csm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int K = T.K, L = T.L;
    uint32_t* sp = csm;            // moduli
    uint32_t* spi = sp + K;        // -p^-1 mod 2^32
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
        sp[j] = T.moduli[j];
        spi[j] = T.pinv[j];
    }
    __syncthreads();
    uint32_t* D = csm + 2 * K + (size_t)warp * crt_lanes_warp_words(K, L);   // digits, then M - x
    uint32_t* X = D + (size_t)kCrtPitch * (K > L ? K : L);                   // limbs of x
    const int groups = (n + 31) / 32;
    for (int g = blockIdx.x * wpb + warp; g < groups; g += gridDim.x * wpb) {
        const int j0 = g * 32;
        const int cnt = min(32, n - j0);
        // every lane loads one value's input offset and output row; the rows
        // then go around by shuffles, so the warp's residue loads (and limb
        // stores) are independent of one another instead of each waiting for
        // its own offset load
        const int jl = j0 + (lane < cnt ? lane : 0);
        const uint64_t my_in = in_off ? in_off[jl] : (uint64_t)jl * K;
        const uint32_t my_row = out_idx ? out_idx[jl] : (uint32_t)jl;
        // residues of the warp's values, one value's row at a time (coalesced)
#pragma unroll 4
        for (int v = 0; v < cnt; ++v) {
            const uint32_t* a = residues + __shfl_sync(0xffffffffu, my_in, v);
            for (int k = lane; k < K; k += 32) D[k * kCrtPitch + v] = __ldg(a + k);
        }
        __syncwarp();
        // digits: digit k takes rows i = 0 .. k-1 in order, each needing the
        // final digit i.  Columns go in groups of kCrtCols: the rows below a
        // group update its columns independently (interleaved Montgomery
        // chains, kCrtCols times the instruction-level parallelism), then
        // the group's own rows finish it column by column.
        const uint32_t t0 = D[lane];                 // raw, as the reference starts from it
        for (int k = 1; k < K; k += kCrtCols) {
            uint32_t d[kCrtCols], pc[kCrtCols], pic[kCrtCols];
#pragma unroll
            for (int c = 0; c < kCrtCols; ++c) {
                const int kk = k + c < K ? k + c : K - 1;   // past K: a duplicate, never stored
                const uint32_t p = sp[kk];
                pc[c] = p;
                pic[c] = spi[kk];
                uint32_t x = D[kk * kCrtPitch + lane];
                x = umin32(x, x - 2u * p);           // a_k < 2^32 < 4p: reduce mod p
                x = umin32(x, x - p);
                uint32_t t = umin32(t0, t0 - 2u * p);   // t_0 < 2^32: t_0 mod p
                t = umin32(t, t - p);
                d[c] = mmul(subm(x, t, p), __ldg(T.garner + kk), Mont{p, pic[c], 0u, 0u});   // row 0
            }
            for (int i = 1; i < k; ++i) {
                const uint32_t ti = D[i * kCrtPitch + lane];                 // < p_i < 2 p_k
                const uint32_t* g = T.garner + (size_t)i * K;
#pragma unroll
                for (int c = 0; c < kCrtCols; ++c) {
                    const int kk = k + c < K ? k + c : K - 1;
                    const uint32_t p = pc[c];
                    d[c] = mmul(subm(d[c], umin32(ti, ti - p), p), __ldg(g + kk), Mont{p, pic[c], 0u, 0u});
                }
            }
#pragma unroll
            for (int c = 0; c < kCrtCols; ++c) {
                if (k + c >= K) break;
                // row k + c: digit k + c is final; it updates the later columns
#pragma unroll
                for (int c2 = c + 1; c2 < kCrtCols; ++c2) {
                    if (k + c2 >= K) break;
                    const uint32_t p = pc[c2];
                    d[c2] = mmul(subm(d[c2], umin32(d[c], d[c] - p), p),
                                 __ldg(T.garner + (size_t)(k + c) * K + (k + c2)), Mont{p, pic[c2], 0u, 0u});
                }
                D[(k + c) * kCrtPitch + lane] = d[c];
            }
        }
        // x = t_0 + p_0 (t_1 + p_1 (t_2 + ...)): Horner from the top digit;
        // the limb count grows when some lane's carry needs a new limb
        int len = 1;
        X[lane] = D[(K - 1) * kCrtPitch + lane];
        for (int i = K - 2; i >= 0; --i) {
            const uint32_t p = sp[i];
            uint64_t c = D[i * kCrtPitch + lane];
            for (int l = 0; l < len; ++l) {
                const uint64_t t = (uint64_t)X[l * kCrtPitch + lane] * p + c;
                X[l * kCrtPitch + lane] = (uint32_t)t;
                c = t >> 32;
            }
            if (len < L && __any_sync(0xffffffffu, c != 0)) X[len++ * kCrtPitch + lane] = (uint32_t)c;
        }
        for (int l = len; l < L; ++l) X[l * kCrtPitch + lane] = 0u;
        __syncwarp();
        if (ulimbs)
            for (int v = 0; v < cnt; ++v) {
                uint32_t* uo = ulimbs + (size_t)__shfl_sync(0xffffffffu, my_row, v) * stride;
                for (int l = lane; l < stride; l += 32) uo[l] = l < L ? X[l * kCrtPitch + v] : 0u;
            }
        // centring (runner.py:79-81): x - M if x > M // 2, else x.  d = M - x;
        // x >= M when that borrows or is zero; otherwise 2x > M (M odd) when
        // x > d, i.e. when x - d does not borrow
        uint32_t bd = 0, dz = 0;
        for (int l = 0; l < L; ++l) {
            const uint32_t m = __ldg(T.Mtotal + l), x = X[l * kCrtPitch + lane];
            const uint32_t s = m - x, dl = s - bd;
            bd = (m < x) | (s < bd);
            D[l * kCrtPitch + lane] = dl;
            dz |= dl;
        }
        const bool ge = bd || dz == 0u;
        uint32_t be = 0;
        for (int l = 0; l < L; ++l) {
            const uint32_t x = X[l * kCrtPitch + lane], dl = D[l * kCrtPitch + lane];
            const uint32_t s = x - dl;
            be = (x < dl) | (s < be);
        }
        const bool neg = !ge && !be;                  // 2x > M: the value is -(M - x)
        uint32_t bm = 0;
        int nl = 0;
        for (int l = 0; l < L; ++l) {
            const uint32_t x = X[l * kCrtPitch + lane];
            uint32_t o;
            if (ge) {                                 // x - M
                const uint32_t m = __ldg(T.Mtotal + l), s = x - m;
                o = s - bm;
                bm = (x < m) | (s < bm);
            } else {
                o = neg ? D[l * kCrtPitch + lane] : x;
            }
            X[l * kCrtPitch + lane] = o;
            if (o) nl = l + 1;
        }
        __syncwarp();
        if (lane < cnt) {
            sign_out[my_row] = nl ? (neg ? -1 : 1) : 0;
            if (nlimbs_out) nlimbs_out[my_row] = nl;
        }
        for (int v = 0; v < cnt; ++v) {
            uint32_t* out = limbs + (size_t)__shfl_sync(0xffffffffu, my_row, v) * stride;
            for (int l = lane; l < stride; l += 32) out[l] = l < L ? X[l * kCrtPitch + v] : 0u;
        }
        __syncwarp();
    }
}

// ---- host launchers -----------------------------------------------------
cudaError_t launch_crt_setup(const uint32_t* moduli, int K, int L, uint32_t* pinv, uint32_t* r2,
                             uint32_t* ginv, uint32_t* Mlimbs, uint32_t* Mtotal, uint32_t* garner,
                             cudaStream_t st) {
    k_crt_setup<<<1, 256, 0, st>>>(moduli, K, L, pinv, r2, ginv, Mlimbs, Mtotal, garner);
    return cudaGetLastError();
}

static cudaError_t launch_crt_lanes(const uint32_t* res, int n, const CrtTables& T, uint32_t* limbs,
                                    int stride, int32_t* sign, int32_t* nl, uint32_t* ul, int sms,
                                    cudaStream_t st, const uint64_t* in_off, const uint32_t* out_idx) {
    const size_t per_warp = 4 * crt_lanes_warp_words(T.K, T.L);
    int wpb = (int)std::min<size_t>(4, std::max<size_t>(1, (96 * 1024) / per_warp));
    const size_t smem = 4ull * 2 * T.K + (size_t)wpb * per_warp;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_crt_lanes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int groups = (n + 31) / 32;
    int blocks = (groups + wpb - 1) / wpb;
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_crt_lanes, 32 * wpb, smem);
    if (e != cudaSuccess) return e;
    blocks = std::max(1, std::min(blocks, std::max(occ, 1) * sms));
    k_crt_lanes<<<blocks, 32 * wpb, smem, st>>>(res, n, T, limbs, stride, sign, nl, ul, in_off, out_idx);
    return cudaGetLastError();
}

template <int OWN>
static cudaError_t launch_crt_t(const uint32_t* res, int n, const CrtTables& T, uint32_t* limbs,
                                int stride, int32_t* sign, int32_t* nl, uint32_t* ul, int sms,
                                cudaStream_t st, const uint64_t* in_off, const uint32_t* out_idx) {
    const int wpb = 4;
    const size_t smem = 4 * (crt_block_words(T.K) + wpb * crt_warp_words(T.K, T.L));
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_crt<OWN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    int blocks = (n + wpb - 1) / wpb;
    const int cap = sms * 8;
    if (blocks > cap) blocks = cap;
    k_crt<OWN><<<blocks, 32 * wpb, smem, st>>>(res, n, T, limbs, stride, sign, nl, ul, in_off, out_idx);
    return cudaGetLastError();
}

cudaError_t launch_crt(const uint32_t* res, int n, const CrtTables& T, uint32_t* limbs, int stride,
                       int32_t* sign, int32_t* nl, uint32_t* ul, int sms, cudaStream_t st,
                       const uint64_t* in_off, const uint32_t* out_idx) {
    if (n <= 0) return cudaSuccess;
    if (T.garner && T.K <= kCrtLanesMaxK)
        return launch_crt_lanes(res, n, T, limbs, stride, sign, nl, ul, sms, st, in_off, out_idx);
    const int own = (T.K + 31) / 32;
    if (own <= 1) return launch_crt_t<1>(res, n, T, limbs, stride, sign, nl, ul, sms, st, in_off, out_idx);
    if (own <= 2) return launch_crt_t<2>(res, n, T, limbs, stride, sign, nl, ul, sms, st, in_off, out_idx);
    if (own <= 4) return launch_crt_t<4>(res, n, T, limbs, stride, sign, nl, ul, sms, st, in_off, out_idx);
    if (own <= 8) return launch_crt_t<8>(res, n, T, limbs, stride, sign, nl, ul, sms, st, in_off, out_idx);
    if (own <= 16) return launch_crt_t<16>(res, n, T, limbs, stride, sign, nl, ul, sms, st, in_off, out_idx);
    if (own <= 32) return launch_crt_t<32>(res, n, T, limbs, stride, sign, nl, ul, sms, st, in_off, out_idx);
    return cudaErrorInvalidValue;
}

}  // namespace dr

// ---- allocation-free CRT ----------------------------------------------------
// For callers that may not allocate device memory themselves, for instance code
// that runs under a framework which owns every byte of device memory through
// its own pool, or that must not trigger the device-wide synchronisation a
// cudaFree implies.  The per-moduli tables that dr_crt_batch_device keeps in
// cudaMalloc'd buffers live here in one file-scope device array instead:
// every GPU that loads the library holds it (about 130 KB) until the process
// exits, and every call rebuilds the tables in it, so calls that overlap on
// the GPU race on its contents.
namespace dr {

constexpr int kStaticCrtMaxK = 128;
constexpr int kStaticCrtL = (31 * kStaticCrtMaxK + 31) / 32 + 2;
constexpr int kStaticCrtWords = 4 * kStaticCrtMaxK + kStaticCrtMaxK * kStaticCrtL + kStaticCrtL +
                                kStaticCrtMaxK * kStaticCrtMaxK;

static __device__ __align__(256) uint32_t g_crt_static[kStaticCrtWords];

// The moduli travel by value as a kernel argument (512 bytes), so a call
// makes no host-to-device copy; this kernel stores them at the head of the
// static array, where k_crt_setup then reads them.
struct CrtModuli {
    uint32_t p[kStaticCrtMaxK];
};

__global__ void k_crt_static_moduli(const CrtModuli mods, int K) {
    for (int j = threadIdx.x; j < K; j += blockDim.x) g_crt_static[j] = mods.p[j];
}

namespace {
std::mutex g_static_mu;
void* g_static_addr[64] = {nullptr};   // host view of g_crt_static's device address, per device
}  // namespace

}  // namespace dr

extern "C" int dr_crt_batch_device_noalloc(const uint32_t* residues_d, int32_t K, int32_t n,
                                           uint32_t* limbs_d, int32_t limb_stride, int32_t* sign_d,
                                           void* stream) {
    using namespace dr;
    if (K < 1 || K > kStaticCrtMaxK) {
        set_error("dr_crt_batch_device_noalloc: K must be in 1..128 (size of its static tables)");
        return K < 1 ? DR_ERR_ARG : DR_ERR_UNSUPPORTED;
    }
    if (n < 0 || (n > 0 && (!residues_d || !limbs_d || !sign_d))) {
        set_error("dr_crt_batch_device_noalloc: null buffer");
        return DR_ERR_ARG;
    }
    const int L = (31 * K + 31) / 32 + 2;
    if (limb_stride < L) {
        set_error("dr_crt_batch_device_noalloc: limb_stride below ceil(31K/32)+2");
        return DR_ERR_ARG;
    }
    if (n == 0) return DR_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("dr_crt_batch_device_noalloc: no current device");
        return DR_ERR_CUDA;
    }
    uint32_t* base = nullptr;
    {
        // first call on each device: the array's device address, with that device current
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_crt_static);
            if (e != cudaSuccess || !p) {
                set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return DR_ERR_CUDA;
            }
            g_static_addr[dev] = p;
        }
        base = static_cast<uint32_t*>(g_static_addr[dev]);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // layout: moduli[K] pinv[K] r2[K] ginv[K] Mlimbs[K*L] Mtotal[L] garner[K*K]
    uint32_t* moduli = base;
    uint32_t* pinv = base + K;
    uint32_t* r2 = base + 2 * K;
    uint32_t* ginv = base + 3 * K;
    uint32_t* Ml = base + 4 * K;
    uint32_t* Mt = Ml + (size_t)K * L;
    uint32_t* gar = Mt + L;
    // the moduli, copied under the prime table's lock (another thread may
    // grow the table meanwhile), go to the device as a kernel argument
    CrtModuli mods{};
    if (prime_table_copy(K, mods.p) != DR_OK) {
        set_error("dr_crt_batch_device_noalloc: prime table");
        return DR_ERR_UNSUPPORTED;
    }
    k_crt_static_moduli<<<1, 128, 0, st>>>(mods, K);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_crt_setup(moduli, K, L, pinv, r2, ginv, Ml, Mt, gar, st);
    if (e != cudaSuccess) {
        set_error(std::string("dr_crt_batch_device_noalloc setup: ") + cudaGetErrorString(e));
        return DR_ERR_CUDA;
    }
    CrtTables T{moduli, pinv, r2, ginv, Ml, Mt, K, L, gar};
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = launch_crt(residues_d, n, T, limbs_d, limb_stride, sign_d, nullptr, nullptr, sms, st);
    if (e != cudaSuccess) {
        set_error(std::string("dr_crt_batch_device_noalloc: ") + cudaGetErrorString(e));
        return DR_ERR_CUDA;
    }
    return DR_OK;
}
