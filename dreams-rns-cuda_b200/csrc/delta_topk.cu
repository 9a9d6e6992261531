// Dreams delta from exact limbs, and top-k selection.
//
// delta = -(1 + ln|p/q - L| / ln|q|) (reference runner.py:103-125).  With the
// target as a ratio L = Lnum / Lden of integers (a dyadic Lden = 2^e for a
// decimal/binary target), the error is computed without cancellation:
//     |p/q - L| = |p*Lden - Lnum*q| / (|q| * Lden)
// where the numerator is an exact big-integer difference.  Each logarithm is
// taken from the leading three limbs (relative error ~2^-53), so delta is
// accurate to ~1e-13, far inside the 1e-9 tolerance against mpmath.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/dreams_b200.h"
#include "dr_types.h"
#include "launch.h"

namespace dr {

__device__ __forceinline__ int top_limb(const uint32_t* x, int n) {
    int t = n - 1;
    while (t >= 0 && x[t] == 0u) --t;
    return t;  // -1 for zero
}

__device__ __forceinline__ double ln_big(const uint32_t* x, int t) {
    // t = index of the top non-zero limb (>= 0)
    double v = (double)x[t];
    int e = 0;
    if (t >= 1) { v = v * 4294967296.0 + (double)x[t - 1]; }
    if (t >= 2) { v = v * 4294967296.0 + (double)x[t - 2]; e = 32 * (t - 2); }
    return log(v) + (double)e * 0.69314718055994530942;
}

// out[0..na+nb) = a * b (column sums per lane, then one carry pass by lane 0)
__device__ void big_mul(const uint32_t* a, int na, const uint32_t* b, int nb, uint32_t* out,
                        uint64_t* col, int lane) {
    const int nr = na + nb;
    for (int l = lane; l < nr; l += 32) {
        uint64_t lo = 0, hi = 0;
        const int i0 = l - (nb - 1) > 0 ? l - (nb - 1) : 0;
        const int i1 = l < na - 1 ? l : na - 1;
        for (int i = i0; i <= i1; ++i) {
            const uint64_t pr = (uint64_t)a[i] * b[l - i];
            lo += pr;
            hi += (lo < pr);
        }
        col[2 * l] = lo;
        col[2 * l + 1] = hi;
    }
    __syncwarp();
    if (lane == 0) {
        unsigned __int128 c = 0;
        for (int l = 0; l < nr; ++l) {
            const unsigned __int128 t = (((unsigned __int128)col[2 * l + 1]) << 64) + col[2 * l] + c;
            out[l] = (uint32_t)t;
            c = t >> 32;
        }
    }
    __syncwarp();
}

// per warp smem: A[maxlen] B[maxlen] col[2*maxlen] (u64)
__global__ void __launch_bounds__(128) k_delta(DeltaArgs D) {
    extern __shared__ uint64_t dsmem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int ML = D.maxlen;
    uint64_t* col = dsmem + (size_t)warp * (2 * ML + ML);
    uint32_t* A = reinterpret_cast<uint32_t*>(col + 2 * ML);
    uint32_t* B = A + ML;
    for (int v = blockIdx.x * wpb + warp; v < D.n; v += gridDim.x * wpb) {
        size_t row = (size_t)v;
        int ti = D.per_item ? v : 0;
        if (D.bank_n > 0) {
            row = D.rows ? D.rows[v / D.bank_n] : (uint32_t)(v / D.bank_n);
            ti = v % D.bank_n;
        }
        const uint32_t* p = D.p + row * D.istride;
        const uint32_t* q = D.q + row * D.istride;
        const uint32_t* ln = D.ln + (size_t)ti * D.listride;
        const uint32_t* ld = D.ld + (size_t)ti * D.listride;
        const int ps = D.ps[row * D.sstride], qs = D.qs[row * D.sstride];
        const int lns = D.lns[(size_t)ti * D.lsstride] * (D.lds ? D.lds[(size_t)ti * D.lsstride] : 1);
        const int tp = top_limb(p, D.nl), tq = top_limb(q, D.nl);
        const int tn = top_limb(ln, D.lnl), td = top_limb(ld, D.lnl);
        double result;
        if (tq < 0 || qs == 0) {
            result = -INFINITY;                                  // q == 0
        } else if (td < 0) {
            result = NAN;                                        // target denominator 0
        } else {
            const int np = tp + 1, nq = tq + 1, nn = tn + 1, nd = td + 1;
            // A = |p| * Lden, B = |Lnum| * |q|
            const int na = (np > 0 && nd > 0) ? np + nd : 0;
            const int nb = (nn > 0) ? nn + nq : 0;
            if (na) big_mul(p, np, ld, nd, A, col, lane);
            if (nb) big_mul(ln, nn, q, nq, B, col, lane);
            if (lane == 0) {
                const int sa = na ? ps : 0;
                const int sb = nb ? lns * qs : 0;
                const int n = na > nb ? na : nb;
                for (int l = na; l < n; ++l) A[l] = 0u;
                for (int l = nb; l < n; ++l) B[l] = 0u;
                // |D| = |sa*A - sb*B| into A
                if (sa == 0 || sb == 0 || sa != sb) {
                    if (sb != 0 && sa != 0) {  // opposite signs: A + B
                        uint64_t c = 0;
                        for (int l = 0; l < n; ++l) {
                            const uint64_t t = (uint64_t)A[l] + B[l] + c;
                            A[l] = (uint32_t)t;
                            c = t >> 32;
                        }
                        // the sum of two n-limb numbers fits in n+1 limbs; ML has room
                        A[n] = (uint32_t)c;
                    } else if (sa == 0) {
                        for (int l = 0; l < n; ++l) A[l] = B[l];
                        A[n] = 0u;
                    } else {
                        A[n] = 0u;
                    }
                } else {                        // same sign: |A - B|
                    int cmp = 0;
                    for (int l = n - 1; l >= 0; --l)
                        if (A[l] != B[l]) { cmp = A[l] > B[l] ? 1 : -1; break; }
                    const uint32_t* big = cmp >= 0 ? A : B;
                    const uint32_t* sml = cmp >= 0 ? B : A;
                    int64_t br = 0;
                    for (int l = 0; l < n; ++l) {
                        const int64_t d = (int64_t)big[l] - (int64_t)sml[l] - br;
                        br = d < 0;
                        A[l] = (uint32_t)(d + (br ? (1ll << 32) : 0));
                    }
                    A[n] = 0u;
                }
                const int tD = top_limb(A, n + 1);
                if (tD < 0) {
                    result = INFINITY;                           // p/q == L exactly
                } else if (tq == 0 && q[0] <= 1u) {
                    result = -INFINITY;                          // |q| <= 1
                } else {
                    const double lq = ln_big(q, tq);
                    const double lerr = ln_big(A, tD) - lq - ln_big(ld, td);
                    result = -(1.0 + lerr / lq);
                }
                D.out[v] = result;
            }
            __syncwarp();
            continue;
        }
        if (lane == 0) D.out[v] = result;
        __syncwarp();
    }
}

// CRT overflow test (reference euler2ai_full_verify.py:152-167): the ratio of
// the reconstructed p and q must agree with the float shadow's p_f / q_f to 1%
// (relative when |p_f/q_f| > 1e-10, absolute otherwise); q = 0 or a
// non-finite ratio also counts as overflow.  One thread per (walk, final or
// checkpoint); rows 4w+0..3 of limbs hold p, q, checkpoint p, checkpoint q.
__global__ void k_crt_check(const uint32_t* __restrict__ limbs, const int32_t* __restrict__ signs,
                            int L, int n, const DevWalk* __restrict__ walks,
                            const double* __restrict__ shadow, uint32_t* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n) return;
    const int w = i >> 1, cp = i & 1;
    const DevWalk W = walks[w];
    if (!(W.flags & DR_WALK_SHADOW) || (cp && !W.checkpoint)) return;
    const double* sh = shadow + 3 * ((size_t)(cp ? n : 0) + w);
    const double est = sh[0] / sh[1];
    const uint32_t* p = limbs + (size_t)(4 * w + 2 * cp) * L;
    const uint32_t* q = p + L;
    const int tp = top_limb(p, L), tq = top_limb(q, L);
    bool bad;
    if (tq < 0 || !isfinite(est)) {
        bad = true;
    } else {
        double ratio = 0.0;
        if (tp >= 0) {
            const double lr = (ln_big(p, tp) - ln_big(q, tq)) * 1.4426950408889634;   // log2 |p/q|
            ratio = lr > 1024.0 ? INFINITY : exp2(lr);
            if (signs[4 * w + 2 * cp] * signs[4 * w + 2 * cp + 1] < 0) ratio = -ratio;
        }
        if (!isfinite(ratio)) bad = true;
        else if (fabs(est) > 1e-10) bad = fabs(ratio - est) / fabs(est) > 0.01;
        else bad = fabs(ratio - est) > 0.01;
    }
    if (bad) atomicOr(status + w, cp ? DR_STATUS_CP_CRT_OVERFLOW : DR_STATUS_CRT_OVERFLOW);
}

cudaError_t launch_crt_check(const uint32_t* limbs, const int32_t* signs, int L, int n,
                             const DevWalk* walks, const double* shadow, uint32_t* status,
                             cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_crt_check<<<(2 * n + 127) / 128, 128, 0, st>>>(limbs, signs, L, n, walks, shadow, status);
    return cudaGetLastError();
}

cudaError_t launch_delta(const DeltaArgs& D, int sms, cudaStream_t st) {
    if (D.n <= 0) return cudaSuccess;
    const int wpb = 4;
    const size_t smem = (size_t)wpb * (3 * (size_t)D.maxlen) * 8;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_delta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int blocks = (D.n + wpb - 1) / wpb;
    if (blocks > sms * 8) blocks = sms * 8;
    k_delta<<<blocks, 32 * wpb, smem, st>>>(D);
    return cudaGetLastError();
}

// ---- top-k -----------------------------------------------------------------
// Keys order doubles descending (+inf first, NaN last); ties by lower index.
__device__ __forceinline__ uint64_t desc_key(double d) {
    if (d != d) return 0ull;                                   // NaN last
    if (d == 0.0) d = 0.0;                                     // -0 equals +0: a tie, by index
    uint64_t b = (uint64_t)__double_as_longlong(d);
    b = (b >> 63) ? ~b : (b | 0x8000000000000000ull);          // ascending order key
    return b;                                                  // larger = better
}

// before(a, b): a ranks ahead of b
__device__ __forceinline__ bool ranks_before(uint64_t ka, uint32_t ia, uint64_t kb, uint32_t ib) {
    return ka > kb || (ka == kb && ia < ib);
}

constexpr int kTopkTile = 4096;

// Compare-exchange of the pair (a, b) of one bitonic stage, a the lower
// index: a takes the better one in an ascending ("best first") segment.
__device__ __forceinline__ void cmpx_pair(uint64_t& ka, uint32_t& ia, uint64_t& kb, uint32_t& ib, bool up) {
    const bool sw = up ? ranks_before(kb, ib, ka, ia) : ranks_before(ka, ia, kb, ib);
    if (sw) {
        const uint64_t tk = ka; ka = kb; kb = tk;
        const uint32_t ti = ia; ia = ib; ib = ti;
    }
}

// Register stage of stride RS * T (T threads): both elements of a pair live
// in one thread (elements e = r * T + tid, r < 4).
template <int RS, int T>
__device__ __forceinline__ void topk_reg_stage(uint64_t (&K)[4], uint32_t (&I)[4], int tid, int size) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
        if ((r & RS) == 0) cmpx_pair(K[r], I[r], K[r | RS], I[r | RS], ((r * T + tid) & size) == 0);
}

// Sort one tile of TILE (key, index) pairs, keep the first k.  Bitonic
// network, TILE / 4 threads holding 4 elements each (element e = r * T +
// tid): strides of T and 2T pair elements of one thread (registers), strides
// below 32 pair lanes of one warp (shuffles), and only strides from 32 to T/2
// go through shared memory, so one SM's shared-memory bandwidth no longer
// bounds the tile.  The order is total (key, then index), so the result is
// the same as any other correct sort's, whatever the tile size.
template <int TILE>
__global__ void __launch_bounds__(TILE / 4) k_topk_tile(const double* __restrict__ vals,
                                                        const uint64_t* __restrict__ in_keys,
                                                        const uint32_t* __restrict__ in_idx, int n,
                                                        int k, uint64_t* __restrict__ out_keys,
                                                        uint32_t* __restrict__ out_idx) {
    constexpr int T = TILE / 4;
    static_assert(T >= 64 && (T & (T - 1)) == 0, "a power-of-two block of at least two warps");
    __shared__ uint64_t sk[TILE];
    __shared__ uint32_t si[TILE];
    const int tid = threadIdx.x;
    const int base = blockIdx.x * TILE;
    uint64_t K[4];
    uint32_t I[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int g = base + r * T + tid;
        if (g < n) {
            K[r] = in_keys ? in_keys[g] : desc_key(vals[g]);
            I[r] = in_idx ? in_idx[g] : (uint32_t)g;
        } else {
            K[r] = 0ull;
            I[r] = 0xffffffffu;
        }
    }
    for (int size = 2; size <= TILE; size <<= 1) {
        int stride = size >> 1;
        if (stride == 2 * T) { topk_reg_stage<2, T>(K, I, tid, size); stride >>= 1; }
        if (stride == T) { topk_reg_stage<1, T>(K, I, tid, size); stride >>= 1; }
        if (stride >= 32) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                sk[r * T + tid] = K[r];
                si[r * T + tid] = I[r];
            }
            __syncthreads();
            for (; stride >= 32; stride >>= 1) {
                for (int i = tid; i < TILE; i += T) {
                    const int j = i ^ stride;
                    if (j > i) {
                        uint64_t ka = sk[i], kb = sk[j];
                        uint32_t ia = si[i], ib = si[j];
                        const bool up = (i & size) == 0;
                        const bool sw = up ? ranks_before(kb, ib, ka, ia) : ranks_before(ka, ia, kb, ib);
                        if (sw) {
                            sk[i] = kb; sk[j] = ka;
                            si[i] = ib; si[j] = ia;
                        }
                    }
                }
                __syncthreads();
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                K[r] = sk[r * T + tid];
                I[r] = si[r * T + tid];
            }
            __syncthreads();   // the next size writes sk / si again
        }
        for (; stride > 0; stride >>= 1) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int e = r * T + tid;
                const uint64_t pk = __shfl_xor_sync(0xffffffffu, K[r], stride);
                const uint32_t pi = __shfl_xor_sync(0xffffffffu, I[r], stride);
                // the lower element of the pair keeps the better one in an
                // ascending segment; the higher keeps it in a descending one
                const bool keep_better = ((e & stride) == 0) == ((e & size) == 0);
                const bool partner_better = ranks_before(pk, pi, K[r], I[r]);
                if (partner_better == keep_better) {
                    K[r] = pk;
                    I[r] = pi;
                }
            }
        }
    }
    const int keep = k < TILE ? k : TILE;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int e = r * T + tid;
        if (e < keep) {
            out_keys[(size_t)blockIdx.x * keep + e] = K[r];
            out_idx[(size_t)blockIdx.x * keep + e] = I[r];
        }
    }
}

// Small inputs sort in tiles of 1024 (256 threads each, several blocks at
// once), larger ones in tiles of 4096.
constexpr int kTopkSmallTile = 1024;
int topk_tile_for(int n, int k) { return (n <= 16384 && 2 * k <= kTopkSmallTile) ? kTopkSmallTile : kTopkTile; }

cudaError_t launch_topk_tile(const double* vals, const uint64_t* in_keys, const uint32_t* in_idx,
                             int n, int k, uint64_t* out_keys, uint32_t* out_idx, cudaStream_t st) {
    const int tile = topk_tile_for(n, k);
    const int tiles = (n + tile - 1) / tile;
    if (tile == kTopkSmallTile)
        k_topk_tile<kTopkSmallTile><<<tiles, kTopkSmallTile / 4, 0, st>>>(vals, in_keys, in_idx, n, k, out_keys, out_idx);
    else
        k_topk_tile<kTopkTile><<<tiles, kTopkTile / 4, 0, st>>>(vals, in_keys, in_idx, n, k, out_keys, out_idx);
    return cudaGetLastError();
}

int topk_tile_size() { return kTopkTile; }

// ---- top-k of a large array: threshold filter --------------------------------
// Sorting every tile costs far more than reading the values once.  For large
// n the host picks a threshold from a strided sample (its r-th best key, r
// chosen so that several times k values are expected to reach it), one pass
// over all n values keeps the (key, index) pairs at or above it, and only
// those go through the tile sort.  The result is exact whenever at least k
// values pass and the candidate buffer holds all of them; the host checks
// the count and otherwise sorts every value.

// sample_keys[j] = key of vals[j * stride], j < s
__global__ void k_topk_sample(const double* __restrict__ vals, int64_t stride, int s,
                              uint64_t* __restrict__ sample_keys, uint32_t* __restrict__ sample_idx) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < s; j += gridDim.x * blockDim.x) {
        sample_keys[j] = desc_key(vals[(int64_t)j * stride]);
        sample_idx[j] = (uint32_t)j;
    }
}

// Appends (key, index) of every value whose key is >= *thr to the candidate
// buffer (warp-aggregated: one atomic per warp and pass); *count counts all
// of them, also those beyond cap, which are not written.
__global__ void __launch_bounds__(256) k_topk_filter(const double* __restrict__ vals, int n,
                                                     const uint64_t* __restrict__ thr,
                                                     uint64_t* __restrict__ cand_keys,
                                                     uint32_t* __restrict__ cand_idx, int cap,
                                                     unsigned int* __restrict__ count) {
    const uint64_t t = *thr;
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int i = base + threadIdx.x;
        uint64_t key = 0;
        bool keep = false;
        if (i < n) {
            key = desc_key(__ldcs(vals + i));   // streamed once: no reuse to cache
            keep = key >= t;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (m == 0u) continue;
        unsigned pos = 0;
        if (lane == __ffs(m) - 1) pos = atomicAdd(count, (unsigned)__popc(m));
        pos = __shfl_sync(0xffffffffu, pos, __ffs(m) - 1) + __popc(m & ((1u << lane) - 1u));
        if (keep && pos < (unsigned)cap) {
            cand_keys[pos] = key;
            cand_idx[pos] = (uint32_t)i;
        }
    }
}

// vals_out[j] = vals[idx[j]], j < k
__global__ void k_topk_gather(const double* __restrict__ vals, const uint32_t* __restrict__ idx, int k,
                              double* __restrict__ vals_out, int32_t* __restrict__ idx_out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
        const uint32_t i = idx[j];
        if (idx_out) idx_out[j] = (int32_t)i;
        if (vals_out) vals_out[j] = vals[i];
    }
}

cudaError_t launch_topk_sample(const double* vals, int64_t stride, int s, uint64_t* keys, uint32_t* idx,
                               cudaStream_t st) {
    k_topk_sample<<<(s + 255) / 256, 256, 0, st>>>(vals, stride, s, keys, idx);
    return cudaGetLastError();
}

cudaError_t launch_topk_filter(const double* vals, int n, const uint64_t* thr, uint64_t* cand_keys,
                               uint32_t* cand_idx, int cap, unsigned int* count, int sms, cudaStream_t st) {
    int blocks = (n + 255) / 256;
    if (blocks > sms * 8) blocks = sms * 8;
    k_topk_filter<<<blocks, 256, 0, st>>>(vals, n, thr, cand_keys, cand_idx, cap, count);
    return cudaGetLastError();
}

cudaError_t launch_topk_gather(const double* vals, const uint32_t* idx, int k, double* vals_out,
                               int32_t* idx_out, cudaStream_t st) {
    k_topk_gather<<<(k + 255) / 256, 256, 0, st>>>(vals, idx, k, vals_out, idx_out);
    return cudaGetLastError();
}

}  // namespace dr
