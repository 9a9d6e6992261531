// FP64 shadow walk (reference runner.py:429-446, cmf_walk.py:400-416):
//     P_f <- P_f @ M_f(s);  if max|P_f| > 1e10: P_f /= max, log_scale += ln(max)
// The recurrence is inherently sequential (the rescale points depend on the
// running values), so each walk's chain runs step by step; what is spread over
// lanes is the evaluation of M_f.  numpy's m x m product rounds as
//     c = a[i][0]*b[0][j];  c = fma(a[i][k], b[k][j], c) for k = 1..m-1
// and is reproduced with explicit IEEE intrinsics (no contraction).
//
// Two modes:
//   interpreted  one warp per walk; lane j evaluates M_f(s0 + j) for 32 steps
//                with the float interpreter, then all lanes run the 32-step
//                chain (redundantly, so nothing diverges).
//   integer      lane = walk, 32 walks per warp: when the host has bounded every
//                intermediate of the reference's float evaluation below 2^53
//                (no INV, integer axes) all those floats are exact integers, so
//                M_f(s) equals the exact integer entries, which advance by
//                int64 forward differences.  Bit-identical to the reference.
#pragma once
#include <stdint.h>

#include "../../include/dreams_b200.h"
#include "dr_types.h"
#include "interp.cuh"

namespace dr {

struct ShadowArgs {
    const DevProgram* progs;
    const uint4* code;
    const int64_t* consts;
    const DevWalk* walks;
    const int64_t* axis;
    const DevShadowSeg* segs;   // segments of this launch
    uint32_t n_items;           // interpreted: segments; integer: groups of 32 segments
    uint32_t n_list;            // segments
    uint32_t* queue;
    double* shadow;             // [3*w] final, [3*(n_walks + w)] checkpoint
    uint32_t n_walks;
    uint32_t* status;
    double* state;              // resident chain state [slot][kShadowStateStride]
    uint32_t rows_regs;         // per-warp smem: doubles, 32 per row
    uint32_t rows_per_warp;
};

constexpr int kShadowStateStride = 72;   // m*m <= 64 entries, then mantissa, exponent, nan flag

// log_scale = sum of ln(max) over the rescale points.  The logarithm is taken
// once at the end: the product of the maxima is carried as mantissa * 2^exp
// (frexp after every rescale, so it cannot overflow), which keeps the
// transcendental off the per-step dependency chain.  The result equals the
// reference's running sum to within its own per-term rounding (~1e-15
// relative).
// x / b rounded to nearest for b > 1e10 finite, given y = RN(1/b): Markstein's
// correction (q0 = RN(x*y), r = x - b*q0 exactly by FMA, q = RN(q0 + r*y) is
// the correctly rounded quotient when it is a normal number; P. Markstein,
// IBM J. Res. Dev. 34(1), 1990).  Zero keeps its sign; subnormal quotients
// take the IEEE division.  One reciprocal serves every entry of a rescale.
__device__ __forceinline__ double div_by(double x, double b, double y) {
    if (x == 0.0) return x;
    const double q0 = __dmul_rn(x, y);
    const double r = __fma_rn(-q0, b, x);
    const double q = __fma_rn(r, y, q0);
    return fabs(q) >= 2.2250738585072014e-308 ? q : __ddiv_rn(x, b);
}

template <int M_>
__device__ __forceinline__ void rescale(double (&P)[M_][M_], double mx) {
    if (isinf(mx)) {
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) P[i][j] = __ddiv_rn(P[i][j], mx);
        return;
    }
    const double y = __drcp_rn(mx);
#pragma unroll
    for (int i = 0; i < M_; ++i)
#pragma unroll
        for (int j = 0; j < M_; ++j) P[i][j] = div_by(P[i][j], mx, y);
}

template <int M_>
struct FChain {
    double P[M_][M_];
    double sc_m;     // product of rescale maxima: sc_m * 2^sc_e
    int sc_e;
    bool nan_seen;

    __device__ __forceinline__ void init(const DevWalk& W) {
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) P[i][j] = (i == j) ? 1.0 : 0.0;
        if ((W.flags & DR_WALK_INIT_PCF) && M_ >= 2) P[0][1] = __ll2double_rn(W.a0);
        sc_m = 1.0;
        sc_e = 0;
        nan_seen = false;
    }
    // P <- P @ X with numpy's rounding, then the max-abs rescale
    __device__ __forceinline__ void step(const double (&X)[M_][M_]) {
        double C[M_][M_];
        double mx = 0.0;
        bool has_nan = false;
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) {
                double c = __dmul_rn(P[i][0], X[0][j]);
#pragma unroll
                for (int k = 1; k < M_; ++k) c = __fma_rn(P[i][k], X[k][j], c);
                C[i][j] = c;
                const double a = fabs(c);
                has_nan |= (a != a);
                mx = fmax(mx, a);
            }
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) P[i][j] = C[i][j];
        if (!has_nan && mx > 1e10) {
            rescale<M_>(P, mx);
            int e;
            sc_m = frexp(__dmul_rn(sc_m, mx), &e);
            sc_e += e;
        }
        nan_seen |= has_nan;
    }
    // companion step: columns shift left, last column = P @ c (same rounding as
    // the dense product with exact 0/1 entries for finite P)
    __device__ __forceinline__ void step_companion(const double (&c)[M_]) {
        double last[M_];
        // the shifted columns are known before the new one: their max and NaN
        // test stay off the dependency chain
        double mx = 0.0;
        bool has_nan = false;
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 1; j < M_; ++j) {
                const double a = fabs(P[i][j]);
                has_nan |= (a != a);
                mx = fmax(mx, a);
            }
#pragma unroll
        for (int i = 0; i < M_; ++i) {
            double v = __dmul_rn(P[i][0], c[0]);
#pragma unroll
            for (int k = 1; k < M_; ++k) v = __fma_rn(P[i][k], c[k], v);
            last[i] = v;
        }
        double mn = 0.0;
#pragma unroll
        for (int i = 0; i < M_; ++i) {
#pragma unroll
            for (int j = 0; j + 1 < M_; ++j) P[i][j] = P[i][j + 1];
            P[i][M_ - 1] = last[i];
            const double a = fabs(last[i]);
            has_nan |= (a != a);
            mn = fmax(mn, a);
        }
        mx = fmax(mx, mn);
        if (!has_nan && mx > 1e10) {
            rescale<M_>(P, mx);
            int e;
            sc_m = frexp(__dmul_rn(sc_m, mx), &e);
            sc_e += e;
        }
        nan_seen |= has_nan;
    }
    __device__ __forceinline__ void load(const double* st) {
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) P[i][j] = st[i * M_ + j];
        sc_m = st[64];
        sc_e = (int)st[65];
        nan_seen = st[66] != 0.0;
    }
    __device__ __forceinline__ void store(double* st) const {
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) st[i * M_ + j] = P[i][j];
        st[64] = sc_m;
        st[65] = (double)sc_e;
        st[66] = nan_seen ? 1.0 : 0.0;
    }
    // start of a segment: the walk's initial matrix at step 0, else the state
    __device__ __forceinline__ void begin(const DevWalk& W, const DevShadowSeg& g, const double* state) {
        if (g.s0 == 0 || g.state == kNoState) init(W);
        else load(state + (size_t)g.state * kShadowStateStride);
    }
    // end of a segment: final outputs, or the state for the next segment
    __device__ __forceinline__ void end(const DevWalk& W, const DevShadowSeg& g, double* state,
                                        double* shadow, uint32_t* status, uint32_t w) const {
        if (g.s1 >= W.depth || g.state == kNoState) {
            write(shadow + 3 * (size_t)w, W);
            if (nan_seen || !isfinite(P[0][M_ - 1])) atomicOr(status + w, DR_STATUS_SHADOW_NAN);
        } else {
            store(state + (size_t)g.state * kShadowStateStride);
        }
    }
    __device__ __forceinline__ void write(double* out, const DevWalk& W) const {
        double q = P[0][M_ - 1];
#pragma unroll
        for (int i = 0; i < M_; ++i)
            if ((uint32_t)i == W.q_row) q = P[i][M_ - 1];
        out[0] = P[0][M_ - 1];
        out[1] = q;
        out[2] = __dadd_rn(log(sc_m), (double)sc_e * 0.69314718055994530942);
    }
};

// LOAD_X in float: float(sn*td + s*tn*sd) / float(sd*td) (cmf_walk.py:278-281);
// the host guarantees these integers fit in int64 for the whole walk.
__device__ __forceinline__ double axis_f64(const int64_t* ax, int64_t s) {
    const int64_t k = ax[0] * ax[3] + s * ax[2] * ax[1];
    return __ddiv_rn(__ll2double_rn(k), __ll2double_rn(ax[1] * ax[3]));
}

template <int M_>
__global__ void __launch_bounds__(128) k_shadow_interp(const ShadowArgs A) {
    extern __shared__ double dsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    double* base = dsm + (size_t)warp * A.rows_per_warp * 32;
    double* rf = base;
    double* axv = rf + A.rows_regs * 32;
    double* mf = axv + kMaxAxes * 32;   // [entry][32 steps]
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const DevShadowSeg g = A.segs[it];
        const uint32_t w = g.walk;
        const DevWalk W = A.walks[w];
        const DevProgram G = A.progs[W.prog];
        FChain<M_> ch;
        ch.begin(W, g, A.state);
        const int64_t* ax = A.axis + W.axis_off;
        if (G.zero_reg != 0xffffffffu) rf[G.zero_reg * 32 + lane] = 0.0;
        for (uint64_t s0 = g.s0; s0 < g.s1; s0 += 32) {
            const int64_t s = (int64_t)(s0 + lane);
            for (uint32_t a = 0; a < G.dim; ++a) axv[a * 32 + lane] = axis_f64(ax + 4 * a, s);
            for (int e = 0; e < M_ * M_; ++e) mf[e * 32 + lane] = 0.0;
            __syncwarp();
            interp_f64(A.code + G.op_off, G.n_ops, rf, A.consts + G.c_off, axv, (double)s, mf, lane);
            __syncwarp();
            const uint32_t n = (uint32_t)min((uint64_t)32, g.s1 - s0);
            for (uint32_t j = 0; j < n; ++j) {
                double X[M_][M_];
#pragma unroll
                for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = mf[e * 32 + j];
                ch.step(X);
                if (W.checkpoint && s0 + j + 1 == W.checkpoint && lane == 0)
                    ch.write(A.shadow + 3 * ((size_t)A.n_walks + w), W);
            }
            __syncwarp();
        }
        if (lane == 0) ch.end(W, g, A.state, A.shadow, A.status, w);
        __syncwarp();
    }
}

// Integer-difference shadow: NS streams of depth D per walk, lane = walk.
template <int CLS, int M_, int D>
__global__ void __launch_bounds__(128) k_shadow_intfd(const ShadowArgs A) {
    constexpr int NS = (CLS == CLS_COMPANION) ? M_ : M_ * M_;
    extern __shared__ double dsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    int64_t* base = reinterpret_cast<int64_t*>(dsm + (size_t)warp * A.rows_per_warp * 32);
    int64_t* rf = base;
    int64_t* axv = rf + A.rows_regs * 32;
    int64_t* stage = axv + kMaxAxes * 32;      // [(j*NS + i)][32 walks]
    int64_t* outv = stage + (D + 1) * NS * 32; // [stream][32 steps]
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const uint32_t first = it * 32;
        const uint32_t count = min(32u, A.n_list - first);
        // difference tables: lane j evaluates segment w's walk at step s0 + j
        for (uint32_t w = 0; w < count; ++w) {
            const DevShadowSeg g = A.segs[first + w];
            const DevWalk W = A.walks[g.walk];
            const DevProgram G = A.progs[W.prog];
            const int64_t* ax = A.axis + W.axis_off;
            const int64_t s = (int64_t)g.s0 + lane;
            for (uint32_t a = 0; a < G.dim; ++a) axv[a * 32 + lane] = ax[0 + 4 * a] + s * ax[2 + 4 * a];
            __syncwarp();
            interp_i64(A.code + G.dop_off, G.dn_ops, rf, A.consts + G.c_off, axv, s, outv, lane);
            __syncwarp();
            if ((uint32_t)lane <= G.degree) {
#pragma unroll
                for (int i = 0; i < NS; ++i) stage[(lane * NS + i) * 32 + w] = outv[i * 32 + lane];
            }
            __syncwarp();
        }
        const bool active = (uint32_t)lane < count;
        const DevShadowSeg g = A.segs[first + (active ? lane : 0)];
        const uint32_t wi = g.walk;
        const DevWalk W = A.walks[wi];
        const DevProgram G = A.progs[W.prog];
        int64_t fd[NS][D + 1];
#pragma unroll
        for (int j = 0; j <= D; ++j)
#pragma unroll
            for (int i = 0; i < NS; ++i) fd[i][j] = ((uint32_t)j <= G.degree && active) ? stage[(j * NS + i) * 32 + lane] : 0;
#pragma unroll
        for (int lvl = 1; lvl <= D; ++lvl)
#pragma unroll
            for (int j = D; j >= lvl; --j)
                if ((uint32_t)j <= G.degree)
#pragma unroll
                    for (int i = 0; i < NS; ++i) fd[i][j] -= fd[i][j - 1];
        FChain<M_> ch;
        ch.begin(W, g, A.state);
        const uint64_t s_end = active ? g.s1 : g.s0;
        for (uint64_t s = g.s0; s < s_end; ++s) {
            if (CLS == CLS_COMPANION) {
                double c[M_];
#pragma unroll
                for (int i = 0; i < M_; ++i) c[i] = __ll2double_rn(fd[i][0]);
                ch.step_companion(c);
            } else {
                double X[M_][M_];
#pragma unroll
                for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = __ll2double_rn(fd[e][0]);
                ch.step(X);
            }
#pragma unroll
            for (int i = 0; i < NS; ++i)
#pragma unroll
                for (int j = 0; j < D; ++j) fd[i][j] += fd[i][j + 1];
            if (W.checkpoint && s + 1 == W.checkpoint) ch.write(A.shadow + 3 * ((size_t)A.n_walks + wi), W);
        }
        if (active) ch.end(W, g, A.state, A.shadow, A.status, wi);
        __syncwarp();
    }
}

}  // namespace dr
