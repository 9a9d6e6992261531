// FP64 shadow walk (reference runner.py:381-398, cmf_walk.py:400-416):
//     P_f <- P_f @ M_f(s);  if max|P_f| > 1e10: P_f /= max, log_scale += ln(max)
// The recurrence is inherently sequential (the rescale points depend on the
// running values), so each walk's chain runs step by step; what is spread over
// lanes is the evaluation of M_f.  numpy's m x m product rounds as
//     c = a[i][0]*b[0][j];  c = fma(a[i][k], b[k][j], c) for k = 1..m-1
// and is reproduced with explicit IEEE intrinsics (no contraction).
//
// Two modes:
//   interpreted  two kernels.  k_shadow_eval evaluates M_f(s) for every step of
//                every segment in parallel (work items of kEvalSteps steps,
//                lane = step, the float interpreter on U sub-blocks at once)
//                and stores the entries the chain needs (the last column when
//                the float matrix has the companion shape, else all m*m) in a
//                step-matrix buffer.  k_shadow_chain then runs the sequential
//                recurrence with lane = segment, 32 segments per warp, streaming
//                its steps' entries through shared memory with cp.async double
//                buffering, so the serial chain never waits on the interpreter.
//   integer      lane = walk, 32 walks per warp: when the host has bounded every
//                intermediate of the reference's float evaluation below 2^53
//                (no INV, integer axes) all those floats are exact integers, so
//                M_f(s) equals the exact integer entries, which advance by
//                int64 forward differences.  Bit-identical to the reference.
//
// Per step the chain's critical path is the product, the max-abs test and,
// when it fires, one correctly rounded reciprocal plus a three-operation
// correction per entry; the max / NaN / threshold tests run on the integer
// pipe (magnitude keys) so the FP64 pipe only carries the arithmetic.
//
// Fast chunks.  The chains run in chunks of steps (the staged chunk of the
// interpreted mode, 8 steps of the integer mode) on a fast path with no
// division branch: every lane computes the Markstein quotients and keeps
// them where it rescales, and records whether it left the Markstein domain.
// A chunk where any lane of the warp did is run again from its saved start
// with the exact steps (IEEE division outside the domain) in a function that
// is not inlined, so that code stays out of the fast loop; both paths give
// bit-identical results inside the domain.  Chains that share their SMs
// with the walk kernels (co-located) run the exact steps throughout: they
// skip the rescale work on steps without one, and issue slots there belong
// to the walks.
#pragma once
#include <stdint.h>

#include <type_traits>

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
    uint32_t n_items;           // evaluation items, or groups of 32 segments (chain, integer)
    uint32_t n_list;            // segments
    double* mf;                 // step-matrix buffer of the interpreted mode
    const uint32_t* eval_items; // segment (index into segs) of every evaluation item
    uint32_t rows_axes;         // evaluation: axis rows per sub-block
    unsigned long long* tstamp; // diagnostics: [start, end] of this launch, or null
    uint32_t* queue;
    double* shadow;             // [3*w] final, [3*(n_walks + w)] checkpoint
    uint32_t n_walks;
    uint32_t* status;
    double* state;              // resident chain state [slot][kShadowStateStride]
    uint32_t rows_regs;         // per-warp smem: doubles, 32 per row
    uint32_t rows_per_warp;
    uint32_t lean;              // chains co-located with walks: exact steps only
    // diagnostics, chain launches: per item [start ns, tables built / state
    // loaded ns, end ns, exact chunk re-runs << 32 | exact steps or chunks], or null
    unsigned long long* item_log;
};

constexpr int kShadowStateStride = 72;   // m*m <= 64 entries, then mantissa, exponent, nan flag

// log_scale = sum of ln(max) over the rescale points.  The logarithm is taken
// once at the end: the product of the maxima is carried as mantissa * 2^exp
// (renormalised by its exponent bits after every rescale, so it cannot overflow), which keeps the
// transcendental off the per-step dependency chain.  The result equals the
// reference's running sum to within its own per-term rounding (~1e-15
// relative).
// IEEE division for the rare entries outside the Markstein domain; not
// inlined so that the common path never pays for it.
static __device__ __noinline__ double div_slow(double x, double b) { return __ddiv_rn(x, b); }

// Biased exponent field of x (0 for zeros and subnormals).
__device__ __forceinline__ int bexp(double x) { return (__double2hiint(x) >> 20) & 0x7ff; }

// Magnitude key: |x| as an integer with the order of |x| (the sign bit
// cleared).  For non-NaN x the key order is the order of |x|; NaN keys exceed
// kInfKey, so the max key of a set of entries also tells whether any is NaN.
__device__ __forceinline__ unsigned long long mag_key(double x) {
    return (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
}
constexpr unsigned long long kInfKey = 0x7ff0000000000000ull;
constexpr unsigned long long kRescaleKey = 0x4202a05f20000000ull;   // key of 1e10

// Markstein quotient q = RN(x / mx) from y = RN(1/mx) (P. Markstein, IBM J.
// Res. Dev. 34(1), 1990): q0 = RN(x*y); the residual x - q0*mx is exact by
// FMA; q = RN(q0 + residual*y).  Written with the residual negated,
// rn = q0*mx - x and q = RN(q0 - rn*y), which equals the above for every x
// and also gives a zero x its own sign (q0 = +-0, rn = +0, -rn*y + q0 keeps
// q0's sign) -- numpy's 0/mx.
__device__ __forceinline__ double markstein_q(double x, double y, double mx) {
    const double q0 = __dmul_rn(x, y);
    const double rn = __fma_rn(q0, mx, -x);
    return __fma_rn(-rn, y, q0);
}

// Whether every quotient x/mx of the entries is exact by markstein_q: y, the
// residual and q are normal numbers when mx < 2^1022 (biased exponent
// em < 2045), the biased exponent ex of x is >= 60 (residual ~ 2^-52 |x|)
// and ex >= em - 1000 (|x/mx| > 2^(ex - em - 1)); zero entries are exact.
// Only exponent bits are read, on the integer pipe.
template <int N_>
__device__ __forceinline__ bool markstein_domain(const double (&P)[N_], double mx) {
    const int em = bexp(mx);
    const int t_hi = max(60, em - 1000) << 20;
    bool out = em >= 2045;
#pragma unroll
    for (int i = 0; i < N_; ++i) {
        const int ahi = __double2hiint(P[i]) & 0x7fffffff;
        out |= (ahi < t_hi) & ((ahi | __double2loint(P[i])) != 0);
    }
    return !out;
}

// Exact rescale: P /= mx entrywise, each quotient rounded to nearest; the
// Markstein quotient inside its domain, the IEEE division outside it (and for
// an infinite mx).
template <int N_>
__device__ __forceinline__ void rescale_n(double (&P)[N_], double mx) {
    const double y = __drcp_rn(mx);
    if (__builtin_expect(!markstein_domain<N_>(P, mx), 0)) {
#pragma unroll
        for (int i = 0; i < N_; ++i) P[i] = div_slow(P[i], mx);
        return;
    }
#pragma unroll
    for (int i = 0; i < N_; ++i) P[i] = markstein_q(P[i], y, mx);
}

template <int M_>
__device__ __forceinline__ void rescale(double (&P)[M_][M_], double mx) {
    rescale_n<M_ * M_>(reinterpret_cast<double (&)[M_ * M_]>(P), mx);
}

// sc_m * 2^sc_e *= mx with sc_m kept in [0.5, 1) (frexp by exponent bits: the
// product of sc_m >= 0.5 and mx > 1e10 is a normal number or infinite).
__device__ __forceinline__ void scale_acc(double& sc_m, int& sc_e, double mx) {
    const double p = __dmul_rn(sc_m, mx);
    const int hi = __double2hiint(p);
    const bool inf = (hi & 0x7ff00000) == 0x7ff00000;
    sc_e += inf ? 0 : ((hi >> 20) & 0x7ff) - 1022;
    sc_m = inf ? p : __hiloint2double((hi & 0x800fffff) | 0x3fe00000, __double2loint(p));
}

// sc_m * 2^sc_e as the same value with sc_m in [0.5, 1) (exact: only the
// exponent moves; an infinite sc_m stays as it is).
__device__ __forceinline__ void scale_norm(double& sc_m, int& sc_e) {
    const int hi = __double2hiint(sc_m);
    const int e = (hi >> 20) & 0x7ff;
    if (e == 0x7ff) return;
    sc_e += e - 1022;
    sc_m = __hiloint2double((hi & 0x800fffff) | 0x3fe00000, __double2loint(sc_m));
}

// Fast rescale of the chunked chains.  Every lane computes the Markstein
// quotients and keeps them where it rescales (rs), with no branch; the scale
// takes the significand of mx in [1, 2) and its exponent separately
// (sc_m * significand rounds to the same significand as sc_m * mx, since the
// two differ by a power of two; scale_norm after at most a chunk of steps
// keeps sc_m finite).  Returns whether this lane rescaled outside the
// Markstein domain: the caller then redoes the chunk with the exact steps.
template <int N_>
__device__ __forceinline__ bool rescale_fast(double (&P)[N_], bool rs, double mx, double& sc_m, int& sc_e) {
    // lanes that do not rescale (their quotients are discarded) take the
    // reciprocal of 2: a tiny, zero or subnormal max would send the
    // reciprocal down its slow special-case path on every step
    const double y = __drcp_rn(rs ? mx : 2.0);
    const bool out = rs & !markstein_domain<N_>(P, mx);
#pragma unroll
    for (int i = 0; i < N_; ++i) {
        const double q = markstein_q(P[i], y, mx);
        P[i] = rs ? q : P[i];
    }
    const int hi = __double2hiint(mx);
    sc_e += rs ? ((hi >> 20) & 0x7ff) - 1023 : 0;
    sc_m = rs ? __dmul_rn(sc_m, __hiloint2double((hi & 0x000fffff) | 0x3ff00000, __double2loint(mx))) : sc_m;
    return out;
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
    // P <- P @ X with numpy's rounding; returns the max magnitude key of the
    // new entries (above kInfKey when one is NaN, numpy's NaN max).
    __device__ __forceinline__ unsigned long long product(const double (&X)[M_][M_]) {
        double C[M_][M_];
        unsigned long long mb = 0;
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) {
                double c = __dmul_rn(P[i][0], X[0][j]);
#pragma unroll
                for (int k = 1; k < M_; ++k) c = __fma_rn(P[i][k], X[k][j], c);
                C[i][j] = c;
                mb = max(mb, mag_key(c));
            }
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) P[i][j] = C[i][j];
        return mb;
    }
    // companion product: X's first m-1 columns are the shifted identity and
    // its last column is c.  The shifted entries use the dense product's own
    // operations with the exact 0 and 1 (so signed zeros, infinities and NaNs
    // come out as numpy's, inf * 0 included); they depend only on the old P
    // and stay off the dependency chain.
    __device__ __forceinline__ unsigned long long product_companion(const double (&c)[M_]) {
        double last[M_];
        double sh[M_][M_ > 1 ? M_ - 1 : 1];
        unsigned long long mb = 0;
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j + 1 < M_; ++j) {
                double v = __dmul_rn(P[i][0], j + 1 == 0 ? 1.0 : 0.0);
#pragma unroll
                for (int k = 1; k < M_; ++k) v = __fma_rn(P[i][k], k == j + 1 ? 1.0 : 0.0, v);
                sh[i][j] = v;
                mb = max(mb, mag_key(v));
            }
#pragma unroll
        for (int i = 0; i < M_; ++i) {
            double v = __dmul_rn(P[i][0], c[0]);
#pragma unroll
            for (int k = 1; k < M_; ++k) v = __fma_rn(P[i][k], c[k], v);
            last[i] = v;
            mb = max(mb, mag_key(v));
        }
#pragma unroll
        for (int i = 0; i < M_; ++i) {
#pragma unroll
            for (int j = 0; j + 1 < M_; ++j) P[i][j] = sh[i][j];
            P[i][M_ - 1] = last[i];
        }
        return mb;
    }
    // the max-abs rescale after a product, exactly (IEEE division outside the
    // Markstein domain); sc_m stays in [0.5, 1)
    __device__ __forceinline__ void finish(unsigned long long mb) {
        const bool nan = mb > kInfKey;
        if (!nan && mb > kRescaleKey) {
            const double mx = __longlong_as_double((long long)mb);
            rescale<M_>(P, mx);
            scale_acc(sc_m, sc_e, mx);
        }
        nan_seen |= nan;
    }
    // the same on the fast path (rescale_fast); out |= this lane left the
    // Markstein domain
    __device__ __forceinline__ void finish_fast(unsigned long long mb, bool& out) {
        const bool nan = mb > kInfKey;
        out |= rescale_fast<M_ * M_>(reinterpret_cast<double (&)[M_ * M_]>(P), !nan && mb > kRescaleKey,
                                     __longlong_as_double((long long)mb), sc_m, sc_e);
        nan_seen |= nan;
    }
    __device__ __forceinline__ void step(const double (&X)[M_][M_]) { finish(product(X)); }
    __device__ __forceinline__ void step_companion(const double (&c)[M_]) { finish(product_companion(c)); }
    __device__ __forceinline__ void step_fast(const double (&X)[M_][M_], bool& out) { finish_fast(product(X), out); }
    __device__ __forceinline__ void step_companion_fast(const double (&c)[M_], bool& out) {
        finish_fast(product_companion(c), out);
    }
    __device__ __forceinline__ void renorm() { scale_norm(sc_m, sc_e); }
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
        double m = sc_m;
        int e = sc_e;
        scale_norm(m, e);
        st[64] = m;
        st[65] = (double)e;
        st[66] = nan_seen ? 1.0 : 0.0;
    }
    // start of a segment: the walk's initial matrix at step 0, else the state
    __device__ __forceinline__ void begin(const DevWalk& W, const DevShadowSeg& g, const double* state,
                                          const int64_t* /*axis*/) {
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
        double p = P[0][M_ - 1], q = P[0][M_ - 1];
#pragma unroll
        for (int i = 0; i < M_; ++i) {
            if ((uint32_t)i == W.p_row) p = P[i][M_ - 1];
            if ((uint32_t)i == W.q_row) q = P[i][M_ - 1];
        }
        double m = sc_m;
        int e = sc_e;
        scale_norm(m, e);
        out[0] = p;
        out[1] = q;
        out[2] = __dadd_rn(log(m), (double)e * 0.69314718055994530942);
    }
};

// State-vector shadow (reference cmf_walk.py:514-522): v <- M_f(s) @ v in
// increasing s, then v /= max|v| when that exceeds 1e10.  numpy's float64
// matrix @ vector goes through BLAS gemv; the summation order below is the one
// the reference's numpy/OpenBLAS produced for m = 2, 3, 4 (checked against
// numpy on random inputs): m = 2: a1*v1 then fma(a0, v0, .); m = 3: the same
// then fma(a2, v2, .); m = 4: (a0v0 + a2v2) + (a1v1 + a3v3) with rounded
// products; other m: a0*v0 then fma(a_k, v_k, .).  A NaN anywhere in v
// reaches every new entry (NaN * x is NaN), so the new entries decide the
// NaN case.
template <int M_>
struct FVec {
    double v[M_];
    double sc_m;
    int sc_e;
    bool nan_seen;

    __device__ __forceinline__ void init(const DevWalk& W, const int64_t* axis) {
        const int64_t* f = axis + W.vec_off + (uint64_t)M_ * W.K;
#pragma unroll
        for (int i = 0; i < M_; ++i) v[i] = __longlong_as_double(__ldg(f + i));
        sc_m = 1.0;
        sc_e = 0;
        nan_seen = false;
    }
    __device__ __forceinline__ static double dot(const double* a, const double* x) {
        if (M_ == 1) return __dmul_rn(a[0], x[0]);
        if (M_ == 2) return __fma_rn(a[0], x[0], __dmul_rn(a[1], x[1]));
        if (M_ == 3) return __fma_rn(a[2], x[2], __fma_rn(a[0], x[0], __dmul_rn(a[1], x[1])));
        if (M_ == 4)
            return __dadd_rn(__dadd_rn(__dmul_rn(a[0], x[0]), __dmul_rn(a[2], x[2])),
                             __dadd_rn(__dmul_rn(a[1], x[1]), __dmul_rn(a[3], x[3 % M_])));
        double c = __dmul_rn(a[0], x[0]);
#pragma unroll
        for (int k = 1; k < M_; ++k) c = __fma_rn(a[k], x[k], c);
        return c;
    }
    // v <- X @ v; returns the max magnitude key of the new entries
    __device__ __forceinline__ unsigned long long product(const double (&X)[M_][M_]) {
        double w[M_];
        unsigned long long mb = 0;
#pragma unroll
        for (int i = 0; i < M_; ++i) {
            w[i] = dot(X[i], v);
            mb = max(mb, mag_key(w[i]));
        }
#pragma unroll
        for (int i = 0; i < M_; ++i) v[i] = w[i];
        return mb;
    }
    // companion-shaped step matrix from its last column: the dense product
    // with the exact 0 and 1 entries
    __device__ __forceinline__ unsigned long long product_companion(const double (&c)[M_]) {
        double X[M_][M_];
#pragma unroll
        for (int i = 0; i < M_; ++i)
#pragma unroll
            for (int j = 0; j < M_; ++j) X[i][j] = (j == M_ - 1) ? c[i] : (i == j + 1 ? 1.0 : 0.0);
        return product(X);
    }
    __device__ __forceinline__ void finish(unsigned long long mb) {
        const bool nan = mb > kInfKey;
        if (!nan && mb > kRescaleKey) {
            const double mx = __longlong_as_double((long long)mb);
            rescale_n<M_>(v, mx);
            scale_acc(sc_m, sc_e, mx);
        }
        nan_seen |= nan;
    }
    __device__ __forceinline__ void finish_fast(unsigned long long mb, bool& out) {
        const bool nan = mb > kInfKey;
        out |= rescale_fast<M_>(v, !nan && mb > kRescaleKey, __longlong_as_double((long long)mb), sc_m, sc_e);
        nan_seen |= nan;
    }
    __device__ __forceinline__ void step(const double (&X)[M_][M_]) { finish(product(X)); }
    __device__ __forceinline__ void step_companion(const double (&c)[M_]) { finish(product_companion(c)); }
    __device__ __forceinline__ void step_fast(const double (&X)[M_][M_], bool& out) { finish_fast(product(X), out); }
    __device__ __forceinline__ void step_companion_fast(const double (&c)[M_], bool& out) {
        finish_fast(product_companion(c), out);
    }
    __device__ __forceinline__ void renorm() { scale_norm(sc_m, sc_e); }
    __device__ __forceinline__ void load(const double* st) {
#pragma unroll
        for (int i = 0; i < M_; ++i) v[i] = st[i];
        sc_m = st[64];
        sc_e = (int)st[65];
        nan_seen = st[66] != 0.0;
    }
    __device__ __forceinline__ void store(double* st) const {
#pragma unroll
        for (int i = 0; i < M_; ++i) st[i] = v[i];
        double m = sc_m;
        int e = sc_e;
        scale_norm(m, e);
        st[64] = m;
        st[65] = (double)e;
        st[66] = nan_seen ? 1.0 : 0.0;
    }
    __device__ __forceinline__ void begin(const DevWalk& W, const DevShadowSeg& g, const double* state,
                                          const int64_t* axis) {
        if (g.s0 == 0 || g.state == kNoState) init(W, axis);
        else load(state + (size_t)g.state * kShadowStateStride);
    }
    __device__ __forceinline__ void write(double* out, const DevWalk& W) const {
        double p = v[0], q = v[0];
#pragma unroll
        for (int i = 0; i < M_; ++i) {
            if ((uint32_t)i == W.p_row) p = v[i];
            if ((uint32_t)i == W.q_row) q = v[i];
        }
        double m = sc_m;
        int e = sc_e;
        scale_norm(m, e);
        out[0] = p;
        out[1] = q;
        out[2] = __dadd_rn(log(m), (double)e * 0.69314718055994530942);
    }
    __device__ __forceinline__ void end(const DevWalk& W, const DevShadowSeg& g, double* state,
                                        double* shadow, uint32_t* status, uint32_t w) const {
        if (g.s1 >= W.depth || g.state == kNoState) {
            write(shadow + 3 * (size_t)w, W);
            double pq[3];
            write(pq, W);
            if (nan_seen || !isfinite(pq[0])) atomicOr(status + w, DR_STATUS_SHADOW_NAN);
        } else {
            store(state + (size_t)g.state * kShadowStateStride);
        }
    }
};

// LOAD_X in float: float(sn*td + s*tn*sd) / float(sd*td) (cmf_walk.py:278-281);
// the host guarantees these integers fit in int64 for the whole walk.
__device__ __forceinline__ double axis_f64(const int64_t* ax, int64_t s) {
    const int64_t k = ax[0] * ax[3] + s * ax[2] * ax[1];
    const int64_t d = ax[1] * ax[3];
    return d == 1 ? __ll2double_rn(k) : __ddiv_rn(__ll2double_rn(k), __ll2double_rn(d));
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Steps per staged chunk of the chain kernel (entries * steps = 16 doubles
// per lane and buffer, at least two steps): a chunk of chain steps takes
// thousands of cycles, far more than the copy of the next one, so small
// buffers suffice (longer chunks measured slower).
__host__ __device__ constexpr int chain_chunk_steps(int ne) { return ne >= 8 ? 2 : 16 / ne; }
// Staging buffers per chain warp (double buffering: one chunk in flight while
// one is consumed; deeper pipelines measured slower).
__host__ __device__ constexpr int chain_buffers(int /*ne*/) { return 2; }

// Evaluation: each warp takes items of kEvalSteps steps of one segment and
// runs the float interpreter on U sub-blocks of 32 steps at a time.  The
// per-warp shared memory holds the register file, the axis values and the
// m*m outputs, each as [row][U][32] doubles; every lane touches only its own
// column, so no warp synchronisation is needed.
template <int U>
__global__ void __launch_bounds__(128) k_shadow_eval(const ShadowArgs A) {
    // the chain launch that follows may place its blocks from now on; it
    // waits for this grid's completion before it reads the step matrices
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    extern __shared__ double dsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    double* rf = dsm + (size_t)warp * A.rows_per_warp * 32;
    double* axv = rf + (size_t)A.rows_regs * U * 32;
    double* outv = axv + (size_t)A.rows_axes * U * 32;
    stamp_begin(A.tstamp);
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const DevShadowSeg g = A.segs[A.eval_items[it]];
        const DevWalk W = A.walks[g.walk];
        const DevProgram G = A.progs[W.prog];
        const int64_t* ax = A.axis + W.axis_off;
        const uint32_t m = G.m;
        const bool comp = G.fcomp != 0;
        const uint32_t ne = comp ? m : m * m;
        if (G.zero_reg != 0xffffffffu)
#pragma unroll
            for (int u = 0; u < U; ++u) rf[(G.zero_reg * U + u) * 32 + lane] = 0.0;
        for (uint32_t e = 0; e < m * m; ++e)
#pragma unroll
            for (int u = 0; u < U; ++u) outv[(e * U + u) * 32 + lane] = 0.0;
        const uint64_t len = g.s1 - g.s0;
        const uint64_t t_item = (uint64_t)(it - g.item0) * kEvalSteps;
        double* dst = A.mf + g.mf_off;
        for (int pass = 0; pass < kEvalSteps / (32 * U); ++pass) {
            const uint64_t t0 = t_item + (uint64_t)pass * 32 * U;
            if (t0 >= len) break;
            const int64_t s_lane = (int64_t)(g.s0 + t0) + lane;
            for (uint32_t a = 0; a < G.dim; ++a)
#pragma unroll
                for (int u = 0; u < U; ++u) axv[(a * U + u) * 32 + lane] = axis_f64(ax + 4 * a, s_lane + 32 * u);
            interp_f64<U>(A.code + G.op_off, G.n_ops, rf, A.consts + G.c_off, axv, s_lane, outv, lane);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t t = t0 + 32 * u + lane;
                if (t < len) {
                    double* d = dst + t * ne;
                    for (uint32_t e = 0; e < ne; ++e) {
                        const uint32_t slot = comp ? e * m + m - 1 : e;
                        d[e] = outv[(slot * U + u) * 32 + lane];
                    }
                }
            }
        }
    }
    stamp_end(A.tstamp);
}

template <int M_, bool COMP, class Chain>
__device__ __forceinline__ void chain_step(Chain& ch, const double (&X)[COMP ? M_ : M_ * M_]) {
    if (COMP) {
        double cv[M_];
#pragma unroll
        for (int i = 0; i < M_; ++i) cv[i] = X[i];
        ch.step_companion(cv);
    } else {
        double Xm[M_][M_];
#pragma unroll
        for (int e = 0; e < M_ * M_; ++e) Xm[e / M_][e % M_] = X[e];
        ch.step(Xm);
    }
}

template <int M_, bool COMP, class Chain>
__device__ __forceinline__ void chain_step_fast(Chain& ch, const double (&X)[COMP ? M_ : M_ * M_], bool& out) {
    if (COMP) {
        double cv[M_];
#pragma unroll
        for (int i = 0; i < M_; ++i) cv[i] = X[i];
        ch.step_companion_fast(cv, out);
    } else {
        double Xm[M_][M_];
#pragma unroll
        for (int e = 0; e < M_ * M_; ++e) Xm[e / M_][e % M_] = X[e];
        ch.step_fast(Xm, out);
    }
}

// The exact steps of one staged chunk (rarely run: only when a lane of the
// warp left the Markstein domain on the fast path).  Not inlined, and taking
// and returning the chain by value, so that its IEEE division code stays out
// of the fast loop's registers and schedule.
template <int M_, bool COMP, class Chain, int CS>
__device__ __noinline__ Chain chain_chunk_exact(Chain ch, const double* buf, int lane) {
    constexpr int NE = COMP ? M_ : M_ * M_;
#pragma unroll 1
    for (int t = 0; t < CS; ++t) {
        double X[NE];
#pragma unroll
        for (int e = 0; e < NE; ++e) X[e] = buf[(t * NE + e) * 32 + lane];
        chain_step<M_, COMP, Chain>(ch, X);
    }
    return ch;
}

template <int M_, bool COMP, class Chain, int CS>
__device__ __noinline__ Chain chain_chunk_partial(Chain ch, const double* buf, int lane, uint64_t base, uint64_t len,
                                                  uint64_t cp_rel, double* cp_out, const DevWalk* Wp) {
    constexpr int NE = COMP ? M_ : M_ * M_;
#pragma unroll 1
    for (int t = 0; t < CS; ++t) {
        const uint64_t rel = base + t;
        if (rel < len) {
            double X[NE];
#pragma unroll
            for (int e = 0; e < NE; ++e) X[e] = buf[(t * NE + e) * 32 + lane];
            chain_step<M_, COMP, Chain>(ch, X);
            if (rel == cp_rel) ch.write(cp_out, *Wp);
        }
    }
    return ch;
}

// Chain: lane = segment, 32 segments per warp, every warp of the block on
// its own items.  The
// warp's entries for the next chunk of steps are copied into shared memory
// ([buffer][step][entry][lane]) while the current chunk runs; every lane only
// reads what it copied itself, so the per-thread cp.async group wait is the
// only synchronisation.
// FLAGS: bit 0 the float step matrix has the companion shape (only its last
// column is stored), bit 1 state-vector walks, bit 2 lean: chains co-located
// with walk kernels run the exact steps, which skip the rescale work on
// steps without one (fewest instructions, as they share issue slots with the
// walks); the others run the fast chunks.
template <int M_, int FLAGS>
__global__ void __launch_bounds__(256) k_shadow_chain(const ShadowArgs A) {
    constexpr bool COMP = (FLAGS & 1) != 0;
    constexpr bool VEC = (FLAGS & 2) != 0;
    constexpr bool LEAN = (FLAGS & 4) != 0;
    using Chain = typename std::conditional<VEC, FVec<M_>, FChain<M_>>::type;
    constexpr int NE = COMP ? M_ : M_ * M_;
    constexpr int CS = chain_chunk_steps(NE);
    extern __shared__ double dsm_all[];
    const int lane = threadIdx.x & 31;
    constexpr int NB = chain_buffers(NE);
    double* dsm = dsm_all + (size_t)(threadIdx.x >> 5) * NB * CS * NE * 32;
    // launched as a programmatic dependent of the evaluation kernel: wait for
    // that grid to complete (and its step matrices to be visible); returns at
    // once when there is no such prerequisite
    asm volatile("griddepcontrol.wait;" ::: "memory");
    stamp_begin(A.tstamp);
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const uint32_t first = it * 32;
        const uint32_t count = min(32u, A.n_list - first);
        unsigned long long* ilog = A.item_log ? A.item_log + 4ull * it : nullptr;
        uint32_t reruns = 0, exact_chunks = 0;
        if (ilog && lane == 0) ilog[0] = global_ns();
        const bool active = (uint32_t)lane < count;
        const DevShadowSeg g = A.segs[first + (active ? lane : 0)];
        const DevWalk W = A.walks[g.walk];
        Chain ch;
        ch.begin(W, g, A.state, A.axis);
        if (ilog && lane == 0) ilog[1] = global_ns();
        const uint64_t len = active ? g.s1 - g.s0 : 0;
        // lanes past the item's segments stream lane 0's step matrices (their
        // results are dropped): stale shared memory could hold values that
        // take slow special-case paths and hold up the whole warp
        const uint64_t load_len = g.s1 - g.s0;
        const double* src = A.mf + g.mf_off;
        unsigned long long mlen = len;
        // chunks every lane runs in full, and the chunk holding any lane's
        // checkpoint, are warp-uniform facts: full chunks without a
        // checkpoint run without per-step tests
        unsigned long long minlen = active ? len : ~0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mlen = max(mlen, __shfl_xor_sync(0xffffffffu, mlen, o));
            minlen = min(minlen, __shfl_xor_sync(0xffffffffu, minlen, o));
        }
        const uint64_t cp_rel = (active && W.checkpoint > g.s0 && W.checkpoint <= g.s1)
                                    ? W.checkpoint - g.s0 - 1 : ~0ull;
        const uint64_t nch = (mlen + CS - 1) / CS;
        auto issue = [&](uint64_t c) {
            double* buf = dsm + (size_t)(c % NB) * CS * NE * 32;
#pragma unroll 1
            for (int t = 0; t < CS; ++t) {
                const uint64_t rel = c * CS + t;
                if (rel < load_len)
#pragma unroll
                    for (int e = 0; e < NE; ++e) cp_async8(buf + (t * NE + e) * 32 + lane, src + rel * NE + e);
            }
        };
        // chunk c goes to buffer c % NB, one commit group per chunk (empty
        // past the end), so waiting until NB - 1 groups are pending means
        // chunk c has landed; chunk c + NB - 1 is issued into the buffer
        // chunk c - 1 has left
#pragma unroll 1
        for (int c0 = 0; c0 + 1 < NB; ++c0) {
            if ((uint64_t)c0 < nch) issue(c0);
            cp_async_commit();
        }
        for (uint64_t c = 0; c < nch; ++c) {
            if (c + NB - 1 < nch) issue(c + NB - 1);
            cp_async_commit();
            cp_async_wait<NB - 1>();
            const double* buf = dsm + (size_t)(c % NB) * CS * NE * 32;
            const uint64_t base = c * CS;
            const bool cp_here = __any_sync(0xffffffffu, cp_rel >= base && cp_rel < base + CS);
            if (LEAN && base + CS <= minlen && !cp_here) {
                double X[NE];
#pragma unroll
                for (int e = 0; e < NE; ++e) X[e] = buf[e * 32 + lane];
#pragma unroll 2
                for (int t = 0; t < CS; ++t) {
                    double Y[NE];
                    const int tn = t + 1 < CS ? t + 1 : t;
#pragma unroll
                    for (int e = 0; e < NE; ++e) Y[e] = buf[(tn * NE + e) * 32 + lane];
                    chain_step<M_, COMP, Chain>(ch, X);
#pragma unroll
                    for (int e = 0; e < NE; ++e) X[e] = Y[e];
                }
            } else if (!LEAN && base + CS <= minlen && !cp_here) {
                // fast steps (no division branch); a chunk where any lane
                // rescaled outside the Markstein domain runs again exactly
                // from its saved start
                const Chain saved = ch;
                bool out = false;
                double X[NE];
#pragma unroll
                for (int e = 0; e < NE; ++e) X[e] = buf[e * 32 + lane];
#pragma unroll
                for (int t = 0; t < CS; ++t) {
                    double Y[NE];
                    const int tn = t + 1 < CS ? t + 1 : t;
#pragma unroll
                    for (int e = 0; e < NE; ++e) Y[e] = buf[(tn * NE + e) * 32 + lane];
                    chain_step_fast<M_, COMP, Chain>(ch, X, out);
#pragma unroll
                    for (int e = 0; e < NE; ++e) X[e] = Y[e];
                }
                ch.renorm();
                if (__any_sync(0xffffffffu, out && active)) {
                    ch = chain_chunk_exact<M_, COMP, Chain, CS>(saved, buf, lane);
                    ++reruns;
                }
            } else {
                ch = chain_chunk_partial<M_, COMP, Chain, CS>(ch, buf, lane, base, len, cp_rel,
                                                               A.shadow + 3 * ((size_t)A.n_walks + g.walk), A.walks + g.walk);
                ++exact_chunks;
            }
        }
        cp_async_wait<0>();
        if (active) ch.end(W, g, A.state, A.shadow, A.status, g.walk);
        if (ilog && lane == 0) {
            ilog[2] = global_ns();
            ilog[3] = ((unsigned long long)reruns << 32) | exact_chunks;
        }
    }
    stamp_end(A.tstamp);
}

// Chain state and difference table of one integer-difference shadow lane.
template <int M_, int NS, int D>
struct FdChain {
    FChain<M_> ch;
    int64_t fd[NS][D + 1];
};

// n exact steps of the integer-difference shadow, with the checkpoint write
// when step s0 + t + 1 is the checkpoint.  Rarely run (segment ends,
// checkpoints, chunks that left the Markstein domain); not inlined and by
// value so that the IEEE division code stays out of the fast loop.
template <int CLS, int M_, int NS, int D>
__device__ __noinline__ FdChain<M_, NS, D> intfd_exact(FdChain<M_, NS, D> st, int n, uint64_t s0,
                                                       uint64_t checkpoint, double* cp_out, const DevWalk* Wp) {
#pragma unroll 1
    for (int t = 0; t < n; ++t) {
        if (CLS == CLS_COMPANION) {
            double c[M_];
#pragma unroll
            for (int i = 0; i < M_; ++i) c[i] = __ll2double_rn(st.fd[i][0]);
            st.ch.step_companion(c);
        } else {
            double X[M_][M_];
#pragma unroll
            for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = __ll2double_rn(st.fd[e][0]);
            st.ch.step(X);
        }
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j < D; ++j) st.fd[i][j] += st.fd[i][j + 1];
        if (checkpoint && s0 + t + 1 == checkpoint) st.ch.write(cp_out, *Wp);
    }
    return st;
}

// Integer-difference shadow: NS streams of depth D per walk, lane = walk.
// LEAN: co-located with walk kernels, the exact steps inline (they skip the
// rescale work on steps without one); otherwise fast chunks.
template <int CLS, int M_, int D, bool LEAN>
__global__ void __launch_bounds__(256) k_shadow_intfd(const ShadowArgs A) {
    constexpr int NS = (CLS == CLS_COMPANION) ? M_ : M_ * M_;
    extern __shared__ double dsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    int64_t* base = reinterpret_cast<int64_t*>(dsm + (size_t)warp * A.rows_per_warp * 32);
    int64_t* rf = base;
    int64_t* axv = rf + A.rows_regs * 32;
    int64_t* stage = axv + kMaxAxes * 32;      // [(j*NS + i)][32 walks]
    int64_t* outv = stage + (D + 1) * NS * 32; // [stream][32 walks]
    stamp_begin(A.tstamp);
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const uint32_t first = it * 32;
        const uint32_t count = min(32u, A.n_list - first);
        unsigned long long* ilog = A.item_log ? A.item_log + 4ull * it : nullptr;
        uint32_t reruns = 0, exact_steps = 0;
        if (ilog && lane == 0) ilog[0] = global_ns();
        // Lanes past the item's walks run a copy of lane 0's walk (same
        // table, same steps) and drop its results.  Left at their start
        // state, they made the whole warp of a partial item ~1.6x slower
        // per step than the warps of full items.
        const bool active = (uint32_t)lane < count;
        const int src = active ? lane : 0;
        const DevShadowSeg g = A.segs[first + src];
        const uint32_t wi = g.walk;
        const DevWalk W = A.walks[wi];
        const DevProgram G = A.progs[W.prog];
        // difference tables: every lane evaluates its own walk at steps
        // s0 .. s0 + degree (the 32 walks at once, each in its own column of
        // the register file, the programs' opcodes applied by selection)
        {
            const int64_t* ax = A.axis + W.axis_off;
            const uint32_t nmax = __reduce_max_sync(0xffffffffu, G.dn_ops);
            for (uint32_t j = 0; j <= G.degree; ++j) {
                const int64_t s = (int64_t)g.s0 + j;
                for (uint32_t a = 0; a < G.dim; ++a) axv[a * 32 + lane] = ax[0 + 4 * a] + s * ax[2 + 4 * a];
                interp_i64_lanes(A.code + G.dop_off, G.dn_ops, nmax, rf, A.consts + G.c_off, axv, s, outv, lane);
#pragma unroll
                for (int i = 0; i < NS; ++i) stage[(j * NS + i) * 32 + lane] = outv[i * 32 + lane];
            }
        }
        FdChain<M_, NS, D> st;
#pragma unroll
        for (int j = 0; j <= D; ++j)
#pragma unroll
            for (int i = 0; i < NS; ++i) st.fd[i][j] = ((uint32_t)j <= G.degree) ? stage[(j * NS + i) * 32 + lane] : 0;
#pragma unroll
        for (int lvl = 1; lvl <= D; ++lvl)
#pragma unroll
            for (int j = D; j >= lvl; --j)
                if ((uint32_t)j <= G.degree)
#pragma unroll
                    for (int i = 0; i < NS; ++i) st.fd[i][j] -= st.fd[i][j - 1];
        st.ch.begin(W, g, A.state, A.axis);
        if (ilog && lane == 0) ilog[1] = global_ns();
        const uint64_t s_end = g.s1;
        const uint64_t cp_step = active ? W.checkpoint : 0;   // copies write no checkpoint
        double* cp_out = A.shadow + 3 * ((size_t)A.n_walks + wi);
        // Chunks of kFdChunk fast steps while every lane that still has steps
        // has a whole chunk left with no checkpoint inside it; a chunk where a
        // lane rescaled outside the Markstein domain runs again exactly from
        // its saved start.  Other steps (segment ends, checkpoints) run exactly.
        constexpr int kFdChunk = 32;
        uint64_t s = g.s0;
        if (LEAN) {
            for (; s < s_end; ++s) {
                if (CLS == CLS_COMPANION) {
                    double c[M_];
#pragma unroll
                    for (int i = 0; i < M_; ++i) c[i] = __ll2double_rn(st.fd[i][0]);
                    st.ch.step_companion(c);
                } else {
                    double X[M_][M_];
#pragma unroll
                    for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = __ll2double_rn(st.fd[e][0]);
                    st.ch.step(X);
                }
#pragma unroll
                for (int i = 0; i < NS; ++i)
#pragma unroll
                    for (int j = 0; j < D; ++j) st.fd[i][j] += st.fd[i][j + 1];
                if (cp_step && s + 1 == cp_step) st.ch.write(cp_out, W);
            }
        }
        if (!LEAN) {
            for (;;) {
                const bool left = s < s_end;
                if (!__any_sync(0xffffffffu, left)) break;
                const bool cp_in = W.checkpoint > s && W.checkpoint <= s + kFdChunk;
                if (__all_sync(0xffffffffu, !left || (s + kFdChunk <= s_end && !cp_in))) {
                    const FdChain<M_, NS, D> saved = st;
                    bool out = false;
#pragma unroll 8
                    for (int t = 0; t < kFdChunk; ++t) {
                        if (CLS == CLS_COMPANION) {
                            double c[M_];
#pragma unroll
                            for (int i = 0; i < M_; ++i) c[i] = __ll2double_rn(st.fd[i][0]);
                            st.ch.step_companion_fast(c, out);
                        } else {
                            double X[M_][M_];
#pragma unroll
                            for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = __ll2double_rn(st.fd[e][0]);
                            st.ch.step_fast(X, out);
                        }
#pragma unroll
                        for (int i = 0; i < NS; ++i)
#pragma unroll
                            for (int j = 0; j < D; ++j) st.fd[i][j] += st.fd[i][j + 1];
                    }
                    st.ch.renorm();
                    if (__any_sync(0xffffffffu, out && left)) {
                        st = intfd_exact<CLS, M_, NS, D>(saved, kFdChunk, s, 0, cp_out, A.walks + wi);
                        ++reruns;
                    }
                    if (left) s += kFdChunk;
                    else st = saved;      // lanes without steps keep their state
                } else {
                    if (left) {
                        st = intfd_exact<CLS, M_, NS, D>(st, 1, s, cp_step, cp_out, A.walks + wi);
                        ++s;
                    }
                    ++exact_steps;
                }
            }
        }
        const FChain<M_>& ch = st.ch;
        if (active) ch.end(W, g, A.state, A.shadow, A.status, wi);
        if (ilog && lane == 0) {
            ilog[2] = global_ns();
            ilog[3] = ((unsigned long long)reruns << 32) | exact_steps;
        }
        __syncwarp();
    }
    stamp_end(A.tstamp);
}


// Split shadow: walks whose float intermediates stay below 2^53 only over
// their first steps (a quartic b(n) with large coefficients, say).  A lane
// runs one walk: the integer-difference chain of k_shadow_intfd (exact int64
// forward differences, bit-identical to the float evaluation while every
// intermediate is an integer below 2^53) from step 0 up to the item's switch
// step g.s0, then the same FChain goes on with the step matrices that
// k_shadow_eval wrote for steps g.s0 .. g.s1, as k_shadow_chain does.  The
// host sorts the walks by their bound, so the 32 walks of an item have
// nearly the same switch step (the smallest of theirs).  Nothing crosses a
// launch: the head costs the integer chain's step, only the tail the
// interpreted chain's.  Shared memory per warp: the head's rows, reused by
// the tail's staging buffers once the head is done.
template <int CLS, int M_, int D>
__global__ void __launch_bounds__(256) k_shadow_split(const ShadowArgs A) {
    constexpr int NS = (CLS == CLS_COMPANION) ? M_ : M_ * M_;
    constexpr bool COMP = CLS == CLS_COMPANION;
    constexpr int NE = COMP ? M_ : M_ * M_;
    constexpr int CS = chain_chunk_steps(NE);
    constexpr int NB = chain_buffers(NE);
    using Chain = FChain<M_>;
    extern __shared__ double dsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    double* wbase = dsm + (size_t)warp * A.rows_per_warp * 32;
    int64_t* rf = reinterpret_cast<int64_t*>(wbase);
    int64_t* axv = rf + A.rows_regs * 32;
    int64_t* stage = axv + kMaxAxes * 32;      // [(j*NS + i)][32 walks]
    int64_t* outv = stage + (D + 1) * NS * 32; // [stream][32 walks]
    double* sbuf = wbase;                      // tail staging, after the head
    // a programmatic dependent of the evaluation kernel: its step matrices
    // are complete and visible past this point
    asm volatile("griddepcontrol.wait;" ::: "memory");
    stamp_begin(A.tstamp);
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const uint32_t first = it * 32;
        const uint32_t count = min(32u, A.n_list - first);
        unsigned long long* ilog = A.item_log ? A.item_log + 4ull * it : nullptr;
        uint32_t reruns = 0, exact = 0;
        if (ilog && lane == 0) ilog[0] = global_ns();
        // lanes past the item's walks run a copy of lane 0's walk and drop
        // its results (as in k_shadow_intfd)
        const bool active = (uint32_t)lane < count;
        const int srcl = active ? lane : 0;
        const DevShadowSeg g = A.segs[first + srcl];
        const uint32_t wi = g.walk;
        const DevWalk W = A.walks[wi];
        const DevProgram G = A.progs[W.prog];
        // head tables: every lane evaluates its own walk at steps 0 .. degree
        // (as in k_shadow_intfd)
        {
            const int64_t* ax = A.axis + W.axis_off;
            const uint32_t nmax = __reduce_max_sync(0xffffffffu, G.dn_ops);
            for (uint32_t j = 0; j <= G.degree; ++j) {
                const int64_t s = j;
                for (uint32_t a = 0; a < G.dim; ++a) axv[a * 32 + lane] = ax[0 + 4 * a] + s * ax[2 + 4 * a];
                interp_i64_lanes(A.code + G.dop_off, G.dn_ops, nmax, rf, A.consts + G.c_off, axv, s, outv, lane);
#pragma unroll
                for (int i = 0; i < NS; ++i) stage[(j * NS + i) * 32 + lane] = outv[i * 32 + lane];
            }
        }
        FdChain<M_, NS, D> st;
#pragma unroll
        for (int j = 0; j <= D; ++j)
#pragma unroll
            for (int i = 0; i < NS; ++i) st.fd[i][j] = ((uint32_t)j <= G.degree) ? stage[(j * NS + i) * 32 + lane] : 0;
#pragma unroll
        for (int lvl = 1; lvl <= D; ++lvl)
#pragma unroll
            for (int j = D; j >= lvl; --j)
                if ((uint32_t)j <= G.degree)
#pragma unroll
                    for (int i = 0; i < NS; ++i) st.fd[i][j] -= st.fd[i][j - 1];
        st.ch.init(W);
        if (ilog && lane == 0) ilog[1] = global_ns();
        const uint64_t s_sw = g.s0;                              // the same on every lane of the item
        const uint64_t cp_step = active ? W.checkpoint : 0;      // copies write no checkpoint
        double* cp_out = A.shadow + 3 * ((size_t)A.n_walks + wi);
        constexpr int kFdChunk = 32;
        uint64_t s = 0;
        while (s < s_sw) {
            const bool cp_in = W.checkpoint > s && W.checkpoint <= s + kFdChunk;
            if (__all_sync(0xffffffffu, s + kFdChunk <= s_sw && !cp_in)) {
                const FdChain<M_, NS, D> saved = st;
                bool out = false;
#pragma unroll 8
                for (int t = 0; t < kFdChunk; ++t) {
                    if (CLS == CLS_COMPANION) {
                        double c[M_];
#pragma unroll
                        for (int i = 0; i < M_; ++i) c[i] = __ll2double_rn(st.fd[i][0]);
                        st.ch.step_companion_fast(c, out);
                    } else {
                        double X[M_][M_];
#pragma unroll
                        for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = __ll2double_rn(st.fd[e][0]);
                        st.ch.step_fast(X, out);
                    }
#pragma unroll
                    for (int i = 0; i < NS; ++i)
#pragma unroll
                        for (int j = 0; j < D; ++j) st.fd[i][j] += st.fd[i][j + 1];
                }
                st.ch.renorm();
                if (__any_sync(0xffffffffu, out)) {
                    st = intfd_exact<CLS, M_, NS, D>(saved, kFdChunk, s, 0, cp_out, A.walks + wi);
                    ++reruns;
                }
                s += kFdChunk;
            } else {
                st = intfd_exact<CLS, M_, NS, D>(st, 1, s, cp_step, cp_out, A.walks + wi);
                ++s;
                ++exact;
            }
        }
        // tail: steps s_sw .. g.s1 from the step-matrix buffer
        Chain ch = st.ch;
        __syncwarp();            // the head's rows are no longer read: the staging reuses them
        const uint64_t len = active ? g.s1 - g.s0 : 0;
        const uint64_t load_len = g.s1 - g.s0;
        const double* src = A.mf + g.mf_off;
        unsigned long long mlen = len;
        unsigned long long minlen = active ? len : ~0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mlen = max(mlen, __shfl_xor_sync(0xffffffffu, mlen, o));
            minlen = min(minlen, __shfl_xor_sync(0xffffffffu, minlen, o));
        }
        const uint64_t cp_rel = (active && W.checkpoint > g.s0 && W.checkpoint <= g.s1)
                                    ? W.checkpoint - g.s0 - 1 : ~0ull;
        const uint64_t nch = (mlen + CS - 1) / CS;
        auto issue = [&](uint64_t c) {
            double* buf = sbuf + (size_t)(c % NB) * CS * NE * 32;
#pragma unroll 1
            for (int t = 0; t < CS; ++t) {
                const uint64_t rel = c * CS + t;
                if (rel < load_len)
#pragma unroll
                    for (int e = 0; e < NE; ++e) cp_async8(buf + (t * NE + e) * 32 + lane, src + rel * NE + e);
            }
        };
#pragma unroll 1
        for (int c0 = 0; c0 + 1 < NB; ++c0) {
            if ((uint64_t)c0 < nch) issue(c0);
            cp_async_commit();
        }
        for (uint64_t c = 0; c < nch; ++c) {
            if (c + NB - 1 < nch) issue(c + NB - 1);
            cp_async_commit();
            cp_async_wait<NB - 1>();
            const double* buf = sbuf + (size_t)(c % NB) * CS * NE * 32;
            const uint64_t base = c * CS;
            const bool cp_here = __any_sync(0xffffffffu, cp_rel >= base && cp_rel < base + CS);
            if (base + CS <= minlen && !cp_here) {
                const Chain saved = ch;
                bool out = false;
                double X[NE];
#pragma unroll
                for (int e = 0; e < NE; ++e) X[e] = buf[e * 32 + lane];
#pragma unroll
                for (int t = 0; t < CS; ++t) {
                    double Y[NE];
                    const int tn = t + 1 < CS ? t + 1 : t;
#pragma unroll
                    for (int e = 0; e < NE; ++e) Y[e] = buf[(tn * NE + e) * 32 + lane];
                    chain_step_fast<M_, COMP, Chain>(ch, X, out);
#pragma unroll
                    for (int e = 0; e < NE; ++e) X[e] = Y[e];
                }
                ch.renorm();
                if (__any_sync(0xffffffffu, out && active)) {
                    ch = chain_chunk_exact<M_, COMP, Chain, CS>(saved, buf, lane);
                    ++reruns;
                }
            } else {
                ch = chain_chunk_partial<M_, COMP, Chain, CS>(ch, buf, lane, base, len, cp_rel, cp_out,
                                                               A.walks + wi);
                ++exact;
            }
        }
        cp_async_wait<0>();
        __syncwarp();            // every lane's copies have landed before the next item's tables
        if (active) ch.end(W, g, A.state, A.shadow, A.status, wi);
        if (ilog && lane == 0) {
            ilog[2] = global_ns();
            ilog[3] = ((unsigned long long)reruns << 32) | exact;
        }
    }
    stamp_end(A.tstamp);
}

}  // namespace dr
