// Persistent walk kernels.
//
// Work unit = tile: one depth chunk [s0, s1) of one (walk, block of <= 32
// primes).  Each warp of a persistent grid pops tiles from a device counter
// (tiles are sorted longest first on the host) and runs the whole chunk in
// registers, lane = prime.  A chunk computes the product of its step
// matrices, starting from the walk's initial matrix (chunk 0) or I.  The
// warp that completes the last chunk of a (walk, prime block) -- detected by
// an atomic counter, so nobody ever waits -- multiplies the chunk products in
// order (matrix products are associative and the arithmetic is exact mod p),
// divides out the accumulated denominator once, and writes the residues.
//
// Per step the step matrix comes from forward-difference streams (classes
// COMPANION, RATIONAL, DENSE; streams initialised by interpreting the derived
// program at D+1 steps) or from the bytecode interpreter (class INTERP).
#pragma once
#include <stdint.h>

#include "../../include/dreams_b200.h"
#include "debug_check.cuh"
#include "dr_types.h"
#include "interp.cuh"
#include "modarith.cuh"

namespace dr {

constexpr unsigned kFull = 0xffffffffu;

struct WalkArgs {
    const DevProgram* progs;
    const uint4* code;          // instructions of every program
    const int64_t* consts;      // constant pools
    const DevWalk* walks;
    const int64_t* axis;        // 4 int64 per axis per walk
    const DevTile* tiles;       // this launch's tiles
    const DevGroup* groups;
    uint32_t n_tiles;
    uint32_t* queue;            // tile counter of this launch (zeroed before launch)
    uint32_t* group_done;       // per-group completion counters (self re-arming)
    uint32_t* chunk_P;          // [slot][m*m][32], slots chunk_stride words apart
    uint32_t chunk_stride;      // words per slot: max m*m of the batch times 32
    uint32_t* chunk_sig;        // [slot][32]
    uint32_t* state_P;          // resident running products [state][chunk_stride words]
    uint32_t* state_sig;        // resident denominators [state][32]
    const uint32_t* primes;     // prime table and Montgomery constants
    const uint32_t* pinv;
    const uint32_t* r2;
    uint32_t* p_res;
    uint32_t* q_res;
    uint32_t* status;
    // per-warp shared memory layout, in 32-word rows; rows_axes rows each for
    // the axis start values, steps and current values (the launch's most axes)
    uint32_t rows_regs, rows_consts, rows_stage;
    uint32_t rows_per_warp;
    uint32_t rows_axes;
    unsigned long long* tstamp;   // diagnostics: [start, end] of this launch, or null
    // sizes of the tables above, for the bounds checks of DR_DEBUG builds
    uint32_t n_progs, n_walks, n_groups, n_slots;
    uint64_t n_code, n_consts, n_axis, n_res;
    uint32_t* dbg;                // DR_DEBUG builds: the first failed check (debug_check.cuh)
};

struct WarpMem {
    uint32_t* rf;
    uint32_t* cst;
    uint32_t* x0;
    uint32_t* dx;
    uint32_t* cur;
    uint32_t* stage;
};

__device__ __forceinline__ WarpMem warp_mem(const WalkArgs& A, uint32_t* smem, int warp) {
    WarpMem w;
    uint32_t* base = smem + (size_t)warp * A.rows_per_warp * 32;
    w.rf = base;
    w.cst = w.rf + A.rows_regs * 32;
    w.x0 = w.cst + A.rows_consts * 32;
    w.dx = w.x0 + A.rows_axes * 32;
    w.cur = w.dx + A.rows_axes * 32;
    w.stage = w.cur + A.rows_axes * 32;
    return w;
}

// Per-lane setup at the start of a tile: modulus, constants and axis
// progressions in Montgomery form.  LOAD_X of axis a at step s is
// x0_a + s * dx_a with x0 = sn*td*inv(sd*td), dx = tn*sd*inv(sd*td)
// (reference cmf_walk.py:221-224, 348-358: the same residues).
__device__ __forceinline__ Mont tile_setup(const WalkArgs& A, const DevTile& T, const DevWalk& W,
                                           const DevProgram& G, const WarpMem& wm, int lane) {
    const uint32_t k = T.prime0 + min((uint32_t)lane, T.nprimes - 1u);
    const Mont M = make_mont(__ldg(A.primes + k), __ldg(A.pinv + k), __ldg(A.r2 + k));
    for (uint32_t i = 0; i < G.n_consts; ++i)
        wm.cst[i * 32 + lane] = to_mont_i64(__ldg(A.consts + G.c_off + i), M);
    for (uint32_t a = 0; a < G.dim; ++a) {
        const int64_t* ax = A.axis + W.axis_off + 4 * a;
        const uint32_t sn = to_mont_i64(__ldg(ax + 0), M), sd = to_mont_i64(__ldg(ax + 1), M);
        const uint32_t tn = to_mont_i64(__ldg(ax + 2), M), td = to_mont_i64(__ldg(ax + 3), M);
        // inv(sd*td); the reference skips the inverse when sd*td == 1
        const uint32_t icd = (__ldg(ax + 1) == 1 && __ldg(ax + 3) == 1) ? M.one : minv(mmul(sd, td, M), M);
        uint32_t x0 = mmul(mmul(sn, td, M), icd, M);
        uint32_t dx = mmul(mmul(tn, sd, M), icd, M);
        if (W.flags & DR_WALK_VEC) {
            // state-vector walk: steps run depth-1 .. 0, so the axis
            // progression starts at x(depth-1) and moves by -dx
            x0 = addm(x0, mmul(to_mont_u64(W.depth - 1, M), dx, M), M.p);
            dx = negm(dx, M.p);
        }
        wm.x0[a * 32 + lane] = x0;
        wm.dx[a * 32 + lane] = dx;
    }
    if (G.zero_reg != 0xffffffffu) wm.rf[G.zero_reg * 32 + lane] = 0u;
    __syncwarp();
    return M;
}

// LOAD_N value (Montgomery) at walk position s: the step index itself, or
// depth-1-s for a state-vector walk, whose product runs M(depth-1) ... M(0).
__device__ __forceinline__ uint32_t step_mont(const DevWalk& W, uint64_t s, const Mont& M) {
    return to_mont_u64((W.flags & DR_WALK_VEC) ? W.depth - 1 - s : s, M);
}

// Axis values at walk position t with x0/dx from tile_setup (already reversed
// for a state-vector walk).
__device__ __forceinline__ void set_axes_at(const WarpMem& wm, uint32_t dim, uint64_t t,
                                            const Mont& M, int lane) {
    const uint32_t t_m = to_mont_u64(t, M);
    for (uint32_t a = 0; a < dim; ++a)
        wm.cur[a * 32 + lane] = addm(wm.x0[a * 32 + lane], mmul(t_m, wm.dx[a * 32 + lane], M), M.p);
}

// Evaluate the original program at step s into stage[entry][lane] (m*m entries,
// zero where not stored, as the reference's fresh zero matrix).
__device__ __forceinline__ bool eval_original(const WalkArgs& A, const DevWalk& W, const DevProgram& G,
                                              const WarpMem& wm, uint64_t s, const Mont& M,
                                              int lane) {
    const uint32_t s_m = step_mont(W, s, M);
    set_axes_at(wm, G.dim, s, M, lane);
    for (uint32_t e = 0; e < G.m * G.m; ++e) wm.stage[e * 32 + lane] = 0u;
    // the derived program may have used the zero register's slot
    if (G.zero_reg != 0xffffffffu) wm.rf[G.zero_reg * 32 + lane] = 0u;
    __syncwarp();
    const bool z = interp_modp(A.code + G.op_off, G.n_ops, wm.rf, wm.cst, wm.cur, s_m, wm.stage, M, lane);
    __syncwarp();
    return z;
}

// Initial chunk matrix: P0 of the walk for chunk 0, else I (Montgomery form).
template <int M_>
__device__ __forceinline__ void init_P(uint32_t (&P)[M_][M_], const DevWalk& W, bool first,
                                       const Mont& M) {
#pragma unroll
    for (int i = 0; i < M_; ++i)
#pragma unroll
        for (int j = 0; j < M_; ++j) P[i][j] = (i == j) ? M.one : 0u;
    if (first && (W.flags & DR_WALK_INIT_PCF) && M_ >= 2) P[0][1] = to_mont_i64(W.a0, M);
}

// P <- P * X for a dense X given per lane
template <int M_>
__device__ __forceinline__ void mat_mul_dense(uint32_t (&P)[M_][M_], const uint32_t (&X)[M_][M_],
                                              const Mont& M) {
    uint32_t R[M_][M_];
#pragma unroll
    for (int i = 0; i < M_; ++i)
#pragma unroll
        for (int j = 0; j < M_; ++j) {
            uint32_t col[M_];
#pragma unroll
            for (int k = 0; k < M_; ++k) col[k] = X[k][j];
            R[i][j] = mdot<M_>(P[i], col, M);
        }
#pragma unroll
    for (int i = 0; i < M_; ++i)
#pragma unroll
        for (int j = 0; j < M_; ++j) P[i][j] = R[i][j];
}

// P <- P * X for X read from stage[entry][lane]
template <int M_>
__device__ __forceinline__ void mat_mul_stage(uint32_t (&P)[M_][M_], const uint32_t* stage,
                                              const Mont& M, int lane) {
    uint32_t X[M_][M_];
#pragma unroll
    for (int i = 0; i < M_; ++i)
#pragma unroll
        for (int j = 0; j < M_; ++j) X[i][j] = stage[(i * M_ + j) * 32 + lane];
    mat_mul_dense<M_>(P, X, M);
}

// Write p = P[0][m-1], q = P[q_row][m-1] divided by sig (Montgomery) as plain
// residues for the active lanes.
template <int M_>
__device__ __forceinline__ void emit(const WalkArgs& A, const DevTile& T, const DevWalk& W,
                                     uint64_t res_off, const uint32_t (&P)[M_][M_], uint32_t sig,
                                     bool scaled, const Mont& M, int lane) {
    uint32_t pv = P[0][M_ - 1];
    uint32_t qv = P[0][M_ - 1];
    if (W.flags & DR_WALK_VEC) {
        // v = P v(0): the two requested entries as dot products with the
        // walk's initial state residues for this prime
        const uint32_t k = T.prime0 + min((uint32_t)lane, T.nprimes - 1u);
        uint32_t w[M_];
#pragma unroll
        for (int j = 0; j < M_; ++j) w[j] = to_mont_i64(__ldg(A.axis + W.vec_off + (uint64_t)j * W.K + k), M);
#pragma unroll
        for (int i = 0; i < M_; ++i) {
            if ((uint32_t)i == W.p_row) pv = mdot<M_>(P[i], w, M);
            if ((uint32_t)i == W.q_row) qv = mdot<M_>(P[i], w, M);
        }
    } else {
#pragma unroll
        for (int i = 0; i < M_; ++i) {
            if ((uint32_t)i == W.p_row) pv = P[i][M_ - 1];
            if ((uint32_t)i == W.q_row) qv = P[i][M_ - 1];
        }
    }
    if (scaled) {
        const uint32_t iv = minv(sig, M);
        pv = mmul(pv, iv, M);
        qv = mmul(qv, iv, M);
    }
    if ((uint32_t)lane < T.nprimes) {
        A.p_res[res_off + T.prime0 + lane] = from_mont(pv, M);
        A.q_res[res_off + T.prime0 + lane] = from_mont(qv, M);
    }
}

// End of a tile: write outputs directly (single chunk) or publish the chunk
// product; the last chunk of the group combines all chunks in order.
template <int M_>
__device__ __forceinline__ void finish_tile(const WalkArgs& A, const DevTile& T, const DevWalk& W,
                                            const uint32_t (&P)[M_][M_], uint32_t sig, bool scaled,
                                            const Mont& M, int lane) {
    const DevGroup Gr = A.groups[T.group];
    const bool resident = Gr.state != kNoState;
    if (Gr.n_chunks == 1 && !resident) {
        emit<M_>(A, T, W, W.res_off, P, sig, scaled, M, lane);
        return;
    }
    uint32_t* dst = A.chunk_P + (size_t)T.slot * A.chunk_stride;
#pragma unroll
    for (int e = 0; e < M_ * M_; ++e) __stcg(dst + e * 32 + lane, P[e / M_][e % M_]);
    if (scaled) __stcg(A.chunk_sig + (size_t)T.slot * 32 + lane, sig);
    __threadfence();
    __syncwarp();
    uint32_t old = 0;
    if (lane == 0) old = atomicAdd(A.group_done + T.group, 1u);
    old = __shfl_sync(kFull, old, 0);
    if (old != Gr.n_chunks - 1) return;
    __threadfence();
    // running product: the resident state of earlier segments, else I (the
    // walk's first chunk already started from its initial matrix)
    uint32_t Q[M_][M_];
    uint32_t acc = M.one;
    const bool from_state = resident && !(Gr.flags & GROUP_FIRST);
    if (from_state) {
        const uint32_t* sp = A.state_P + (size_t)Gr.state * A.chunk_stride;
#pragma unroll
        for (int e = 0; e < M_ * M_; ++e) Q[e / M_][e % M_] = __ldcg(sp + e * 32 + lane);
        acc = __ldcg(A.state_sig + (size_t)Gr.state * 32 + lane);
    }
    for (uint32_t c = 0; c < Gr.n_chunks; ++c) {
        const uint32_t* src = A.chunk_P + (size_t)(Gr.slot0 + c) * A.chunk_stride;
        if (c == 0 && !from_state) {
#pragma unroll
            for (int e = 0; e < M_ * M_; ++e) Q[e / M_][e % M_] = __ldcg(src + e * 32 + lane);
        } else {
            uint32_t X[M_][M_];
#pragma unroll
            for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = __ldcg(src + e * 32 + lane);
            mat_mul_dense<M_>(Q, X, M);
        }
        if (scaled) acc = mmul(acc, __ldcg(A.chunk_sig + (size_t)(Gr.slot0 + c) * 32 + lane), M);
        if (c + 1 == Gr.cp_chunks) emit<M_>(A, T, W, W.cp_res_off, Q, acc, scaled, M, lane);
    }
    if (!resident || (Gr.flags & GROUP_FINAL)) {
        emit<M_>(A, T, W, W.res_off, Q, acc, scaled, M, lane);
    } else {
        uint32_t* sp = A.state_P + (size_t)Gr.state * A.chunk_stride;
#pragma unroll
        for (int e = 0; e < M_ * M_; ++e) __stcg(sp + e * 32 + lane, Q[e / M_][e % M_]);
        __stcg(A.state_sig + (size_t)Gr.state * 32 + lane, acc);
    }
    if (lane == 0) A.group_done[T.group] = 0u;  // re-armed for the next run of this batch
}

// Difference tables: fd[i][j] = Delta^j stream_i(s0), from the derived
// program evaluated at s0 .. s0+Dp (Dp = program degree <= D).
template <int NS, int D>
__device__ __forceinline__ bool fd_init(uint32_t (&fd)[NS][D + 1], const WalkArgs& A, const DevWalk& W,
                                        const DevProgram& G, const WarpMem& wm, uint64_t s0,
                                        const Mont& M, int lane) {
    const uint32_t Dp = G.degree;
    bool inv0 = false;
    for (uint32_t j = 0; j <= Dp; ++j) {
        const uint32_t s_m = step_mont(W, s0 + j, M);
        set_axes_at(wm, G.dim, s0 + j, M, lane);
        __syncwarp();
        inv0 |= interp_modp(A.code + G.dop_off, G.dn_ops, wm.rf, wm.cst, wm.cur, s_m,
                            wm.stage + j * NS * 32, M, lane);
        __syncwarp();
    }
#pragma unroll
    for (int j = 0; j <= D; ++j)
#pragma unroll
        for (int i = 0; i < NS; ++i) fd[i][j] = ((uint32_t)j <= Dp) ? wm.stage[(j * NS + i) * 32 + lane] : 0u;
#pragma unroll
    for (int lvl = 1; lvl <= D; ++lvl)
#pragma unroll
        for (int j = D; j >= lvl; --j)
            if ((uint32_t)j <= Dp)
#pragma unroll
                for (int i = 0; i < NS; ++i) fd[i][j] = subm(fd[i][j], fd[i][j - 1], M.p);
    __syncwarp();
    return inv0;
}

template <int NS, int D>
__device__ __forceinline__ void fd_step(uint32_t (&fd)[NS][D + 1], uint32_t p) {
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) fd[i][j] = addm(fd[i][j], fd[i][j + 1], p);
}

// ---- class bodies -----------------------------------------------------------

// COMPANION: new column j = old column j+1, new last column = P * c.
template <int M_, int D>
__device__ __forceinline__ void tile_companion(const WalkArgs& A, const DevTile& T, const DevWalk& W,
                                               const DevProgram& G, const WarpMem& wm, int lane) {
    const Mont M = tile_setup(A, T, W, G, wm, lane);
    uint32_t fd[M_][D + 1];
    bool inv0 = fd_init<M_, D>(fd, A, W, G, wm, T.s0, M, lane);
    uint32_t P[M_][M_];
    init_P<M_>(P, W, T.s0 == 0, M);
    const uint32_t n = (uint32_t)(T.s1 - T.s0);
    // 8 steps per loop trip (benchmark walk-only replay, m = 2: 1.56 ms
    // unrolled 1x, 1.34 ms 2x, 1.32 ms 4x, 1.24 ms 8x; 16x spills registers)
#pragma unroll 8
    for (uint32_t t = 0; t < n; ++t) {
        uint32_t c[M_];
#pragma unroll
        for (int i = 0; i < M_; ++i) c[i] = fd[i][0];
        uint32_t nc[M_];
#pragma unroll
        for (int i = 0; i < M_; ++i) nc[i] = mdot<M_>(P[i], c, M);
#pragma unroll
        for (int i = 0; i < M_; ++i) {
#pragma unroll
            for (int j = 0; j + 1 < M_; ++j) P[i][j] = P[i][j + 1];
            P[i][M_ - 1] = nc[i];
        }
        fd_step<M_, D>(fd, M.p);
    }
    if (__any_sync(kFull, inv0 && (uint32_t)lane < T.nprimes) && lane == 0)
        atomicOr(A.status + T.walk, DR_STATUS_INV0);
    finish_tile<M_>(A, T, W, P, M.one, false, M, lane);
}

// RATIONAL: M' = g*M with streams c'_0..c'_{m-1} (last column) and g (stream m).
template <int M_, int D>
__device__ __forceinline__ void tile_rational(const WalkArgs& A, const DevTile& T, const DevWalk& W,
                                              const DevProgram& G, const WarpMem& wm, int lane) {
    const Mont M = tile_setup(A, T, W, G, wm, lane);
    uint32_t fd[M_ + 1][D + 1];
    bool inv0 = fd_init<M_ + 1, D>(fd, A, W, G, wm, T.s0, M, lane);
    uint32_t P[M_][M_];
    init_P<M_>(P, W, T.s0 == 0, M);
    uint32_t sig = M.one;
    const uint32_t n = (uint32_t)(T.s1 - T.s0);
#pragma unroll 1
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t g = fd[M_][0];
        if (__any_sync(kFull, g == 0u)) {
            // some denominator is 0 mod p: the reference's INV(0) -> 0 step,
            // re-evaluated exactly from the original bytecode
            inv0 = true;
            eval_original(A, W, G, wm, T.s0 + t, M, lane);
            mat_mul_stage<M_>(P, wm.stage, M, lane);
        } else {
            uint32_t c[M_];
#pragma unroll
            for (int i = 0; i < M_; ++i) c[i] = fd[i][0];
            uint32_t nc[M_];
#pragma unroll
            for (int i = 0; i < M_; ++i) nc[i] = mdot<M_>(P[i], c, M);
#pragma unroll
            for (int i = 0; i < M_; ++i) {
#pragma unroll
                for (int j = 0; j + 1 < M_; ++j) P[i][j] = mmul(P[i][j + 1], g, M);
                P[i][M_ - 1] = nc[i];
            }
            sig = mmul(sig, g, M);
        }
        fd_step<M_ + 1, D>(fd, M.p);
    }
    if (__any_sync(kFull, inv0 && (uint32_t)lane < T.nprimes) && lane == 0)
        atomicOr(A.status + T.walk, DR_STATUS_INV0);
    finish_tile<M_>(A, T, W, P, sig, true, M, lane);
}

// DENSE: every entry is a stream; full P * M.
template <int M_, int D>
__device__ __forceinline__ void tile_dense(const WalkArgs& A, const DevTile& T, const DevWalk& W,
                                           const DevProgram& G, const WarpMem& wm, int lane) {
    const Mont M = tile_setup(A, T, W, G, wm, lane);
    uint32_t fd[M_ * M_][D + 1];
    bool inv0 = fd_init<M_ * M_, D>(fd, A, W, G, wm, T.s0, M, lane);
    uint32_t P[M_][M_];
    init_P<M_>(P, W, T.s0 == 0, M);
    const uint32_t n = (uint32_t)(T.s1 - T.s0);
#pragma unroll 1
    for (uint32_t t = 0; t < n; ++t) {
        uint32_t X[M_][M_];
#pragma unroll
        for (int e = 0; e < M_ * M_; ++e) X[e / M_][e % M_] = fd[e][0];
        mat_mul_dense<M_>(P, X, M);
        fd_step<M_ * M_, D>(fd, M.p);
    }
    if (__any_sync(kFull, inv0 && (uint32_t)lane < T.nprimes) && lane == 0)
        atomicOr(A.status + T.walk, DR_STATUS_INV0);
    finish_tile<M_>(A, T, W, P, M.one, false, M, lane);
}

// INTERP: the bytecode is interpreted at every step (reference semantics
// directly).
template <int M_>
__device__ __forceinline__ void tile_interp(const WalkArgs& A, const DevTile& T, const DevWalk& W,
                                            const DevProgram& G, const WarpMem& wm, int lane) {
    const Mont M = tile_setup(A, T, W, G, wm, lane);
    uint32_t P[M_][M_];
    init_P<M_>(P, W, T.s0 == 0, M);
    bool inv0 = false;
    // axis values advance by dx per step; the step counter by one (down by
    // one for a state-vector walk)
    uint32_t s_m = step_mont(W, T.s0, M);
    set_axes_at(wm, G.dim, T.s0, M, lane);
    const bool rev = (W.flags & DR_WALK_VEC) != 0;
    const uint32_t n = (uint32_t)(T.s1 - T.s0);
#pragma unroll 1
    for (uint32_t t = 0; t < n; ++t) {
        for (uint32_t e = 0; e < (uint32_t)(M_ * M_); ++e) wm.stage[e * 32 + lane] = 0u;
        __syncwarp();
        inv0 |= interp_modp(A.code + G.op_off, G.n_ops, wm.rf, wm.cst, wm.cur, s_m, wm.stage, M, lane);
        __syncwarp();
        mat_mul_stage<M_>(P, wm.stage, M, lane);
        s_m = rev ? subm(s_m, M.one, M.p) : addm(s_m, M.one, M.p);
        for (uint32_t a = 0; a < G.dim; ++a)
            wm.cur[a * 32 + lane] = addm(wm.cur[a * 32 + lane], wm.dx[a * 32 + lane], M.p);
        __syncwarp();
    }
    if (__any_sync(kFull, inv0 && (uint32_t)lane < T.nprimes) && lane == 0)
        atomicOr(A.status + T.walk, DR_STATUS_INV0 | DR_STATUS_FALLBACK);
    else if (lane == 0 && T.s0 == 0)
        atomicOr(A.status + T.walk, DR_STATUS_FALLBACK);
    finish_tile<M_>(A, T, W, P, M.one, false, M, lane);
}

// DR_DEBUG builds: every index the tile takes from the batch's tables, checked
// before it is used (each lane computes the same answer; lane 0 records).
static __device__ __noinline__ bool tile_ok(const WalkArgs& A, const DevTile& T, int lane) {
    uint32_t* d = lane == 0 ? A.dbg : nullptr;
    if (!dbg_check(d, DBG_TILE_WALK, T.walk, A.n_walks) || !dbg_check(d, DBG_TILE_GROUP, T.group, A.n_groups))
        return false;
    const DevWalk& W = A.walks[T.walk];
    if (!dbg_check(d, DBG_WALK_PROGRAM, W.prog, A.n_progs)) return false;
    const DevProgram& G = A.progs[W.prog];
    const DevGroup& Gr = A.groups[T.group];
    bool ok = dbg_check(d, DBG_TILE_PRIMES, T.nprimes - 1u, 32) &
              dbg_check(d, DBG_TILE_PRIMES, (uint64_t)T.prime0 + T.nprimes, (uint64_t)W.K + 1);
    if (Gr.n_chunks > 1 || Gr.state != kNoState) ok &= dbg_check(d, DBG_TILE_SLOT, T.slot, A.n_slots);
    ok &= dbg_check(d, DBG_WALK_OUTPUT, W.res_off + W.K, A.n_res + 1);
    if (W.checkpoint) ok &= dbg_check(d, DBG_WALK_OUTPUT, W.cp_res_off + W.K, A.n_res + 1);
    ok &= dbg_check(d, DBG_WALK_AXES, W.axis_off + 4ull * G.dim, A.n_axis + 1) &
          dbg_check(d, DBG_OPERAND_AXIS, G.dim, A.rows_axes + 1);
    ok &= dbg_check(d, DBG_PROGRAM_CODE, (uint64_t)G.op_off + G.n_ops, A.n_code + 1) &
          dbg_check(d, DBG_PROGRAM_CODE, (uint64_t)G.dop_off + G.dn_ops, A.n_code + 1) &
          dbg_check(d, DBG_PROGRAM_CONSTS, (uint64_t)G.c_off + G.n_consts, A.n_consts + 1) &
          dbg_check(d, DBG_OPERAND_CONSTANT, G.n_consts, A.rows_consts + 1);
    if (!ok) return false;
    const uint32_t zr = G.zero_reg;
    ok &= zr == 0xffffffffu || dbg_check(d, DBG_OPERAND_REGISTER, zr, A.rows_regs);
    ok &= dbg_program(d, A.code + G.op_off, G.n_ops, A.rows_regs, A.rows_consts, G.dim, G.m * G.m) &
          dbg_program(d, A.code + G.dop_off, G.dn_ops, A.rows_regs, A.rows_consts, G.dim,
                      G.n_streams ? G.n_streams : G.m * G.m);
    return ok;
}

// ---- persistent kernel ----------------------------------------------------
// DR_WALK_MIN_BLOCKS (a build define; 0 = the compiler's choice) asks for that
// many resident 128-thread blocks per SM, which caps the registers per thread.
#ifndef DR_WALK_MIN_BLOCKS
#define DR_WALK_MIN_BLOCKS 0
#endif
#if DR_WALK_MIN_BLOCKS > 0
#define DR_WALK_BOUNDS __launch_bounds__(128, DR_WALK_MIN_BLOCKS)
#else
#define DR_WALK_BOUNDS __launch_bounds__(128)
#endif
template <int CLS, int M_, int D>
__global__ void DR_WALK_BOUNDS k_walk(const WalkArgs A) {
    extern __shared__ uint32_t smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const WarpMem wm = warp_mem(A, smem, warp);
    stamp_begin(A.tstamp);
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(A.queue, 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= A.n_tiles) break;
        const DevTile T = A.tiles[t];
        if (kDebugChecks && A.dbg && !tile_ok(A, T, lane)) continue;   // recorded; the host reports it
        const DevWalk W = A.walks[T.walk];
        const DevProgram G = A.progs[W.prog];
        if (CLS == CLS_COMPANION) tile_companion<M_, D>(A, T, W, G, wm, lane);
        else if (CLS == CLS_RATIONAL) tile_rational<M_, D>(A, T, W, G, wm, lane);
        else if (CLS == CLS_DENSE) tile_dense<M_, D>(A, T, W, G, wm, lane);
        else tile_interp<M_>(A, T, W, G, wm, lane);
        __syncwarp();
    }
    stamp_end(A.tstamp);
}

}  // namespace dr
