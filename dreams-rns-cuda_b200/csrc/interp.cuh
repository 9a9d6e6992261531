// Warp-uniform bytecode interpreters.
//
// All 32 lanes of a warp run the same program at the same time, so every
// dispatch (instruction fetch from global memory through the read-only path,
// jump on the opcode) is uniform and never diverges; lanes differ only in
// their data (one prime per lane for the residue interpreter, one step or one
// walk per lane for the float interpreters).  The register file lives in
// shared memory as [register][lane], so every access is bank-conflict free.
// Programs arrive compacted by the host planner (a few live registers, NOPs
// and everything after END removed, STORE's operand b = output slot).
#pragma once
#include <stdint.h>

#include "dr_types.h"
#include "modarith.cuh"

namespace dr {

// Residue interpreter (reference runner.py:198-260): registers, constants and
// axis values are Montgomery residues [slot*32 + lane].  Returns true when an
// INV met a zero operand (the reference's "dead lane", config.h:166-169).
__device__ __forceinline__ bool interp_modp(const uint4* __restrict__ code, uint32_t n,
                                            uint32_t* __restrict__ rf,
                                            const uint32_t* __restrict__ cst,
                                            const uint32_t* __restrict__ axv, uint32_t step_m,
                                            uint32_t* __restrict__ out, const Mont& M, int lane) {
    bool inv0 = false;
#pragma unroll 1
    for (uint32_t pc = 0; pc < n; ++pc) {
        const uint4 in = __ldg(code + pc);
        switch (in.x) {
            case OP_LOAD_X: rf[in.z * 32 + lane] = axv[in.y * 32 + lane]; break;
            case OP_LOAD_C: rf[in.z * 32 + lane] = cst[in.y * 32 + lane]; break;
            case OP_LOAD_N: rf[in.y * 32 + lane] = step_m; break;
            case OP_ADD: rf[in.w * 32 + lane] = addm(rf[in.y * 32 + lane], rf[in.z * 32 + lane], M.p); break;
            case OP_SUB: rf[in.w * 32 + lane] = subm(rf[in.y * 32 + lane], rf[in.z * 32 + lane], M.p); break;
            case OP_MUL: rf[in.w * 32 + lane] = mmul(rf[in.y * 32 + lane], rf[in.z * 32 + lane], M); break;
            case OP_NEG: rf[in.z * 32 + lane] = negm(rf[in.y * 32 + lane], M.p); break;
            case OP_POW2: {
                const uint32_t v = rf[in.y * 32 + lane];
                rf[in.z * 32 + lane] = mmul(v, v, M);
                break;
            }
            case OP_POW3: {
                const uint32_t v = rf[in.y * 32 + lane];
                rf[in.z * 32 + lane] = mmul(mmul(v, v, M), v, M);
                break;
            }
            case OP_INV: {
                const uint32_t v = rf[in.y * 32 + lane];
                inv0 |= (v == 0u);
                rf[in.z * 32 + lane] = minv(v, M);
                break;
            }
            case OP_STORE: out[in.z * 32 + lane] = rf[in.y * 32 + lane]; break;
            default: break;
        }
    }
    return inv0;
}

// x^3 rounded once to nearest from the exact product (error-free
// transformations), the rounding the reference's float64 x**3 delivers
// whenever the platform pow is correctly rounded.
__device__ __forceinline__ double cube_rn(double x) {
    const double h = __dmul_rn(x, x);
    const double e = __fma_rn(x, x, -h);        // x*x = h + e exactly
    const double p1 = __dmul_rn(h, x);
    const double e1 = __fma_rn(h, x, -p1);      // h*x = p1 + e1 exactly
    return __dadd_rn(p1, __fma_rn(e, x, e1));
}

// Float64 interpreter (reference runner.py:263-316, cmf_walk.py:261-313),
// U sub-blocks of 32 steps at once: every decoded instruction is applied to
// U independent values per lane, so the shared-memory round trips of one
// sub-block overlap those of the others.  Register r of sub-block u for this
// lane lives at rf[(r*U + u)*32 + lane]; axv and out use the same layout.
// The next instruction is fetched while the current one executes.  No
// contraction: every operation is an explicit IEEE op.
template <int U>
__device__ __forceinline__ void interp_f64(const uint4* __restrict__ code, uint32_t n,
                                           double* __restrict__ rf,
                                           const int64_t* __restrict__ consts,
                                           const double* __restrict__ axv, int64_t s_lane,
                                           double* __restrict__ out, int lane) {
    if (n == 0) return;
    uint4 nx = __ldg(code);
#pragma unroll 1
    for (uint32_t pc = 0; pc < n; ++pc) {
        const uint4 in = nx;
        if (pc + 1 < n) nx = __ldg(code + pc + 1);
#define R_(r, u) rf[((r) * U + (u)) * 32 + lane]
        switch (in.x) {
            case OP_LOAD_X:
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.z, u) = axv[(in.y * U + u) * 32 + lane];
                break;
            case OP_LOAD_C: {
                const double c = __ll2double_rn(__ldg(consts + in.y));
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.z, u) = c;
                break;
            }
            case OP_LOAD_N:
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.y, u) = __ll2double_rn(s_lane + 32 * u);
                break;
            case OP_ADD:
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.w, u) = __dadd_rn(R_(in.y, u), R_(in.z, u));
                break;
            case OP_SUB:
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.w, u) = __dsub_rn(R_(in.y, u), R_(in.z, u));
                break;
            case OP_MUL:
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.w, u) = __dmul_rn(R_(in.y, u), R_(in.z, u));
                break;
            case OP_NEG:
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.z, u) = -R_(in.y, u);
                break;
            case OP_POW2:
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double v = R_(in.y, u);
                    R_(in.z, u) = __dmul_rn(v, v);
                }
                break;
            case OP_POW3:
#pragma unroll
                for (int u = 0; u < U; ++u) R_(in.z, u) = cube_rn(R_(in.y, u));
                break;
            case OP_INV:
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double v = R_(in.y, u);
                    R_(in.z, u) = fabs(v) > 1e-300 ? __ddiv_rn(1.0, v) : 0.0;
                }
                break;
            case OP_STORE:
#pragma unroll
                for (int u = 0; u < U; ++u) out[(in.z * U + u) * 32 + lane] = R_(in.y, u);
                break;
            default: break;
        }
#undef R_
    }
}

// Exact int64 interpreter for programs without INV whose values the host has
// bounded below 2^53 (integer-valued float shadow), with one program per lane
// (the exception to the uniform dispatch above: the lanes evaluate 32
// different walks, whose programs differ in their op sequences).  Every lane
// fetches its own instruction and the opcode selects the result and its
// destination instead of a jump, so the warp stays converged however the
// programs differ.  nmax = the warp's longest program; a lane past its own n
// writes nothing.  Operand rows are read at row 0 where the opcode has no
// such operand, so every access stays inside the register file and axis
// rows.  The instructions (and the
// constants they load) come in batches of kBatch independent loads: with the
// chain kernels' shared memory taking most of the SM, the lanes' 32 programs
// do not stay in L1, and one fetch at a time waited on L2 for every op.
__device__ __forceinline__ void interp_i64_lanes(const uint4* __restrict__ code, uint32_t n, uint32_t nmax,
                                                 int64_t* __restrict__ rf,
                                                 const int64_t* __restrict__ consts,
                                                 const int64_t* __restrict__ axv, int64_t step,
                                                 int64_t* __restrict__ out, int lane) {
    constexpr int kBatch = 8;
#pragma unroll 1
    for (uint32_t pc0 = 0; pc0 < nmax; pc0 += kBatch) {
        uint4 ins[kBatch];
        int64_t cv[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k)
            ins[k] = pc0 + k < n ? __ldg(code + pc0 + k) : make_uint4(OP_NOP, 0u, 0u, 0u);
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            cv[k] = 0;
            if (ins[k].x == OP_LOAD_C) cv[k] = __ldg(consts + ins[k].y);
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint4 in = ins[k];
            const uint32_t op = in.x;
            const bool bin = op == OP_ADD || op == OP_SUB || op == OP_MUL;
            const bool un = op == OP_NEG || op == OP_POW2 || op == OP_POW3;
            const int64_t a = rf[((bin || un || op == OP_STORE) ? in.y : 0u) * 32 + lane];
            const int64_t b = rf[(bin ? in.z : 0u) * 32 + lane];
            const int64_t x = axv[(op == OP_LOAD_X ? in.y : 0u) * 32 + lane];
            const int64_t sq = a * a;
            const int64_t r = op == OP_ADD ? a + b
                            : op == OP_SUB ? a - b
                            : op == OP_MUL ? a * b
                            : op == OP_NEG ? -a
                            : op == OP_POW2 ? sq
                            : op == OP_POW3 ? sq * a
                            : op == OP_LOAD_X ? x
                            : op == OP_LOAD_C ? cv[k]
                            : step;                                  // OP_LOAD_N
            const uint32_t dst = bin ? in.w : op == OP_LOAD_N ? in.y : in.z;
            if (bin || un || op == OP_LOAD_X || op == OP_LOAD_C || op == OP_LOAD_N) rf[dst * 32 + lane] = r;
            if (op == OP_STORE) out[in.z * 32 + lane] = a;
        }
    }
}

}  // namespace dr
