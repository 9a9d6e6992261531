// Bounds checks of DR_DEBUG builds (python dreams-rns-cuda_b200/build.py --debug).
//
// The host validates every program, descriptor and offset before a launch,
// so in a normal build the kernels index their tables without checks.  A
// debug build re-checks on the device every index a walk tile takes from
// its tables -- the walk, its program and combine group, the chunk slot, the
// prime block, the residue outputs, and every register, constant, axis and
// output operand of its bytecode -- before using any of them.  The first
// failed check is recorded in a four-word buffer {site, index, bound, count}
// and the tile is skipped (no out-of-range access is made); the host reads
// the buffer after the run and returns DR_ERR_INDEX.  In normal builds the
// checks compile to nothing.
#pragma once
#include <stdint.h>

#include "dr_types.h"

namespace dr {

// failure sites (first word of the record)
enum DebugSite : uint32_t {
    DBG_TILE_WALK = 1, DBG_TILE_GROUP = 2, DBG_TILE_SLOT = 3, DBG_WALK_PROGRAM = 4,
    DBG_TILE_PRIMES = 5, DBG_WALK_OUTPUT = 6, DBG_PROGRAM_CODE = 7, DBG_PROGRAM_CONSTS = 8,
    DBG_OPERAND_REGISTER = 9, DBG_OPERAND_CONSTANT = 10, DBG_OPERAND_AXIS = 11,
    DBG_OPERAND_OUTPUT = 12, DBG_WALK_AXES = 13,
};

#ifdef DR_DEBUG
constexpr bool kDebugChecks = true;
#else
constexpr bool kDebugChecks = false;
#endif

// idx < bound, else record {site, idx, bound} (first failure wins) and count it
__device__ __forceinline__ bool dbg_check(uint32_t* dbg, uint32_t site, uint64_t idx, uint64_t bound) {
    if (idx < bound) return true;
    if (dbg) {
        if (atomicCAS(dbg, 0u, site) == 0u) {
            dbg[1] = (uint32_t)(idx > 0xffffffffull ? 0xffffffffull : idx);
            dbg[2] = (uint32_t)(bound > 0xffffffffull ? 0xffffffffull : bound);
        }
        atomicAdd(dbg + 3, 1u);
    }
    return false;
}

// Every operand of n instructions at code: registers below regs rows,
// constants below consts, axes below axes, outputs below outs.  STORE's
// second operand is its output slot; the operand layout is the compacted
// one the host planner emits.
__device__ __forceinline__ bool dbg_program(uint32_t* dbg, const uint4* code, uint32_t n, uint32_t regs,
                                            uint32_t consts, uint32_t axes, uint32_t outs) {
    bool ok = true;
    for (uint32_t pc = 0; pc < n; ++pc) {
        const uint4 in = code[pc];
        switch (in.x) {
            case OP_LOAD_X: ok &= dbg_check(dbg, DBG_OPERAND_AXIS, in.y, axes) &
                                  dbg_check(dbg, DBG_OPERAND_REGISTER, in.z, regs); break;
            case OP_LOAD_C: ok &= dbg_check(dbg, DBG_OPERAND_CONSTANT, in.y, consts) &
                                  dbg_check(dbg, DBG_OPERAND_REGISTER, in.z, regs); break;
            case OP_LOAD_N: ok &= dbg_check(dbg, DBG_OPERAND_REGISTER, in.y, regs); break;
            case OP_ADD: case OP_SUB: case OP_MUL:
                ok &= dbg_check(dbg, DBG_OPERAND_REGISTER, in.y, regs) &
                      dbg_check(dbg, DBG_OPERAND_REGISTER, in.z, regs) &
                      dbg_check(dbg, DBG_OPERAND_REGISTER, in.w, regs);
                break;
            case OP_NEG: case OP_POW2: case OP_POW3: case OP_INV:
                ok &= dbg_check(dbg, DBG_OPERAND_REGISTER, in.y, regs) &
                      dbg_check(dbg, DBG_OPERAND_REGISTER, in.z, regs);
                break;
            case OP_STORE: ok &= dbg_check(dbg, DBG_OPERAND_REGISTER, in.y, regs) &
                                 dbg_check(dbg, DBG_OPERAND_OUTPUT, in.z, outs); break;
            default: break;
        }
    }
    return ok;
}

}  // namespace dr
