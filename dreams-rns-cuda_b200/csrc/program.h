// Host-side program handling: blob parsing, validation, register compaction
// and the step-matrix planner that picks an execution class.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "dr_types.h"

namespace dr {

struct Insn {
    uint32_t op, a, b, c;
};

// A program exactly as serialized (reference compiler.py:53-62).
struct RawProgram {
    uint32_t m = 0, dim = 0;
    std::vector<Insn> ops;
    std::vector<int64_t> consts;
    std::vector<int32_t> dirs;
};

// The executable form of one program.
struct Plan {
    uint32_t m = 0, dim = 0;
    Class cls = CLS_INTERP;
    uint32_t degree = 0;            // max degree in the step index over the streams
    std::vector<Insn> ops;          // executed prefix, NOPs dropped, compacted registers,
                                    // STORE operand b = row*m + col
    uint32_t n_regs = 1, zero_reg = 0;
    std::vector<Insn> dops;         // derived stream program (STORE b = stream slot)
    uint32_t dn_regs = 0;
    uint32_t n_streams = 0;
    std::vector<int64_t> consts;    // constant pool shared by both programs
    bool has_inv = false;           // the executed prefix contains INV
    std::vector<Insn> exec;         // executed prefix, uncompacted (bounds analysis)
    std::vector<int32_t> dirs;
    bool fcomp = false;             // float_companion_shape(*this), set once planned
    uint32_t code_id = 0;           // equal ids: identical ops and dops (shared device code)
    std::string blob;               // the program bytes (plan cache key storage)
};

// Status codes mirror the public DR_ERR_* values.
int parse_blob(const uint8_t* blob, uint64_t size, RawProgram* out, std::string* err);
int plan_program(const RawProgram& raw, Plan* out, std::string* err);

// True when the reference's float evaluation of the (compacted) program gives
// every non-last-column entry as an exact constant of the companion shape
// (1.0 on the sub-diagonal, 0.0 elsewhere): the entries are stored straight
// from LOAD_C of that constant (or never stored, which leaves 0.0).
bool float_companion_shape(const Plan& plan);

// log2 of a bound on |value| of every register the reference float evaluator
// produces for steps [0, depth) with integer axes (sd = td = 1); +inf when the
// program has INV or the bound is not finite.
double float_bound_log2(const Plan& plan, const int64_t* axis, uint64_t depth);

}  // namespace dr
