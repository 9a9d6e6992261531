// Internal types shared by the host planner and the device kernels.
#pragma once
#include <stdint.h>

namespace dr {

// Opcode numbers of the program wire format (reference compiler.py:14-28).
enum Opcode : uint32_t {
    OP_NOP = 0, OP_LOAD_X = 1, OP_LOAD_C = 2, OP_LOAD_N = 3, OP_ADD = 4, OP_SUB = 5,
    OP_MUL = 6, OP_NEG = 7, OP_POW2 = 8, OP_POW3 = 9, OP_INV = 10, OP_STORE = 11, OP_END = 12
};

// How a program is executed.
enum Class : uint32_t {
    CLS_COMPANION = 1,   // M = [[0..0 c0],[1 ..  c1],...]: sub-diagonal exactly 1, no INV
                         // of step-dependent values; entries advanced by forward
                         // differences, P*M is a column shift plus one mat-vec.
    CLS_RATIONAL = 2,    // companion with rational last column: M = M'/g, g = product of
                         // the denominators; P' advances with polynomial M', the scalar
                         // g is accumulated and divided out once per chunk combine.
    CLS_DENSE = 3,       // dense polynomial matrix, every entry by forward differences.
    CLS_INTERP = 4,      // anything else: bytecode interpreted every step.
};

// Per-program record in device memory.  Instructions are uint4 {op, a, b, c}
// with compacted registers; STORE's second operand is the entry slot
// row*m + col (original program) or the stream slot (derived program).
struct DevProgram {
    uint32_t m, dim, cls, degree;      // degree: max degree in s of the streams
    uint32_t op_off, n_ops, n_regs;    // original program (compacted)
    uint32_t dop_off, dn_ops, dn_regs; // derived stream program (FD classes)
    uint32_t c_off, n_consts;          // int64 constant pool
    uint32_t n_streams;                // derived outputs
    uint32_t zero_reg;                 // compacted register that always holds 0
    uint32_t shadow_fd;                // 1: float shadow may use integer differences
    uint32_t fcomp;                    // 1: float step matrix has the companion shape
};

// Per-walk record in device memory.
struct DevWalk {
    uint32_t prog, K, flags, q_row;
    int64_t a0;
    uint64_t depth, checkpoint;
    uint64_t axis_off;                 // into the int64 axis parameter array
    uint64_t res_off, cp_res_off;      // residue output offsets
    uint32_t shadow_mode;              // 0 none, 1 interpret, 2 integer differences
    uint32_t p_row;                    // row (state-vector walk: entry) of p
    uint64_t vec_off;                  // state-vector walk: v(0) in the axis array
};

// One unit of walk work: a depth chunk of one (walk, prime block).
struct DevTile {
    uint32_t walk;
    uint32_t group;        // (walk, prime block) combine group
    uint32_t prime0;       // first prime index of the block
    uint32_t nprimes;      // primes in this block (<= 32)
    uint32_t chunk;        // chunk index within the group
    uint32_t slot;         // chunk-product slot (unused when the group has one chunk)
    uint64_t s0, s1;       // step range [s0, s1)
};

// Combine group: the chunks of one (walk, prime block) in one launch.  With a
// resident state slot (serving) the chunks are one segment of a longer walk:
// the running product and denominator are read from the slot (unless this is
// the first segment), multiplied by the chunk products, and written back (or
// emitted on the final segment).
constexpr uint32_t kNoState = 0xffffffffu;
constexpr uint32_t GROUP_FIRST = 1u, GROUP_FINAL = 2u;
struct DevGroup {
    uint32_t walk, prime0, nprimes, n_chunks;
    uint32_t slot0;        // first chunk-product slot
    uint32_t cp_chunks;    // chunks covering [0, checkpoint) (0 = no checkpoint)
    uint32_t state;        // resident state slot or kNoState
    uint32_t flags;        // GROUP_FIRST | GROUP_FINAL
};

// Shadow work item: steps [s0, s1) of one walk; state is a resident slot
// (segments of a longer walk) or kNoState (the walk runs from step 0 to its
// depth).  Interpreted segments also own a range of the step-matrix buffer
// (mf_off, in doubles: (s1 - s0) steps of ne entries) and the evaluation
// items item0 .. item0 + ceil((s1 - s0) / kEvalSteps) - 1.
struct DevShadowSeg {
    uint32_t walk, state;
    uint64_t s0, s1;
    uint64_t mf_off;
    uint32_t item0, pad;
};

// Steps per evaluation work item of the interpreted shadow.
constexpr int kEvalSteps = 128;

// Entries of the float step matrix the chain reads per step: the last column
// when the reference's float evaluation yields exactly the companion shape
// (sub-diagonal 1.0, other non-last columns 0.0), else all m*m.
inline uint32_t shadow_entries(uint32_t m, bool float_companion) {
    return float_companion ? m : m * m;
}

enum ShadowMode : uint32_t { SHADOW_NONE = 0, SHADOW_INTERP = 1, SHADOW_INTFD = 2 };

// Diagnostics: when a launch carries a timestamp pair, the first instruction
// of every block lowers [0] and the last raises [1] to the global timer (ns),
// so a concurrent run shows when each kernel actually held the GPU.
#ifdef __CUDACC__
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void stamp_begin(unsigned long long* ts) {
    if (ts && threadIdx.x == 0) atomicMin(ts, (unsigned long long)global_ns());
}
__device__ __forceinline__ void stamp_end(unsigned long long* ts) {
    if (ts) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(ts + 1, (unsigned long long)global_ns());
    }
}
#endif

constexpr int kMaxM = 8;
constexpr int kMaxAxes = 8;
constexpr int kMaxDegree = 16;
constexpr int kMaxConsts = 512;
constexpr int kMaxCompactRegs = 160;
constexpr int kMaxFdRegs = 72;     // streams * (D + 1) held in registers per lane

// Difference-table depths with a compiled kernel.
constexpr int kTemplateDegrees[] = {1, 2, 3, 4, 6, 8, 12, 16};

inline int streams_for(uint32_t cls, uint32_t m) {
    return cls == CLS_COMPANION ? (int)m : cls == CLS_RATIONAL ? (int)m + 1
         : cls == CLS_DENSE ? (int)(m * m) : 0;
}

// Smallest compiled difference depth >= degree for (cls, m), or -1 if the
// program must run on the interpreter.  Must agree with the instantiation
// list in walk_kernels.cu.
inline int template_degree(uint32_t cls, uint32_t m, uint32_t degree) {
    bool m_ok = (cls == CLS_COMPANION && m >= 2 && m <= 6) ||
                (cls == CLS_RATIONAL && m >= 2 && m <= 4) ||
                (cls == CLS_DENSE && m >= 2 && m <= 3);
    if (!m_ok) return -1;
    for (int d : kTemplateDegrees) {
        if ((uint32_t)d < degree) continue;
        if (streams_for(cls, m) * (d + 1) > kMaxFdRegs) return -1;
        return d;
    }
    return -1;
}

}  // namespace dr
