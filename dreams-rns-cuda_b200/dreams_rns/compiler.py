"""Bytecode ISA, program wire format and the sympy -> bytecode compiler.

The bytecode is the interface between the host and the walk kernels, so the
opcode numbering, the 16-byte instruction record and the program blob layout
are kept identical to the reference (python/dreams_rns/compiler.py:14-89).
The compiler below is written independently but must emit the same
instruction stream, register numbers and constant order as the reference
compiler (compiler.py:92-306) for the same sympy expression, because users
serialize programs and the walk results are defined by that exact stream:

* every sympy node gets a fresh virtual register, allocated *after* its
  operands have been compiled (compiler.py:116-122, 153-198);
* the register counter restarts at 0 after each STORE (compiler.py:280-289);
* the allocator refuses the register whose allocation would bring the count
  to 512 (compiler.py:105, 120-121);
* constants are de-duplicated in first-use order (compiler.py:124-128).
"""

from __future__ import annotations

import struct
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Dict, List, Optional, Tuple

__all__ = [
    "Opcode",
    "Instruction",
    "CmfProgram",
    "CmfCompiler",
    "compile_cmf",
    "compile_cmf_from_dict",
    "compile_pcf",
]


class Opcode(IntEnum):
    """Opcode numbers of the walk bytecode (reference compiler.py:14-28)."""

    NOP = 0
    LOAD_X = 1   # LOAD_X axis, dest      : axis value at this step
    LOAD_C = 2   # LOAD_C index, dest     : program constant
    LOAD_N = 3   # LOAD_N dest            : step counter (0-based)
    ADD = 4      # ADD a, b, dest
    SUB = 5      # SUB a, b, dest
    MUL = 6      # MUL a, b, dest
    NEG = 7      # NEG a, dest
    POW2 = 8     # POW2 a, dest
    POW3 = 9     # POW3 a, dest
    INV = 10     # INV a, dest            : a^(p-2) mod p, so INV(0) == 0
    STORE = 11   # STORE reg, row, col    : matrix entry
    END = 12


_INSN = struct.Struct("<IIII")
_HEADER = _INSN


@dataclass
class Instruction:
    """One 16-byte instruction: opcode and three unsigned 32-bit operands."""

    op: Opcode
    arg0: int = 0
    arg1: int = 0
    arg2: int = 0

    def pack(self) -> bytes:
        return _INSN.pack(int(self.op), self.arg0, self.arg1, self.arg2)


@dataclass
class CmfProgram:
    """A compiled step-matrix program.

    Blob layout (little-endian, reference compiler.py:53-62):
    ``u32 m, u32 dim, u32 n_ops, u32 n_consts`` then ``n_ops`` records of
    ``u32 op, arg0, arg1, arg2``, then ``n_consts`` ``i64`` constants, then
    ``dim`` ``i32`` walk directions.
    """

    m: int
    dim: int
    opcodes: List[Instruction] = field(default_factory=list)
    constants: List[int] = field(default_factory=list)
    directions: List[int] = field(default_factory=list)

    def serialize(self) -> bytes:
        parts = [_HEADER.pack(self.m, self.dim, len(self.opcodes), len(self.constants))]
        parts.extend(ins.pack() for ins in self.opcodes)
        parts.extend(struct.pack("<q", c) for c in self.constants)
        parts.extend(struct.pack("<i", d) for d in self.directions)
        return b"".join(parts)

    @classmethod
    def deserialize(cls, data: bytes) -> "CmfProgram":
        m, dim, n_ops, n_consts = _HEADER.unpack_from(data, 0)
        pos = _HEADER.size
        ops = []
        for _ in range(n_ops):
            op, a0, a1, a2 = _INSN.unpack_from(data, pos)
            ops.append(Instruction(Opcode(op), a0, a1, a2))
            pos += _INSN.size
        consts = list(struct.unpack_from("<%dq" % n_consts, data, pos))
        pos += 8 * n_consts
        dirs = list(struct.unpack_from("<%di" % dim, data, pos))
        return cls(m=m, dim=dim, opcodes=ops, constants=consts, directions=dirs)


class CmfCompiler:
    """Tree-walking sympy -> bytecode compiler with one register per node.

    Public methods and their emission order follow the reference
    (compiler.py:92-306) so that programs are byte-identical.
    """

    MAX_REGS = 512

    def __init__(self, m: int, dim: int, directions: Optional[List[int]] = None):
        self.m = m
        self.dim = dim
        self.directions = directions or [1] * dim
        self.opcodes: List[Instruction] = []
        self.constants: Dict[int, int] = {}
        self.next_reg = 0
        self.entry_regs: Dict[Tuple[int, int], int] = {}

    # -- emission primitives -------------------------------------------------
    def _alloc_reg(self) -> int:
        reg = self.next_reg
        self.next_reg = reg + 1
        if self.next_reg >= self.MAX_REGS:
            raise RuntimeError("Out of registers")
        return reg

    def _add_const(self, value: int) -> int:
        return self.constants.setdefault(value, len(self.constants))

    def _emit(self, op: Opcode, arg0: int = 0, arg1: int = 0, arg2: int = 0) -> None:
        self.opcodes.append(Instruction(op, arg0, arg1, arg2))

    def _unary(self, op: Opcode, r: int) -> int:
        dest = self._alloc_reg()
        self._emit(op, r, dest)
        return dest

    def _binary(self, op: Opcode, r1: int, r2: int) -> int:
        dest = self._alloc_reg()
        self._emit(op, r1, r2, dest)
        return dest

    def load_axis(self, axis: int) -> int:
        reg = self._alloc_reg()
        self._emit(Opcode.LOAD_X, axis, reg)
        return reg

    def load_const(self, value: int) -> int:
        idx = self._add_const(value)
        reg = self._alloc_reg()
        self._emit(Opcode.LOAD_C, idx, reg)
        return reg

    def load_n(self) -> int:
        reg = self._alloc_reg()
        self._emit(Opcode.LOAD_N, reg)
        return reg

    def add(self, r1: int, r2: int) -> int:
        return self._binary(Opcode.ADD, r1, r2)

    def sub(self, r1: int, r2: int) -> int:
        return self._binary(Opcode.SUB, r1, r2)

    def mul(self, r1: int, r2: int) -> int:
        return self._binary(Opcode.MUL, r1, r2)

    def neg(self, r: int) -> int:
        return self._unary(Opcode.NEG, r)

    def pow2(self, r: int) -> int:
        return self._unary(Opcode.POW2, r)

    def pow3(self, r: int) -> int:
        return self._unary(Opcode.POW3, r)

    def inv(self, r: int) -> int:
        return self._unary(Opcode.INV, r)

    def store(self, r: int, row: int, col: int) -> None:
        self._emit(Opcode.STORE, r, row, col)
        self.entry_regs[(row, col)] = r

    # -- sympy tree walk -----------------------------------------------------
    def _fold(self, op, operands, axis_symbols) -> int:
        """Left fold of ``op`` over compiled operands, emitting as it goes."""
        acc = self.compile_sympy_expr(operands[0], axis_symbols)
        for term in operands[1:]:
            acc = op(acc, self.compile_sympy_expr(term, axis_symbols))
        return acc

    def _power_chain(self, base, count: int, axis_symbols) -> int:
        r = self.compile_sympy_expr(base, axis_symbols)
        acc = r
        for _ in range(count - 1):
            acc = self.mul(acc, r)
        return acc

    def compile_sympy_expr(self, expr, axis_symbols: Dict[str, int]) -> int:
        """Compile ``expr``; return the register that holds its value."""
        import sympy as sp

        if isinstance(expr, (int, sp.Integer)):
            return self.load_const(int(expr))
        if isinstance(expr, sp.Symbol):
            name = str(expr)
            if name == "n":
                return self.load_n()
            if name in axis_symbols:
                return self.load_axis(axis_symbols[name])
            raise ValueError(f"Unknown symbol: {name}")
        if isinstance(expr, sp.Add):
            return self._fold(self.add, expr.args, axis_symbols)
        if isinstance(expr, sp.Mul):
            args = expr.args
            if args[0] == -1:
                return self.neg(self.compile_sympy_expr(sp.Mul(*args[1:]), axis_symbols))
            return self._fold(self.mul, args, axis_symbols)
        if isinstance(expr, sp.Pow):
            base, exp = expr.args
            if exp == 2:
                return self.pow2(self.compile_sympy_expr(base, axis_symbols))
            if exp == 3:
                return self.pow3(self.compile_sympy_expr(base, axis_symbols))
            if exp == -1:
                return self.inv(self.compile_sympy_expr(base, axis_symbols))
            if isinstance(exp, (int, sp.Integer)):
                e = int(exp)
                if e > 0:
                    return self._power_chain(base, e, axis_symbols)
                if e < -1:
                    return self.inv(self._power_chain(base, -e, axis_symbols))
            raise ValueError(f"Unsupported power: {expr}")
        if isinstance(expr, sp.Rational):
            num = self.load_const(int(expr.p))
            den = self.load_const(int(expr.q))
            return self.mul(num, self.inv(den))
        raise ValueError(f"Unsupported expression type: {type(expr)}")

    def compile_matrix_entry(self, row: int, col: int, expr, axis_symbols: Dict[str, int]) -> None:
        reg = self.compile_sympy_expr(expr, axis_symbols)
        self.store(reg, row, col)
        self.next_reg = 0

    def build(self) -> CmfProgram:
        self._emit(Opcode.END)
        consts = [0] * len(self.constants)
        for value, idx in self.constants.items():
            consts[idx] = value
        return CmfProgram(m=self.m, dim=self.dim, opcodes=list(self.opcodes),
                          constants=consts, directions=list(self.directions))


def compile_cmf(cmf, axis_names: Optional[List[str]] = None) -> CmfProgram:
    """Compile an object exposing a sympy matrix as ``.M`` or ``.matrix``.

    Same contract as reference compiler.py:309-364: zero entries are skipped,
    axis names default to ``cmf.symbols`` or the sorted free symbols other
    than ``n``, and ``cmf.directions`` is used when present.
    """
    if hasattr(cmf, "M"):
        mat = cmf.M
    elif hasattr(cmf, "matrix"):
        mat = cmf.matrix
    else:
        raise ValueError("CMF object must have 'M' or 'matrix' attribute")
    m = mat.rows
    if axis_names is None:
        if hasattr(cmf, "symbols"):
            axis_names = [str(s) for s in cmf.symbols]
        else:
            axis_names = sorted(str(s) for s in mat.free_symbols if str(s) != "n")
    dim = len(axis_names)
    axis_symbols = {name: i for i, name in enumerate(axis_names)}
    directions = list(cmf.directions) if hasattr(cmf, "directions") else [1] * dim
    comp = CmfCompiler(m=m, dim=dim, directions=directions)
    for i in range(m):
        for j in range(m):
            entry = mat[i, j]
            if entry != 0:
                comp.compile_matrix_entry(i, j, entry, axis_symbols)
    return comp.build()


def compile_cmf_from_dict(matrix_dict: Dict[Tuple[int, int], str], m: int, dim: int,
                          axis_names: Optional[List[str]] = None,
                          directions: Optional[List[int]] = None) -> CmfProgram:
    """Compile ``{(row, col): "expr"}`` in dict order (reference compiler.py:367-404).

    Every listed entry is compiled, zeros included; ``n`` always parses as the
    step symbol.
    """
    import sympy as sp

    if axis_names is None:
        axis_names = [f"x{i}" for i in range(dim)]
    axis_symbols = {name: i for i, name in enumerate(axis_names)}
    local_ns = {name: sp.Symbol(name) for name in axis_names}
    local_ns["n"] = sp.Symbol("n")
    comp = CmfCompiler(m=m, dim=dim, directions=directions or [1] * dim)
    for (row, col), text in matrix_dict.items():
        comp.compile_matrix_entry(row, col, sp.sympify(text, locals=local_ns), axis_symbols)
    return comp.build()


def compile_pcf(a_str: str, b_str: str) -> Optional[CmfProgram]:
    """Companion bytecode of PCF(a, b) (reference runner.py:130-166): n is axis
    0 with direction 1, entries (0,1)=b, (1,0)=1, (1,1)=a; None for imaginary
    input.  Pure Python: it needs neither the native library nor a GPU."""
    import sympy as sp
    from sympy.abc import n

    a_expr = sp.sympify(a_str)
    b_expr = sp.sympify(b_str)
    if a_expr.has(sp.I) or b_expr.has(sp.I):
        return None
    s = sp.Symbol("_s")
    a_expr = a_expr.subs(n, s)
    b_expr = b_expr.subs(n, s)
    comp = CmfCompiler(m=2, dim=1, directions=[1])
    axes = {"_s": 0}
    comp.compile_matrix_entry(0, 1, b_expr, axes)
    comp.compile_matrix_entry(1, 0, sp.Integer(1), axes)
    comp.compile_matrix_entry(1, 1, a_expr, axes)
    return comp.build()
