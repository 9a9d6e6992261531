"""The bytecode compiler emits exactly the reference's programs (golden blobs)."""

import pytest

from dreams_rns import compile_cmf_from_dict, compile_pcf
from dreams_rns.cmf_walk import compile_cmf_spec
from dreams_rns.compiler import CmfProgram, Instruction, Opcode


def test_pcf_programs_match_reference(golden):
    n = 0
    for case in golden["compiler"]:
        if case["kind"] != "pcf":
            continue
        prog = compile_pcf(case["a"], case["b"])
        if case["blob"] is None:
            assert prog is None, case
        else:
            assert prog.serialize().hex() == case["blob"], (case["a"], case["b"])
        n += 1
    assert n >= 20


def test_dict_and_spec_programs_match_reference(golden):
    for case in golden["compiler"]:
        if case["kind"] == "dict":
            mat = {(r, c): e for r, c, e in case["matrix"]}
            prog = compile_cmf_from_dict(mat, m=case["m"], dim=case["dim"],
                                         axis_names=case["axis_names"],
                                         directions=case["directions"])
            assert prog.serialize().hex() == case["blob"]
        elif case["kind"] == "spec":
            prog = compile_cmf_spec(case["spec"], case["trajectory"])
            assert prog.serialize().hex() == case["blob"]


def test_compiler_errors_match_reference(golden):
    for case in golden["compiler_errors"]:
        if case["error"] is None:
            compile_pcf(case["a"], case["b"])
        else:
            with pytest.raises(Exception) as ei:
                compile_pcf(case["a"], case["b"])
            assert type(ei.value).__name__ == case["error"]


def test_serialize_roundtrip(golden):
    for case in golden["compiler"]:
        if case["blob"] in (None, "?"):
            continue
        blob = bytes.fromhex(case["blob"])
        assert CmfProgram.deserialize(blob).serialize() == blob


def test_out_of_registers():
    from dreams_rns.compiler import CmfCompiler
    c = CmfCompiler(m=2, dim=1)
    with pytest.raises(RuntimeError, match="Out of registers"):
        for _ in range(600):
            c.load_n()


def test_unknown_opcode_rejected_by_deserialize():
    prog = CmfProgram(m=2, dim=1, opcodes=[Instruction(Opcode.END)], constants=[], directions=[1])
    blob = bytearray(prog.serialize())
    blob[16] = 99
    with pytest.raises(ValueError):
        CmfProgram.deserialize(bytes(blob))
