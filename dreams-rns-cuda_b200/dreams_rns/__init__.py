"""dreams_rns on B200: the RNS walk engine of Dreams-RNS-CUDA, sm_100a-native.

Drop-in for the reference package's walk path (python/dreams_rns/__init__.py):
the bytecode compiler and program format are unchanged; walks, CRT and the
exact delta run in hand-written CUDA behind libdreams_b200.so.

    M(n) = [[0, b(n)], [1, a(n)]]          companion form
    P(N) = A * M(1) * M(2) * ... * M(N)    A = [[1, a(0)], [0, 1]]
    p = P[0, m-1],  q = P[1, m-1]          last column
    delta = -(1 + log|p/q - L| / log|q|)
"""

from .compiler import CmfCompiler, CmfProgram, Instruction, Opcode, compile_cmf, compile_cmf_from_dict
from .engine import (WalkBatch, WalkRequest, autotune, cmf_request, pcf_request, run_walks,
                     stage_times, sweep, sweep_many, vec_request)
from .gpu_walk import (gpu_available, run_cmf_walk_batch_gpu, run_cmf_walk_gpu,
                       run_pcf_walk_batch_gpu, run_pcf_walk_gpu)
from .runner import (WalkConfig, centered, compile_pcf, compute_dreams_delta_exact,
                     compute_dreams_delta_float, crt_batch, crt_overflowed, crt_reconstruct,
                     delta_batch, estimate_K, generate_rns_primes, pcf_initial_values,
                     run_pcf_walk, verify_pcf)
from .cmf_walk import compile_cmf_spec, run_cmf_walk, run_cmf_walk_vec
from . import cmf_sweep, constants, runner, synth

__version__ = "1.0.0"
__all__ = [
    "compile_cmf", "compile_cmf_from_dict", "CmfCompiler", "CmfProgram", "Opcode", "Instruction",
    "WalkConfig", "generate_rns_primes", "crt_reconstruct", "centered",
    "compute_dreams_delta_float", "compute_dreams_delta_exact", "compile_pcf",
    "pcf_initial_values", "run_pcf_walk", "verify_pcf",
    "gpu_available", "run_pcf_walk_gpu", "run_pcf_walk_batch_gpu", "run_cmf_walk_gpu",
    "run_cmf_walk_batch_gpu", "run_cmf_walk", "run_cmf_walk_vec", "vec_request", "compile_cmf_spec",
    "WalkBatch", "WalkRequest", "pcf_request", "cmf_request", "run_walks", "sweep", "sweep_many", "autotune", "crt_batch",
    "delta_batch", "estimate_K", "crt_overflowed", "stage_times",
]
