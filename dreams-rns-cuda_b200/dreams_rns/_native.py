"""ctypes binding of libdreams_b200.so (the sm_100a engine's C ABI).

The library is required: importing the walk API without it, or calling it
without a CUDA device, raises immediately -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# DREAMS_B200_DEBUG=1 selects the DR_DEBUG build (device bounds checks; built
# by `python dreams-rns-cuda_b200/build.py --debug`); DREAMS_B200_LIB names
# another build of the same library explicitly
LIB_PATH = os.environ.get("DREAMS_B200_LIB") or os.path.join(
    _HERE, "_native", "libdreams_b200_debug.so"
    if os.environ.get("DREAMS_B200_DEBUG", "") not in ("", "0") else "libdreams_b200.so")

DR_OK = 0
DR_ERR_CUDA = -1
DR_ERR_ARG = -2
DR_ERR_BLOB = -3
DR_ERR_OPCODE = -4
DR_ERR_INDEX = -5
DR_ERR_UNSUPPORTED = -6
DR_ERR_NOMEM = -7
DR_ERR_NOT_INIT = -8
DR_ERR_HANDLE = -9
DR_ERR_TIMEOUT = -10
DR_ERR_MODULUS = -11
DR_ERR_BUSY = -12

DR_WALK_INIT_PCF = 0x1
DR_WALK_SHADOW = 0x2
DR_WALK_VEC = 0x4

DR_STATUS_INV0 = 0x1
DR_STATUS_SHADOW_NAN = 0x2
DR_STATUS_FALLBACK = 0x4
DR_STATUS_CRT_OVERFLOW = 0x8
DR_STATUS_CP_CRT_OVERFLOW = 0x10

DR_ENGINE_AUTO = 0
DR_ENGINE_INTERP = 1
DR_ENGINE_PLAIN = 2

DR_INJECT_ADMIT_NOMEM = 1
DR_INJECT_WAVE_NOMEM = 2

DR_MAX_K = 8192


class WalkDesc(ctypes.Structure):
    """Mirror of ``dr_walk_desc`` in include/dreams_b200.h."""

    _fields_ = [
        ("program", ctypes.c_uint32),
        ("K", ctypes.c_uint32),
        ("depth", ctypes.c_uint64),
        ("checkpoint", ctypes.c_uint64),
        ("a0", ctypes.c_int64),
        ("flags", ctypes.c_uint32),
        ("q_row", ctypes.c_uint32),
        ("axis_offset", ctypes.c_uint64),
        ("res_offset", ctypes.c_uint64),
        ("cp_res_offset", ctypes.c_uint64),
        ("p_row", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("vec_offset", ctypes.c_uint64),
    ]


WALK_DTYPE = np.dtype([("program", "<u4"), ("K", "<u4"), ("depth", "<u8"), ("checkpoint", "<u8"),
                       ("a0", "<i8"), ("flags", "<u4"), ("q_row", "<u4"), ("axis_offset", "<u8"),
                       ("res_offset", "<u8"), ("cp_res_offset", "<u8"), ("p_row", "<u4"),
                       ("reserved", "<u4"), ("vec_offset", "<u8")], align=True)
assert WALK_DTYPE.itemsize == ctypes.sizeof(WalkDesc)


class Tune(ctypes.Structure):
    _fields_ = [("chunk_steps", ctypes.c_uint32), ("warps_per_block", ctypes.c_uint32),
                ("engine", ctypes.c_uint32), ("shadow_buffer_mb", ctypes.c_uint32),
                ("chain_pack_depth", ctypes.c_uint32)]


class Pipeline(ctypes.Structure):
    """Mirror of ``dr_pipeline``."""

    _fields_ = [("crt", ctypes.c_int32), ("delta_mode", ctypes.c_int32), ("topk", ctypes.c_int32),
                ("l_limbs", ctypes.c_int32), ("lnum", ctypes.c_void_p), ("lden", ctypes.c_void_p),
                ("lnum_sign", ctypes.c_int32), ("reserved", ctypes.c_int32)]


DR_DELTA_NONE = 0
DR_DELTA_FIXED = 1
DR_DELTA_SELF = 2


class ServeConfig(ctypes.Structure):
    _fields_ = [("mem_cap_bytes", ctypes.c_uint64), ("max_inflight", ctypes.c_uint32),
                ("chunk_steps", ctypes.c_uint32), ("max_wave_tiles", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32 * 3)]


class DreamsError(RuntimeError):
    """Error status returned by the native library."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I32 = ctypes.c_int32
_U64 = ctypes.c_uint64
_I64 = ctypes.c_int64

_SIGNATURES = {
    "dr_init": (ctypes.c_int, [ctypes.c_int]),
    "dr_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "dr_last_error": (ctypes.c_char_p, []),
    "dr_version": (ctypes.c_int, []),
    "dr_prime_table": (ctypes.c_int, [ctypes.c_int, _P]),
    "dr_stage_times": (ctypes.c_int, [_P, _P, _I32, _I32]),
    "dr_program_info": (ctypes.c_int, [ctypes.c_char_p, _U64, _P, _P, _P]),
    "dr_walk_batch": (ctypes.c_int, [_P, _I32, _P, _P, _I32, _P, _U64, _P, _P, _P, _U64, _P, _P]),
    "dr_batch_create": (ctypes.c_int, [_P, _I32, _P, _P, _I32, _P, _U64, _P, _P]),
    "dr_batch_run": (ctypes.c_int, [_I32, _P]),
    "dr_stream_create": (ctypes.c_int, [_P]),
    "dr_stream_destroy": (ctypes.c_int, [_P]),
    "dr_batch_read": (ctypes.c_int, [_I32, _P, _P, _U64, _P, _P]),
    "dr_batch_stats": (ctypes.c_int, [_I32, _P, _P, _P, _P]),
    "dr_batch_destroy": (ctypes.c_int, [_I32]),
    "dr_batch_set_pipeline": (ctypes.c_int, [_I32, _P]),
    "dr_batch_profile": (ctypes.c_int, [_I32, _I32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "dr_autotune": (ctypes.c_int, [_P, _I32, _P, _P, _I32, _P, _U64, _P, _P]),
    "dr_batch_set_bank": (ctypes.c_int, [_I32, _I32, _I32, _P, _P, _P]),
    "dr_batch_read_bank": (ctypes.c_int, [_I32, _P, _I32]),
    "dr_batch_read_pipeline": (ctypes.c_int, [_I32, _P, _P, _P, _P, _P, _I32]),
    "dr_crt_batch": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I32, _P, _P, _P]),
    "dr_crt_batch_device": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _I32, _P, _P, _P]),
    "dr_crt_batch_device_noalloc": (ctypes.c_int, [_P, _I32, _I32, _P, _I32, _P, _P]),
    "dr_delta_batch": (ctypes.c_int, [_P, _P, _P, _P, _I32, _I32, _P, _P, _P, _I32, _I32, _P]),
    "dr_topk": (ctypes.c_int, [_P, _I32, _I32, _P, _P]),
    "dr_topk_device": (ctypes.c_int, [_P, _I32, _I32, _P, _P, _P, _P]),
    "dr_serve_open": (ctypes.c_int, [_P, _P]),
    "dr_serve_submit": (ctypes.c_int, [_I32, _P, ctypes.c_char_p, _U64, _P, _P]),
    "dr_serve_poll": (ctypes.c_int, [_I32, _I64, _P, _P, _P, _P, _P]),
    "dr_serve_cancel": (ctypes.c_int, [_I32, _I64]),
    "dr_serve_stats": (ctypes.c_int, [_I32, _P, _P, _P, _P]),
    "dr_serve_close": (ctypes.c_int, [_I32]),
    "dr_bench_int_peak": (ctypes.c_int, [_I32, _P]),
    "dr_bench_chain_step": (ctypes.c_int, [_I32, _P]),
    "dr_debug_host_pool": (ctypes.c_int, [_I32, _U64, _I32, _P, _P]),
    "dr_debug_rescale": (ctypes.c_int, [_P, _P, _I32, _P]),
    "dr_debug_batch_timeline": (ctypes.c_int, [_I32, _I32, _P, _P]),
    "dr_debug_chain_items": (ctypes.c_int, [_I32, _I32, _P, _P]),
    "dr_debug_serve_waves": (ctypes.c_int, [_I32, _I32, _P, _P]),
    "dr_debug_serve_inject": (ctypes.c_int, [_I32, _I32, _I32, _P]),
    "dr_debug_build_phases": (ctypes.c_int, [_P, _I32]),
    "dr_debug_sim_walk": (ctypes.c_int, [ctypes.c_char_p, _U64, _I32, _U64, _U64, _P, _I32, _I64,
                                         _U32, _U64, _I32, _P, _P, _P, _P]),
}

_lib = None
_lock = threading.RLock()
_initialised = False


def lib():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(
                        f"libdreams_b200.so not found at {LIB_PATH}; build it with "
                        "`python dreams-rns-cuda_b200/build.py` (this engine has no CPU fallback)")
                L = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in _SIGNATURES.items():
                    if not hasattr(L, name):
                        continue
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status == DR_OK:
        return
    L = lib()
    msg = L.dr_last_error().decode(errors="replace") or L.dr_strerror(status).decode()
    text = f"{what}: {msg}" if what else msg
    if status in (DR_ERR_OPCODE, DR_ERR_BLOB):
        raise ValueError(text)
    if status == DR_ERR_INDEX:
        raise IndexError(text)
    if status == DR_ERR_NOMEM:
        raise MemoryError(text)
    raise DreamsError(status, text)


def init(device: int = 0) -> None:
    """Bind the engine to a CUDA device (idempotent)."""
    global _initialised
    if _initialised:
        return
    L = lib()
    with _lock:
        if not _initialised:
            check(L.dr_init(device), "dr_init")
            _initialised = True


def ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def prime_table(K: int) -> np.ndarray:
    out = np.zeros(max(K, 1), dtype=np.uint32)
    check(lib().dr_prime_table(K, ptr(out)), "dr_prime_table")
    return out[:K]


def program_info(blob: bytes):
    c, d, r = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(lib().dr_program_info(blob, len(blob), ctypes.byref(c), ctypes.byref(d), ctypes.byref(r)),
          "dr_program_info")
    return {"class": c.value, "degree": d.value, "n_regs": r.value}
