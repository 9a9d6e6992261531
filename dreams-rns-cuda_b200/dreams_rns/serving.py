"""Continuous-batching walk server (C ABI dr_serve_*).

    srv = WalkServer()
    rid = srv.submit(pcf_request(program, a0, depth, K))
    ...
    res = srv.poll(rid)          # None until done, then the walk's result dict
    srv.close()

Requests that arrive while earlier ones are on the GPU join the next wave;
long walks are cut into segments that resume from device-resident state.
Admission is bounded by a device-memory cap (running products, shadow
state and outputs of the admitted walks).
"""

from __future__ import annotations

import ctypes
import time
from typing import Dict, Iterable, List, Optional

import numpy as np

from . import _native as N
from .engine import WalkRequest

__all__ = ["WalkServer"]


class WalkServer:
    def __init__(self, mem_cap_bytes: int = 0, max_inflight: int = 2, chunk_steps: int = 0,
                 max_wave_tiles: int = 0):
        N.init()
        cfg = N.ServeConfig()
        cfg.mem_cap_bytes = mem_cap_bytes
        cfg.max_inflight = max_inflight
        cfg.chunk_steps = chunk_steps
        cfg.max_wave_tiles = max_wave_tiles
        h = ctypes.c_int32()
        N.check(N.lib().dr_serve_open(ctypes.byref(cfg), ctypes.byref(h)), "dr_serve_open")
        self.handle = h.value
        self._K: Dict[int, int] = {}
        self._primes: Dict[int, np.ndarray] = {}

    def submit(self, req: WalkRequest) -> int:
        d = N.WalkDesc()
        d.program = 0
        d.K = req.K
        d.depth = max(int(req.depth), 0)
        d.checkpoint = 0
        d.a0 = int(req.a0)
        d.flags = (N.DR_WALK_INIT_PCF if req.pcf_init else 0) | (N.DR_WALK_SHADOW if req.shadow else 0)
        d.q_row = req.q_row
        axis = np.array([v for t in req.axis for v in t] or [0], dtype=np.int64)
        rid = ctypes.c_int64()
        N.check(N.lib().dr_serve_submit(self.handle, ctypes.byref(d), req.blob, len(req.blob),
                                        N.ptr(axis), ctypes.byref(rid)), "dr_serve_submit")
        self._K[rid.value] = req.K
        return rid.value

    def poll(self, rid: int) -> Optional[dict]:
        K = self._K[rid]
        p = np.zeros(K, dtype=np.uint32)
        q = np.zeros(K, dtype=np.uint32)
        sh = np.zeros(3, dtype=np.float64)
        st = ctypes.c_uint32()
        lat = ctypes.c_double()
        rc = N.lib().dr_serve_poll(self.handle, rid, N.ptr(p), N.ptr(q), N.ptr(sh), ctypes.byref(st),
                                   ctypes.byref(lat))
        if rc == N.DR_ERR_BUSY:
            return None
        if rc != N.DR_OK:
            self._K.pop(rid, None)     # the request ended with an error of its own
        N.check(rc, "dr_serve_poll")
        del self._K[rid]
        if K not in self._primes:
            self._primes[K] = N.prime_table(K).astype(np.int64)
        return {"p_residues": p.astype(np.int64), "q_residues": q.astype(np.int64),
                "p_float": float(sh[0]), "q_float": float(sh[1]), "log_scale": float(sh[2]),
                "primes": self._primes[K], "status": int(st.value), "latency_s": float(lat.value)}

    def wait(self, rids: Iterable[int], timeout: float = 60.0) -> Dict[int, dict]:
        """Poll until every request is done (or raise TimeoutError)."""
        left = list(rids)
        out: Dict[int, dict] = {}
        t0 = time.monotonic()
        while left:
            nxt = []
            for r in left:
                res = self.poll(r)
                if res is None:
                    nxt.append(r)
                else:
                    out[r] = res
            left = nxt
            if left:
                if time.monotonic() - t0 > timeout:
                    raise TimeoutError(f"{len(left)} requests still running")
                time.sleep(0.0002)
        return out

    def inject_failures(self, admissions: int = 0, waves: int = 0) -> int:
        """Test hook: the next ``admissions`` admissions and ``waves`` wave
        launches fail as if their device allocation had failed; the affected
        requests raise MemoryError from poll/wait and the server serves the
        rest.  Returns the number of requests that have failed so far."""
        failed = ctypes.c_uint64()
        N.check(N.lib().dr_debug_serve_inject(self.handle, N.DR_INJECT_ADMIT_NOMEM, int(admissions),
                                              ctypes.byref(failed)), "dr_debug_serve_inject")
        N.check(N.lib().dr_debug_serve_inject(self.handle, N.DR_INJECT_WAVE_NOMEM, int(waves),
                                              ctypes.byref(failed)), "dr_debug_serve_inject")
        return failed.value

    def cancel(self, rid: int) -> None:
        N.check(N.lib().dr_serve_cancel(self.handle, rid), "dr_serve_cancel")
        self._K.pop(rid, None)

    def stats(self) -> dict:
        c, ps, ab, qd = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        N.check(N.lib().dr_serve_stats(self.handle, ctypes.byref(c), ctypes.byref(ps), ctypes.byref(ab),
                                       ctypes.byref(qd)), "dr_serve_stats")
        return {"completed": c.value, "prime_steps": ps.value, "admitted_bytes": ab.value,
                "queue_depth": qd.value}

    def wave_log(self) -> np.ndarray:
        """Scheduler record of the wave launches, one row each: selection, launch-issued
        and harvest times (ms after open), device ms, requests, long-request wave, wave
        slot, walk tiles, longest shadow segment, then the times (ms after open) at which
        the wave's host build finished its geometry, allocation/upload and launches."""
        n = ctypes.c_int32()
        N.check(N.lib().dr_debug_serve_waves(self.handle, 0, ctypes.byref(n), None), "dr_debug_serve_waves")
        rows = np.zeros((max(n.value, 1), 12))
        N.check(N.lib().dr_debug_serve_waves(self.handle, n.value, ctypes.byref(n), rows.ctypes.data),
                "dr_debug_serve_waves")
        return rows[:n.value]

    def close(self) -> None:
        if self.handle:
            N.lib().dr_serve_close(self.handle)
            self.handle = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
