"""Build libdreams_b200.so (sm_100a) in-tree.

    python dreams-rns-cuda_b200/build.py [--force] [--jobs N] [--debug]

Each translation unit under csrc/ is compiled by nvcc in parallel into
_build/, then linked into dreams_rns/_native/libdreams_b200.so (the CUDA
runtime is linked statically, so the library only needs the driver).
--debug builds the same sources with -DDR_DEBUG (device bounds checks on
every table index a walk tile uses; see csrc/debug_check.cuh) into
_build_debug/ and dreams_rns/_native/libdreams_b200_debug.so, which the
package loads instead when DREAMS_B200_DEBUG=1.
csrc/pack.c (request packing, CPython API) is compiled by the C compiler
into dreams_rns/_pack.*.so.
Rebuilds a unit when it or any header in csrc/ or include/ is newer than its
object file.
"""

from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "dreams_rns", "_native")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libdreams_b200.so")
OBJ_DEBUG = os.path.join(HERE, "_build_debug")
LIB_DEBUG = os.path.join(OUT_DIR, "libdreams_b200_debug.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I", os.path.join(REPO, "include"), "-I", SRC]


def _headers():
    return (glob.glob(os.path.join(SRC, "*.h")) + glob.glob(os.path.join(SRC, "*.cuh")) +
            glob.glob(os.path.join(REPO, "include", "*.h")))


def _units():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))


def _compile(src: str, force: bool, verbose_ptxas: bool, obj_dir: str, defines) -> str:
    obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [NVCC] + ARCH + COMMON + list(defines)
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    cmd += ["-c", src, "-o", obj + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}")
    if verbose_ptxas:
        with open(obj + ".ptxas.txt", "w") as f:
            f.write(res.stderr)
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, jobs: int = 0, verbose_ptxas: bool = False, debug: bool = False) -> str:
    obj_dir, lib = (OBJ_DEBUG, LIB_DEBUG) if debug else (OBJ, LIB)
    defines = ["-DDR_DEBUG=1"] if debug else []
    os.makedirs(obj_dir, exist_ok=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    units = _units()
    jobs = jobs or min(len(units), os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose_ptxas, obj_dir, defines), units))
    stale = [o for o in glob.glob(os.path.join(obj_dir, "*.o")) if o not in objs]
    for o in stale:          # objects of removed sources must not be linked
        os.remove(o)
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-cudart", "static",
                               "-o", lib + ".tmp"] + objs + ["-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link failed")
        os.replace(lib + ".tmp", lib)
    build_pack(force)
    return lib


PACK_SRC = os.path.join(SRC, "pack.c")
PACK = os.path.join(HERE, "dreams_rns", "_pack" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def build_pack(force: bool = False) -> str:
    """The request-packing extension (plain C against the CPython API)."""
    newest = max(os.path.getmtime(PACK_SRC), os.path.getmtime(os.path.join(REPO, "include", "dreams_b200.h")))
    if not force and os.path.exists(PACK) and os.path.getmtime(PACK) >= newest:
        return PACK
    cc = os.environ.get("CC", "gcc")
    cmd = [cc, "-O2", "-shared", "-fPIC", "-Wall", "-I", sysconfig.get_paths()["include"],
           "-I", os.path.join(REPO, "include"), PACK_SRC, "-o", PACK + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("compiling pack.c failed")
    os.replace(PACK + ".tmp", PACK)
    return PACK


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--ptxas", action="store_true", help="keep -Xptxas -v reports next to objects")
    ap.add_argument("--debug", action="store_true", help="DR_DEBUG build (device bounds checks)")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.ptxas, a.debug))
