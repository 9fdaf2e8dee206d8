"""Build the engine in-tree.

Produces, next to this file:
  libdokigpu.so        -- the C-ABI library (include/dokigpu.h): CUDA kernels for
                          sm_100a + host runtime + planner
  doki<EXT_SUFFIX>     -- the CPython `doki` module, linked to libdokigpu.so

Usage: python -m doki_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I", INC, "-I", CSRC]

CU_SOURCES = ["dk_kernels.cu", "dk_runtime.cu", "dk_noalloc.cu", "dk_batch.cu"]
C_SOURCES = ["dk_plan.c"]
HEADERS = ["dk_internal.h", "dk_kernels.h", "dk_device.cuh"]

LIB = os.path.join(HERE, "libdokigpu.so")
# Debug build: the kernels check every index they compute
# (-DDK_DEBUG_CHECKS) and export dk_debug_checks; only dk_kernels.cu differs.
LIB_DBG = os.path.join(HERE, "libdokigpu_dbg.so")
DBG_SOURCE = "dk_kernels.cu"
EXT = os.path.join(HERE, "doki" + sysconfig.get_config_var("EXT_SUFFIX"))


def _cc() -> str:
    # The image exports CC pointing at a gcc without libgomp; the system gcc
    # is complete.
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")
    return r


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> None:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + \
        [os.path.join(INC, "dokigpu.h")]
    objs = []
    nvcc = _nvcc()
    dsrc = os.path.join(CSRC, DBG_SOURCE)
    dobj = os.path.join(OBJ, DBG_SOURCE + ".dbg.o")
    dproc = None
    if force or _stale(dobj, [dsrc] + hdrs):
        # compiled beside the release objects, in parallel with them
        dproc = subprocess.Popen([nvcc, *ARCH, *NVCC_FLAGS, "-DDK_DEBUG_CHECKS", "-c", dsrc,
                                  "-o", dobj], stdout=subprocess.PIPE,
                                 stderr=subprocess.PIPE, text=True)
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            r = _run(cmd)
            if verbose:
                sys.stderr.write(r.stderr)
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + hdrs):
            # -mpopcnt: the planner counts bits everywhere (one instruction
            # instead of a libgcc call on x86-64 hosts)
            _run([_cc(), "-O2", "-std=c11", "-fPIC", "-Wall", "-mpopcnt", "-I", INC, "-I", CSRC,
                  "-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs,
              "-Xlinker", "-rpath=/usr/local/cuda/lib64"])
    if dproc is not None:
        out, err = dproc.communicate()
        if dproc.returncode != 0:
            sys.stderr.write(out + err)
            raise RuntimeError(f"build step failed: debug {DBG_SOURCE} ({dproc.returncode})")
    dobjs = [dobj if o.endswith(DBG_SOURCE + ".o") else o for o in objs]
    if force or _stale(LIB_DBG, dobjs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB_DBG, *dobjs,
              "-Xlinker", "-rpath=/usr/local/cuda/lib64", "-Xlinker", "-Bsymbolic"])
    msrc = os.path.join(CSRC, "doki_module.c")
    if force or _stale(EXT, [msrc, LIB, os.path.join(INC, "dokigpu.h")]):
        pyinc = sysconfig.get_paths()["include"]
        _run([_cc(), "-O2", "-std=c11", "-shared", "-fPIC", "-Wall",
              "-Wno-unused-parameter", "-I", pyinc, "-I", INC, msrc, "-o", EXT,
              "-L", HERE, "-ldokigpu", "-Wl,-rpath,$ORIGIN"])


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", LIB, EXT)
