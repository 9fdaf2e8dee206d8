"""NVTX ranges over the C-ABI calls (tracing), on CPU.

Every call of libdokigpu.so that launches device work or copies pushes an
NVTX range named after the function.  With no profiler attached NVTX does
nothing; with one, the ranges group the kernels by the call that launched
them.  This test attaches a small recording tool through NVTX's public
injection interface (NVTX_INJECTION64_PATH names a library exporting
InitializeInjectionNvtx2, which installs its own RangePushA / RangePop) and
checks the names recorded for calls that fail early without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
import textwrap

import pytest

from tests.conftest import ROOT

RECORDER = r"""
#include <stdio.h>
#include <stdlib.h>
#include <nvtx3/nvToolsExt.h>

static FILE *out;
static int depth;

static int push_a(const char *msg)
{
	if (out) {
		fprintf(out, "push %d %s\n", depth, msg);
		fflush(out);
	}
	return depth++;
}

static int pop(void)
{
	if (out) {
		fprintf(out, "pop %d\n", --depth);
		fflush(out);
	}
	return depth;
}

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get)
{
	const NvtxExportTableCallbacks *cb =
		(const NvtxExportTableCallbacks *)get(NVTX_ETID_CALLBACKS);
	NvtxFunctionTable table = 0;
	unsigned int size = 0;
	if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size) ||
	    size <= NVTX_CBID_CORE_RangePop)
		return 0;
	out = fopen(getenv("DK_NVTX_LOG"), "w");
	*table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)push_a;
	*table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)pop;
	return 1;
}
"""

CALLS = textwrap.dedent("""
    import ctypes, sys
    lib = ctypes.CDLL(sys.argv[1])
    out = ctypes.c_void_p()
    lib.dk_state_new.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.dk_marginals.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.dk_sync.argtypes = []
    rcs = [lib.dk_state_new(4, 2, ctypes.byref(out)), lib.dk_marginals(None, None)]
    assert all(rc != 0 for rc in rcs), rcs   # no GPU here, or invalid arguments
    lib.dk_sync()
""")


def _cuda_include():
    for d in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        if d and os.path.exists(os.path.join(d, "include", "nvtx3", "nvToolsExt.h")):
            return os.path.join(d, "include")
    return None


def test_c_abi_calls_push_named_ranges(tmp_path):
    inc = _cuda_include()
    if inc is None:
        pytest.skip("NVTX headers not found")
    src = tmp_path / "recorder.c"
    src.write_text(RECORDER)
    lib = tmp_path / "librecorder.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-O1", "-I", inc, str(src), "-o", str(lib)],
                   check=True, capture_output=True)
    log = tmp_path / "ranges.txt"
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(lib), DK_NVTX_LOG=str(log),
               CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", CALLS,
                        os.path.join(ROOT, "doki_b200", "libdokigpu.so")],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = log.read_text().split("\n")
    pushed = [ln.split()[2] for ln in lines if ln.startswith("push 0 ")]
    assert pushed[:1] == ["dk_state_new"] and "dk_marginals" in pushed and \
        pushed[-1] == "dk_sync", pushed
    # every range is closed, top level back at depth 0
    assert sum(ln.startswith("push") for ln in lines) == sum(ln.startswith("pop") for ln in lines)
    assert [ln for ln in lines if ln.startswith("pop")][-1] == "pop 0"
