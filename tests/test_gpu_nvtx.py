"""NVTX ranges of the step's phases: a small NVTX injection library (built
here with gcc against the NVTX v3 headers, loaded through the documented
NVTX_INJECTION64_PATH hook) records every range pushed by a process that
steps a workpiece; the ranges are balanced, the launches of the fused
schedule nest inside their step call, and each phase is named."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

INJECT = r"""
#include <stdio.h>
#include <stdlib.h>
#include <nvtx3/nvToolsExt.h>

static FILE* out;
static int push(const char* m) { if (out) { fprintf(out, "push %s\n", m); fflush(out); } return 0; }
static int pop(void) { if (out) { fprintf(out, "pop\n"); fflush(out); } return 0; }

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get) {
    const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable table = 0;
    unsigned int size = 0;
    if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size)) return 0;
    if (size <= NVTX_CBID_CORE_RangePop) return 0;
    *table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)push;
    *table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)pop;
    out = fopen(getenv("MPM_NVTX_LOG"), "w");
    return out != 0;
}
"""

RUN = r"""
import sys
sys.path.insert(0, sys.argv[1])
from mpm_b200 import Solver, capi as A, workpiece as W
case = W.config1(cells=(12, 8, 8), speed=20.0)
b = case["box"]
s = Solver(W.to_mpm_params(case, precision=A.PREC_F32), 12 * 8 * 8 * b["ppc"])
s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], 0, b["fixed_layers"], b["T0"], tool=case["tool"])
s.step(case["dt"], 3)
s.metrics()
s.download()
s.checkpoint()
s.close()
"""


def test_step_phases_are_named_ranges(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    cuda_inc = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"
    lib = tmp_path / "libinject.so"
    src = tmp_path / "inject.c"
    src.write_text(INJECT)
    r = subprocess.run(["gcc", "-shared", "-fPIC", "-O1", "-I", str(cuda_inc), str(src), "-o", str(lib)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    log = tmp_path / "ranges.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(lib), MPM_NVTX_LOG=str(log))
    run = subprocess.run([sys.executable, "-c", RUN, str(ROOT / "edegpredict-engine-rotary_b200")], env=env,
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr[-3000:]
    stack, seen, nested = [], set(), []
    for line in log.read_text().splitlines():
        if line.startswith("push "):
            name = line[5:]
            if name.startswith("mpm.launch."):
                nested.append("mpm.step" in stack)
            stack.append(name)
            seen.add(name)
        else:
            assert stack, "pop without push"
            stack.pop()
    assert not stack, stack
    for name in ("mpm.init_box", "mpm.step", "mpm.rebin", "mpm.launch.p2g", "mpm.launch.g2p_p2g",
                 "mpm.launch.g2p", "mpm.metrics", "mpm.download", "mpm.checkpoint_save"):
        assert name in seen, (name, sorted(seen))
    assert nested and all(nested)
