"""The C++ drop-in adapter (edegpredict-engine-rotary_b200/adapter/MPMSolverB200)
compiles against the reference's own headers (IPhysicsSolver.h, Types.h,
Config.h): every `override` matches the reference interface.  A small program
links it with libmpm_b200.so and runs the calls that need no GPU.  Skipped
unless MPM_REFERENCE_SRC names the reference source tree."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT
from mpm_b200 import capi as A

REF = Path(os.environ.get("MPM_REFERENCE_SRC", "") or "/nonexistent")
ADAPTER = ROOT / "edegpredict-engine-rotary_b200" / "adapter"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

pytestmark = pytest.mark.skipif(not (REF / "include" / "IPhysicsSolver.h").exists() or shutil.which("g++") is None,
                                reason="MPM_REFERENCE_SRC does not name the reference source tree, or g++ is missing")

MAIN = r"""
#include <cstdio>
#include "MPMSolverB200.h"
using namespace edgepredict;
int main() {
    MPMSolverB200 s(1000);
    IPhysicsSolver* base = &s;
    IMetricsProvider* metrics = &s;
    IThermalCoupling* thermal = &s;
    // nothing runs before initialize(), as in the reference
    s.initializeParticleBox(Vec3(0, 0, 0), Vec3(1e-3, 1e-3, 1e-3), 1e-4);
    base->step(1e-9);
    std::printf("%s %d %d %.1f %.1f %d\n", base->getName().c_str(), (int)base->isInitialized(),
                base->getParticleCount(), metrics->getMaxStress(), thermal->getTemperatureAt(0, 0, 0),
                (int)s.lastStatus());
    return 0;
}
"""


def _compile(tmp_path, src: Path, obj: Path):
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-c", str(src), "-o", str(obj), "-I", str(ADAPTER),
           "-I", str(REF / "include"), "-I", str(ROOT / "include"), "-I", str(CUDA / "include")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_adapter_compiles_against_reference_interface(tmp_path):
    _compile(tmp_path, ADAPTER / "MPMSolverB200.cpp", tmp_path / "adapter.o")


def test_adapter_links_and_runs_without_gpu(tmp_path):
    _compile(tmp_path, ADAPTER / "MPMSolverB200.cpp", tmp_path / "adapter.o")
    (tmp_path / "main.cpp").write_text(MAIN)
    _compile(tmp_path, tmp_path / "main.cpp", tmp_path / "main.o")
    lib = A.LIB_PATH
    exe = tmp_path / "adapter_main"
    cmd = ["g++", str(tmp_path / "main.o"), str(tmp_path / "adapter.o"), "-o", str(exe), "-L", str(lib.parent),
           f"-Wl,-rpath,{lib.parent}", "-lmpm_b200", "-L", str(CUDA / "lib64"), f"-Wl,-rpath,{CUDA / 'lib64'}",
           "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    name, inited, count, smax, temp, status = out.stdout.split()
    assert name == "MPMSolverB200" and inited == "0" and count == "0" and status == "0"
    assert float(smax) == 0.0 and float(temp) == 25.0
