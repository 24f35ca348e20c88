"""Build recipe of libmpm_b200.so (sm_100a) -- in-tree, no JIT cache.

    python edegpredict-engine-rotary_b200/build.py [--force] [--checked]
    MPM_REFERENCE_SRC=<reference tree> python edegpredict-engine-rotary_b200/build.py --adapter

Compiles every .cu under csrc/ with nvcc for sm_100a and links one shared
library next to the Python package (mpm_b200/libmpm_b200.so).  Objects go to
_build/ (git-ignored).  Incremental: a source newer than its object, or any
header newer than the library, triggers a rebuild.  --checked builds the
bounds-checked variant (-DMPMB_CHECKED, mpm_b200/libmpm_b200_checked.so,
objects in _build_checked/) instead.  --adapter builds the drop-in adapter
(adapter/MPMSolverB200.cpp) with its C driver (adapter/adapter_driver.cpp)
into adapter/_build/libmpm_adapter.so: it compiles against the reference's
own headers and links the reference's src/Config.cpp (initialize(Config)),
so it needs the reference source tree, as building the adapter inside the
reference does.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
BUILD = HERE / "_build"
LIB = HERE / "mpm_b200" / "libmpm_b200.so"
LIB_CHECKED = HERE / "mpm_b200" / "libmpm_b200_checked.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]
# Per-file flags.  The step kernel's FP32 divisions and square roots use the
# compiler's approximate forms and FP32 denormals flush to zero (the reference
# builds everything with --use_fast_math, which does both): 4 % and 2.5 % off
# the fused step on the 33.5M-particle workload, within the FP32 tolerances of
# the parity tests.  FP64 arithmetic is unaffected; every other file stays
# IEEE.
FILE_FLAGS = {"mpm_step.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newest(paths) -> float:
    return max((p.stat().st_mtime for p in paths), default=0.0)


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> Path:
    out_dir = HERE / "_build_checked" if checked else BUILD
    lib = LIB_CHECKED if checked else LIB
    extra = ["-DMPMB_CHECKED"] if checked else []
    out_dir.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    hdr_time = _newest(headers)
    objs = []
    for src in sources:
        obj = out_dir / (src.stem + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_time):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(src.name, []), *extra, "-I", str(INCLUDE), "-c",
                   str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or not lib.exists() or lib.stat().st_mtime < _newest(objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return lib


ADAPTER = HERE / "adapter"
ADAPTER_LIB = ADAPTER / "_build" / "libmpm_adapter.so"


def build_adapter(reference_src: str, force: bool = False, verbose: bool = False) -> Path:
    """adapter/_build/libmpm_adapter.so from the adapter, its C driver and the
    reference's src/Config.cpp, linked against libmpm_b200.so (rpath to it)."""
    ref = Path(reference_src)
    cfg = ref / "src" / "Config.cpp"
    if not cfg.exists():
        raise RuntimeError(f"{cfg} not found: pass the reference source tree")
    lib = build()
    out = ADAPTER_LIB
    out.parent.mkdir(exist_ok=True)
    srcs = [ADAPTER / "MPMSolverB200.cpp", ADAPTER / "adapter_driver.cpp", cfg]
    deps = srcs + [ADAPTER / "MPMSolverB200.h", INCLUDE / "mpm_capi.h", lib]
    if force or not out.exists() or out.stat().st_mtime < _newest(deps):
        cuda = Path(nvcc()).resolve().parent.parent
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", str(out), *map(str, srcs), "-I", str(ADAPTER),
               "-I", str(ref / "include"), "-I", str(INCLUDE), "-I", str(cuda / "include"), "-L", str(lib.parent),
               "-Wl,-rpath,$ORIGIN/../../mpm_b200", "-lmpm_b200", "-L", str(cuda / "lib64"),
               f"-Wl,-rpath,{cuda / 'lib64'}", "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    if "--adapter" in sys.argv:
        print(build_adapter(os.environ.get("MPM_REFERENCE_SRC", ""), force="--force" in sys.argv, verbose=True))
    else:
        print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
