"""The C ABI library without a GPU: it loads, exports every entry point that
include/*.h declares, fills defaults, validates parameters and fails cleanly
(an error status, no crash) when no device is present."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT, has_gpu
from mpm_b200 import capi as A, workpiece as W


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(?:mpm_status|const char \*|void)\s*\*?\s*(mpm_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "mpm_step" in names and "mpm_create" in names and len(names) >= 20


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    lib = A.lib()
    assert hasattr(lib, name), name


def test_exports_are_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", str(A.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (mpm_\w+)", out))
    assert set(declared_functions()) <= exported


def test_params_default_are_reference_constants():
    p = A.default_params()
    assert p.abi_version == A.MPM_ABI_VERSION
    assert (p.apic_dinv_factor, p.apic_decay, p.deps_cap, p.dT_cap) == (3.0, 0.99, 0.05, 50.0)
    assert (p.gravity_z, p.mass_threshold, p.fixture_damping, p.chip_every) == (-9.81, 1e-12, 1e7, 2)
    assert (p.E, p.nu, p.jc_A, p.jc_B, p.jc_n, p.jc_C, p.jc_m) == (200e9, 0.3, 595e6, 580e6, 0.133, 0.023, 1.03)


def test_struct_sizes_match_header():
    """The ctypes mirrors must have the C layout (compiled probe)."""
    src = r'''
#include <stdio.h>
#include "mpm_capi.h"
#include <stddef.h>
int main(void){printf("%zu %zu %zu %zu %zu %zu\n", sizeof(mpm_params), sizeof(mpm_tool_desc), sizeof(mpm_particles_soa),
 sizeof(mpm_metrics), sizeof(mpm_tool_sdf), offsetof(mpm_tool_sdf, angle));return 0;}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "probe.c"
        c.write_text(src)
        exe = Path(d) / "probe"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), str(c), "-o", str(exe)], check=True)
        sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert sizes == [C.sizeof(A.MpmParams), C.sizeof(A.MpmToolDesc), C.sizeof(A.MpmParticlesSoa),
                     C.sizeof(A.MpmMetrics), C.sizeof(A.MpmToolSdf), A.MpmToolSdf.angle.offset]


def test_invalid_params_rejected_before_device_use():
    p = A.default_params()
    h = C.c_void_p()
    st = A.lib().mpm_create(C.byref(p), 10, None, C.byref(h))  # nx = 0
    assert st == A.MPM_INVALID_ARG and not h.value
    assert b"grid" in A.lib().mpm_last_error(None)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    case = W.config1(cells=(8, 8, 8))
    p = W.to_mpm_params(case)
    h = C.c_void_p()
    st = A.lib().mpm_create(C.byref(p), 100, None, C.byref(h))
    assert st in (A.MPM_CUDA_ERROR, A.MPM_OOM) and not h.value


def test_null_handle_is_refused():
    lib = A.lib()
    assert lib.mpm_step(None, 1e-9, 1) == A.MPM_INVALID_ARG
    assert lib.mpm_destroy(None) == A.MPM_OK
