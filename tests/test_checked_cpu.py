"""The bounds-checked build (libmpm_b200_checked.so, -DMPMB_CHECKED) without a
GPU: it exports exactly the default library's entry points, and the default
library's mpm_check_report answers MPM_NOT_SUPPORTED (it has no checks)."""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess

import pytest

from conftest import ROOT
from mpm_b200 import capi as A

PKG = ROOT / "edegpredict-engine-rotary_b200" / "mpm_b200"


def exports(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    return sorted(l.split()[-1] for l in out.splitlines() if l.split()[-1].startswith("mpm_"))


@pytest.mark.skipif(shutil.which("nm") is None, reason="nm not available")
def test_checked_library_exports_the_same_entry_points():
    default, checked = PKG / "libmpm_b200.so", PKG / "libmpm_b200_checked.so"
    assert checked.exists(), "build with edegpredict-engine-rotary_b200/build.py --checked"
    assert exports(default) == exports(checked)
    assert "mpm_check_report" in exports(default)


def test_default_library_has_no_checks():
    v, s, i = C.c_int64(7), C.c_int32(7), C.c_int64(7)
    assert A.lib().mpm_check_report(C.byref(v), C.byref(s), C.byref(i), 0) == A.MPM_NOT_SUPPORTED
    assert (v.value, s.value, i.value) == (0, 0, 0)
