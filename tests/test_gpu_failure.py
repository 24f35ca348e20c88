"""Failure detection without a GPU fault: the bounded device-side wait that
guards the step kernel's tile loads gives up when nothing completes it, the
host reads MPM_TIMEOUT, and the context stays usable (a step right after
matches the oracle).  The wait is limited to 50 ms; no copy is in flight."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

from mpm_b200 import Solver, capi as A, workpiece as W


def test_selftest_argument_checks_need_no_gpu():
    L = A.lib()
    assert L.mpm_selftest_bounded_wait(0, None) == A.MPM_INVALID_ARG
    assert L.mpm_selftest_bounded_wait(2_000_000_000, None) == A.MPM_INVALID_ARG


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_context_survives(oracle):
    L = A.lib()
    t0 = time.perf_counter()
    st = L.mpm_selftest_bounded_wait(50_000_000, None)
    el = time.perf_counter() - t0
    assert st == A.MPM_TIMEOUT, L.mpm_last_error(None)
    assert b"gave up" in L.mpm_last_error(None)
    assert el < 5.0
    # the context is usable: a small run right after matches the oracle
    case = W.config1(cells=(12, 8, 8), speed=20.0)
    st0 = W.full_state(W.generate_box(case), case)
    ref, rc = oracle.step(case, st0, 4)
    assert rc == 0
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), len(st0["x"]))
    try:
        s.set_tool(case["tool"])
        s.upload(st0)
        s.step(case["dt"], 4)
        out = s.download()
    finally:
        s.close()
    assert np.abs(out["x"] - ref["x"]).max() <= 1e-9 * case["params"]["dx"]
    assert (out["status"] == ref["status"]).all()
