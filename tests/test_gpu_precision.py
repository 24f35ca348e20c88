"""Precision: the FP32 state (with FP64 Johnson-Cook Newton solve and FP64
conservation reductions) against an FP64 run of the same kernels from the
same seeded state, through chip formation.

Target: relative error <= 1e-4 on total momentum (its norm) and on kinetic +
internal energy after 1000 steps; peak von Mises stress within 1e-3; the same
chip count within 0.1 % of the particles.
"""
from __future__ import annotations

import numpy as np
import pytest

from mpm_b200 import Solver, capi as A, workpiece as W

pytestmark = pytest.mark.gpu


def run(case, prec, n):
    b = case["box"]
    s = Solver(W.to_mpm_params(case, precision=prec), int(np.prod(np.subtract(b["c1"], b["c0"]))) * b["ppc"])
    try:
        s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], 0, b["fixed_layers"], b["T0"], tool=case["tool"])
        s.step(case["dt"], n)
        return s.metrics()
    finally:
        s.close()


@pytest.mark.parametrize("plasticity", [A.PLAST_EXPLICIT, A.PLAST_NEWTON])
def test_fp32_within_1e4_of_fp64_through_chip_formation(plasticity):
    case = W.config4(cells=(64, 32, 32))
    case["params"]["plasticity"] = plasticity
    m32 = run(case, A.PREC_F32, 1000)
    m64 = run(case, A.PREC_F64, 1000)
    assert m64["n_chip"] > 0   # the run goes through chip separation
    p32, p64 = np.array(m32["momentum"]), np.array(m64["momentum"])
    assert np.linalg.norm(p32 - p64) / np.linalg.norm(p64) <= 1e-4
    e32 = m32["kinetic"] + m32["internal_elastic"]
    e64 = m64["kinetic"] + m64["internal_elastic"]
    assert abs(e32 - e64) / e64 <= 1e-4
    assert abs(m32["max_von_mises"] - m64["max_von_mises"]) / m64["max_von_mises"] <= 1e-3
    n = m64["n_active"] + m64["n_chip"] + m64["n_fixed"]
    assert abs(m32["n_chip"] - m64["n_chip"]) <= max(1, n // 1000)
    assert abs(m32["mass"] - m64["mass"]) / m64["mass"] <= 1e-6


def run_state(case, prec, n, det):
    b = case["box"]
    s = Solver(W.to_mpm_params(case, precision=prec), int(np.prod(np.subtract(b["c1"], b["c0"]))) * b["ppc"])
    try:
        s.set_launch_config(deterministic=det)
        s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], 0, b["fixed_layers"], b["T0"], tool=case["tool"])
        s.step(case["dt"], n)
        return s.metrics(), s.download(("x", "vx", "plastic_strain", "status"))
    finally:
        s.close()


def test_config4_full_size_deterministic_fp32_within_1e4():
    """The full config-4 workload (128x64x64 cells, 4.17M particles, 1000
    steps through chip formation).  Default-mode FP32 runs differ from run to
    run (float atomics), and under the tool edge a fracture event can branch
    on a 1e-7 difference; the deterministic mode gives one FP32 result for
    this build and input, so this check holds on every run: momentum and
    kinetic + internal energy within 1e-4 of FP64, and a second FP32 run equal
    bit for bit."""
    case = W.config4()
    m64, _ = run_state(case, A.PREC_F64, 1000, True)
    m32, s32 = run_state(case, A.PREC_F32, 1000, True)
    assert m64["n_chip"] > 0
    p32, p64 = np.array(m32["momentum"]), np.array(m64["momentum"])
    assert np.linalg.norm(p32 - p64) / np.linalg.norm(p64) <= 1e-4
    e32 = m32["kinetic"] + m32["internal_elastic"]
    e64 = m64["kinetic"] + m64["internal_elastic"]
    assert abs(e32 - e64) / e64 <= 1e-4
    _, s32b = run_state(case, A.PREC_F32, 1000, True)
    for k in s32:
        assert np.array_equal(s32[k], s32b[k]), k
