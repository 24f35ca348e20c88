"""The step kernel's pass size (mpm_launch_config.pass_size: 128, 256 or 512
FP32 particles staged per pass) and the persistent grid's clamp to the CTAs
that fit on an SM.

- Every pass size matches the FP64 oracle within the FP32 tolerances of the
  parity tests (positions 2e-4 cell, velocities 1e-3, other fields 2e-3;
  status equal for >= 99.9 % of the particles), and gives the same bits on a
  second run (deterministic node sums) and at another CTA count.
- 512-particle passes need more shared memory than four CTAs per SM can hold:
  the launch clamps the grid to the CTAs that fit, so asking for 8 CTAs per
  SM still gives the same bits.
- An unknown pass size is refused.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from scenarios import SCENARIOS  # noqa: E402
from mpm_b200 import Solver, capi as A, workpiece as W  # noqa: E402
from test_gpu_batch import assert_same  # noqa: E402

pytestmark = pytest.mark.gpu

STATE = ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "stress", "plastic_strain", "strain_rate",
         "temperature", "damage", "residual_stress", "status")


def run(case, st, n, pass_size, ctas=4):
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F32), len(st["x"]) + 64)
    try:
        s.set_launch_config(ctas_per_sm=ctas, pass_size=pass_size)
        assert s.launch_config()["pass_size"] == pass_size
        s.set_tool(case["tool"])
        s.upload(st)
        s.step(case["dt"], n)
        return s.download()
    finally:
        s.close()


@pytest.mark.parametrize("pass_size", [128, 256, 512])
def test_pass_size_matches_the_oracle_and_repeats(oracle, pass_size):
    case, st, n, extf = SCENARIOS["plastic_damage_chip"]()
    ref, rc = oracle.step(case, st, n, extf=extf)
    assert rc == 0
    a = run(case, st, n, pass_size)
    assert_same(a, ref, case, A.PREC_F32)
    for b in (run(case, st, n, pass_size), run(case, st, n, pass_size, ctas=8 if pass_size == 512 else 2)):
        for k in STATE:
            assert np.array_equal(a[k], b[k], equal_nan=True), (pass_size, k)


def test_unknown_pass_size_is_refused():
    case, st, n, _ = SCENARIOS["elastic_raster"]()
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F32), len(st["x"]) + 64)
    try:
        with pytest.raises(A.MpmError) as e:
            s.set_launch_config(pass_size=384)
        assert e.value.status == A.MPM_INVALID_ARG
    finally:
        s.close()
