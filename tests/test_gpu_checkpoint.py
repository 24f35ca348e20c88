"""Checkpoint and resume of a workpiece (mpm_checkpoint_*): a checkpoint taken
mid-run and loaded into a fresh handle gives back exactly the saved state
(every field of the download equal, the step count and clock equal), and the
resumed run matches the uninterrupted one.

Tolerances of the resumed run (the reload re-bins, so the order of the
particles within a cell and of the atomic grid sums may differ):
  FP64: 1e-9 of each field's scale, status identical
  FP32: the batched form's tolerances (positions 2e-4 cell, velocities 1e-3,
        other fields 2e-3; status equal for >= 99.9 % of the particles)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from scenarios import SCENARIOS  # noqa: E402
from mpm_b200 import Batch, Solver, capi as A, workpiece as W  # noqa: E402
from test_gpu_batch import assert_same, cap_of, init_i, small_cases  # noqa: E402

pytestmark = pytest.mark.gpu

STATE = ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "stress", "backstress", "plastic_strain",
         "strain_rate", "temperature", "damage", "residual_stress", "status", "id")


def start(case, st, prec):
    s = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
    s.set_tool(case["tool"])
    if case["tool"].get("sdf") is not None:
        s.set_tool_sdf(case["tool"]["sdf"])
    s.upload(st)
    if "ext" in case:
        e = case["ext"]
        s.apply_external_force(e["center"], e["radius"], e["force"])
    return s


def same_state(a, b):
    for k in STATE:
        if k in a:
            assert np.array_equal(a[k], b[k], equal_nan=True), k


@pytest.mark.parametrize("prec,name", [(A.PREC_F64, "elastic_raster"), (A.PREC_F64, "plastic_damage_chip"),
                                       (A.PREC_F64, "lod_kinematic_extf"), (A.PREC_F64, "adiabatic_shear"),
                                       (A.PREC_F32, "plastic_damage_chip")])
def test_resume_matches_the_uninterrupted_run(prec, name):
    """Raster tool samples, damage and chips, backstress, LOD and the shear
    counter all travel in the checkpoint."""
    case, st, n, _ = SCENARIOS[name]()
    k1 = max(n // 2, 1)
    k2 = max(n - k1, 1)
    a = start(case, st, prec)
    try:
        a.step(case["dt"], k1)
        ck = a.checkpoint()
        saved = a.download()
        counts = a.counts()
        a.step(case["dt"], k2)
        ref = a.download()
        ref_counts = a.counts()
    finally:
        a.close()
    b = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
    try:
        b.restore(ck)
        if case["tool"].get("sdf") is not None:
            b.set_tool_sdf(case["tool"]["sdf"])
        assert b.counts() == counts
        same_state(b.download(), saved)
        assert b.status() == A.MPM_OK
        b.step(case["dt"], k2)
        out = b.download()
        assert b.counts() == ref_counts
    finally:
        b.close()
    assert_same(out, ref, case, prec)


def test_checkpoint_moves_between_batches():
    """Instance 1 of one batch is saved and loaded into instance 0 of another
    batch with the same grid; both then step on and agree with each other."""
    cases = small_cases(3, seed=9)
    prec = A.PREC_F64
    b1 = Batch([W.to_mpm_params(c, precision=prec) for c in cases], [cap_of(c) for c in cases])
    b2 = Batch([W.to_mpm_params(c, precision=prec) for c in (cases[1], cases[0])],
               [cap_of(cases[1]), cap_of(cases[0])])
    try:
        for i, c in enumerate(cases):
            init_i(b1, i, c)
        init_i(b2, 1, cases[0])
        b1.step_all([c["dt"] for c in cases], 5)
        ck = b1.checkpoint(1)
        b2.restore(ck, 0)
        assert b2.counts_i(0) == b1.counts_i(1)
        same_state(b2.download_i(0), b1.download_i(1))
        b1.step_all([c["dt"] for c in cases], 4)
        b2.step_all([cases[1]["dt"], cases[0]["dt"]], 4)
        assert_same(b2.download_i(0), b1.download_i(1), cases[1], prec)
        # a grid of another size is refused and leaves the instance as it was
        before = b2.download_i(1)
        with pytest.raises(A.MpmError) as e:
            b2.restore(ck, 1)
        assert e.value.status == A.MPM_INVALID_ARG and "grid" in str(e.value)
        same_state(b2.download_i(1), before)
    finally:
        b1.close()
        b2.close()


def test_corrupt_checkpoint_is_refused():
    case, st, n, _ = SCENARIOS["plastic_damage_chip"]()
    s = start(case, st, A.PREC_F64)
    try:
        s.step(case["dt"], 3)
        ck = s.checkpoint()
        before = s.download()
        bad = ck.copy()
        bad[len(bad) // 2] ^= 0x40
        with pytest.raises(A.MpmError) as e:
            s.restore(bad)
        assert e.value.status == A.MPM_INVALID_ARG and "checksum" in str(e.value)
        with pytest.raises(A.MpmError):
            s.restore(ck[:-8])
        same_state(s.download(), before)
        s.restore(ck)
        same_state(s.download(), before)
    finally:
        s.close()


@pytest.mark.parametrize("prec", [A.PREC_F32, A.PREC_F64])
def test_deterministic_resume_is_identical_bit_for_bit(prec):
    """In deterministic mode the reload re-bins in the saved slot order, so the
    resumed run gives the uninterrupted run's bits exactly."""
    case, st, n, _ = SCENARIOS["plastic_damage_chip"]()
    k1, k2 = n // 2, n - n // 2

    def fresh():
        s = start(case, st, prec)
        s.set_launch_config(deterministic=True)
        return s

    a = fresh()
    try:
        a.step(case["dt"], k1)
        ck = a.checkpoint()
        a.step(case["dt"], k2)
        ref = a.download()
    finally:
        a.close()
    b = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
    try:
        b.set_launch_config(deterministic=True)
        b.restore(ck)
        b.step(case["dt"], k2)
        out = b.download()
    finally:
        b.close()
    same_state(out, ref)
