"""Deterministic mode (mpm_launch_config.deterministic): the same workpiece
gives the same state bit for bit on every run, at every launch shape, and
alone or inside a batch; and it still matches the oracle.

The mode runs the fused step kernel: each work item's node tile is stored
and k_node_sum adds the tiles of a node in a fixed order; particles whose
stencil left their bin's tile add to the grid in fixed point; the re-bin
puts each cell's particles in the order of their old slots.

Tolerances against the oracle (as tests/test_gpu_parity.py):
  FP64: 1e-9 of each field's scale, status identical
  FP32: positions 2e-4 cell, velocities 1e-3, other fields 2e-3; status equal
        for >= 99.9 % of the particles
Between deterministic runs: exact equality of every downloaded field.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from scenarios import PARITY_SCENARIOS, SCENARIOS  # noqa: E402
from mpm_b200 import Batch, Solver, capi as A, workpiece as W  # noqa: E402
from test_gpu_batch import assert_same, cap_of, init_i, small_cases  # noqa: E402
from test_gpu_parity import field_errors  # noqa: E402

pytestmark = pytest.mark.gpu

STATE = ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "stress", "plastic_strain", "strain_rate",
         "temperature", "damage", "residual_stress", "status", "id")


def run_det(case, st, n, prec, ctas=4, splits=None):
    s = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
    try:
        s.set_launch_config(ctas_per_sm=ctas, deterministic=True)
        assert s.launch_config()["deterministic"] == 1
        s.set_tool(case["tool"])
        s.upload(st)
        if "ext" in case:
            e = case["ext"]
            s.apply_external_force(e["center"], e["radius"], e["force"])
        for k in (splits or [n]):
            s.step(case["dt"], k)
        out = s.download()
        out["metrics"] = s.metrics()
    finally:
        s.close()
    return out


def identical(a, b):
    for k in STATE:
        assert np.array_equal(a[k], b[k], equal_nan=True), k


@pytest.mark.parametrize("name", ["plastic_damage_chip", "boundary_mix"])
def test_runs_are_identical_bit_for_bit(name):
    """FP32, where the atomic mode's sums differ from run to run: two
    runs, a third with another CTA count and a fourth split into two step
    calls give the same bits."""
    case, st, n, _ = SCENARIOS[name]()
    a = run_det(case, st, n, A.PREC_F32)
    b = run_det(case, st, n, A.PREC_F32)
    c = run_det(case, st, n, A.PREC_F32, ctas=2)
    d = run_det(case, st, n, A.PREC_F32, splits=[n // 2, n - n // 2])
    for o in (b, c, d):
        identical(a, o)


@pytest.mark.parametrize("name", ["elastic_raster", "plastic_damage_chip", "boundary_mix", "lod_kinematic_extf"])
def test_matches_the_oracle_fp64(oracle, name):
    case, st, n, extf = SCENARIOS[name]()
    ref, rc = oracle.step(case, st, n, extf=extf)
    assert rc == 0
    out = run_det(case, st, n, A.PREC_F64)
    assert (out["status"] == ref["status"]).all()
    err = field_errors(out, ref, case)
    assert max(err.values()) < 1e-9, err


def test_matches_the_oracle_fp32(oracle):
    case, st, n, extf = SCENARIOS["plastic_damage_chip"]()
    ref, rc = oracle.step(case, st, n, extf=extf)
    assert rc == 0
    assert_same(run_det(case, st, n, A.PREC_F32), ref, case, A.PREC_F32)


def test_batched_instance_is_identical_to_its_run_alone():
    """The sums of an instance's nodes run over its own particles in its own
    slot order, so a workpiece in a batch gives the bits it gives alone."""
    prec = A.PREC_F32
    cases = small_cases(3, seed=21, precision=prec)
    n = 8
    bt = Batch([W.to_mpm_params(c, precision=prec) for c in cases], [cap_of(c) for c in cases])
    try:
        bt.set_launch_config(deterministic=True)
        for i, c in enumerate(cases):
            init_i(bt, i, c)
        bt.step_all([c["dt"] for c in cases], n)
        outs = [bt.download_i(i) for i in range(3)]
    finally:
        bt.close()
    for i, c in enumerate(cases):
        s = Solver(W.to_mpm_params(c, precision=prec), cap_of(c))
        try:
            s.set_launch_config(deterministic=True)
            b = c["box"]
            s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], b["instance"], b["fixed_layers"], b["T0"],
                       tool=c["tool"])
            s.step(c["dt"], n)
            identical(outs[i], s.download())
        finally:
            s.close()


@pytest.mark.parametrize("name", ["adiabatic_shear", "heat_conduction"])
def test_extensions_run_deterministically(name):
    """The adiabatic shear model and grid heat conduction (the kernel variant
    with the T m channel in its stored tiles): FP32 runs are identical, and
    FP64 agrees with the atomic path within 1e-9."""
    from test_gpu_parity import run_ours
    case, st, n, _ = PARITY_SCENARIOS[name]()
    a = run_det(case, st, n, A.PREC_F32)
    b = run_det(case, st, n, A.PREC_F32, ctas=2)
    identical(a, b)
    det = run_det(case, st, n, A.PREC_F64)
    atomic = run_ours(case, st, n, prec=A.PREC_F64, atomic=True)
    assert (det["status"] == atomic["status"]).all()
    err = field_errors(det, atomic, case)
    assert max(err.values()) < 1e-9, err


def test_escaped_particles_sum_in_fixed_point():
    """A re-bin cadence longer than the scenario leaves particles whose
    stencil left their bin's tile; their fixed-point sums keep runs identical
    and agree with the atomic path (FP64 within 1e-9)."""
    from test_gpu_parity import run_ours
    case, st, n, _ = SCENARIOS["plastic_damage_chip"]()

    def run(prec, det, ctas=4):
        s = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
        try:
            s.set_launch_config(ctas_per_sm=ctas, sort_every=1024, deterministic=det)
            s.set_tool(case["tool"])
            s.upload(st)
            s.step(case["dt"], n)
            out = s.download()
            out["metrics"] = s.metrics()
        finally:
            s.close()
        return out

    a, b = run(A.PREC_F32, True), run(A.PREC_F32, True, ctas=3)
    assert a["metrics"]["n_escaped"] > 0
    identical(a, b)
    det, atomic = run(A.PREC_F64, True), run(A.PREC_F64, False)
    assert (det["status"] == atomic["status"]).all()
    err = field_errors(det, atomic, case)
    assert max(err.values()) < 1e-9, err


@pytest.mark.parametrize("name", ["plastic_damage_chip", "lod_kinematic_extf"])
def test_matches_the_atomic_path_fp64(name):
    """The deterministic sums against the default atomic path (fused
    schedule): FP64 within 1e-9, status identical."""
    from test_gpu_parity import run_ours
    case, st, n, _ = SCENARIOS[name]()
    atomic = run_ours(case, st, n, prec=A.PREC_F64, atomic=True)
    det = run_det(case, st, n, A.PREC_F64)
    assert (det["status"] == atomic["status"]).all()
    err = field_errors(det, atomic, case)
    assert max(err.values()) < 1e-9, err
