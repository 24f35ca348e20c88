"""MPMWorkpieceSolver's semantics (the reference's other MPM solver,
src/MPMWorkpieceSolver.cu, which its engine never constructs): trilinear PIC,
hypoelastic stress with the Johnson-Cook return at the old plastic strain,
the nearest-tool-sample normal projection with contact heating, strain-rate
damage, its CHIP criteria and its chip separation.

- CPU: the oracle's restatement (orc_ws_step) against the reference kernels'
  own output on the workpiece_solver scenario (tests/golden/workpiece/
  workpiece_solver.npz, made by tests/golden/make_golden.py on a GPU):
  every field within 1e-9 of its scale (the reference sums with FP64
  atomics in arrival order; its run-to-run spread is stored and shown),
  statuses equal.
- GPU: the same against the reference kernels live; the CUDA path
  (mpm_set_workpiece_semantics) against the oracle: FP64 within 1e-9 of each
  field's scale, FP32 within the plain parity tolerances; the per-particle
  force through mpm_import_aos; the semantics switched off again returns to
  MPMSolver's step.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
from scenarios import WS_SCENARIOS  # noqa: E402

from mpm_b200 import Solver, capi as A, workpiece as W  # noqa: E402

FIX = HERE / "golden" / "workpiece" / "workpiece_solver.npz"
WS_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "stress", "backstress", "plastic_strain", "strain_rate", "temperature",
             "damage", "residual_stress")
FP32_TOL = dict(x=2e-4, y=2e-4, z=2e-4, vx=1e-3, vy=1e-3, vz=1e-3)


def ws_errors(out, ref, case):
    """max |out - ref| over each field's scale: dx for positions, the largest
    of |v| and the tool speed for velocities, the temperature rise for T, the
    field's peak otherwise."""
    dx = case["params"]["dx"]
    Tamb = case["params"]["Tamb"]
    vt = float(np.linalg.norm(case["tool"]["velocity"]))
    err = {}
    for k in WS_FIELDS:
        a = np.asarray(out[k], np.float64)
        b = np.asarray(ref[k], np.float64)
        if k in ("x", "y", "z"):
            sc = dx
        elif k in ("vx", "vy", "vz"):
            sc = max(np.abs(b).max(), vt)
        elif k == "temperature":
            a, b = a - Tamb, b - Tamb
            sc = max(np.abs(b).max(), 1e-6)
        else:
            sc = max(np.abs(b).max(), 1e-30)
        err[k] = float(np.abs(a - b).max() / sc)
    return err


def test_fixture_present():
    assert FIX.exists(), "run tests/golden/make_golden.py <dir> workpiece_solver on a GPU"


def test_oracle_matches_reference_kernels_fixture(oracle):
    d = np.load(FIX)
    meta = json.loads(bytes(d["meta"]).decode())
    case, st, n, extf = WS_SCENARIOS["workpiece_solver"]()
    for k in WS_FIELDS + ("status", "id"):
        assert np.array_equal(np.asarray(st[k]), d[f"in_{k}"]), k
    assert n == meta["nsteps"]
    out, force = oracle.ws_step(case, st, n, extf=extf.copy())
    ref = {k: d[f"out_{k}"] for k in WS_FIELDS + ("status",)}
    assert (out["status"] == ref["status"]).all()
    err = ws_errors(out, ref, case)
    print("\nreference spread:", meta["spread"], "\noracle vs reference:", err)
    assert max(err.values()) < 1e-9, err
    assert abs(force - d["contact_force"][0]) <= 1e-9 * abs(d["contact_force"][0])
    # the scenario reaches the branches
    assert (ref["status"] == A.CHIP).sum() > 100 and (ref["plastic_strain"] > 0).sum() > 100
    dmg = ref["damage"][ref["status"] == A.ACTIVE]
    assert ((dmg > 0.7) & (dmg < 1.0)).sum() > 10
    assert (np.abs(ref["backstress"]).max(axis=1) > 0).sum() > 100 and d["contact_force"][0] > 0


def _ours(case, st, n, extf, prec):
    s = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
    try:
        s.set_tool(case["tool"])
        s.upload(st)
        s.set_workpiece_semantics(case["ws"])
        if extf is not None:
            rec = s.export_aos().view(A.MPM_PARTICLE).copy()
            rec["ext_fx"], rec["ext_fy"], rec["ext_fz"] = extf[:, 0], extf[:, 1], extf[:, 2]
            s.import_aos(rec.view(np.uint8), A.AOS_EXT_FORCE)
        s.step(case["dt"], n)
        out = s.download()
        out["metrics"] = s.metrics()
    finally:
        s.close()
    return out


@pytest.mark.gpu
def test_reference_kernels_match_oracle_live(oracle):
    from oracle.oracle import RefKern

    case, st, n, extf = WS_SCENARIOS["workpiece_solver"]()
    ref, rforce = RefKern().ws_step(case, st, n, extf=extf.copy())
    out, force = oracle.ws_step(case, st, n, extf=extf.copy())
    assert (out["status"] == ref["status"]).all()
    err = ws_errors(out, ref, case)
    assert max(err.values()) < 1e-9, err
    assert abs(force - rforce) <= 1e-9 * abs(rforce)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [A.PREC_F64, A.PREC_F32])
def test_cuda_matches_oracle(prec, oracle):
    case, st, n, extf = WS_SCENARIOS["workpiece_solver"]()
    ref, force = oracle.ws_step(case, st, n, extf=extf.copy())
    out = _ours(case, st, n, extf, prec)
    err = ws_errors(out, ref, case)
    print(f"\nprec {prec}: {err}; contact force {out['metrics']['contact_force']:.6e} vs {force:.6e}")
    if prec == A.PREC_F64:
        assert (out["status"] == ref["status"]).all()
        assert max(err.values()) < 1e-9, err
        assert abs(out["metrics"]["contact_force"] - force) <= 1e-9 * abs(force)
    else:
        assert (out["status"] == ref["status"]).mean() >= 0.999
        # FP32 keeps the absolute temperature: each step rounds it to a float
        # spacing of T (3.05e-5 K at 293 K), which against this scenario's
        # 0.08 K rise is 4e-4 a step.  The temperature bound is therefore n
        # steps of that spacing, or 2e-3 of the rise when that is larger.
        Tmax = float(np.max(ref["temperature"]))
        rise = max(Tmax - case["params"]["Tamb"], 1e-30)
        tol = dict(FP32_TOL, temperature=max(2e-3, n * float(np.spacing(np.float32(Tmax))) / rise))
        bad = {k: v for k, v in err.items() if v > tol.get(k, 2e-3)}
        assert not bad, (bad, err, tol["temperature"])


@pytest.mark.gpu
def test_switching_back_runs_mpmsolver_semantics(oracle):
    """After mpm_set_workpiece_semantics(NULL) the handle steps with
    MPMSolver's semantics again (the oracle's orc_step from the same state)."""
    case, st, n, extf = WS_SCENARIOS["workpiece_solver"]()
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), len(st["x"]) + 64)
    try:
        s.set_tool(case["tool"])
        s.upload(st)
        s.set_workpiece_semantics(case["ws"])
        s.step(case["dt"], 4)
        mid = s.download()
        s.set_workpiece_semantics(None)
        s.step(case["dt"], 4)
        out = s.download()
    finally:
        s.close()
    mid["id"] = st["id"]
    ref, rc = oracle.step(case, mid, 4, step0=4, t0=4 * case["dt"])
    assert rc == 0
    assert (out["status"] == ref["status"]).all()
    from test_gpu_parity import field_errors
    err = field_errors(out, ref, case)
    assert max(err.values()) < 1e-9, err
