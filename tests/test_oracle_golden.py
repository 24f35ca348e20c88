"""The oracle against the reference's own kernels: tests/golden/*.npz hold the
input state and the state the reference's CUDA kernels (src/MPMSolver.cu,
built from its sources, run by tests/golden/make_golden.py on a B200)
produced after n steps.  The reference accumulates with FP64 atomics, so the
tolerance (1e-9 of each field's scale) sits well above its own run-to-run
spread, which the fixture records."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from conftest import max_rel

GOLDEN = Path(__file__).resolve().parent / "golden"
FILES = sorted(GOLDEN.glob("*.npz"))
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "stress", "backstress", "plastic_strain",
          "strain_rate", "temperature", "damage", "residual_stress")


def load(path):
    d = np.load(path)
    meta = json.loads(bytes(d["meta"]).decode())
    case = dict(meta["case"])
    case["tool"] = meta["tool"]
    if "samples" in case["tool"]:
        case["tool"]["samples"] = np.asarray(case["tool"]["samples"])
    case["params"]["origin"] = tuple(case["params"]["origin"])
    st = {k: d[f"in_{k}"] for k in FIELDS + ("status", "id")}
    ref = {k: d[f"out_{k}"] for k in FIELDS + ("status", "id")}
    if "in_asb" in d:   # adiabatic shear counters (MPMParticle::asbCounter)
        st["asb"], ref["asb"] = d["in_asb"], d["out_asb"]
    extf = d["extf"] if "extf" in d else None
    return case, st, ref, meta, extf, d["ref_stats"]


def test_fixtures_present():
    assert len(FILES) >= 4, "tests/golden/*.npz missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", FILES, ids=[f.stem for f in FILES])
def test_oracle_reproduces_reference(path, oracle):
    case, st, ref, meta, extf, _ = load(path)
    out, rc = oracle.step(case, st, meta["nsteps"], extf=extf)
    assert rc == 0
    assert (out["status"] == ref["status"]).all()
    if "asb" in ref:
        assert (out["asb"] == ref["asb"]).all()
    dx = case["params"]["dx"]
    for k in FIELDS:
        scale = dx if k in ("x", "y", "z") else max(np.abs(ref[k]).max(), 1e-30)
        if k == "temperature":
            T0 = case["params"]["Tamb"]
            e = max_rel(out[k] - T0, ref[k] - T0, max(np.abs(ref[k] - T0).max(), 1e-6))
        elif k in ("F", "Fp"):
            eye = np.tile(np.eye(3).reshape(1, 9), (len(ref[k]), 1))
            e = max_rel(out[k] - eye, ref[k] - eye, max(np.abs(ref[k] - eye).max(), 1e-12))
        else:
            e = max_rel(out[k], ref[k], scale)
        assert e < 1e-9, (k, e, meta["spread"].get(k))


@pytest.mark.parametrize("path", FILES, ids=[f.stem for f in FILES])
def test_oracle_metrics_match_reference_stats(path, oracle):
    """computeParticleStatsKernel's four numbers on the reference's output."""
    case, st, ref, meta, extf, ref_stats = load(path)
    m = oracle.metrics(case, ref)
    mine = [m["ref_max_stress"], m["ref_max_T"], m["ref_kinetic"], m["ref_internal"]]
    for a, b in zip(mine, ref_stats):
        assert abs(a - b) <= 1e-12 * max(abs(b), 1e-30) + 1e-300, (mine, list(ref_stats))


def test_fixture_spread_is_small():
    """The reference's own run-to-run spread (FP64 atomic order), relative to
    each field's scale, is far below the parity tolerance."""
    for path in FILES:
        _, _, ref, meta, _, _ = load(path)
        for k, v in meta["spread"].items():
            if k in ("status", "id", "asb"):
                assert v == 0, (path.stem, k)
                continue
            scale = max(float(np.abs(ref[k]).max()), 1e-30)
            assert v / scale < 1e-11, (path.stem, k, v, scale)
