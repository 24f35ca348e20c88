"""Adiabatic shear band heating: AdiabaticShearModel::update
(src/AdiabaticShearModel.cu:262-279), i.e. applyAdiabaticHeatingKernel
(:104-177), run after g2p when asb_enabled is set (src/MPMSolver.cu:1130-1132).

- CPU: the oracle's single pass against tests/golden/kernels/asb_heating.npz,
  the reference kernels' own output on crafted particles that reach every
  branch (counters exact, temperatures to 1e-12 relative);
- CPU: the branch rules on hand-built particles with values worked out here;
- GPU: the reference kernels live against the oracle on the crafted
  particles, and the fused CUDA step with the model on against the oracle
  (counters read back through the AoS export).  The field parity of the
  adiabatic_shear scenario runs with the other scenarios in
  test_gpu_parity.py.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE / "golden"))
from mpm_b200 import capi as A  # noqa: E402
from make_golden import ASB_DT, asb_pass_inputs  # noqa: E402

FIXTURE = HERE / "golden" / "kernels" / "asb_heating.npz"


def test_fixture_present():
    assert FIXTURE.exists(), "run tests/golden/make_golden.py on a GPU (writes kernels/asb_heating.npz)"


def test_oracle_pass_matches_reference_fixture(oracle):
    d = np.load(FIXTURE)
    case, st = asb_pass_inputs()
    # the fixture was made from these inputs
    assert (st["status"] == d["in_status"]).all() and (st["asb"] == d["in_asb"]).all()
    assert np.array_equal(st["temperature"], d["in_temperature"])
    assert np.array_equal(st["strain_rate"], d["in_strain_rate"]) and np.array_equal(st["stress"], d["in_stress"])
    out = oracle.asb_heat(case, st, float(d["dt"]))
    assert (out["asb"] == d["out_asb"]).all()
    rise = d["out_temperature"] - d["in_temperature"]
    assert np.abs(rise).max() > 0, "the crafted pass heats some particles"
    err = np.abs(out["temperature"] - d["out_temperature"]) / np.maximum(np.abs(d["out_temperature"]), 1.0)
    assert err.max() < 1e-12, err.max()


def _one(status, T, edot, asb, sxx=1e9, dt=ASB_DT):
    case, _ = asb_pass_inputs()
    z = np.zeros(1)
    st = dict(x=z.copy(), y=z.copy(), z=z.copy(), vx=z.copy(), vy=z.copy(), vz=z.copy(),
              F=np.eye(3).reshape(1, 9), Fp=np.eye(3).reshape(1, 9), C=np.zeros((1, 9)),
              stress=np.array([[sxx, 0, 0, 0, 0, 0]], float), backstress=np.zeros((1, 6)), plastic_strain=z.copy(),
              strain_rate=np.array([edot]), temperature=np.array([T]), damage=z.copy(), residual_stress=z.copy(),
              status=np.array([status], np.int32), id=np.zeros(1, np.int32), asb=np.array([asb], np.int32))
    return case, st, dt


def _base_rise(case, sxx, edot, dt):
    p = case["params"]
    # uniaxial stress: von Mises = |sxx|
    return p["asb_taylor_quinney"] * abs(sxx) * edot * dt / (p["rho_phys"] * p["cp"])


@pytest.mark.parametrize("status,T,edot,asb,want_asb,heated", [
    (A.CHIP, 300.0, 2e4, 7, 0, False),        # CHIP: counter reset, nothing else
    (A.FIXED, 300.0, 2e4, 4, 4, False),       # not ACTIVE: untouched
    (A.BOUNDARY, 300.0, 2e4, 4, 4, False),
    (A.INACTIVE, 300.0, 2e4, 4, 4, False),
    (A.ACTIVE, 25.5, 2e4, 4, 4, False),       # at the 25.5 guard: untouched
    (A.ACTIVE, 30.0, 4999.0, 2, 1, False),    # below the 5000 /s floor: counter decays
    (A.ACTIVE, 30.0, 4999.0, 0, 0, False),
    (A.ACTIVE, 30.0, 5000.0, 0, 1, True),     # at the floor: heated, counter ramps
    (A.ACTIVE, 30.0, 2e4, 5, 6, True),        # localisation on, then capped at the base rise
    (A.ACTIVE, 30.0, 2e4, 10, 10, True),      # counter saturates at 10
])
def test_oracle_branches(oracle, status, T, edot, asb, want_asb, heated):
    case, st, dt = _one(status, T, edot, asb)
    out = oracle.asb_heat(case, st, dt)
    assert int(out["asb"][0]) == want_asb
    if heated:
        want = T + _base_rise(case, 1e9, edot, dt)
        assert abs(out["temperature"][0] - want) <= 1e-12 * want
    else:
        assert out["temperature"][0] == T


def test_oracle_caps():
    from oracle.oracle import Oracle
    o = Oracle()
    # per-step cap: 100 K
    case, st, _ = _one(A.ACTIVE, 30.0, 1e6, 0, sxx=2e9, dt=1e-3)
    assert _base_rise(case, 2e9, 1e6, 1e-3) > 100
    assert o.asb_heat(case, st, 1e-3)["temperature"][0] == pytest.approx(130.0, rel=1e-15)
    # temperature cap 0.9 Tm = 1494, which also lowers a particle already above it
    case, st, dt = _one(A.ACTIVE, 1493.99, 2e4, 0)
    assert o.asb_heat(case, st, dt)["temperature"][0] == pytest.approx(1494.0, rel=1e-15)
    case, st, dt = _one(A.ACTIVE, 1500.0, 2e4, 0)
    assert o.asb_heat(case, st, dt)["temperature"][0] == pytest.approx(1494.0, rel=1e-15)


@pytest.mark.gpu
def test_reference_pass_matches_oracle(oracle):
    from oracle.oracle import RefKern
    case, st = asb_pass_inputs()
    ref = RefKern().asb_heat(case, st, ASB_DT)
    out = oracle.asb_heat(case, st, ASB_DT)
    assert (out["asb"] == ref["asb"]).all()
    err = np.abs(out["temperature"] - ref["temperature"]) / np.maximum(np.abs(ref["temperature"]), 1.0)
    assert err.max() < 1e-12


# MPMParticle::asbCounter in the 504-byte AoS record
_ASB_OFFSET = 17 * 8 + 27 * 8 + 12 * 8 + 4 * 8 + 5 * 4


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [A.PREC_F64, A.PREC_F32])
def test_step_with_shear_model_matches_oracle(oracle, prec):
    from mpm_b200 import Solver, workpiece as W
    from scenarios import SCENARIOS
    case, st, n, _ = SCENARIOS["adiabatic_shear"]()
    ref, rc = oracle.step(case, st, n)
    assert rc == 0
    s = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
    try:
        s.set_tool(case["tool"])
        s.upload(st)
        s.step(case["dt"], n)
        out = s.download()
        m = s.metrics()
        aos = s.export_aos().reshape(-1, 504)
    finally:
        s.close()
    assert m["n_asb_heated"] > 0
    asb = aos[:, _ASB_OFFSET].astype(np.int32)
    same = (asb == ref["asb"]).mean()
    assert same >= (0.999 if prec == A.PREC_F64 else 0.99), same
    assert ref["asb"].max() >= 3, "the scenario reaches the localisation branch"
    # heating by the model, seen in the temperatures (FP64: the oracle's, to 1e-9 of the rise)
    Tamb = case["params"]["Tamb"]
    scale = max(np.abs(ref["temperature"] - Tamb).max(), 1e-6)
    err = np.abs((out["temperature"] - Tamb) - (ref["temperature"] - Tamb)).max() / scale
    assert err < (1e-9 if prec == A.PREC_F64 else 2e-3), err
