"""Grid heat conduction, as the reference's MPMWorkpieceSolver does it (T m
scattered with the mass, src/MPMWorkpieceSolver.cu:118; one explicit
diffusion step on the grid, mpmDiffuseTemperatureKernel :208-262; the
temperature gather of mpmG2PKernel :282-306), run on this solver's quadratic
weights when heat_conduction is set.

- CPU: the oracle's diffusion step against tests/golden/kernels/heat_diffusion.npz,
  the reference kernel's own output on a crafted grid (1e-13 relative);
- CPU: properties of the oracle's step with conduction (a workpiece at
  ambient stays there; hot spots spread and their peak falls);
- GPU: the reference kernel live against the oracle on the crafted grid.
  The fused CUDA step with conduction on runs against the oracle in
  test_gpu_parity.py (scenario heat_conduction).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE / "golden"))
from make_golden import HEAT_DT, heat_pass_inputs  # noqa: E402

FIXTURE = HERE / "golden" / "kernels" / "heat_diffusion.npz"


def _check(mass, tm_in, tm_out, tn):
    upd = mass >= 1e-15
    # nodes the kernel updates: its temperatureMass / mass against the oracle's T
    ref_T = tm_out[upd] / mass[upd]
    assert np.abs(tn[upd] - ref_T).max() <= 1e-13 * np.abs(ref_T).max()
    # lighter nodes are left as they were
    assert np.array_equal(tm_out[~upd], tm_in[~upd])
    light = (~upd) & (mass > 0)
    assert np.allclose(tn[light], tm_in[light] / mass[light], rtol=1e-15, atol=0)


def test_fixture_present():
    assert FIXTURE.exists(), "run tests/golden/make_golden.py on a GPU (writes kernels/heat_diffusion.npz)"


def test_oracle_diffusion_matches_reference_fixture(oracle):
    d = np.load(FIXTURE)
    case, mass, tm = heat_pass_inputs()
    assert np.array_equal(mass, d["mass"]) and np.array_equal(tm, d["tm_in"])
    tn = oracle.heat_diffuse(case, mass, tm, float(d["dt"]))
    # the step moved the temperatures: the comparison is not trivial
    upd = mass >= 1e-15
    assert np.abs(d["tm_out"][upd] - d["tm_in"][upd]).max() > 0
    _check(d["mass"], d["tm_in"], d["tm_out"], tn)


def test_uniform_ambient_stays():
    """Every node at ambient: the empty-node neighbours pull the surface nodes
    below ambient, and the gather's clamp at Tamb brings the particles back, so
    an elastic workpiece at ambient keeps its temperature."""
    from oracle.oracle import Oracle
    from scenarios import elastic_raster
    case, st, n, _ = elastic_raster()
    case["params"].update(heat_conduction=1, thermal_conductivity=42.6)
    out, rc = Oracle().step(case, st, 5)
    assert rc == 0
    live = out["status"] != 1
    # up to the rounding of (T m)/m and of the weighted mean
    dev = out["temperature"][live] - case["params"]["Tamb"]
    assert dev.min() >= 0.0 and dev.max() < 1e-9


def test_hot_spots_spread(oracle):
    from scenarios import heat_conduction
    case, st, n, _ = heat_conduction()
    case["params"]["jc_A"] = 1e12        # elastic: no plastic heating in this check
    out, rc = oracle.step(case, st, 4)
    assert rc == 0
    Tamb = case["params"]["Tamb"]
    live = out["status"] != 1
    hot0 = st["temperature"] > Tamb
    # the peak falls and heat reaches particles that started at ambient
    assert out["temperature"][live].max() < st["temperature"].max()
    assert (out["temperature"][live & ~hot0] > Tamb).any()
    # the same run without conduction leaves the particles that started at ambient there
    case0, st0, _, _ = heat_conduction()
    case0["params"].update(jc_A=1e12, heat_conduction=0)
    out0, _ = oracle.step(case0, st0, 4)
    assert (out0["temperature"][(out0["status"] != 1) & ~hot0] == Tamb).all()


@pytest.mark.gpu
def test_reference_diffusion_matches_oracle(oracle):
    from oracle.oracle import RefKern
    case, mass, tm = heat_pass_inputs()
    out = RefKern().heat_diffuse(case, mass, tm, HEAT_DT)
    tn = oracle.heat_diffuse(case, mass, tm, HEAT_DT)
    _check(mass, tm, out, tn)
