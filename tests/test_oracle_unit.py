"""Properties of the FP64 oracle restatement (src/MPMSolver.cu semantics) that
hold independent of the reference run: B-spline partition of unity, exact
mass conservation, momentum conservation without tool and gravity, elastic
response, the Johnson-Cook return and its Newton form, and the generator."""
from __future__ import annotations

import math

import numpy as np
import pytest

from mpm_b200 import capi as A, workpiece as W


def weights(xi):
    """getWeightsAndGradients (src/MPMSolver.cu:20-34) in cell units."""
    b = math.floor(xi - 0.5)
    d0 = xi - b
    w = [0.5 * (1.5 - d0) ** 2, 0.75 - (d0 - 1) ** 2, 0.5 * (d0 - 0.5) ** 2]
    dw = [-(1.5 - d0), -2 * (d0 - 1), d0 - 0.5]
    return b, w, dw


@pytest.mark.parametrize("xi", np.random.default_rng(0).uniform(1, 50, 64))
def test_bspline_partition_of_unity(xi):
    b, w, dw = weights(xi)
    assert abs(sum(w) - 1.0) < 1e-14
    assert abs(sum(wi * (b + i - xi) for i, wi in enumerate(w))) < 1e-14  # first moment
    assert abs(sum(dw)) < 1e-14
    assert abs(sum(dwi * (b + i - xi) for i, dwi in enumerate(dw)) - 1.0) < 1e-14


def quiet_case(**over):
    """No tool, gravity, fixture or chip separation."""
    case = W.config1(cells=(8, 8, 8), tool_mode=A.TOOL_NONE)
    case["params"].update(gravity_z=0.0, fixture_thickness=0.0, chip_every=0)
    case["params"].update(over)
    return case


def test_mass_exact_and_momentum_conserved(oracle):
    """With the empty-node mass threshold at 0 linear momentum is conserved to
    round-off.  (The reference's 1e-12 kg threshold drops the momentum of
    nearly empty edge nodes: a drift of ~1e-5 per 20 steps at this size.)"""
    case = quiet_case(mass_threshold=0.0)
    st = W.full_state(W.generate_box(case), case)
    st["status"][:] = A.ACTIVE
    rng = np.random.default_rng(1)
    n = len(st["x"])
    st["vx"] = rng.normal(0, 1e-2, n)
    st["vy"] = rng.normal(0, 1e-2, n)
    st["vz"] = rng.normal(0, 1e-2, n)
    m0 = oracle.metrics(case, st)
    out, rc = oracle.step(case, st, 20)
    m1 = oracle.metrics(case, out)
    assert rc == 0
    assert m1["mass"] == m0["mass"]
    pscale = m0["mass"] * 1e-2
    for k in ("px", "py", "pz"):
        assert abs(m1[k] - m0[k]) < 1e-12 * pscale


def test_uniform_translation_is_preserved(oracle):
    """A uniformly moving block: particles whose stencils are beyond the reach
    of the free-surface disturbance (two steps, the centre cells) keep v."""
    case = quiet_case()
    st = W.full_state(W.generate_box(case), case)
    st["status"][:] = A.ACTIVE
    st["vx"][:] = 0.5
    out, rc = oracle.step(case, st, 2)
    dx = case["params"]["dx"]
    c = [out[k] / dx for k in ("x", "y", "z")]
    inner = np.logical_and.reduce([(ci > 3) & (ci < 5) for ci in c])
    assert inner.sum() > 20
    assert np.allclose(out["vx"][inner], 0.5, rtol=1e-12, atol=1e-12)
    assert np.abs(out["vz"][inner]).max() < 1e-12


def test_uniaxial_elastic_stress(oracle):
    """F = diag(1+e, 1, 1) with F_p = I: sigma = mu/J (B - I) + lambda (J - 1) I."""
    case = quiet_case(jc_A=1e12)
    st = W.full_state(W.generate_box(case), case)
    st["status"][:] = A.ACTIVE
    e = 1e-4
    st["F"][:, 0] = 1.0 + e
    out, _ = oracle.step(case, st, 1, dt=1e-30)
    p = case["params"]
    mu = p["E"] / (2 * (1 + p["nu"]))
    lam = p["E"] * p["nu"] / ((1 + p["nu"]) * (1 - 2 * p["nu"]))
    J = 1 + e
    sxx = mu / J * ((1 + e) ** 2 - 1) + lam * (J - 1)
    syy = lam * (J - 1)
    assert np.allclose(out["stress"][:, 0], sxx, rtol=1e-9)
    assert np.allclose(out["stress"][:, 1], syy, rtol=1e-9)


def jc_flow(p, eps, edot, dT):
    Ts = min(max(dT / max(p["Tm"] - p["Tamb"], 1.0), 0.0), 1.0)
    es = max(edot / max(p["edot0"], 1e-12), 1e-5)
    return (p["jc_A"] + p["jc_B"] * eps ** p["jc_n"]) * (1 + p["jc_C"] * math.log(es)) * (1 - Ts ** p["jc_m"])


@pytest.mark.parametrize("mode", [A.PLAST_EXPLICIT, A.PLAST_NEWTON])
def test_radial_return_on_yield_surface(oracle, mode):
    """A shear state above yield: after the step the deviatoric stress lies on
    the JC surface (Newton: at the updated strain; explicit: at the old one)."""
    case = quiet_case(jc_A=100e6, jc_B=200e6, jc_n=0.4, plasticity=mode, D_th=1e9)
    st = W.full_state(W.generate_box(case), case)
    st["status"][:] = A.ACTIVE
    g = 4e-3
    st["F"][:, 1] = g
    st["strain_rate"][:] = 1e3
    out, rc = oracle.step(case, st, 1, dt=1e-30)
    assert rc == 0
    p = case["params"]
    s = out["stress"]
    tr = s[:, :3].sum(1) / 3
    dev = s[:, :3] - tr[:, None]
    q = np.sqrt(1.5 * ((dev ** 2).sum(1) + 2 * (s[:, 3:] ** 2).sum(1)))
    eps = out["plastic_strain"]
    assert (eps > 0).all()
    if mode == A.PLAST_NEWTON:
        Y = np.array([jc_flow(p, e, 1e3, 0.0) for e in eps])
    else:
        Y = np.full(len(eps), jc_flow(p, 0.0, 1e3, 0.0))
    assert np.allclose(q, Y, rtol=1e-9)


def test_plastic_heating_and_melt_cap(oracle):
    case = quiet_case(jc_A=50e6, jc_B=0.0, D_th=1e9)
    st = W.full_state(W.generate_box(case), case)
    st["status"][:] = A.ACTIVE
    st["F"][:, 1] = 2e-2
    out, _ = oracle.step(case, st, 1, dt=1e-30)
    p = case["params"]
    dT = out["temperature"] - p["Tamb"]
    expect = np.minimum(p["beta"] * jc_flow(p, 0.0, 0.0, 0.0) * out["plastic_strain"] / (p["rho_phys"] * p["cp"]), 50.0)
    assert np.allclose(dT, expect, rtol=1e-9)
    assert (out["temperature"] <= p["Tm"]).all()


def test_philox_matches_c(oracle):
    rng = np.random.default_rng(5)
    for _ in range(16):
        seed = int(rng.integers(0, 2 ** 63))
        c = [int(x) for x in rng.integers(0, 2 ** 32, 4)]
        mine = np.array([u[0] for u in W.philox4x32_10(seed & 0xFFFFFFFF, seed >> 32, *[np.array([x]) for x in c])])
        assert np.array_equal(mine, oracle.philox(seed, *c))


def test_philox_known_answer():
    """Philox4x32-10 with zero counter and key, and with the all-ones pattern
    (Random123 known-answer vectors, as 24-bit uniforms)."""
    u = W.philox4x32_10(0, 0, np.array([0]), np.array([0]), np.array([0]), np.array([0]))
    words = [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert [float(x[0]) for x in u] == [float(np.float32((w >> 8) / 16777216.0)) for w in words]
    m = 0xFFFFFFFF
    u = W.philox4x32_10(m, m, np.array([m]), np.array([m]), np.array([m]), np.array([m]))
    words = [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert [float(x[0]) for x in u] == [float(np.float32((w >> 8) / 16777216.0)) for w in words]


def test_tool_sdf_matches_c(oracle):
    import ctypes as C
    from oracle.oracle import orc_params
    for case in (W.config1(cells=(16, 8, 8)), W.config2(cells=(32, 8, 16))):
        p = orc_params(case)
        rng = np.random.default_rng(9)
        x = rng.uniform(-1e-3, 2e-3, 200)
        z = rng.uniform(-1e-3, 2e-3, 200)
        pr = (C.c_double * 3)(*case["tool"]["position"])
        mine = W.tool_sdf(case["tool"], x, z, case["tool"]["position"][0], case["tool"]["position"][2])
        theirs = np.array([oracle.L.orc_tool_sdf(C.byref(p), pr, xi, 0.0, zi) for xi, zi in zip(x, z)])
        assert np.allclose(mine, theirs, rtol=0, atol=1e-15)
