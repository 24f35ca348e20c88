"""C ABI behaviour on the GPU: the device generator, upload/download round
trips, the reference-layout AoS export, metrics, error returns and edge cases."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from mpm_b200 import Solver, capi as A, workpiece as W

pytestmark = pytest.mark.gpu

# MPMParticle (include/Types.h:199-266) as a numpy record, 504 bytes
AOS = A.MPM_PARTICLE


def small_case(**kw):
    args = dict(cells=(12, 8, 8), speed=20.0)
    args.update(kw)
    return W.config1(**args)


@pytest.mark.parametrize("prec", [A.PREC_F64, A.PREC_F32])
def test_device_generator_matches_host_mirror(prec):
    case = small_case()
    host = W.generate_box(case)
    b = case["box"]
    s = Solver(W.to_mpm_params(case, precision=prec), 8 * 12 * 8 * 8)
    n = s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], b["instance"], b["fixed_layers"], b["T0"], tool=case["tool"])
    out = s.download(fields=("x", "y", "z", "status", "id", "temperature"))
    s.close()
    assert n == len(host["x"])
    tol = 1e-12 if prec == A.PREC_F64 else 1e-6
    for k in ("x", "y", "z"):
        assert np.abs(out[k] - host[k]).max() <= tol * case["params"]["dx"] * 100
    assert (out["status"] == host["status"]).all() and (out["id"] == host["id"]).all()
    assert np.allclose(out["temperature"], host["temperature"])


@pytest.mark.parametrize("prec,tol", [(A.PREC_F64, 0.0), (A.PREC_F32, 2e-7)])
def test_upload_download_roundtrip(prec, tol):
    case = small_case()
    st = W.full_state(W.generate_box(case), case)
    rng = np.random.default_rng(3)
    n = len(st["x"])
    st["vx"] = rng.normal(0, 1, n)
    st["C"] = rng.normal(0, 10, (n, 9))
    st["F"] = st["F"] + rng.normal(0, 1e-3, (n, 9))
    st["stress"] = rng.normal(0, 1e8, (n, 6))
    st["damage"] = rng.uniform(0, 0.5, n)
    st["status"][::7] = A.CHIP
    s = Solver(W.to_mpm_params(case, precision=prec), n)
    s.upload(st)
    out = s.download()
    s.close()
    for k in ("x", "y", "z", "vx", "C", "F", "stress", "damage", "temperature"):
        scale = np.abs(st[k]).max()
        assert np.abs(out[k] - st[k]).max() <= tol * scale + (1e-15 * scale), k
    assert (out["status"] == st["status"]).all() and (out["id"] == st["id"]).all()


def test_export_aos_layout():
    case = small_case()
    st = W.full_state(W.generate_box(case), case)
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), len(st["x"]))
    s.set_tool(case["tool"])
    s.upload(st)
    s.step(case["dt"], 4)
    soa = s.download()
    raw = s.export_aos()
    s.close()
    rec = raw.view(AOS)
    assert len(rec) == len(st["x"])
    for a, b in (("x", "x"), ("vz", "vz"), ("temperature", "temperature"), ("plasticStrain", "plastic_strain"),
                 ("strainRate", "strain_rate"), ("damage", "damage"), ("residualStress", "residual_stress")):
        assert np.array_equal(rec[a], soa[b]), a
    assert np.array_equal(rec["F"], soa["F"]) and np.array_equal(rec["C"], soa["C"])
    assert np.array_equal(rec["stress"], soa["stress"])
    assert (rec["status"] == soa["status"]).all() and (rec["id"] == soa["id"]).all()
    assert np.allclose(rec["mass"], case["params"]["particle_mass"])


def test_empty_workpiece_steps():
    case = small_case()
    s = Solver(W.to_mpm_params(case), 16)
    s.upload({"x": np.zeros(0), "y": np.zeros(0), "z": np.zeros(0)})
    s.step(case["dt"], 5)
    m = s.metrics()
    s.close()
    assert m["mass"] == 0.0 and m["n_active"] == 0


def test_error_returns_do_not_crash():
    case = small_case()
    p = W.to_mpm_params(case)
    bad = W.to_mpm_params(case)
    bad.nx = 2
    with pytest.raises(A.MpmError) as e:
        Solver(bad, 10)
    assert e.value.status == A.MPM_INVALID_ARG
    s = Solver(p, 10)
    with pytest.raises(A.MpmError) as e:
        s.upload({"x": np.zeros(100), "y": np.zeros(100), "z": np.zeros(100)})
    assert e.value.status == A.MPM_CAPACITY
    with pytest.raises(A.MpmError) as e:
        s.step(-1.0, 1)
    assert e.value.status == A.MPM_INVALID_ARG
    # a NULL handle is refused, not dereferenced
    st = A.lib().mpm_step(None, 1e-9, 1)
    assert st == A.MPM_INVALID_ARG
    s.close()


def test_mass_scaling_and_temperatures():
    case = small_case()
    st = W.full_state(W.generate_box(case), case)
    n = len(st["x"])
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), n)
    s.upload(st)
    m0 = s.metrics()["mass"]
    s.set_mass_scaling(4.0)
    m1 = s.metrics()["mass"]
    assert abs(m1 / m0 - 4.0) < 1e-12
    T = np.linspace(300.0, 900.0, n)
    s.set_temperatures(T)
    out = s.download(fields=("temperature",))
    s.close()
    assert np.allclose(out["temperature"], T)


def test_stable_dt_is_cfl():
    case = small_case()
    s = Solver(W.to_mpm_params(case), 8)
    dt = s.stable_dt(0.3)
    s.close()
    assert abs(dt / case["dt"] - 1.0) < 1e-12
