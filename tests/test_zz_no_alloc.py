"""mpm_metrics_aos_noalloc -- workpiece metrics of a device MPMParticle array
with no handle and no allocation (scratch in a static device array) --
against mpm_sync_metrics on a handle holding the same particles.

Tolerances: sums (mass, momentum, energies, heat, mean plastic strain) within
1e-9 of their magnitude (FP64 sums in another order), the heat term also
within 1e-12 K of total heat capacity (the record stores T = Tamb + dT, which
rounds dT); maxima and bounds within 1e-12 relative; counts exact.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from scenarios import SCENARIOS  # noqa: E402

from mpm_b200 import Solver, capi as A, workpiece as W  # noqa: E402
from mpm_b200.solver import metrics_aos_noalloc  # noqa: E402

SUMS = ("mass", "kinetic", "internal_elastic", "ref_kinetic", "ref_internal", "mean_plastic_strain")
MAXES = ("max_von_mises", "max_plastic_strain", "ref_max_stress", "ref_max_temperature", "max_temperature")
COUNTS = ("n_active", "n_chip", "n_fixed", "n_inactive")


def assert_metrics_match(got, ref, heat_capacity):
    for k in SUMS:
        assert abs(got[k] - ref[k]) <= 1e-9 * max(abs(ref[k]), 1e-300), (k, got[k], ref[k])
    pscale = max(abs(v) for v in ref["momentum"]) or 1e-300
    for a in range(3):
        assert abs(got["momentum"][a] - ref["momentum"][a]) <= 1e-9 * pscale
    assert abs(got["thermal"] - ref["thermal"]) <= 1e-9 * abs(ref["thermal"]) + 1e-12 * heat_capacity
    for k in MAXES:
        assert abs(got[k] - ref[k]) <= 1e-12 * max(abs(ref[k]), 1e-300), (k, got[k], ref[k])
    for k in ("bounds_min", "bounds_max"):
        assert np.allclose(got[k], ref[k], rtol=1e-12, atol=0), (k, got[k], ref[k])
    for k in COUNTS:
        assert got[k] == ref[k], (k, got[k], ref[k])
    assert got["n_escaped"] == 0 and got["n_sorts"] == 0 and got["n_yielded"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [A.PREC_F32, A.PREC_F64])
def test_noalloc_metrics_match_handle_metrics(prec):
    import torch

    case, st, n, extf = SCENARIOS["plastic_damage_chip"]()
    p = W.to_mpm_params(case, precision=prec)
    s = Solver(p, len(st["x"]) + 64)
    try:
        s.set_tool(case["tool"])
        s.upload(st)
        count = s.counts()[0]
        dev = torch.empty(count * 504, dtype=torch.uint8, device="cuda")
        heat_capacity = p.rho_phys * p.cp * p.particle_volume * count
        # two calls in a row, each on a new state of the workpiece
        for _ in range(2):
            s.step(case["dt"], max(n // 2, 1))
            ref = s.metrics()
            s._check(s._lib.mpm_export_aos(s.h, C.c_void_p(dev.data_ptr()), dev.numel()))
            got = metrics_aos_noalloc(p, dev.data_ptr(), count)
            assert got["n_active"] + got["n_chip"] > 0
            assert_metrics_match(got, ref, heat_capacity)
    finally:
        s.close()


def test_noalloc_refuses_counts_above_scratch_limit():
    """Refused before any CUDA call (runs without a GPU); the pointer is never
    dereferenced."""
    p = A.default_params()
    m = A.MpmMetrics()
    st = A.lib().mpm_metrics_aos_noalloc(C.byref(p), C.c_void_p(4096), 67_108_865, None, C.byref(m))
    assert st == A.MPM_CAPACITY
    msg = A.lib().mpm_last_error(None).decode()
    assert "67108864" in msg and "mpm_sync_metrics" in msg
    assert A.lib().mpm_metrics_aos_noalloc(None, None, 0, None, C.byref(m)) == A.MPM_INVALID_ARG
    assert A.lib().mpm_metrics_aos_noalloc(C.byref(p), None, -1, None, C.byref(m)) == A.MPM_INVALID_ARG
    assert A.lib().mpm_metrics_aos_noalloc(C.byref(p), None, 10, None, C.byref(m)) == A.MPM_INVALID_ARG


@pytest.mark.gpu
def test_noalloc_metrics_across_reduction_blocks():
    """Each reduction block takes 16,384 records; the records of one workpiece
    repeated six times (36,390 records: two full blocks and a partial third)
    make the final combine join several partial rows: sums and counts come
    out six times the handle's, maxima and bounds the same."""
    import torch

    case, st, n, extf = SCENARIOS["plastic_damage_chip"]()
    p = W.to_mpm_params(case, precision=A.PREC_F32)
    s = Solver(p, len(st["x"]) + 64)
    try:
        s.set_tool(case["tool"])
        s.upload(st)
        s.step(case["dt"], n)
        count = s.counts()[0]
        ref = s.metrics()
        one = torch.empty(count * 504, dtype=torch.uint8, device="cuda")
        s._check(s._lib.mpm_export_aos(s.h, C.c_void_p(one.data_ptr()), one.numel()))
        k = 2 * 16384 // count + 1
        assert count * k > 2 * 16384 and (count * k) % 16384 != 0
        tiled = one.repeat(k)
        heat_capacity = p.rho_phys * p.cp * p.particle_volume * count * k
        scaled = dict(ref)
        for key in ("mass", "kinetic", "internal_elastic", "thermal", "ref_kinetic", "ref_internal",
                    "n_active", "n_chip", "n_fixed", "n_inactive"):
            scaled[key] = ref[key] * k
        scaled["momentum"] = [v * k for v in ref["momentum"]]
        scaled["n_escaped"] = scaled["n_sorts"] = scaled["n_yielded"] = 0
        for _ in range(2):
            got = metrics_aos_noalloc(p, tiled.data_ptr(), count * k)
            assert_metrics_match(got, scaled, heat_capacity)
    finally:
        s.close()


@pytest.mark.gpu
def test_noalloc_metrics_of_no_particles():
    """n = 0 (no pointer needed): the same result as a handle holding no
    particles -- zero sums and counts, the reductions' empty seeds."""
    case, st, n, extf = SCENARIOS["plastic_damage_chip"]()
    p = W.to_mpm_params(case, precision=A.PREC_F32)
    s = Solver(p, 64)
    try:
        empty = {k: v[:0] for k, v in st.items()}
        s.upload(empty)
        ref = s.metrics()
    finally:
        s.close()
    got = metrics_aos_noalloc(p, 0, 0)
    for key in SUMS + ("thermal",) + COUNTS:
        assert got[key] == 0, (key, got[key])
    assert got["momentum"] == [0.0, 0.0, 0.0]
    for key in MAXES + COUNTS + SUMS + ("thermal", "momentum", "bounds_min", "bounds_max"):
        assert got[key] == ref[key], (key, got[key], ref[key])
