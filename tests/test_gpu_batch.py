"""Batched form (mpm_batch_*): several uneven workpieces in one handle give the
same results as each one run alone through the plain handle; instances can be
dropped and added between steps without disturbing the others; the CUDA-graph
replay and the autotuner change nothing but the launch shape.

Tolerances (per instance, fields scaled as in test_gpu_parity.field_errors):
  FP64: 1e-9 (only the order of the atomic grid sums differs)
  FP32: positions 2e-4 cell, velocities 1e-3, other fields 2e-3; status equal
        for >= 99.9 % of particles
"""
from __future__ import annotations

import numpy as np
import pytest

from mpm_b200 import Batch, Solver, capi as A, workpiece as W
from test_gpu_parity import field_errors

pytestmark = pytest.mark.gpu

TOL32 = dict(x=2e-4, y=2e-4, z=2e-4, vx=1e-3, vy=1e-3, vz=1e-3)


def small_cases(n, seed=11, precision=A.PREC_F64):
    rng = np.random.default_rng(seed)
    return [W.config3_case(rng, i, cells_lo=6, cells_hi=12, steps=12, precision=precision) for i in range(n)]


def cap_of(case):
    b = case["box"]
    return int(np.prod(np.subtract(b["c1"], b["c0"]))) * b["ppc"]


def init_i(bt, i, case):
    b = case["box"]
    return bt.init_box_i(i, b["c0"], b["c1"], b["ppc"], b["seed"], b["instance"], b["fixed_layers"], b["T0"],
                         tool=case["tool"])


def run_alone(case, nsteps, precision):
    s = Solver(W.to_mpm_params(case, precision=precision), cap_of(case))
    try:
        b = case["box"]
        s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], b["instance"], b["fixed_layers"], b["T0"], tool=case["tool"])
        for k in nsteps if isinstance(nsteps, (list, tuple)) else [nsteps]:
            s.step(case["dt"], k)
        return s.download()
    finally:
        s.close()


def assert_same(out, ref, case, precision):
    if precision == A.PREC_F64:
        assert (out["status"] == ref["status"]).all()
        err = field_errors(out, ref, case)
        assert max(err.values()) < 1e-9, err
    else:
        assert (out["status"] == ref["status"]).mean() >= 0.999
        err = field_errors(out, ref, case)
        bad = {k: v for k, v in err.items() if v > TOL32.get(k, 2e-3)}
        assert not bad, (bad, err)


@pytest.mark.parametrize("precision", [A.PREC_F64, A.PREC_F32])
def test_batch_matches_instances_alone(precision):
    cases = small_cases(5, precision=precision)
    n = 12
    bt = Batch([W.to_mpm_params(c, precision=precision) for c in cases], [cap_of(c) for c in cases])
    try:
        assert bt.count() == 5
        for i, c in enumerate(cases):
            assert init_i(bt, i, c) > 0
        bt.step_all([c["dt"] for c in cases], n)
        outs = [bt.download_i(i) for i in range(len(cases))]
        counts = [bt.counts_i(i) for i in range(len(cases))]
    finally:
        bt.close()
    for i, c in enumerate(cases):
        assert counts[i][1] == n and abs(counts[i][2] - n * c["dt"]) < 1e-18
        assert_same(outs[i], run_alone(c, n, precision), c, precision)


def test_batch_change_keeps_other_instances():
    """Drop instance 1 and add a new one after 5 steps; the kept instances
    continue as if nothing happened and the new one starts from t = 0."""
    cases = small_cases(4, seed=5)
    extra = small_cases(1, seed=99)[0]
    prec = A.PREC_F64
    bt = Batch([W.to_mpm_params(c, precision=prec) for c in cases[:3]], [cap_of(c) for c in cases[:3]])
    try:
        for i in range(3):
            init_i(bt, i, cases[i])
        bt.step_all([c["dt"] for c in cases[:3]], 5)
        first = bt.change(add_params=[W.to_mpm_params(extra, precision=prec)], add_caps=[cap_of(extra)], remove=[1])
        assert first == 2 and bt.count() == 3
        init_i(bt, 2, extra)
        live = [cases[0], cases[2], extra]
        bt.step_all([c["dt"] for c in live], 7)
        outs = [bt.download_i(i) for i in range(3)]
        steps = [bt.counts_i(i)[1] for i in range(3)]
    finally:
        bt.close()
    assert steps == [12, 12, 7]
    assert_same(outs[0], run_alone(cases[0], [5, 7], prec), cases[0], prec)
    assert_same(outs[1], run_alone(cases[2], [5, 7], prec), cases[2], prec)
    assert_same(outs[2], run_alone(extra, 7, prec), extra, prec)


def test_graph_replay_and_autotune_keep_results():
    cases = small_cases(3, seed=21)
    prec = A.PREC_F64
    dts = [c["dt"] for c in cases]
    ref = []
    bt = Batch([W.to_mpm_params(c, precision=prec) for c in cases], [cap_of(c) for c in cases])
    try:
        for i, c in enumerate(cases):
            init_i(bt, i, c)
        for _ in range(3):
            bt.step_all(dts, 4)
        ref = [bt.download_i(i) for i in range(3)]
    finally:
        bt.close()
    bt = Batch([W.to_mpm_params(c, precision=prec) for c in cases], [cap_of(c) for c in cases])
    try:
        for i, c in enumerate(cases):
            init_i(bt, i, c)
        bt.set_launch_config(ctas_per_sm=4, sort_every=16, use_graph=True)
        assert bt.launch_config()["use_graph"] == 1
        n0 = bt.launches()
        for _ in range(3):   # the second and third calls replay the captured graph
            bt.step_all(dts, 4)
        assert bt.launches() - n0 >= 3 * 5
        got = [bt.download_i(i) for i in range(3)]
        cfg = bt.autotune(dts)
        assert cfg["ctas_per_sm"] in (2, 3, 4) and cfg["sort_every"] in (8, 16, 32)
        assert cfg["pass_size"] in (128, 256, 512)
        # 16 steps per pass size, then one re-bin period per CTAs x cadence
        assert bt.counts_i(0)[1] == 12 + 3 * 16 + 3 * (8 + 16 + 32)
    finally:
        bt.close()
    for i, c in enumerate(cases):
        assert_same(got[i], ref[i], c, prec)
