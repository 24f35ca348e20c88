"""Failure detection without a GPU fault: the bounded device-side wait that
guards the step kernel's tile loads gives up when nothing completes it, the
host reads MPM_TIMEOUT, and the context stays usable (a step right after
matches the oracle).  The wait is limited to 50 ms; no copy is in flight."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

from mpm_b200 import Solver, capi as A, workpiece as W


def test_selftest_argument_checks_need_no_gpu():
    L = A.lib()
    assert L.mpm_selftest_bounded_wait(0, None) == A.MPM_INVALID_ARG
    assert L.mpm_selftest_bounded_wait(2_000_000_000, None) == A.MPM_INVALID_ARG


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_context_survives(oracle):
    L = A.lib()
    t0 = time.perf_counter()
    st = L.mpm_selftest_bounded_wait(50_000_000, None)
    el = time.perf_counter() - t0
    assert st == A.MPM_TIMEOUT, L.mpm_last_error(None)
    assert b"gave up" in L.mpm_last_error(None)
    assert el < 5.0
    # the context is usable: a small run right after matches the oracle
    case = W.config1(cells=(12, 8, 8), speed=20.0)
    st0 = W.full_state(W.generate_box(case), case)
    ref, rc = oracle.step(case, st0, 4)
    assert rc == 0
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), len(st0["x"]))
    try:
        s.set_tool(case["tool"])
        s.upload(st0)
        s.step(case["dt"], 4)
        out = s.download()
    finally:
        s.close()
    assert np.abs(out["x"] - ref["x"]).max() <= 1e-9 * case["params"]["dx"]
    assert (out["status"] == ref["status"]).all()


def active_middle(st) -> int:
    """The middle ACTIVE particle (a FIXED particle's velocity is never used)."""
    act = np.flatnonzero(st["status"] == A.ACTIVE)
    return int(act[len(act) // 2])


@pytest.mark.gpu
def test_nan_velocity_matches_the_oracle(oracle):
    """A NaN velocity of one ACTIVE particle: after one step the grid has
    carried it to the positions of its neighbours, and the next step's kill
    zone deactivates exactly those particles, as the oracle does (FP64: the
    same status, the same NaN pattern, the finite positions within 1e-9 of a
    cell); the error word is set once the kill zone has run."""
    case = W.config1(cells=(12, 8, 8), speed=20.0)
    st0 = W.full_state(W.generate_box(case), case)
    st0["vx"][active_middle(st0)] = np.nan
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), len(st0["x"]))
    try:
        s.set_tool(case["tool"])
        s.upload(st0)
        s.step(case["dt"], 1)
        assert s.status() == A.MPM_OK               # positions NaN, nothing killed yet
        out1 = s.download(strict=False)
        s.step(case["dt"], 3)
        assert s.status() == A.MPM_NUMERIC
        with pytest.raises(A.MpmError) as e:
            s.download()
        assert e.value.status == A.MPM_NUMERIC
        out = s.download(strict=False)
    finally:
        s.close()
    ref1, rc1 = oracle.step(case, st0, 1)
    ref, rc = oracle.step(case, st0, 4)
    assert rc1 == 0 and rc == 0
    assert np.isnan(out1["x"]).sum() == np.isnan(ref1["x"]).sum() > 0
    assert (out1["status"] == ref1["status"]).all()
    assert (ref["status"] == A.INACTIVE).sum() == np.isnan(ref1["x"]).sum()
    assert (out["status"] == ref["status"]).all()
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        assert (np.isnan(out[f]) == np.isnan(ref[f])).all(), f
    ok = ~np.isnan(ref["x"])
    assert np.abs(out["x"][ok] - ref["x"][ok]).max() <= 1e-9 * case["params"]["dx"]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [A.PREC_F64, A.PREC_F32])
def test_nan_in_one_workpiece_marks_only_that_one(precision):
    """One NaN velocity uploaded into instance 1 of three: the grid carries it
    to the positions of its neighbours within a step, the kill zone takes
    them out and only instance 1's error word is set; its metrics report
    MPM_NUMERIC, and instances 0 and 2 match the same workpieces run alone
    (tolerances of the batched form).  A clean upload clears the word;
    dropping the instance leaves the others' words clean and their steps
    unchanged."""
    from mpm_b200 import Batch
    from test_gpu_batch import assert_same, cap_of, init_i, run_alone, small_cases
    cases = small_cases(3, seed=5, precision=precision)
    n, n2 = 6, 4
    bt = Batch([W.to_mpm_params(c, precision=precision) for c in cases], [cap_of(c) for c in cases])
    try:
        for i, c in enumerate(cases):
            assert init_i(bt, i, c) > 0
        bad = W.full_state(W.generate_box(cases[1]), cases[1])
        j = active_middle(bad)
        bad["vx"][j] = np.nan
        bt.upload_i(1, bad)
        assert bt.instance_status() == [A.MPM_OK] * 3
        bt.step_all([c["dt"] for c in cases], n)
        assert bt.instance_status() == [A.MPM_OK, A.MPM_NUMERIC, A.MPM_OK]
        with pytest.raises(A.MpmError) as e:
            bt.metrics_i(1)
        assert e.value.status == A.MPM_NUMERIC and "instance 1" in str(e.value)
        for i in (0, 2):
            assert bt.metrics_i(i)["n_active"] > 0
        outs = [bt.download_i(0), bt.download_i(2)]
        # a clean state clears the word
        bad["vx"][j] = 0.0
        bt.upload_i(1, bad)
        assert bt.instance_status() == [A.MPM_OK] * 3
        # the failed workpiece can also be dropped: the others run on
        bad["vx"][j] = np.nan
        bt.upload_i(1, bad)
        bt.step_all([c["dt"] for c in cases], 2)
        assert bt.instance_status() == [A.MPM_OK, A.MPM_NUMERIC, A.MPM_OK]
        bt.change(remove=[1])
        assert bt.instance_status() == [A.MPM_OK, A.MPM_OK]
        bt.step_all([cases[0]["dt"], cases[2]["dt"]], n2)
        assert bt.instance_status() == [A.MPM_OK, A.MPM_OK]
        outs2 = [bt.download_i(0), bt.download_i(1)]
    finally:
        bt.close()
    for k, i in enumerate((0, 2)):
        assert_same(outs[k], run_alone(cases[i], n, precision), cases[i], precision)
        assert_same(outs2[k], run_alone(cases[i], [n, 2, n2], precision), cases[i], precision)


@pytest.mark.gpu
def test_server_evicts_a_failed_request_and_cancels_another():
    """Three requests of one workpiece share the GPU; one runs the Newton
    return with a single iteration allowed, so its first plastic return does
    not converge.  That request ends FAILED with MPM_NUMERIC and is dropped,
    a second is cancelled while it runs, and the third completes with the
    metrics it has when it runs alone (FP64: 1e-9 relative)."""
    from mpm_b200 import Server
    from mpm_b200.solver import make_request
    case = W.config1(cells=(12, 8, 8), speed=20.0)
    nsteps = 30
    prec = A.PREC_F64

    def serve(cancel_second: bool, with_bad: bool):
        srv = Server(precision=prec, hbm_budget_bytes=1 << 30, max_chunk=5)
        try:
            ids = [srv.submit(case, nsteps)]
            if with_bad:
                r = make_request(case, nsteps, prec)
                r.params.plasticity = A.PLAST_NEWTON
                r.params.newton_maxit = 1
                ids.append(srv.submit_request(r))
            if cancel_second:
                ids.append(srv.submit(case, nsteps))
            srv.tick()
            if cancel_second:
                srv.cancel(ids[-1])
            for _ in range(100):
                if all(srv.poll(i)["state"] not in (A.REQ_QUEUED, A.REQ_RUNNING) for i in ids):
                    break
                srv.tick()
            srv.tick()   # drops the requests that ended in the last tick
            return [srv.poll(i) for i in ids], srv.stats()
        finally:
            srv.close()

    res, st = serve(cancel_second=True, with_bad=True)
    good, bad, cancelled = res
    assert bad["state"] == A.REQ_FAILED and bad["status"] == A.MPM_NUMERIC, bad
    assert 0 < bad["steps_done"] < nsteps
    assert cancelled["state"] == A.REQ_CANCELLED and cancelled["status"] == A.MPM_CANCELLED
    assert cancelled["steps_done"] == 5
    assert good["state"] == A.REQ_DONE and good["steps_done"] == nsteps
    assert st["failed"] == 1 and st["cancelled"] == 1 and st["completed"] == 1 and st["resident"] == 0
    (alone,), _ = serve(cancel_second=False, with_bad=False)
    assert alone["state"] == A.REQ_DONE
    for k in ("mass", "kinetic", "internal_elastic", "max_plastic_strain"):
        a, b = good["metrics"][k], alone["metrics"][k]
        assert abs(a - b) <= 1e-9 * max(abs(b), 1e-300), (k, a, b)
    assert good["metrics"]["n_active"] == alone["metrics"]["n_active"]
