"""Serving loop (mpm_server_*): each request's result is the same when it runs
alone and when it runs in a mix where requests arrive while others are on the
GPU, are admitted between ticks and share launches with them.

Tolerances on the completion metrics:
  FP64: 1e-9 relative on sums (mass, momentum, energies), maxima and bounds;
        counts exact (only the order of the atomic grid sums differs)
  FP32: 1e-4 relative on momentum (scaled by mass x tool speed) and on
        kinetic + internal energy; counts within 0.1 % of the particles
"""
from __future__ import annotations

import numpy as np
import pytest

from mpm_b200 import Server, Solver, capi as A, workpiece as W

pytestmark = pytest.mark.gpu

NSTEPS = [8, 12, 20, 6, 15]
BUDGET = 2 << 30


def cases():
    rng = np.random.default_rng(31)
    return [W.config3_case(rng, i, cells_lo=6, cells_hi=12) for i in range(len(NSTEPS))]


def run_alone(case, n, precision, det=False):
    srv = Server(precision=precision, hbm_budget_bytes=BUDGET, max_chunk=5, deterministic=det)
    try:
        rid = srv.submit(case, n)
        while srv.poll(rid)["state"] not in (A.REQ_DONE, A.REQ_FAILED):
            srv.tick()
        return srv.poll(rid)
    finally:
        srv.close()


def run_mix(cs, precision, det=False):
    srv = Server(precision=precision, hbm_budget_bytes=BUDGET, max_chunk=5, deterministic=det)
    try:
        ids = [srv.submit(cs[k], NSTEPS[k]) for k in range(3)]
        srv.tick()                      # the first three are on the GPU
        assert srv.stats()["resident"] == 3
        ids += [srv.submit(cs[k], NSTEPS[k]) for k in range(3, 5)]   # arrive while they run
        for _ in range(200):
            if all(srv.poll(i)["state"] in (A.REQ_DONE, A.REQ_FAILED) for i in ids):
                break
            srv.tick()
        st = srv.stats()
        return [srv.poll(i) for i in ids], st
    finally:
        srv.close()


def rel(a, b, scale):
    return abs(a - b) / max(scale, 1e-300)


def test_mix_equals_alone_fp64():
    cs = cases()
    mix, st = run_mix(cs, A.PREC_F64)
    assert st["completed"] == 5 and st["failed"] == 0 and st["offered"] == 5
    for k, c in enumerate(cs):
        a = run_alone(c, NSTEPS[k], A.PREC_F64)
        m, r = mix[k], a
        assert m["state"] == A.REQ_DONE and r["state"] == A.REQ_DONE
        assert m["steps_done"] == NSTEPS[k] and m["n_particles"] == r["n_particles"] > 0
        assert m["t_submit"] <= m["t_admit"] <= m["t_done"]
        mm, rm = m["metrics"], r["metrics"]
        for key in ("mass", "kinetic", "internal_elastic", "thermal", "ref_kinetic", "ref_internal",
                    "max_von_mises", "max_plastic_strain", "ref_max_stress", "max_temperature"):
            assert rel(mm[key], rm[key], abs(rm[key])) < 1e-9, (k, key, mm[key], rm[key])
        pscale = rm["mass"] * np.linalg.norm(c["tool"]["velocity"])
        for a_ in range(3):
            assert rel(mm["momentum"][a_], rm["momentum"][a_], pscale) < 1e-9
        for key in ("n_active", "n_chip", "n_fixed", "n_inactive"):
            assert mm[key] == rm[key]


def test_server_matches_plain_handle_fp64():
    """A served request equals the same workpiece stepped through mpm_create."""
    c = cases()[1]
    n = NSTEPS[1]
    served = run_alone(c, n, A.PREC_F64)["metrics"]
    b = c["box"]
    s = Solver(W.to_mpm_params(c, precision=A.PREC_F64), int(np.prod(np.subtract(b["c1"], b["c0"]))) * b["ppc"])
    try:
        s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], b["instance"], b["fixed_layers"], b["T0"], tool=c["tool"])
        s.step(c["dt"], n)
        plain = s.metrics()
    finally:
        s.close()
    for key in ("mass", "kinetic", "internal_elastic", "thermal", "max_von_mises"):
        assert rel(served[key], plain[key], abs(plain[key])) < 1e-9, (key, served[key], plain[key])


def test_mix_equals_alone_fp32():
    cs = cases()
    mix, st = run_mix(cs, A.PREC_F32)
    assert st["completed"] == 5
    for k, c in enumerate(cs):
        r = run_alone(c, NSTEPS[k], A.PREC_F32)["metrics"]
        m = mix[k]["metrics"]
        pscale = r["mass"] * np.linalg.norm(c["tool"]["velocity"])
        for a_ in range(3):
            assert rel(m["momentum"][a_], r["momentum"][a_], pscale) < 1e-4, (k, a_)
        e_m = m["kinetic"] + m["internal_elastic"]
        e_r = r["kinetic"] + r["internal_elastic"]
        assert rel(e_m, e_r, abs(e_r)) < 1e-4, (k, e_m, e_r)
        n = mix[k]["n_particles"]
        for key in ("n_active", "n_chip", "n_fixed"):
            assert abs(m[key] - r[key]) <= max(1, n // 1000)


def test_zero_step_request_and_capacity_refusal():
    c = cases()[0]
    srv = Server(precision=A.PREC_F32, hbm_budget_bytes=1 << 27)
    try:
        rid = srv.submit(c, 0)
        srv.tick()
        res = srv.poll(rid)
        assert res["state"] == A.REQ_DONE and res["steps_done"] == 0 and res["metrics"]["mass"] > 0
        big = W.config1()   # 524k particles: more than a 128 MiB budget holds
        with pytest.raises(A.MpmError) as e:
            srv.submit(big, 10)
        assert e.value.status == A.MPM_CAPACITY
    finally:
        srv.close()


def test_preempted_request_resumes_where_it_stopped():
    """A request preempted after 10 of its 30 steps is saved, dropped from the
    device, admitted again from its checkpoint and finished; its completion
    metrics equal those of its run alone (FP64: 1e-9 relative, counts exact)."""
    case = W.config1(cells=(12, 8, 8), speed=20.0)
    n = 30
    alone = run_alone(case, n, A.PREC_F64)
    srv = Server(precision=A.PREC_F64, hbm_budget_bytes=BUDGET, max_chunk=5)
    try:
        rid = srv.submit(case, n)
        srv.tick()
        srv.tick()                               # 10 steps
        srv.preempt(rid)
        srv.tick()                               # saved, dropped and admitted again from the checkpoint
        assert srv.stats()["preempted"] == 1
        for _ in range(100):
            if srv.poll(rid)["state"] == A.REQ_DONE:
                break
            srv.tick()
        res = srv.poll(rid)
    finally:
        srv.close()
    assert res["state"] == A.REQ_DONE and res["steps_done"] == n
    for k in ("mass", "kinetic", "internal_elastic", "max_plastic_strain", "max_von_mises"):
        a, b = res["metrics"][k], alone["metrics"][k]
        assert rel(a, b, abs(b)) <= 1e-9, (k, a, b)
    for k in ("n_active", "n_chip", "n_inactive"):
        assert res["metrics"][k] == alone["metrics"][k], k


def test_deterministic_mix_equals_alone_bit_for_bit():
    """With the server's deterministic option, FP32 results are the same bits
    alone and in the mix: every per-workpiece metric is equal exactly (the
    cumulative counters of the whole handle are not per workpiece)."""
    cs = cases()
    mix, st = run_mix(cs, A.PREC_F32, det=True)
    assert st["completed"] == 5 and st["failed"] == 0
    handle_wide = {"n_escaped", "n_sorts", "n_yielded", "n_contacts", "contact_work", "contact_force",
                   "n_asb_heated"}
    for k, c in enumerate(cs):
        a = run_alone(c, NSTEPS[k], A.PREC_F32, det=True)
        assert mix[k]["state"] == a["state"] == A.REQ_DONE
        mm, am = mix[k]["metrics"], a["metrics"]
        for key in mm:
            if key not in handle_wide:
                assert mm[key] == am[key], (k, key, mm[key], am[key])

