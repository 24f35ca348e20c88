"""The drop-in adapter MPMSolverB200 (edegpredict-engine-rotary_b200/adapter/)
on the GPU, driven through its C driver (adapter/_build/libmpm_adapter.so,
built against the reference's headers) in SimulationEngine's call pattern
(src/SimulationEngine.cpp:495-536): per macro step setToolPosition,
beginInterpolatedToolMotion on a snapshot of the FEM tool nodes, eight times
interpolateToolForSubStep(nodes, sub/8) + step(microDt),
endInterpolatedToolMotion, syncMetrics.

The FEM tool is a cylinder's surface samples as FEMNodeGPU records in device
memory, translating at the tool speed, so that the blended node positions of
each sub-step equal the oracle's rasterised tool at that step.

Checks:
- the adapter's particles after the macro steps equal the FP64 oracle's
  (rasterizeToolKernel semantics) to 1e-9 of each field's scale, and the
  C-ABI path (mpm_set_tool_nodes + one mpm_step of 8) to 1e-12;
- the eight sub-steps of a macro step run as one call of 9 step launches
  (not 2 per sub-step), with no host copy of the nodes;
- the live device mirror: velocities written into getDeviceParticles() reach
  the next steps, as the reference's d_particles writes do, and the result
  equals the oracle stepping the same mutated state.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from test_gpu_parity import field_errors

from mpm_b200 import Solver, capi as A, workpiece as W
from mpm_b200.adapter import DRIVER, Adapter, fem_node_records

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not DRIVER.exists(), reason="adapter driver not built (build.py --adapter with "
                                                            "MPM_REFERENCE_SRC naming the reference source tree)")]

SUB = 8
MACRO = 3


def _case():
    """Soft material cut by a cylinder moving along +x (no z motion, so the
    chip-separation tip is the pose's z throughout)."""
    case = W.config1(cells=(12, 8, 8), speed=60.0, tool_mode=A.TOOL_RASTER)
    case["params"].update(jc_A=20e6, jc_B=40e6, jc_n=0.5, D1=0.002, D2=0.01, D3=-1.0, D4=0.01, D5=0.5, D_th=0.02)
    case["tool"]["samples"] = W.cylinder_samples(case)
    case["tool"]["tip_dz"] = 0.0
    return case


def _fem_nodes(case, t):
    """FEMNodeGPU records of the tool's samples at the pose of time t, in a
    device buffer (x, y, z and vx, vy, vz set; the rest zero)."""
    import torch

    tool, smp = case["tool"], case["tool"]["samples"]
    pose = np.array([tool["position"][a] + tool["velocity"][a] * t for a in range(3)])
    return torch.from_numpy(fem_node_records(smp + pose, tool["velocity"]).copy()).to("cuda"), len(smp)


def _engine_macro_steps(ad, case, m0, m1, keep, live=False):
    """Macro steps m0..m1-1 in SimulationEngine's pattern (live: the device
    mirror has been handed out, so the queue imports it before the steps and
    exports it after them)."""
    dt = case["dt"]
    tool = case["tool"]
    for m in range(m0, m1):
        t0 = m * SUB * dt
        start, n = _fem_nodes(case, t0)
        end, _ = _fem_nodes(case, t0 + SUB * dt)
        keep += [start, end]
        pose = (C.c_double * 3)(*[tool["position"][a] + tool["velocity"][a] * t0 for a in range(3)])
        ad.L.mad_set_tool_position(ad.a, pose)
        ad.L.mad_begin_interp(ad.a, start.data_ptr(), n)
        sorts0 = ad.sync_metrics()[1].n_sorts
        l0 = ad.launches()
        for sub in range(SUB):
            ad.L.mad_interp_substep(ad.a, end.data_ptr(), sub / SUB)
            ad.L.mad_step(ad.a, dt)
        assert ad.L.mad_pending(ad.a) == SUB       # queued, nothing launched yet
        assert ad.launches() == l0
        ad.L.mad_end_interp(ad.a, end.data_ptr())  # runs the queue: one library call
        steps = ad.launches() - l0
        iface, full = (C.c_double * 4)(), A.MpmMetrics()
        ad.L.mad_sync_metrics(ad.a, iface, C.byref(full))
        ad.ok()
        # 9 step launches, 8 node sums (deterministic mode) and 8 raster
        # launches, not 2 + 1 per sub-step, plus the launches of a re-bin when
        # one fell due (counts, scans, order, scatter, work list: at most 15)
        rebins = full.n_sorts - sorts0
        assert steps <= SUB + 1 + SUB + SUB + 15 * rebins + (2 if live else 0), (steps, rebins)


def _state_of(rec):
    return dict(x=rec["x"].copy(), y=rec["y"].copy(), z=rec["z"].copy(), vx=rec["vx"].copy(), vy=rec["vy"].copy(),
                vz=rec["vz"].copy(), F=rec["F"].copy(), Fp=rec["F_p"].copy(), C=rec["C"].copy(),
                stress=rec["stress"].copy(), backstress=rec["backstress"].copy(),
                plastic_strain=rec["plasticStrain"].copy(), strain_rate=rec["strainRate"].copy(),
                temperature=rec["temperature"].copy(), damage=rec["damage"].copy(),
                residual_stress=rec["residualStress"].copy(), status=rec["status"].astype(np.int32),
                id=rec["id"].astype(np.int32))


def _open(case, prec):
    b = case["box"]
    ad = Adapter(int(np.prod(np.subtract(b["c1"], b["c0"]))) * b["ppc"] + 64)
    p = W.to_mpm_params(case, precision=prec)
    ad.ok(ad.L.mad_initialize_params(ad.a, C.byref(p)))
    c0, c1 = (C.c_int32 * 3)(*b["c0"]), (C.c_int32 * 3)(*b["c1"])
    ad.ok(ad.L.mad_init_seeded_box(ad.a, c0, c1, b["ppc"], b["seed"], b["fixed_layers"], b["T0"], None))
    return ad


def _initial_state(case):
    gen = dict(case)
    gen["tool"] = dict(case["tool"], mode=A.TOOL_NONE)   # the adapter's box keeps every candidate
    return W.full_state(W.generate_box(gen), case)


def test_adapter_engine_pattern_matches_oracle_and_capi(oracle):
    case = _case()
    keep = []
    ad = _open(case, A.PREC_F64)
    try:
        _engine_macro_steps(ad, case, 0, MACRO, keep)
        rec = ad.particles()
    finally:
        ad.close()
    out = _state_of(rec)
    st0 = _initial_state(case)
    ref, rc = oracle.step(case, st0, MACRO * SUB)
    assert rc == 0
    assert (out["status"] == ref["status"]).all()
    err = field_errors(out, ref, case)
    assert max(err.values()) < 1e-9, err
    assert (ref["plastic_strain"] > 0).any()          # the tool engaged the workpiece
    # the C-ABI path doing what the adapter does
    s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), len(st0["x"]) + 64)
    try:
        b = case["box"]
        s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], 0, b["fixed_layers"], b["T0"])
        L = A.lib()
        for m in range(MACRO):
            t0 = m * SUB * case["dt"]
            start, n = _fem_nodes(case, t0)
            end, _ = _fem_nodes(case, t0 + SUB * case["dt"])
            keep += [start, end]
            s.set_tool(dict(mode=A.TOOL_RASTER, position=tuple(case["tool"]["position"][a] +
                                                              case["tool"]["velocity"][a] * t0 for a in range(3)),
                            velocity=(0.0, 0.0, 0.0), tip_dz=0.0))
            tn = A.MpmToolNodes(start.data_ptr(), end.data_ptr(), n, 264, (C.c_int32 * 3)(0, 8, 16),
                                (C.c_int32 * 3)(48, 56, 64), 0.0, 1.0 / SUB)
            A.check(L.mpm_set_tool_nodes(s.h, C.byref(tn)), s.h)
            s.step(case["dt"], SUB)
            s.metrics()
        capi = _state_of(s.export_aos().view(A.MPM_PARTICLE))
    finally:
        s.close()
    err = field_errors(out, capi, case)
    assert max(err.values()) < 1e-12, err


def test_adapter_live_mirror_writes_reach_the_steps(oracle):
    cudart = C.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    case = _case()
    keep = []
    ad = _open(case, A.PREC_F64)
    try:
        _engine_macro_steps(ad, case, 0, 1, keep)
        dev = ad.L.mad_device_particles(ad.a)
        ad.ok()
        n = ad.L.mad_particle_count(ad.a)
        # what ContactSolver / CFD would do on the handed-out array: slow down
        # the particles of the upper half (vx, vy, vz scaled by 0.5)
        raw = np.zeros(n * 504, np.uint8)
        assert cudart.cudaMemcpy(raw.ctypes.data, dev, n * 504, 2) == 0        # device to host
        rec = raw.view(A.MPM_PARTICLE)
        up = rec["z"] > np.median(rec["z"])
        for k in ("vx", "vy", "vz"):
            rec[k][up] *= 0.5
        assert cudart.cudaMemcpy(dev, raw.ctypes.data, n * 504, 1) == 0        # host to device
        rec = rec.copy()
        _engine_macro_steps(ad, case, 1, 2, keep, live=True)
        out = _state_of(ad.particles())
    finally:
        ad.close()
    ref, rc = oracle.step(case, _state_of(rec), SUB, step0=SUB, t0=SUB * case["dt"])
    assert rc == 0
    assert (out["status"] == ref["status"]).all()
    err = field_errors(out, ref, case)
    assert max(err.values()) < 1e-9, err
