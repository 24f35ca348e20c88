"""The writable AoS mirror: mpm_export_aos hands the reference's consumers an
MPMParticle array, they write it in place, and mpm_import_aos reads their
writes back before the next step.

- The reference's own xpbdContactSDFKernel (src/ContactSolver.cu:797-923,
  oracle/_ref) runs on the exported device array and moves positions,
  velocities and temperatures; CFD-like writes add drag to ext_f, cool some
  particles and turn a few into chips.  After the import, two steps of the
  CUDA path match the oracle stepping the same mutated records: FP64 within
  1e-9 of each field's scale, FP32 within the plain parity tolerances.
- An unmodified array imports as a no-op, bit for bit.
- A record with a status outside 0..4 is refused (MPM_INVALID_ARG) and keeps
  its status; its other fields are imported.
- An imported ext_f equals applyExternalForce's (mpm_apply_external_force)
  for the same per-particle force.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from make_golden import cylinder_sdf  # noqa: E402
from scenarios import SCENARIOS  # noqa: E402

from test_gpu_parity import field_errors  # noqa: E402

from mpm_b200 import Solver, capi as A, workpiece as W  # noqa: E402

pytestmark = pytest.mark.gpu

N0, N1 = 10, 2
FP32_TOL = dict(x=2e-4, y=2e-4, z=2e-4, vx=1e-3, vy=1e-3, vz=1e-3)


def _state_from_records(rec):
    """The particle state dict (upload order) of MPMParticle records."""
    return dict(x=rec["x"].copy(), y=rec["y"].copy(), z=rec["z"].copy(), vx=rec["vx"].copy(), vy=rec["vy"].copy(),
                vz=rec["vz"].copy(), F=rec["F"].copy(), Fp=rec["F_p"].copy(), C=rec["C"].copy(),
                stress=rec["stress"].copy(), backstress=rec["backstress"].copy(),
                plastic_strain=rec["plasticStrain"].copy(), strain_rate=rec["strainRate"].copy(),
                temperature=rec["temperature"].copy(), damage=rec["damage"].copy(),
                residual_stress=rec["residualStress"].copy(), status=rec["status"].astype(np.int32),
                id=rec["id"].astype(np.int32), asb=rec["asbCounter"].astype(np.int32))


def _solver(prec):
    case, st, n, extf = SCENARIOS["plastic_damage_chip"]()
    s = Solver(W.to_mpm_params(case, precision=prec), len(st["x"]) + 64)
    s.set_tool(case["tool"])
    s.upload(st)
    s.step(case["dt"], N0)
    return case, s


def _mirror(s):
    import torch

    n = s.counts()[0]
    dev = torch.empty(n * 504, dtype=torch.uint8, device="cuda")
    s.export_aos_device(dev.data_ptr(), dev.numel())
    return dev, n


@pytest.mark.parametrize("prec", [A.PREC_F64, A.PREC_F32])
def test_unmodified_mirror_imports_as_a_no_op(prec):
    case, s = _solver(prec)
    try:
        before = s.download()
        dev, n = _mirror(s)
        s.import_aos(dev.data_ptr(), A.AOS_WRITABLE, dev.numel())
        after = s.download()
        host = s.export_aos()
        s.import_aos(host, A.AOS_WRITABLE)   # from host memory as well
        again = s.download()
    finally:
        s.close()
    for k, v in before.items():
        assert np.array_equal(v, after[k]) and np.array_equal(v, again[k]), k


@pytest.mark.parametrize("prec", [A.PREC_F64, A.PREC_F32])
def test_reference_contact_on_the_mirror_then_steps_match_oracle(prec, oracle):
    import torch

    from oracle.oracle import RefKern

    case, s = _solver(prec)
    try:
        dev, n = _mirror(s)
        p, tool = case["params"], case["tool"]
        dx, t = p["dx"], N0 * case["dt"]
        # the reference's contact pass on the mirror: a voxel cylinder of the
        # tool's radius at the tool's pose of step N0, contact radius 1.5 dx
        R = tool["radius"]
        voxel = dx / 2
        half = int(np.ceil((R + 4 * dx) / voxel))
        dims = (2 * half, 48, 2 * half)
        origin = (-half * voxel, -(4 * dx + tool["position"][1]), -half * voxel)
        sdf = {"v": cylinder_sdf(R, voxel, dims, origin), "origin": origin, "voxel": voxel}
        args = dict(cx=tool["position"][0] + tool["velocity"][0] * t, cy=tool["position"][1],
                    cz=tool["position"][2] + tool["velocity"][2] * t, cos_a=1.0, sin_a=0.0, radius=1.5 * dx,
                    friction=0.3, heat_partition=0.5, dt=case["dt"], cp=p["cp"], rho_phys=p["rho_phys"], Tm=p["Tm"])
        cnt, work, force = RefKern().contact_sdf_device(sdf, args, dev.data_ptr(), n)
        assert cnt > 20
        # CFD-like writes: drag into ext_f, cooling, a few chips
        rec = dev.cpu().numpy().view(A.MPM_PARTICLE).copy()
        rng = np.random.default_rng(11)
        live = np.flatnonzero((rec["status"] == A.ACTIVE) | (rec["status"] == A.CHIP))
        drag = rng.choice(live, len(live) // 5, replace=False)
        for k in ("ext_fx", "ext_fy", "ext_fz"):
            rec[k][drag] = rng.normal(0.0, 1e-3, len(drag))
        cool = rng.choice(live, 40, replace=False)
        rec["temperature"][cool] = np.maximum(rec["temperature"][cool] - 5.0, p["Tamb"])
        chip = rng.choice(np.flatnonzero(rec["status"] == A.ACTIVE), 12, replace=False)
        rec["status"][chip] = A.CHIP
        dev.copy_(torch.from_numpy(rec.view(np.uint8).ravel()).to("cuda"))
        s.import_aos(dev.data_ptr(), A.AOS_WRITABLE, dev.numel())
        s.step(case["dt"], N1)
        out = s.download()
    finally:
        s.close()
    st = _state_from_records(rec)
    extf = np.stack([rec["ext_fx"], rec["ext_fy"], rec["ext_fz"]], axis=1)
    ref, rc = oracle.step(case, st, N1, step0=N0, t0=N0 * case["dt"], extf=extf)
    assert rc == 0
    err = field_errors(out, ref, case)
    if prec == A.PREC_F64:
        assert (out["status"] == ref["status"]).all()
        bad = {k: v for k, v in err.items() if v > 1e-9}
    else:
        assert (out["status"] == ref["status"]).mean() >= 0.999
        bad = {k: v for k, v in err.items() if v > FP32_TOL.get(k, 2e-3)}
    assert not bad, (bad, err)


def test_status_outside_range_is_refused_and_kept():
    case, s = _solver(A.PREC_F64)
    try:
        before = s.download()
        rec = s.export_aos().view(A.MPM_PARTICLE).copy()
        rec["status"][5] = 9
        rec["vx"][5] += 1.0
        with pytest.raises(RuntimeError, match="status outside"):
            s.import_aos(rec.view(np.uint8), A.AOS_WRITABLE)
        after = s.download()
    finally:
        s.close()
    assert after["status"][5] == before["status"][5]
    assert after["vx"][5] == before["vx"][5] + 1.0


def test_imported_ext_force_equals_apply_external_force():
    case, st, n, extf = SCENARIOS["plastic_damage_chip"]()
    c, r, f = (3e-4, 2e-4, 3e-4), 3e-4, (0.0, 0.0, -2e-2)

    def run(mode):
        s = Solver(W.to_mpm_params(case, precision=A.PREC_F64), len(st["x"]) + 64)
        try:
            s.set_tool(case["tool"])
            s.upload(st)
            s.step(case["dt"], N0)
            if mode == "import":
                rec = s.export_aos().view(A.MPM_PARTICLE).copy()
                d = np.sqrt((rec["x"] - c[0]) ** 2 + (rec["y"] - c[1]) ** 2 + (rec["z"] - c[2]) ** 2)
                on = ((rec["status"] == A.ACTIVE) | (rec["status"] == A.CHIP)) & (d < r)
                assert on.sum() > 10
                w = np.where(on, 1.0 - d / r, 0.0)
                for k, fk in zip(("ext_fx", "ext_fy", "ext_fz"), f):
                    rec[k] = fk * w
                s.import_aos(rec.view(np.uint8), A.AOS_EXT_FORCE)
            elif mode == "apply":
                s.apply_external_force(c, r, f)
            s.step(case["dt"], N1)
            return s.download()
        finally:
            s.close()

    a, b, none = run("import"), run("apply"), run("none")
    assert (a["status"] == b["status"]).all()
    err = field_errors(a, b, case)
    assert max(err.values()) < 1e-9, err
    # the force acted: the run without it differs
    assert max(field_errors(none, b, case).values()) > 1e-6
