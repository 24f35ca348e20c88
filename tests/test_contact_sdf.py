"""The reference's SDF contact kernel (xpbdContactSDFKernel,
src/ContactSolver.cu:797-923) on a voxel tool SDF sampled through a 3D texture
set up as ToolSDF::createTexture does.  The oracle restates the kernel with
its float/double arithmetic and emulates the texture unit's trilinear
filtering.

- CPU: the filtering emulation against hardware fetches through the
  reference's texture setup (tests/golden/kernels/tex_probe.npz): exact up to
  float accumulation;
- CPU: the oracle's contact pass against the reference kernel's own output on
  a sampled cylinder with 4000 particles (tests/golden/kernels/contact_sdf.npz).
  The reference is built with --use_fast_math, so its float voxel
  coordinates can land on the other side of a 1/256 weight step than IEEE
  arithmetic does.  A sampled distance then differs by one step (at most
  1/256 of a voxel), so: counts equal; sums to 1e-5; every particle within
  one step (positions 1/128 voxel, velocities and heating 2e-3); 99.5 % of
  particles within 1e-5;
- GPU: both against the reference live.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE / "golden"))
from make_golden import contact_pass_inputs, tex_probe_inputs  # noqa: E402

K = HERE / "golden" / "kernels"


def check_contact(out, metrics, ref, ref_metrics, st, voxel):
    assert metrics[0] == ref_metrics[0] and metrics[0] > 1000
    assert abs(metrics[1] - ref_metrics[1]) <= 1e-5 * ref_metrics[1]
    assert abs(metrics[2] - ref_metrics[2]) <= 1e-5 * ref_metrics[2]
    ep = np.sqrt(sum((out[k] - ref[k]) ** 2 for k in ("x", "y", "z"))) / voxel
    vmax = max(np.abs(ref[k]).max() for k in ("vx", "vy", "vz"))
    ev = np.sqrt(sum((out[k] - ref[k]) ** 2 for k in ("vx", "vy", "vz"))) / vmax
    rise = np.abs(ref["temperature"] - st["temperature"]).max()
    eT = np.abs(out["temperature"] - ref["temperature"]) / rise
    for e, one_step in ((ep, 1.0 / 128), (ev, 2e-3), (eT, 2e-3)):
        assert e.max() <= one_step, e.max()
        assert (e <= 1e-5).mean() >= 0.995, (e <= 1e-5).mean()


def test_fixtures_present():
    assert (K / "tex_probe.npz").exists() and (K / "contact_sdf.npz").exists(), \
        "run tests/golden/make_golden.py on a GPU (contact_pass)"


def test_texture_emulation_matches_hardware(oracle):
    d = np.load(K / "tex_probe.npz")
    sdf, xyz = tex_probe_inputs()
    assert np.array_equal(sdf["v"], d["v"]) and np.array_equal(xyz, d["xyz"])
    assert np.abs(oracle.tex3d(sdf, xyz) - d["out"]).max() < 1e-6


def test_oracle_contact_matches_reference_fixture(oracle):
    d = np.load(K / "contact_sdf.npz")
    case, st, sdf, args = contact_pass_inputs()
    out, m = oracle.contact_sdf(case, st, sdf, args)
    ref = {k: d[f"out_{k}"] for k in ("x", "y", "z", "vx", "vy", "vz", "temperature")}
    check_contact(out, m, ref, tuple(d["metrics"]), st, sdf["voxel"])
    # untouched particles: INACTIVE, FIXED and those out of reach keep their state
    moved = np.abs(out["x"] - st["x"]) > 0
    assert not moved[(st["status"] == 1) | (st["status"] == 4)].any()


@pytest.mark.gpu
def test_texture_emulation_matches_hardware_live(oracle):
    from oracle.oracle import RefKern
    sdf, xyz = tex_probe_inputs()
    assert np.abs(oracle.tex3d(sdf, xyz) - RefKern().tex_probe(sdf, xyz)).max() < 1e-6


@pytest.mark.gpu
def test_reference_contact_matches_oracle_live(oracle):
    from oracle.oracle import RefKern
    case, st, sdf, args = contact_pass_inputs()
    ref, rm = RefKern().contact_sdf(case, st, sdf, args)
    out, m = oracle.contact_sdf(case, st, sdf, args)
    check_contact(out, m, ref, rm, st, sdf["voxel"])
