"""Seeded scenarios used for the golden fixtures and the parity tests.

Each scenario returns (case, state, nsteps, extf) where `state` is a full
particle state (every MPMParticle field) and extf an optional one-step
external force per particle.  The scenarios are chosen to drive every branch
of the reference step (src/MPMSolver.cu): tool contact through the raster
boundary, Johnson-Cook yield with heating and damage, stress degradation,
CHIP transition, chip separation and fracture, the kill zone, the fixture
layer, FIXED and BOUNDARY particles, LOD zones, kinematic hardening and the
one-step external force.
"""
from __future__ import annotations

import numpy as np

from mpm_b200 import capi as A, workpiece as W


def _base(cells=(12, 8, 8), **kw):
    args = dict(cells=cells, speed=20.0, steps=10)
    args.update(kw)
    return W.config1(**args)


def elastic_raster():
    case = _base(tool_mode=A.TOOL_RASTER)
    case["tool"]["samples"] = W.cylinder_samples(case)
    st = W.full_state(W.generate_box(case), case)
    return case, st, 12, None


def plastic_damage_chip():
    """Soft material, fast tool moving down and along x: yield, heating,
    damage, stress degradation, CHIP transition, chip separation, fracture."""
    case = _base(tool_mode=A.TOOL_RASTER, speed=60.0)
    p = case["params"]
    p.update(jc_A=20e6, jc_B=40e6, jc_n=0.5, D1=0.002, D2=0.01, D3=-1.0, D4=0.01, D5=0.5, D_th=0.02)
    case["tool"]["velocity"] = (60.0, 0.0, -15.0)
    case["tool"]["samples"] = W.cylinder_samples(case)
    st = W.full_state(W.generate_box(case), case)
    return case, st, 24, None


def boundary_mix():
    """No tool; kill zone, fixture damping, FIXED/BOUNDARY/CHIP particles,
    pre-deformed F and F_p, nonzero C, stress, damage near and above the
    fracture threshold, random velocities."""
    case = _base(tool_mode=A.TOOL_NONE)
    p = case["params"]
    p.update(jc_A=150e6, jc_B=100e6, fixture_thickness=8 * p["dx"])
    rng = np.random.default_rng(7)
    st = W.full_state(W.generate_box(case), case)
    n = len(st["x"])
    st["vx"] = rng.normal(0, 0.5, n)
    st["vy"] = rng.normal(0, 0.5, n)
    st["vz"] = rng.normal(0, 0.5, n)
    # smooth pre-deformation (a uniform stretch plus small noise) so that the
    # explicit step stays stable over the scenario
    F = np.tile((np.eye(3) + np.diag([1e-3, -4e-4, -4e-4])).reshape(1, 9), (n, 1)) + rng.normal(0, 2e-5, (n, 9))
    Fp = np.tile(np.eye(3).reshape(1, 9), (n, 1)) + rng.normal(0, 1e-5, (n, 9))
    st["F"], st["Fp"] = F, Fp
    st["C"] = rng.normal(0, 1e2, (n, 9))
    st["stress"] = rng.normal(0, 5e7, (n, 6))
    st["plastic_strain"] = rng.uniform(0, 0.2, n)
    st["strain_rate"] = rng.uniform(0, 1e5, n)
    st["temperature"] = p["Tamb"] + rng.uniform(0, 800, n)
    st["damage"] = rng.uniform(0, 1.6, n) * p["D_th"]
    st["residual_stress"] = rng.uniform(0, 1e8, n)
    stat = st["status"].copy()
    pick = rng.uniform(0, 1, n)
    stat[(pick < 0.05) & (stat == A.ACTIVE)] = A.BOUNDARY
    stat[(pick > 0.93) & (stat == A.ACTIVE)] = A.CHIP
    stat[(pick > 0.90) & (pick <= 0.91)] = A.INACTIVE
    st["status"] = stat
    # push a few particles into the kill zone (next to the domain edge)
    edge = rng.choice(n, 20, replace=False)
    st["x"][edge] = p["origin"][0] + rng.uniform(0.2, 1.5, 20) * p["dx"]
    return case, st, 10, None


def sphere_force(st, center, radius, force):
    """Per-particle force of applyExternalForceKernel (src/MPMSolver.cu:611-631):
    force * (1 - d/R) inside the sphere, ACTIVE and CHIP particles only."""
    d = np.sqrt((st["x"] - center[0]) ** 2 + (st["y"] - center[1]) ** 2 + (st["z"] - center[2]) ** 2)
    w = np.where((d < radius) & ((st["status"] == A.ACTIVE) | (st["status"] == A.CHIP)), 1.0 - d / radius, 0.0)
    return np.stack([force[0] * w, force[1] * w, force[2] * w], axis=1)


def lod_kinematic_extf():
    """LOD zones around the tool tip, kinematic hardening, a one-step external
    force (the reference's sphere form)."""
    case = _base(tool_mode=A.TOOL_RASTER, speed=30.0)
    p = case["params"]
    p.update(lod_enabled=1, lod_active_r=3 * p["dx"], lod_near_r=6 * p["dx"], H_kin=5e9, jc_A=60e6, jc_B=80e6)
    case["tool"]["samples"] = W.cylinder_samples(case)
    st = W.full_state(W.generate_box(case), case)
    dx = p["dx"]
    case["ext"] = dict(center=(8 * dx, 4 * dx, 4 * dx), radius=4 * dx, force=(3e-4, -1e-4, 2e-4))
    extf = sphere_force(st, **case["ext"])
    return case, st, 10, extf


def adiabatic_shear():
    """The adiabatic shear model on (AdiabaticShearModel::update after g2p):
    the plastic_damage_chip tool path in degC with the reference's 25 degC
    ambient and 0.5 degC touch guard.  Initial temperatures straddle the guard
    (some exactly at 25.5) and a few lie near the 0.9 Tm cap, so that heating,
    the counter ramp and localisation, the decay, the cap and the CHIP reset
    all occur.  Counters start at 0."""
    case, st, n, _ = plastic_damage_chip()
    p = case["params"]
    p.update(Tamb=25.0, Tm=1660.0, asb_enabled=1, asb_critical_rate=1e4, asb_taylor_quinney=0.9,
             asb_max_temp_ratio=0.9, asb_touch_rise=0.5)
    rng = np.random.default_rng(11)
    nn = len(st["x"])
    pick = rng.uniform(0, 1, nn)
    T = np.where(pick < 0.3, 25.0, np.where(pick < 0.4, 25.5, 25.0 + rng.uniform(0.5, 400.0, nn)))
    T = np.where(pick > 0.98, rng.uniform(1480.0, 1500.0, nn), T)
    st["temperature"] = T
    st["asb"] = np.zeros(nn, np.int32)
    return case, st, n, None


def heat_conduction():
    """Grid heat conduction on (MPMWorkpieceSolver's scatter, diffusion and
    gather on this solver's weights): the plastic_damage_chip tool path with
    hot spots (up to 600 K above ambient) and a conductivity that makes
    alpha dt / dx^2 = 0.05, so that both the diffusion step and the
    temperature gather move temperatures.  The reference's MPMSolver conducts
    no heat, so this scenario is checked against the oracle only."""
    case, st, n, _ = plastic_damage_chip()
    p = case["params"]
    alpha = 0.05 * p["dx"] ** 2 / case["dt"]
    p.update(heat_conduction=1, thermal_conductivity=alpha * p["rho_phys"] * p["cp"])
    rng = np.random.default_rng(13)
    nn = len(st["x"])
    hot = rng.uniform(0, 1, nn) < 0.2
    st["temperature"] = p["Tamb"] + np.where(hot, rng.uniform(0.0, 600.0, nn), 0.0)
    return case, st, n, None


def workpiece_solver():
    """MPMWorkpieceSolver's semantics (src/MPMWorkpieceSolver.cu:98-400,
    :667-725): trilinear PIC, hypoelastic stress with the Johnson-Cook return
    at the old plastic strain, nearest-sample normal projection with contact
    heating.  The soft plastic_damage_chip workpiece flies at -30 m/s in x
    (with noise) into the cylinder's surface samples, so that nodes meet the
    tool with an approaching normal velocity; kinematic hardening; a particle
    force on a tenth of the particles; damage from the strain rate (failure
    strain 0.005, threshold 1) reaching degradation and CHIP, and chip
    separation on even steps.  Conduction off (k = 0): the reference's diffusion updates its grid
    in place, so its result depends on the thread schedule; the diffusion is
    pinned on its own (kernels/heat_diffusion.npz)."""
    case, st, n, _ = plastic_damage_chip()
    p = case["params"]
    p.update(H_kin=2e9, thermal_conductivity=0.0, D_th=1.0)
    case["ws"] = dict(failure_strain=0.005, critical_plastic_strain=0.3, thermal_chip_ratio=0.98,
                      tool_contact_radius=1.5 * p["dx"], contact_damping=0.15, max_contact_temp_rise=25.0,
                      thermal_clamp=1)
    rng = np.random.default_rng(29)
    nn = len(st["x"])
    st["vx"] = -30.0 + rng.normal(0.0, 2.0, nn)
    st["vy"] = rng.normal(0.0, 2.0, nn)
    st["vz"] = rng.normal(0.0, 2.0, nn)
    pick = rng.uniform(0, 1, nn) < 0.1
    extf = np.zeros((nn, 3))
    extf[pick] = rng.normal(0.0, 2e-4, (int(pick.sum()), 3))
    return case, st, 16, extf


# MPMWorkpieceSolver's semantics (the reference's other MPM solver).
WS_SCENARIOS = {
    "workpiece_solver": workpiece_solver,
}

SCENARIOS = {
    "elastic_raster": elastic_raster,
    "plastic_damage_chip": plastic_damage_chip,
    "boundary_mix": boundary_mix,
    "lod_kinematic_extf": lod_kinematic_extf,
    "adiabatic_shear": adiabatic_shear,
}

# Scenarios of this build's extensions that the reference's MPMSolver does not
# have: parity against the oracle only (no reference-kernel fixture).
ORACLE_ONLY = {
    "heat_conduction": heat_conduction,
}

PARITY_SCENARIOS = {**SCENARIOS, **ORACLE_ONLY}
