"""Generates tests/golden/*.npz from the REFERENCE's own CUDA kernels.

    python tests/golden/make_golden.py [outdir] [scenario ...]

Needs a GPU and oracle/_ref/libmpm_ref.so (the reference's src/MPMSolver.cu
and src/AdiabaticShearModel.cu built from their sources by oracle/Makefile).
For every scenario of scenarios.py (or the ones named) it stores the input
state, the reference's state after n steps, and the reference's own stats
kernel (computeParticleStatsKernel) on it.  The reference kernels accumulate
with FP64 atomics, so two runs differ in the last bits; the run-to-run spread
of the reference is stored too.

kernels/asb_heating.npz holds one pass of the reference's adiabatic shear
kernels (detectShearBandsKernel + applyAdiabaticHeatingKernel) over crafted
particles that reach every branch (asb_pass_inputs); it is written when no
scenario is named or when "asb_pass" is.

kernels/tex_probe.npz holds hardware texture fetches through the reference's
SDF texture setup (ToolSDF::createTexture) at crafted coordinates, and
kernels/contact_sdf.npz one launch of the reference's xpbdContactSDFKernel
(src/ContactSolver.cu) on a sampled cylinder SDF with crafted particles
(tex_probe_inputs, contact_pass_inputs); written when no scenario is named or
when "contact_pass" is.

kernels/heat_diffusion.npz holds one launch of the reference's grid heat
diffusion kernel (mpmDiffuseTemperatureKernel, src/MPMWorkpieceSolver.cu) on a
crafted grid (heat_pass_inputs); written when no scenario is named or when
"heat_pass" is.  The kernel updates the grid in place, so in general its result
depends on the thread schedule; on this grid every node it updates (mass >=
1e-15) has only neighbours it never updates, so the result is deterministic.

workpiece_solver.npz holds the reference's MPMWorkpieceSolver kernels
(src/MPMWorkpieceSolver.cu) stepped on the scenario of that name
(scenarios.WS_SCENARIOS); written when no scenario is named or when it is.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1] / "edegpredict-engine-rotary_b200"))
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))

from oracle.oracle import RefKern  # noqa: E402
from scenarios import SCENARIOS, WS_SCENARIOS  # noqa: E402

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "stress", "backstress", "plastic_strain", "strain_rate",
          "temperature", "damage", "residual_stress", "status", "id", "asb")

ASB_DT = 1e-8


def asb_pass_inputs():
    """Crafted particles for one adiabatic shear pass: every status, the
    temperature guard (below, exactly at and above 25.5 degC), strain rates
    below, at and above the 5000 /s floor and the 1e4 /s critical rate,
    counters 0..10, temperatures near and above the 0.9 Tm cap, stresses up to
    2 GPa."""
    case = {"params": dict(nx=8, ny=8, nz=8, dx=1e-4, origin=(0.0, 0.0, 0.0), E=113.8e9, nu=0.34,
                           rho_phys=4430.0, cp=526.3, beta=0.9, Tm=1660.0, Tamb=25.0, jc_A=1e9, jc_B=1e9,
                           jc_n=0.3, jc_C=0.01, jc_m=1.0, edot0=1.0, H_kin=0.0, D1=0.05, D2=3.44, D3=-2.12,
                           D4=0.002, D5=0.61, D_th=1.0, fixture_thickness=0.0, fixture_damping=1e7,
                           gravity_z=-9.81, mass_threshold=1e-12, apic_dinv_factor=3.0, apic_decay=0.99,
                           lod_enabled=0, lod_active_r=0.0, lod_near_r=0.0, deps_cap=0.05, dT_cap=50.0,
                           newton_tol=1e-12, plasticity=0, chip_every=2, newton_maxit=60, particle_mass=1e-9,
                           particle_volume=1e-13, asb_enabled=1, asb_critical_rate=1e4, asb_taylor_quinney=0.9,
                           asb_max_temp_ratio=0.9, asb_touch_rise=0.5),
            "tool": {"mode": 0}}
    rng = np.random.default_rng(23)
    n = 4096
    z = np.zeros(n)
    eye = np.tile(np.eye(3).reshape(1, 9), (n, 1))
    status = rng.choice([0, 0, 0, 0, 0, 0, 1, 2, 3, 4], n).astype(np.int32)
    T = rng.choice([24.0, 25.0, 25.5, 25.5000001, 30.0, 300.0, 1000.0, 1493.9, 1500.0], n) + \
        np.where(rng.uniform(0, 1, n) < 0.5, rng.uniform(0, 5, n), 0.0)
    edot = rng.choice([0.0, 4999.0, 5000.0, 7000.0, 1e4, 1.00001e4, 2e4, 5e4, 1e6], n) * \
        np.where(rng.uniform(0, 1, n) < 0.3, rng.uniform(0.9, 1.1, n), 1.0)
    st = dict(x=z.copy(), y=z.copy(), z=z.copy(), vx=z.copy(), vy=z.copy(), vz=z.copy(), F=eye.copy(),
              Fp=eye.copy(), C=np.zeros((n, 9)), stress=rng.uniform(-2e9, 2e9, (n, 6)) *
              rng.choice([0.0, 1e-3, 1.0], (n, 1)), backstress=np.zeros((n, 6)), plastic_strain=z.copy(),
              strain_rate=edot, temperature=T, damage=z.copy(), residual_stress=z.copy(), status=status,
              id=np.arange(n, dtype=np.int32), asb=rng.integers(0, 11, n).astype(np.int32))
    return case, st


HEAT_DT = 1e-6


def tex_probe_inputs():
    """Random texels on a 9x7x5 grid and fetch points: random ones (some
    outside the grid, where clamping applies), texel centres and integers."""
    rng = np.random.default_rng(41)
    v = rng.uniform(-1.0, 1.0, (5, 7, 9)).astype(np.float32)
    n = np.array([9, 7, 5], np.float32)
    pts = [rng.uniform(-1.5, 1.0, (3000, 3)) * 1.0 + rng.uniform(0, 1, (3000, 3)) * (n + 1.0)]
    pts.append(rng.integers(0, 9, (200, 3)) + 0.5)
    pts.append(rng.integers(-1, 10, (200, 3)).astype(np.float64))
    xyz = np.concatenate(pts).astype(np.float32)
    return {"v": v, "origin": (0.0, 0.0, 0.0), "voxel": 1.0}, xyz


def cylinder_sdf(R: float, voxel: float, dims, origin):
    """A cylinder of radius R along y, centred on the rest frame's origin,
    sampled at voxel centres (float32 [nz, ny, nx])."""
    nx, ny, nz = dims
    xc = origin[0] + (np.arange(nx) + 0.5) * voxel
    zc = origin[2] + (np.arange(nz) + 0.5) * voxel
    r = np.sqrt(xc[None, :] ** 2 + zc[:, None] ** 2) - R
    return np.ascontiguousarray(np.broadcast_to(r[:, None, :], (nz, ny, nx)), dtype=np.float32)


def contact_pass_inputs():
    """A 40x20x40 cylinder SDF (R = 0.3 mm, 20 um voxels) under a tool
    transform (translated, rotated 0.3 rad about z) and 4000 particles within
    +-3 voxels of its surface, a few outside the grid, all statuses; contact
    radius 2 voxels, friction 0.3, heat partition 0.5, dt 1e-5 (so that the
    friction cap binds for some particles and not for others)."""
    case, _ = asb_pass_inputs()
    voxel, R = 2e-5, 3e-4
    dims = (40, 20, 40)
    origin = (-20 * voxel, -10 * voxel, -20 * voxel)
    sdf = {"v": cylinder_sdf(R, voxel, dims, origin), "origin": origin, "voxel": voxel}
    ang = 0.3
    args = dict(cx=1e-3, cy=5e-4, cz=8e-4, cos_a=np.cos(ang), sin_a=np.sin(ang), radius=2 * voxel, friction=0.3,
                heat_partition=0.5, dt=1e-5, cp=526.3, rho_phys=4430.0, Tm=1878.0)
    rng = np.random.default_rng(43)
    n = 4000
    th = rng.uniform(0, 2 * np.pi, n)
    r = R + rng.uniform(-3, 3, n) * voxel
    lx, ly, lz = r * np.cos(th), rng.uniform(-8, 8, n) * voxel, r * np.sin(th)
    ly[:40] = 12 * voxel                     # outside the grid along y
    wx = lx * args["cos_a"] - ly * args["sin_a"] + args["cx"]
    wy = lx * args["sin_a"] + ly * args["cos_a"] + args["cy"]
    wz = lz + args["cz"]
    z = np.zeros(n)
    eye = np.tile(np.eye(3).reshape(1, 9), (n, 1))
    st = dict(x=wx, y=wy, z=wz, vx=rng.uniform(-3, 3, n), vy=rng.uniform(-3, 3, n), vz=rng.uniform(-3, 3, n),
              F=eye.copy(), Fp=eye.copy(), C=np.zeros((n, 9)), stress=np.zeros((n, 6)), backstress=np.zeros((n, 6)),
              plastic_strain=z.copy(), strain_rate=z.copy(), temperature=300.0 + rng.uniform(0, 500, n),
              damage=z.copy(), residual_stress=z.copy(),
              status=rng.choice([0, 0, 0, 0, 0, 0, 1, 2, 3, 4], n).astype(np.int32), id=np.arange(n, dtype=np.int32))
    return case, st, sdf, args


def write_contact_pass(rk, outdir: Path) -> None:
    d = outdir / "kernels"
    d.mkdir(parents=True, exist_ok=True)
    sdf, xyz = tex_probe_inputs()
    np.savez_compressed(d / "tex_probe.npz", v=sdf["v"], xyz=xyz, out=rk.tex_probe(sdf, xyz))
    case, st, sdf, args = contact_pass_inputs()
    out, (cnt, heat, force) = rk.contact_sdf(case, st, sdf, args)
    keys = ("x", "y", "z", "vx", "vy", "vz", "temperature")
    np.savez_compressed(d / "contact_sdf.npz", **{f"out_{k}": out[k] for k in keys},
                        metrics=np.array([cnt, heat, force], np.float64))
    print(f"contact_pass: n={len(st['x'])} contacts={cnt} work={heat:.3e} force={force:.3e}")


def heat_pass_inputs():
    """A 12x10x8 grid for one diffusion step: nodes of even parity i+j+k carry
    1e-9..1e-8 kg (updated), a few of them below 1e-15 (kept); odd nodes carry
    none (an empty neighbour counts as T = 0), 1e-16 or 1e-20 kg (never
    updated).  Temperatures 300..1500 on every massive node; alpha dt / dx^2 =
    0.05."""
    case, _ = asb_pass_inputs()
    p = case["params"]
    nx, ny, nz, dx = 12, 10, 8, 1e-4
    alpha = 0.05 * dx * dx / HEAT_DT
    p.update(nx=nx, ny=ny, nz=nz, dx=dx, heat_conduction=1,
             thermal_conductivity=alpha * p["rho_phys"] * p["cp"])
    rng = np.random.default_rng(31)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    even = ((i + j + k) % 2 == 0).ravel()
    n = nx * ny * nz
    mass = np.where(even, rng.uniform(1e-9, 1e-8, n), rng.choice([0.0, 0.0, 1e-16, 1e-20], n))
    mass = np.where(even & (rng.uniform(0, 1, n) < 0.05), 1e-16, mass)
    T = rng.uniform(300.0, 1500.0, n)
    return case, mass, T * mass


def write_heat_pass(rk, outdir: Path) -> None:
    case, mass, tm = heat_pass_inputs()
    out = rk.heat_diffuse(case, mass, tm, HEAT_DT)
    d = outdir / "kernels"
    d.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(d / "heat_diffusion.npz", mass=mass, tm_in=tm, tm_out=out, dt=np.array(HEAT_DT))
    print(f"heat_pass: nodes={len(mass)} updated={int((mass >= 1e-15).sum())} "
          f"changed={int((out != tm).sum())}")


def write_asb_pass(rk, outdir: Path) -> None:
    case, st = asb_pass_inputs()
    out = rk.asb_heat(case, st, ASB_DT)
    d = outdir / "kernels"
    d.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(d / "asb_heating.npz", in_status=st["status"], in_temperature=st["temperature"],
                        in_strain_rate=st["strain_rate"], in_stress=st["stress"], in_asb=st["asb"],
                        out_temperature=out["temperature"], out_asb=out["asb"], dt=np.array(ASB_DT))
    moved = int((out["temperature"] != st["temperature"]).sum())
    print(f"asb_pass: n={len(st['status'])} heated={moved} counters changed={int((out['asb'] != st['asb']).sum())}")


WS_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "stress", "backstress", "plastic_strain", "strain_rate", "temperature",
             "damage", "residual_stress", "status", "id")


def write_ws(rk, outdir: Path, name: str, fn) -> None:
    """The reference's MPMWorkpieceSolver kernels on a scenario: input and
    output state, the last step's contact force, the run-to-run spread."""
    case, st, n, extf = fn()
    out1, f1 = rk.ws_step(case, st, n, extf=extf.copy())
    out2, f2 = rk.ws_step(case, st, n, extf=extf.copy())
    spread = {k: float(np.abs(out1[k].astype(float) - out2[k].astype(float)).max()) for k in WS_FIELDS}
    arrays = {f"in_{k}": np.asarray(st[k]) for k in WS_FIELDS}
    arrays.update({f"out_{k}": np.asarray(out1[k]) for k in WS_FIELDS})
    arrays["extf"] = extf
    arrays["contact_force"] = np.array([f1, f2])
    meta = {"nsteps": n, "spread": spread}
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    (outdir / "workpiece").mkdir(parents=True, exist_ok=True)
    np.savez_compressed(outdir / "workpiece" / f"{name}.npz", **arrays)
    print(f"{name}: n={len(st['x'])} steps={n} chips={int((out1['status'] == 2).sum())} "
          f"max_eps={out1['plastic_strain'].max():.3e} max_D={out1['damage'].max():.3e} "
          f"contact_force={f1:.3e} spread_x={spread['x']:.2e}")


def main(outdir: Path, names=None) -> None:
    rk = RefKern()
    outdir.mkdir(parents=True, exist_ok=True)
    if not names or "asb_pass" in names:
        write_asb_pass(rk, outdir)
    if not names or "heat_pass" in names:
        write_heat_pass(rk, outdir)
    if not names or "contact_pass" in names:
        write_contact_pass(rk, outdir)
    for name, fn in WS_SCENARIOS.items():
        if not names or name in names:
            write_ws(rk, outdir, name, fn)
    for name, fn in SCENARIOS.items():
        if names and name not in names:
            continue
        case, st, n, extf = fn()
        st["lod"] = np.zeros(len(st["x"]), np.int32)
        st.setdefault("asb", np.zeros(len(st["x"]), np.int32))
        out1 = rk.step(case, st, n, extf=extf)
        out2 = rk.step(case, st, n, extf=extf)
        spread = {k: float(np.abs(out1[k].astype(float) - out2[k].astype(float)).max()) for k in FIELDS if k in out1}
        stats = rk.stats(case, out1)
        arrays = {f"in_{k}": np.asarray(st[k]) for k in FIELDS}
        arrays.update({f"out_{k}": np.asarray(out1[k]) for k in FIELDS})
        if extf is not None:
            arrays["extf"] = extf
        arrays["ref_stats"] = stats
        meta = {"nsteps": n, "spread": spread,
                "case": {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in case.items() if k != "tool"},
                "tool": {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in case["tool"].items()}}
        arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
        np.savez_compressed(outdir / f"{name}.npz", **arrays)
        n_chip = int((out1["status"] == 2).sum())
        print(f"{name}: n={len(st['x'])} steps={n} chips={n_chip} inactive={int((out1['status'] == 1).sum())} "
              f"max_eps={out1['plastic_strain'].max():.3e} spread_x={spread['x']:.2e}")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE, sys.argv[2:])
