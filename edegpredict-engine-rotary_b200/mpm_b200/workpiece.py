"""Synthetic workpieces: material rows, the benchmark configurations and a numpy
mirror of the device-side seeded generator.

A *case* is a plain dict:
    params : mpm_params field values (names as in include/mpm_capi.h)
    tool   : rigid tool (mode, shape, position, velocity, radius, rake,
             clearance, tip_dz[, samples])
    box    : generator box (c0, c1, ppc, seed, instance, fixed_layers, T0)
    dt, steps
The same case drives the CUDA path (through the C ABI) and the oracle.

Workpiece geometry (all configs): the box occupies cells [0, W) on each axis
in world coordinates starting at 0; the grid origin is 4 cells below it on
-x, -y, -z, with 8 cells of pad on +x, 4 on +y and a top pad that clears the
tool.  The bottom `fixed_layers` cell layers are FIXED_BOUNDARY, and the
fixture damping zone spans the pad below the workpiece plus those layers.
"""
from __future__ import annotations

import math
from typing import Dict, Optional

import numpy as np

from . import _capi as A

# ----------------------------------------------------------------- materials

# AISI 4340 (config 1): Johnson-Cook flow row as given; damage constants are
# Johnson & Cook's published 4340 set; cp 475 J/kgK.
AISI_4340 = dict(E=205e9, nu=0.29, rho_phys=7850.0, cp=475.0, beta=0.9, Tm=1793.0, Tamb=293.0,
                 jc_A=792e6, jc_B=510e6, jc_n=0.26, jc_C=0.014, jc_m=1.03, edot0=1.0, H_kin=0.0,
                 D1=0.05, D2=3.44, D3=-2.12, D4=0.002, D5=0.61, D_th=1.0)
# Ti-6Al-4V (configs 2 and 4); damage constants: the widely used Lesuer set;
# cp 526.3 J/kgK (the reference's Ti-6Al-4V default, include/Types.h:517).
TI_6AL_4V = dict(E=113.8e9, nu=0.34, rho_phys=4430.0, cp=526.3, beta=0.9, Tm=1878.0, Tamb=293.0,
                 jc_A=1098e6, jc_B=1092e6, jc_n=0.93, jc_C=0.014, jc_m=1.1, edot0=1.0, H_kin=0.0,
                 D1=-0.09, D2=0.25, D3=-0.5, D4=0.014, D5=3.87, D_th=1.0)

# Kinematics and boundary constants of the reference step (src/MPMSolver.cu:16,
# :174-175, :255, :315, :578-592, :890, :1160).
REFERENCE_KINEMATICS = dict(fixture_damping=1e7, gravity_z=-9.81, mass_threshold=1e-12, apic_dinv_factor=3.0,
                            apic_decay=0.99, deps_cap=0.05, dT_cap=50.0, lod_enabled=0, lod_active_r=0.002,
                            lod_near_r=0.01, chip_every=2, plasticity=A.PLAST_EXPLICIT, newton_tol=1e-12,
                            newton_maxit=60)

PAD_LO = 4
PAD_X_HI = 8
PAD_Y_HI = 4


def make_case(cells, dx, ppc, material, tool_kind, *, doc, speed, radius, steps, cfl=0.3, seed=1234,
              instance=0, fixed_layers=2, rake=0.0, clearance=math.radians(7.0), tool_x_cells=16.0,
              tool_mode=A.TOOL_SDF_STICKY, precision=A.PREC_F32) -> dict:
    """A box workpiece of `cells` (Wx, Wy, Wz) cells with a rigid tool cutting
    along +x at depth `doc` below its top surface."""
    Wx, Wy, Wz = map(int, cells)
    top = Wz * dx
    if tool_kind == "cylinder":
        shape = A.SHAPE_CYLINDER_Y
        pz = top - doc + radius
        reach = 2.0 * radius + doc
    else:
        shape = A.SHAPE_WEDGE_Y
        pz = top - doc + radius
        reach = 2.0 * radius + doc
    pad_top = int(math.ceil(reach / dx)) + 4
    nx = Wx + PAD_LO + PAD_X_HI + 1
    ny = Wy + PAD_LO + PAD_Y_HI + 1
    nz = Wz + PAD_LO + pad_top + 1
    params = dict(REFERENCE_KINEMATICS)
    params.update(material)
    params.update(nx=nx, ny=ny, nz=nz, dx=dx, origin=(-PAD_LO * dx, -PAD_LO * dx, -PAD_LO * dx),
                  particle_mass=material["rho_phys"] * dx ** 3 / ppc, particle_volume=dx ** 3 / ppc,
                  fixture_thickness=(PAD_LO + fixed_layers) * dx, precision=precision)
    c = math.sqrt(material["E"] / material["rho_phys"])
    tool = dict(mode=tool_mode, shape=shape, position=(tool_x_cells * dx, 0.0, pz), velocity=(speed, 0.0, 0.0),
                radius=radius, rake=rake, clearance=clearance, tip_dz=-radius)
    box = dict(c0=(PAD_LO, PAD_LO, PAD_LO), c1=(PAD_LO + Wx, PAD_LO + Wy, PAD_LO + Wz), ppc=ppc, seed=seed,
               instance=instance, fixed_layers=fixed_layers, T0=material["Tamb"])
    return dict(params=params, tool=tool, box=box, dt=cfl * dx / c, steps=steps, cells=(Wx, Wy, Wz))


def config1(**kw) -> dict:
    """Plain small: 64x32x32 cells, dx 0.05 mm, 8 ppc, AISI 4340, cylinder R 0.5 mm
    at 1.67 m/s, depth of cut 0.1 mm, CFL 0.3, 200 steps."""
    args = dict(cells=(64, 32, 32), dx=5e-5, ppc=8, material=AISI_4340, tool_kind="cylinder", doc=1e-4,
                speed=1.67, radius=5e-4, steps=200)
    args.update(kw)
    return make_case(**args)


def config2(**kw) -> dict:
    """Plain large: 256x128x128 cells, dx 0.02 mm, 8 ppc, Ti-6Al-4V, rounded wedge
    (edge radius 0.3 mm, rake 0, clearance 7 deg) at 2.5 m/s, depth of cut
    0.05 mm, 500 steps."""
    args = dict(cells=(256, 128, 128), dx=2e-5, ppc=8, material=TI_6AL_4V, tool_kind="wedge", doc=5e-5,
                speed=2.5, radius=3e-4, steps=500)
    args.update(kw)
    return make_case(**args)


def config4(**kw) -> dict:
    """Precision study: config 2's geometry and material at 128x64x64 cells, 1000 steps."""
    args = dict(cells=(128, 64, 64), dx=2e-5, ppc=8, material=TI_6AL_4V, tool_kind="wedge", doc=5e-5,
                speed=2.5, radius=3e-4, steps=1000)
    args.update(kw)
    return make_case(**args)


def config3_case(rng: np.random.Generator, index: int, *, cells_lo: int = 16, cells_hi: int = 64, steps: int = 300,
                 dx: float = 2e-5, seed: int = 1234, precision=A.PREC_F32, ppc: Optional[int] = None) -> dict:
    """One instance of the batched sweep: cell count log-uniform in
    [cells_lo^3, cells_hi^3] with aspect ratios (Wx/Wz, Wy/Wz) uniform in
    [1, 4], 4-8 ppc, Johnson-Cook A in [300, 1200] MPa, B in [200, 1100] MPa,
    n in [0.1, 0.9], C in [0.005, 0.03], m in [0.8, 1.4], cutting speed in
    [0.5, 5] m/s, depth of cut in [0.02, 0.2] mm (capped at half the height),
    elastic and thermal rows interpolated between AISI 4340 and Ti-6Al-4V;
    rounded wedge with edge radius 2 x depth of cut at mid-length.  `ppc`
    fixes the particles per cell (the serving workload uses 8)."""
    C = math.exp(rng.uniform(math.log(cells_lo ** 3), math.log(cells_hi ** 3)))
    ax, ay = rng.uniform(1.0, 4.0, 2)
    wz = max(4, int(round((C / (ax * ay)) ** (1.0 / 3.0))))
    wx, wy = max(4, int(round(ax * wz))), max(4, int(round(ay * wz)))
    ppc = int(rng.integers(4, 9)) if ppc is None else int(ppc)
    f = rng.uniform()
    mat = {k: (1.0 - f) * AISI_4340[k] + f * TI_6AL_4V[k] for k in ("E", "nu", "rho_phys", "cp", "Tm")}
    mat.update(beta=0.9, Tamb=293.0, edot0=1.0, H_kin=0.0, D1=0.05, D2=3.44, D3=-2.12, D4=0.002, D5=0.61, D_th=1.0,
               jc_A=rng.uniform(300e6, 1200e6), jc_B=rng.uniform(200e6, 1100e6), jc_n=rng.uniform(0.1, 0.9),
               jc_C=rng.uniform(0.005, 0.03), jc_m=rng.uniform(0.8, 1.4))
    speed = rng.uniform(0.5, 5.0)
    doc = min(rng.uniform(2e-5, 2e-4), 0.5 * wz * dx)
    return make_case((wx, wy, wz), dx, ppc, mat, "wedge", doc=doc, speed=speed, radius=max(2.0 * doc, 2.0 * dx),
                     steps=steps, seed=seed, instance=index, tool_x_cells=wx / 2.0, precision=precision)


def config3(n_instances: int = 512, seed: int = 7, **kw) -> list:
    """The batched sweep: n_instances independent workpieces (config3_case)."""
    rng = np.random.default_rng(seed)
    return [config3_case(rng, i, **kw) for i in range(n_instances)]


def to_mpm_params(case: dict, **over) -> A.MpmParams:
    p = A.default_params()
    vals = dict(case["params"])
    vals.update(over)
    for k, v in vals.items():
        if k == "origin":
            for i in range(3):
                p.origin[i] = float(v[i])
        elif hasattr(p, k):
            f = dict(A.MpmParams._fields_)[k]
            setattr(p, k, int(v) if f is A._i32 else float(v))
    return p


# ----------------------------------------------------------------- generator

_M0, _M1, _W0, _W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox4x32_10(k0: int, k1: int, c0, c1, c2, c3):
    """Philox4x32-10 (Salmon et al., SC'11) on uint32 arrays; returns 4 arrays of
    24-bit uniforms in [0,1) as float32 (same as the device generator)."""
    m = np.uint64(0xFFFFFFFF)
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint64) & m for c in (c0, c1, c2, c3))
    k0, k1 = np.uint64(k0 & 0xFFFFFFFF), np.uint64(k1 & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(_M0) * c0
        p1 = np.uint64(_M1) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & m
        hi1, lo1 = p1 >> np.uint64(32), p1 & m
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & m, lo1, (hi0 ^ c3 ^ k1) & m, lo0
        k0 = (k0 + np.uint64(_W0)) & m
        k1 = (k1 + np.uint64(_W1)) & m
    s = np.float32(1.0 / 16777216.0)
    return tuple((c >> np.uint64(8)).astype(np.float32) * s for c in (c0, c1, c2, c3))


def tool_sdf(tool: dict, x: np.ndarray, z: np.ndarray, pr0: float, pr2: float) -> np.ndarray:
    """Analytic tool SDF (cylinder along y, or rounded wedge extruded along y),
    same arithmetic as the device function tool_sdf."""
    qx, qz = x - pr0, z - pr2
    if tool["shape"] == A.SHAPE_CYLINDER_Y:
        return np.sqrt(qx * qx + qz * qz) - tool["radius"]
    sg, cg = math.sin(tool["rake"]), math.cos(tool["rake"])
    sa, ca = math.sin(tool["clearance"]), math.cos(tool["clearance"])
    t1x, t1z, n1x, n1z = -sg, cg, cg, sg
    t2x, t2z, n2x, n2z = -ca, sa, -sa, -ca
    d1, d2 = n1x * qx + n1z * qz, n2x * qx + n2z * qz
    inside = (d1 <= 0) & (d2 <= 0)
    s1 = np.maximum(qx * t1x + qz * t1z, 0.0)
    s2 = np.maximum(qx * t2x + qz * t2z, 0.0)
    l1 = np.sqrt((qx - s1 * t1x) ** 2 + (qz - s1 * t1z) ** 2)
    l2 = np.sqrt((qx - s2 * t2x) ** 2 + (qz - s2 * t2z) ** 2)
    core = np.where(inside, np.maximum(d1, d2), np.minimum(l1, l2))
    return core - tool["radius"]


# Strata of a cell's candidates for ppc <= 8: its octants in this fixed order
# (mpm_aux.cu, gen_offset).
OCTANT_ORDER = (0, 7, 3, 4, 5, 2, 6, 1)


def gen_offset(k: np.ndarray, ppc: int, u) -> list:
    """Offsets in cells of candidates k of a cell (host mirror of gen_offset,
    mpm_aux.cu): a jittered point of the candidate's stratum, an octant of the
    cell for ppc <= 8 (0.5 bit + 0.5 u, exact), else sub-cell 37 k mod n^3
    of the n^3 grid, n the smallest even number with n^3 >= ppc
    ((s + u) / n)."""
    if ppc <= 8:
        o = np.asarray(OCTANT_ORDER, dtype=np.int64)[k & 7]
        return [0.5 * ((o >> a) & 1).astype(np.float64) + 0.5 * u[a].astype(np.float64) for a in range(3)]
    n = 4
    while n ** 3 < ppc:
        n += 2
    q = (37 * k) % (n ** 3)
    sa = (q % n, (q // n) % n, q // (n * n))
    return [(sa[a].astype(np.float64) + u[a].astype(np.float64)) / float(n) for a in range(3)]


def generate_box(case: dict) -> Dict[str, np.ndarray]:
    """Host mirror of mpm_init_box: returns particle arrays in upload order."""
    p, box, tool = case["params"], case["box"], case["tool"]
    c0, c1, ppc = box["c0"], box["c1"], box["ppc"]
    wx, wy, wz = (c1[i] - c0[i] for i in range(3))
    ncell = wx * wy * wz
    cand = np.arange(ncell * ppc, dtype=np.int64)
    cell, k = cand // ppc, cand % ppc
    ix, iy, iz = cell % wx, (cell // wx) % wy, cell // (wx * wy)
    seed = int(box["seed"])
    u = philox4x32_10(seed & 0xFFFFFFFF, seed >> 32, cell, k, np.full_like(cell, box["instance"]),
                      np.zeros_like(cell))
    off = gen_offset(k, ppc, u)
    xi = np.stack([(c0[0] + ix) + off[0], (c0[1] + iy) + off[1], (c0[2] + iz) + off[2]], axis=1)
    dx = p["dx"]
    org = p["origin"]
    x = org[0] + xi[:, 0] * dx
    y = org[1] + xi[:, 1] * dx
    z = org[2] + xi[:, 2] * dx
    keep = np.ones(len(cand), dtype=bool)
    if tool and tool.get("mode", A.TOOL_NONE) != A.TOOL_NONE:
        keep = tool_sdf(tool, x, z, tool["position"][0], tool["position"][2]) > 0.0
    n = int(keep.sum())
    status = np.where(iz[keep] < box["fixed_layers"], A.FIXED, A.ACTIVE).astype(np.int32)
    return dict(x=x[keep], y=y[keep], z=z[keep], status=status, id=np.arange(n, dtype=np.int32),
                temperature=np.full(n, float(box["T0"])))


def full_state(parts: Dict[str, np.ndarray], case: dict) -> Dict[str, np.ndarray]:
    """Complete every MPMParticle field with its default (include/Types.h:245-266)."""
    n = len(parts["x"])
    eye = np.tile(np.eye(3).reshape(1, 9), (n, 1))
    out = dict(vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n), F=eye.copy(), Fp=eye.copy(), C=np.zeros((n, 9)),
               stress=np.zeros((n, 6)), backstress=np.zeros((n, 6)), plastic_strain=np.zeros(n),
               strain_rate=np.zeros(n), temperature=np.full(n, case["params"]["Tamb"]), damage=np.zeros(n),
               residual_stress=np.zeros(n))
    out.update({k: np.array(v, copy=True) for k, v in parts.items()})
    return out


def cylinder_samples(case: dict, spacing_cells: float = 0.5) -> np.ndarray:
    """Tool surface samples (offsets from the tool reference point) for the
    raster boundary: the cylinder surface over the grid's y extent."""
    p, tool = case["params"], case["tool"]
    dx, R = p["dx"], tool["radius"]
    h = spacing_cells * dx
    nth = max(8, int(math.ceil(2 * math.pi * R / h)))
    th = np.arange(nth) * (2 * math.pi / nth)
    ys = p["origin"][1] + np.arange(0.0, (p["ny"] - 1) * dx + 1e-12, h) - tool["position"][1]
    T, Y = np.meshgrid(th, ys, indexing="ij")
    return np.stack([R * np.cos(T).ravel(), Y.ravel(), R * np.sin(T).ravel()], axis=1)


def wedge_samples(case: dict, spacing_cells: float = 0.5) -> np.ndarray:
    """Surface samples of the rounded wedge (offsets from the edge-circle
    centre): the edge arc between the flank and rake normals, the rake face up
    to the top of the grid and the flank face back to the grid's -x side,
    extruded over the grid's y extent."""
    p, tool = case["params"], case["tool"]
    dx, r = p["dx"], tool["radius"]
    h = spacing_cells * dx
    g, a = tool["rake"], tool["clearance"]
    th0, th1 = math.atan2(-math.cos(a), -math.sin(a)), g  # flank normal .. rake normal (exterior arc)
    nth = max(4, int(math.ceil(r * (th1 - th0) / h)) + 1)
    th = np.linspace(th0, th1, nth)
    pts = [np.stack([r * np.cos(th), r * np.sin(th)], axis=1)]
    px, pz = tool["position"][0], tool["position"][2]
    ztop = p["origin"][2] + (p["nz"] - 1) * dx
    up = max(0.0, ztop - (pz + r * math.sin(g)))
    s = np.arange(h, up + h, h)
    pts.append(np.stack([r * math.cos(g) - s * math.sin(g), r * math.sin(g) + s * math.cos(g)], axis=1))
    back = max(0.0, (px - r * math.sin(a)) - p["origin"][0])
    s = np.arange(h, back + h, h)
    pts.append(np.stack([-r * math.sin(a) - s * math.cos(a), -r * math.cos(a) + s * math.sin(a)], axis=1))
    xz = np.concatenate(pts, axis=0)
    ys = p["origin"][1] + np.arange(0.0, (p["ny"] - 1) * dx + 1e-12, h) - tool["position"][1]
    XZ = np.repeat(xz, len(ys), axis=0)
    Y = np.tile(ys, len(xz))
    return np.stack([XZ[:, 0], Y, XZ[:, 1]], axis=1)


def tool_samples(case: dict, spacing_cells: float = 0.5) -> np.ndarray:
    if case["tool"]["shape"] == A.SHAPE_CYLINDER_Y:
        return cylinder_samples(case, spacing_cells)
    return wedge_samples(case, spacing_cells)


def generate_box_chunked(case: dict, zchunk: int = 8):
    """generate_box for large boxes, `zchunk` cell layers at a time; returns
    (x, y, z, status) with the ids implied by the order."""
    box = case["box"]
    c0, c1 = list(box["c0"]), list(box["c1"])
    xs, ys, zs, sts = [], [], [], []
    for z0 in range(c0[2], c1[2], zchunk):
        sub = dict(case)
        b = dict(box)
        b["c0"] = (c0[0], c0[1], z0)
        b["c1"] = (c1[0], c1[1], min(z0 + zchunk, c1[2]))
        b["fixed_layers"] = box["fixed_layers"] - (z0 - c0[2])
        sub["box"] = b
        part = _generate_box_offset(sub, cell_offset=(z0 - c0[2]) * (c1[0] - c0[0]) * (c1[1] - c0[1]))
        xs.append(part["x"]); ys.append(part["y"]); zs.append(part["z"]); sts.append(part["status"])
    return np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), np.concatenate(sts)


def _generate_box_offset(case: dict, cell_offset: int) -> Dict[str, np.ndarray]:
    p, box, tool = case["params"], case["box"], case["tool"]
    c0, c1, ppc = box["c0"], box["c1"], box["ppc"]
    wx, wy, wz = (c1[i] - c0[i] for i in range(3))
    cand = np.arange(wx * wy * wz * ppc, dtype=np.int64)
    cell, k = cand // ppc, cand % ppc
    ix, iy, iz = cell % wx, (cell // wx) % wy, cell // (wx * wy)
    seed = int(box["seed"])
    u = philox4x32_10(seed & 0xFFFFFFFF, seed >> 32, cell + cell_offset, k, np.full_like(cell, box["instance"]),
                      np.zeros_like(cell))
    dx, org = p["dx"], p["origin"]
    off = gen_offset(k, ppc, u)
    x = org[0] + ((c0[0] + ix) + off[0]) * dx
    y = org[1] + ((c0[1] + iy) + off[1]) * dx
    z = org[2] + ((c0[2] + iz) + off[2]) * dx
    keep = np.ones(len(cand), dtype=bool)
    if tool and tool.get("mode", A.TOOL_NONE) != A.TOOL_NONE:
        keep = tool_sdf(tool, x, z, tool["position"][0], tool["position"][2]) > 0.0
    status = np.where(iz[keep] < box["fixed_layers"], A.FIXED, A.ACTIVE).astype(np.int32)
    return dict(x=x[keep], y=y[keep], z=z[keep], status=status)
