"""Python access to the test-only checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg / reference arm.  Never imported by the product.

  Oracle   -- liboracle_mpm.so, the CPU FP64 restatement (mpm_oracle.c)
  RefKern  -- _ref/libmpm_ref.so, the reference's own CUDA kernels
              (src/MPMSolver.cu compiled from its sources, GPU only)

States are dicts of float64 numpy arrays keyed like mpm_particles_soa fields
(x, y, z, vx, vy, vz, F[n,9], Fp[n,9], C[n,9], stress[n,6], backstress[n,6],
plastic_strain, strain_rate, temperature, damage, residual_stress, status, id).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path
from typing import Dict, Optional

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle_mpm.so"
REF_LIB = HERE / "_ref" / "libmpm_ref.so"

_d, _i32, _i64, _vp = C.c_double, C.c_int32, C.c_int64, C.c_void_p
TOOL_NONE, TOOL_RASTER, TOOL_SDF_STICKY, TOOL_SDF_SLIP = 0, 1, 2, 3


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", _i32), ("ny", _i32), ("nz", _i32), ("_pad0", _i32), ("dx", _d), ("ox", _d), ("oy", _d), ("oz", _d),
        ("E", _d), ("nu", _d), ("rho_phys", _d), ("cp", _d), ("beta", _d), ("Tm", _d), ("Tamb", _d),
        ("A", _d), ("B", _d), ("n", _d), ("C", _d), ("m", _d), ("edot0", _d), ("Hkin", _d),
        ("D1", _d), ("D2", _d), ("D3", _d), ("D4", _d), ("D5", _d), ("Dth", _d),
        ("fixture_thickness", _d), ("fixture_damping", _d), ("gravity_z", _d), ("mass_threshold", _d),
        ("apic_dinv_factor", _d), ("apic_decay", _d),
        ("lod_enabled", _i32), ("plasticity_mode", _i32), ("lod_active_r", _d), ("lod_near_r", _d),
        ("deps_cap", _d), ("dT_cap", _d), ("chip_sep_enabled", _i32), ("chip_every", _i32),
        ("tool_mode", _i32), ("tool_shape", _i32), ("tool_p0", _d * 3), ("tool_v", _d * 3), ("tool_r", _d),
        ("tool_rake", _d), ("tool_clear", _d), ("tool_tip_dz", _d), ("newton_tol", _d), ("newton_maxit", _i32),
        ("contact_every", _i32), ("contact_radius", _d), ("contact_friction", _d), ("contact_heat_partition", _d),
        ("asb_enabled", _i32), ("asb_critical_rate", _d), ("asb_taylor_quinney", _d), ("asb_max_temp_ratio", _d),
        ("asb_touch_rise", _d), ("heat_conduction", _i32), ("thermal_conductivity", _d),
        ("tool_sdf", _vp), ("tool_sdf_angle", C.c_float),
    ]


class OrcState(C.Structure):
    _fields_ = [("n", _i32), ("_pad", _i32)] + [
        (k, _vp) for k in ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "sig", "bs", "eps", "edot", "T", "D",
                           "sres", "mass", "vol", "extf", "status", "id", "lod", "asb")
    ]


class OrcSdfGrid(C.Structure):
    _fields_ = [("nx", _i32), ("ny", _i32), ("nz", _i32), ("_pad", _i32), ("v", _vp), ("ox", C.c_float),
                ("oy", C.c_float), ("oz", C.c_float), ("voxel", C.c_float)]


class OrcContactArgs(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("cx", "cy", "cz", "cos_a", "sin_a", "radius", "friction", "heat_partition",
                                         "dt", "_pad")] + [("cp", _d), ("rho_phys", _d), ("Tm", _d)]


def sdf_grid(sdf: dict):
    """(OrcSdfGrid, keep-alive array) from {"v": float32 [nz, ny, nx], "origin": (x, y, z), "voxel": h}."""
    v = np.ascontiguousarray(sdf["v"], dtype=np.float32)
    g = OrcSdfGrid()
    g.nz, g.ny, g.nx = v.shape
    g.v = v.ctypes.data
    g.ox, g.oy, g.oz = (float(c) for c in sdf["origin"])
    g.voxel = float(sdf["voxel"])
    return g, v


def contact_args(a: dict) -> OrcContactArgs:
    o = OrcContactArgs()
    for k in ("cx", "cy", "cz", "cos_a", "sin_a", "radius", "friction", "heat_partition", "dt", "cp", "rho_phys", "Tm"):
        setattr(o, k, float(a[k]))
    return o


class OrcWsParams(C.Structure):
    """orc_ws_params: MPMWorkpieceSolver's own constants."""
    _fields_ = [("failure_strain", _d), ("critical_plastic_strain", _d), ("thermal_chip_ratio", _d),
                ("tool_contact_radius", _d), ("contact_damping", _d), ("max_contact_temp_rise", _d),
                ("thermal_clamp", _i32), ("_pad", _i32)]


def ws_params(w: dict) -> OrcWsParams:
    o = OrcWsParams()
    for k in ("failure_strain", "critical_plastic_strain", "thermal_chip_ratio", "tool_contact_radius",
              "contact_damping", "max_contact_temp_rise"):
        setattr(o, k, float(w[k]))
    o.thermal_clamp = int(w.get("thermal_clamp", 1))
    return o


class OrcTool(C.Structure):
    _fields_ = [("n", _i32), ("_pad", _i32), ("ox", _vp), ("oy", _vp), ("oz", _vp)]


class OrcMetrics(C.Structure):
    _fields_ = [(k, _d) for k in ("mass", "px", "py", "pz", "kinetic", "internal_elastic", "thermal", "max_T",
                                  "max_vm", "max_eps", "sum_eps", "ref_max_stress", "ref_max_T", "ref_kinetic",
                                  "ref_internal")] + \
               [(k, _i64) for k in ("n_active", "n_chip", "n_fixed", "n_inactive")] + \
               [("bmin", _d * 3), ("bmax", _d * 3)]


FIELD_MAP = [("x", "x", 1), ("y", "y", 1), ("z", "z", 1), ("vx", "vx", 1), ("vy", "vy", 1), ("vz", "vz", 1),
             ("F", "F", 9), ("Fp", "Fp", 9), ("C", "C", 9), ("stress", "sig", 6), ("backstress", "bs", 6),
             ("plastic_strain", "eps", 1), ("strain_rate", "edot", 1), ("temperature", "T", 1),
             ("damage", "D", 1), ("residual_stress", "sres", 1)]


def build(ref: bool = False) -> None:
    """make -C oracle [ref]; the reference harness only when its sources exist."""
    targets = ["all"]
    if ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


def orc_params(case: dict) -> OrcParams:
    p, t = case["params"], case["tool"]
    o = OrcParams()
    o.nx, o.ny, o.nz = p["nx"], p["ny"], p["nz"]
    o.dx = p["dx"]
    o.ox, o.oy, o.oz = p["origin"]
    for k in ("E", "nu", "rho_phys", "cp", "beta", "Tm", "Tamb", "edot0", "D1", "D2", "D3", "D4", "D5",
              "fixture_thickness", "fixture_damping", "gravity_z", "mass_threshold", "apic_dinv_factor",
              "apic_decay", "lod_active_r", "lod_near_r", "deps_cap", "dT_cap", "newton_tol"):
        setattr(o, k, float(p[k]))
    o.A, o.B, o.n, o.C, o.m, o.Hkin = p["jc_A"], p["jc_B"], p["jc_n"], p["jc_C"], p["jc_m"], p["H_kin"]
    o.Dth = p["D_th"]
    o.lod_enabled = int(p["lod_enabled"])
    o.plasticity_mode = int(p["plasticity"])
    o.chip_every = int(p["chip_every"])
    o.chip_sep_enabled = 1 if p["chip_every"] > 0 else 0
    o.newton_maxit = int(p["newton_maxit"])
    o.tool_mode = int(t.get("mode", TOOL_NONE))
    o.tool_shape = int(t.get("shape", 0))
    for i in range(3):
        o.tool_p0[i] = t.get("position", (0, 0, 0))[i]
        o.tool_v[i] = t.get("velocity", (0, 0, 0))[i]
    o.tool_r = t.get("radius", 0.0)
    o.tool_rake = t.get("rake", 0.0)
    o.tool_clear = t.get("clearance", 0.0)
    o.tool_tip_dz = t.get("tip_dz", 0.0)
    o.contact_every = int(p.get("contact_every", 0))
    o.contact_radius = float(p.get("contact_radius", 0.0))
    o.contact_friction = float(p.get("contact_friction", 0.0))
    o.contact_heat_partition = float(p.get("contact_heat_partition", 0.0))
    o.asb_enabled = int(p.get("asb_enabled", 0))
    o.asb_critical_rate = float(p.get("asb_critical_rate", 1e4))
    o.asb_taylor_quinney = float(p.get("asb_taylor_quinney", 0.9))
    o.asb_max_temp_ratio = float(p.get("asb_max_temp_ratio", 0.9))
    o.asb_touch_rise = float(p.get("asb_touch_rise", 0.5))
    o.heat_conduction = int(p.get("heat_conduction", 0))
    o.thermal_conductivity = float(p.get("thermal_conductivity", 42.6))
    if t.get("sdf") is not None:
        g, arr = sdf_grid(t["sdf"])
        o._keep = (g, arr)
        o.tool_sdf = C.cast(C.pointer(g), C.c_void_p).value
        o.tool_sdf_angle = float(t["sdf"].get("angle", 0.0))
    return o


class _Bound:
    """Keeps numpy arrays alive while a C call uses them."""

    def __init__(self, case: dict, state: Dict[str, np.ndarray], extf: Optional[np.ndarray] = None):
        n = len(state["x"])
        self.arrs = {}
        s = OrcState()
        s.n = n
        for ext, intn, per in FIELD_MAP:
            a = np.ascontiguousarray(state[ext], dtype=np.float64).reshape((n, per) if per > 1 else (n,)).copy()
            self.arrs[ext] = a
            setattr(s, intn, a.ctypes.data)
        p = case["params"]
        self.arrs["mass"] = np.full(n, float(p["particle_mass"]))
        self.arrs["vol"] = np.full(n, float(p["particle_volume"]))
        s.mass = self.arrs["mass"].ctypes.data
        s.vol = self.arrs["vol"].ctypes.data
        self.arrs["status"] = np.ascontiguousarray(state["status"], dtype=np.int32).copy()
        self.arrs["id"] = np.ascontiguousarray(state["id"], dtype=np.int32).copy()
        lod = state.get("lod")
        self.arrs["lod"] = np.zeros(n, np.int32) if lod is None else np.ascontiguousarray(lod, np.int32).copy()
        asb = state.get("asb")
        self.arrs["asb"] = np.zeros(n, np.int32) if asb is None else np.ascontiguousarray(asb, np.int32).copy()
        s.status = self.arrs["status"].ctypes.data
        s.id = self.arrs["id"].ctypes.data
        s.lod = self.arrs["lod"].ctypes.data
        s.asb = self.arrs["asb"].ctypes.data
        if extf is not None:
            self.arrs["extf"] = np.ascontiguousarray(extf, np.float64).reshape(n, 3).copy()
            s.extf = self.arrs["extf"].ctypes.data
        self.state = s
        samples = case["tool"].get("samples")
        self.tool = OrcTool()
        if samples is not None:
            smp = np.ascontiguousarray(samples, np.float64)
            self.cols = [np.ascontiguousarray(smp[:, k]) for k in range(3)]
            self.tool.n = len(smp)
            self.tool.ox, self.tool.oy, self.tool.oz = (c.ctypes.data for c in self.cols)

    def result(self) -> Dict[str, np.ndarray]:
        out = {k: v for k, v in self.arrs.items() if k not in ("mass", "vol", "extf")}
        return out


class Oracle:
    def __init__(self):
        if not ORACLE_LIB.exists():
            build()
        L = C.CDLL(str(ORACLE_LIB))
        L.orc_grid_doubles.restype = _i64
        L.orc_grid_doubles.argtypes = [C.POINTER(OrcParams)]
        L.orc_step.restype = _i32
        L.orc_step.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcState), C.POINTER(OrcTool), C.POINTER(_d), _d,
                               _i32, _i64, _d, _i32]
        L.orc_metrics_compute.restype = None
        L.orc_metrics_compute.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcState), C.POINTER(OrcMetrics)]
        L.orc_philox_uniform4.restype = None
        L.orc_philox_uniform4.argtypes = [C.c_uint32] * 6 + [C.POINTER(C.c_float)]
        L.orc_tool_sdf.restype = _d
        L.orc_tool_sdf.argtypes = [C.POINTER(OrcParams), C.POINTER(_d), _d, _d, _d]
        L.orc_asb_heat.restype = None
        L.orc_asb_heat.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcState), _d]
        L.orc_heat_diffuse.restype = None
        L.orc_heat_diffuse.argtypes = [C.POINTER(OrcParams), C.POINTER(_d), C.POINTER(_d), C.POINTER(_d), _d]
        L.orc_tex3d.restype = C.c_float
        L.orc_tex3d.argtypes = [C.POINTER(OrcSdfGrid), C.c_float, C.c_float, C.c_float]
        L.orc_tool_sdf_build.restype = _i32
        L.orc_tool_sdf_build.argtypes = [_vp, _i32, _vp, _i32, _vp, _d, _i32, C.POINTER(_i32 * 3),
                                         C.POINTER(C.c_float * 3), C.POINTER(C.c_float), _vp]
        L.orc_ws_grid_doubles.restype = _i64
        L.orc_ws_grid_doubles.argtypes = [C.POINTER(OrcParams)]
        L.orc_ws_step.restype = None
        L.orc_ws_step.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcWsParams), C.POINTER(OrcState),
                                  C.POINTER(OrcTool), C.POINTER(_d), _d, _i32, _i64, _d, C.POINTER(_d)]
        L.orc_contact_sdf.restype = None
        L.orc_contact_sdf.argtypes = [C.POINTER(OrcSdfGrid), C.POINTER(OrcContactArgs), C.POINTER(OrcState),
                                      C.POINTER(_i64), C.POINTER(_d), C.POINTER(_d)]
        self.L = L

    def step(self, case: dict, state: Dict[str, np.ndarray], nsteps: int, step0: int = 0, t0: float = 0.0,
             nthreads: int = 1, dt: Optional[float] = None, extf: Optional[np.ndarray] = None):
        p = orc_params(case)
        b = _Bound(case, state, extf)
        grid = np.zeros(int(self.L.orc_grid_doubles(C.byref(p))), dtype=np.float64)
        rc = self.L.orc_step(C.byref(p), C.byref(b.state), C.byref(b.tool),
                             grid.ctypes.data_as(C.POINTER(_d)), float(dt if dt is not None else case["dt"]),
                             int(nsteps), int(step0), float(t0), int(nthreads))
        return b.result(), rc

    def ws_step(self, case: dict, state: Dict[str, np.ndarray], nsteps: int, step0: int = 0, t0: float = 0.0,
                extf: Optional[np.ndarray] = None):
        """nsteps of MPMWorkpieceSolver's step (case["ws"]: its constants):
        (state after, contact force of the last step)."""
        p = orc_params(case)
        w = ws_params(case["ws"])
        b = _Bound(case, state, extf)
        grid = np.zeros(int(self.L.orc_ws_grid_doubles(C.byref(p))), dtype=np.float64)
        f = _d()
        self.L.orc_ws_step(C.byref(p), C.byref(w), C.byref(b.state), C.byref(b.tool),
                           grid.ctypes.data_as(C.POINTER(_d)), float(case["dt"]), int(nsteps), int(step0), float(t0),
                           C.byref(f))
        out = b.result()
        if extf is not None:
            out["extf"] = b.arrs["extf"]
        return out, f.value

    def asb_heat(self, case: dict, state: Dict[str, np.ndarray], dt: float) -> Dict[str, np.ndarray]:
        """One adiabatic shear heating pass (no grid step)."""
        p = orc_params(case)
        b = _Bound(case, state)
        self.L.orc_asb_heat(C.byref(p), C.byref(b.state), float(dt))
        return b.result()

    def heat_diffuse(self, case: dict, mass: np.ndarray, tm: np.ndarray, dt: float) -> np.ndarray:
        """One grid diffusion step: node masses and T m (x fastest) -> node temperatures."""
        p = orc_params(case)
        m = np.ascontiguousarray(mass, np.float64).ravel()
        q = np.ascontiguousarray(tm, np.float64).ravel()
        out = np.zeros_like(m)
        P = C.POINTER(_d)
        self.L.orc_heat_diffuse(C.byref(p), m.ctypes.data_as(P), q.ctypes.data_as(P), out.ctypes.data_as(P), float(dt))
        return out

    def tex3d(self, sdf: dict, xyz: np.ndarray) -> np.ndarray:
        """Emulated texture fetches at voxel coordinates xyz [n, 3]."""
        g, keep = sdf_grid(sdf)
        q = np.asarray(xyz, np.float32).reshape(-1, 3)
        return np.array([self.L.orc_tex3d(C.byref(g), float(a), float(b), float(c)) for a, b, c in q], np.float32)

    def tool_sdf_build(self, verts, tris, normals, padding: float, voxels_per_axis: int) -> dict:
        """The voxel SDF of a closed mesh as ToolSDF builds it."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        n = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        dims, org, vox = (_i32 * 3)(), (C.c_float * 3)(), C.c_float()
        args = (v.ctypes.data, len(v), t.ctypes.data, len(t), n.ctypes.data, float(padding), int(voxels_per_axis))
        if self.L.orc_tool_sdf_build(*args, C.byref(dims), C.byref(org), C.byref(vox), None) != 0:
            raise ValueError("empty mesh or grid")
        out = np.zeros((dims[2], dims[1], dims[0]), np.float32)
        self.L.orc_tool_sdf_build(*args, C.byref(dims), C.byref(org), C.byref(vox), out.ctypes.data)
        return {"v": out, "origin": tuple(org), "voxel": float(vox.value), "angle": 0.0}

    def contact_sdf(self, case: dict, state: Dict[str, np.ndarray], sdf: dict, args: dict):
        """One xpbdContactSDFKernel pass: (state after, (count, friction work, normal force))."""
        g, keep = sdf_grid(sdf)
        b = _Bound(case, state)
        a = contact_args(args)
        cnt, heat, force = _i64(), _d(), _d()
        self.L.orc_contact_sdf(C.byref(g), C.byref(a), C.byref(b.state), C.byref(cnt), C.byref(heat), C.byref(force))
        return b.result(), (cnt.value, heat.value, force.value)

    def metrics(self, case: dict, state: Dict[str, np.ndarray]) -> dict:
        p = orc_params(case)
        b = _Bound(case, state)
        m = OrcMetrics()
        self.L.orc_metrics_compute(C.byref(p), C.byref(b.state), C.byref(m))
        out = {}
        for name, _ in m._fields_:
            v = getattr(m, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out

    def philox(self, seed: int, c0: int, c1: int, c2: int, c3: int) -> np.ndarray:
        out = (C.c_float * 4)()
        self.L.orc_philox_uniform4(seed & 0xFFFFFFFF, seed >> 32, c0, c1, c2, c3, out)
        return np.array(out[:], dtype=np.float32)


class RefKern:
    """The reference's own CUDA kernels (needs a GPU)."""

    def __init__(self):
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} is missing: build it with `make -C oracle ref` where the reference "
                               "sources are present")
        L = C.CDLL(str(REF_LIB))
        L.ref_last_error.restype = C.c_char_p
        L.ref_device_count.restype = _i32
        L.ref_sizeof_particle.restype = _i32
        L.ref_run.restype = _i32
        L.ref_run.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcState), C.POINTER(OrcTool), _d, _i32, C.c_longlong,
                              _d]
        L.ref_stats.restype = _i32
        L.ref_stats.argtypes = [C.POINTER(OrcState), C.POINTER(_d)]
        L.ref_asb_heat.restype = _i32
        L.ref_asb_heat.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcState), _d]
        L.ref_heat_diffuse.restype = _i32
        L.ref_heat_diffuse.argtypes = [C.POINTER(OrcParams), C.POINTER(_d), C.POINTER(_d), _d]
        L.ref_heat_last_error.restype = C.c_char_p
        L.ref_ws_run.restype = _i32
        L.ref_ws_run.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcWsParams), C.POINTER(OrcState),
                                 C.POINTER(OrcTool), _d, _i32, C.c_longlong, _d, C.POINTER(_d)]
        L.ref_contact_last_error.restype = C.c_char_p
        L.ref_tex_probe.restype = _i32
        L.ref_tex_probe.argtypes = [C.POINTER(OrcSdfGrid), _vp, _i32, _vp]
        L.ref_contact_sdf.restype = _i32
        L.ref_contact_sdf.argtypes = [C.POINTER(OrcSdfGrid), C.POINTER(OrcContactArgs), C.POINTER(OrcState),
                                      C.POINTER(_i64), C.POINTER(_d), C.POINTER(_d)]
        L.ref_contact_sdf_device.restype = _i32
        L.ref_contact_sdf_device.argtypes = [C.POINTER(OrcSdfGrid), C.POINTER(OrcContactArgs), _vp, _i32,
                                             C.POINTER(_i64), C.POINTER(_d), C.POINTER(_d)]
        L.ref_bench.restype = _i32
        L.ref_bench.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcState), C.POINTER(OrcTool), _d, _i32, _i32,
                                C.POINTER(_d)]
        L.ref_bench_positions.restype = _i32
        L.ref_bench_positions.argtypes = [C.POINTER(OrcParams), _vp, _vp, _vp, _vp, _i32, _d, _d, _d,
                                          C.POINTER(OrcTool), _d, _i32, _i32, C.POINTER(_d), C.POINTER(C.c_longlong)]
        self.L = L

    def step(self, case: dict, state: Dict[str, np.ndarray], nsteps: int, step0: int = 0, t0: float = 0.0,
             dt: Optional[float] = None, extf: Optional[np.ndarray] = None):
        p = orc_params(case)
        b = _Bound(case, state, extf)
        rc = self.L.ref_run(C.byref(p), C.byref(b.state), C.byref(b.tool), float(dt if dt is not None else case["dt"]),
                            int(nsteps), int(step0), float(t0))
        if rc != 0:
            raise RuntimeError(f"reference run failed ({rc}): {self.L.ref_last_error().decode()}")
        return b.result()

    def asb_heat(self, case: dict, state: Dict[str, np.ndarray], dt: float) -> Dict[str, np.ndarray]:
        """The reference's detectShearBands + applyAdiabaticHeating kernels once."""
        p = orc_params(case)
        b = _Bound(case, state)
        rc = self.L.ref_asb_heat(C.byref(p), C.byref(b.state), float(dt))
        if rc != 0:
            raise RuntimeError(f"reference shear pass failed ({rc}): {self.L.ref_last_error().decode()}")
        return b.result()

    def ws_step(self, case: dict, state: Dict[str, np.ndarray], nsteps: int, step0: int = 0, t0: float = 0.0,
                extf: Optional[np.ndarray] = None):
        """The reference's MPMWorkpieceSolver kernels for nsteps steps:
        (state after, contact force of the last step)."""
        p = orc_params(case)
        w = ws_params(case["ws"])
        b = _Bound(case, state, extf)
        f = _d()
        rc = self.L.ref_ws_run(C.byref(p), C.byref(w), C.byref(b.state), C.byref(b.tool), float(case["dt"]),
                               int(nsteps), int(step0), float(t0), C.byref(f))
        if rc != 0:
            raise RuntimeError(f"reference workpiece-solver run failed: {self.L.ref_heat_last_error().decode()}")
        out = b.result()
        if extf is not None:
            out["extf"] = b.arrs["extf"]
        return out, f.value

    def heat_diffuse(self, case: dict, mass: np.ndarray, tm: np.ndarray, dt: float) -> np.ndarray:
        """The reference's mpmDiffuseTemperatureKernel once: returns its new T m."""
        p = orc_params(case)
        m = np.ascontiguousarray(mass, np.float64).ravel()
        q = np.ascontiguousarray(tm, np.float64).ravel().copy()
        P = C.POINTER(_d)
        rc = self.L.ref_heat_diffuse(C.byref(p), m.ctypes.data_as(P), q.ctypes.data_as(P), float(dt))
        if rc != 0:
            raise RuntimeError(f"reference diffusion failed ({rc}): {self.L.ref_heat_last_error().decode()}")
        return q

    def tex_probe(self, sdf: dict, xyz: np.ndarray) -> np.ndarray:
        """Hardware texture fetches (the reference's texture setup) at voxel coordinates xyz [n, 3]."""
        g, keep = sdf_grid(sdf)
        q = np.ascontiguousarray(np.asarray(xyz, np.float32).reshape(-1, 3))
        out = np.zeros(len(q), np.float32)
        rc = self.L.ref_tex_probe(C.byref(g), q.ctypes.data, len(q), out.ctypes.data)
        if rc != 0:
            raise RuntimeError(self.L.ref_contact_last_error().decode())
        return out

    def contact_sdf(self, case: dict, state: Dict[str, np.ndarray], sdf: dict, args: dict):
        """The reference's xpbdContactSDFKernel once: (state after, (count, friction work, normal force))."""
        g, keep = sdf_grid(sdf)
        b = _Bound(case, state)
        a = contact_args(args)
        cnt, heat, force = _i64(), _d(), _d()
        rc = self.L.ref_contact_sdf(C.byref(g), C.byref(a), C.byref(b.state), C.byref(cnt), C.byref(heat),
                                    C.byref(force))
        if rc != 0:
            raise RuntimeError(self.L.ref_contact_last_error().decode())
        return b.result(), (cnt.value, heat.value, force.value)

    def contact_sdf_device(self, sdf: dict, args: dict, d_particles: int, n: int):
        """The reference's xpbdContactSDFKernel once, in place on n MPMParticle
        records at device address d_particles: (count, friction work, normal force)."""
        g, keep = sdf_grid(sdf)
        a = contact_args(args)
        cnt, heat, force = _i64(), _d(), _d()
        rc = self.L.ref_contact_sdf_device(C.byref(g), C.byref(a), C.c_void_p(int(d_particles)), int(n),
                                           C.byref(cnt), C.byref(heat), C.byref(force))
        if rc != 0:
            raise RuntimeError(self.L.ref_contact_last_error().decode())
        return cnt.value, heat.value, force.value

    def stats(self, case: dict, state: Dict[str, np.ndarray]) -> np.ndarray:
        b = _Bound(case, state)
        out = (C.c_double * 4)()
        rc = self.L.ref_stats(C.byref(b.state), out)
        if rc != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return np.array(out[:])

    def bench(self, case: dict, state: Dict[str, np.ndarray], warmup: int, steps: int, dt: Optional[float] = None):
        p = orc_params(case)
        b = _Bound(case, state)
        ms = C.c_double()
        rc = self.L.ref_bench(C.byref(p), C.byref(b.state), C.byref(b.tool),
                              float(dt if dt is not None else case["dt"]), int(warmup), int(steps), C.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference bench failed ({rc}): {self.L.ref_last_error().decode()}")
        return ms.value, b.result()

    def bench_positions(self, case: dict, x, y, z, status, warmup: int, steps: int, samples=None):
        """Time the reference kernels on particles given by position and status
        (MPMParticle defaults elsewhere), with the tool rasterised from
        `samples`.  Returns (device ms of the timed steps, live particles)."""
        p = orc_params(case)
        if samples is not None:
            p.tool_mode = TOOL_RASTER
        arrs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z)]
        st = np.ascontiguousarray(status, np.int32)
        tool = OrcTool()
        cols = []
        if samples is not None:
            smp = np.ascontiguousarray(samples, np.float64)
            cols = [np.ascontiguousarray(smp[:, k]) for k in range(3)]
            tool.n = len(smp)
            tool.ox, tool.oy, tool.oz = (c.ctypes.data for c in cols)
        ms, live = C.c_double(), C.c_longlong()
        pr = case["params"]
        rc = self.L.ref_bench_positions(C.byref(p), arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data,
                                        st.ctypes.data, len(st), float(pr["particle_mass"]),
                                        float(pr["particle_volume"]), float(case["box"]["T0"]), C.byref(tool),
                                        float(case["dt"]), int(warmup), int(steps), C.byref(ms), C.byref(live))
        if rc != 0:
            raise RuntimeError(f"reference bench failed ({rc}): {self.L.ref_last_error().decode()}")
        return ms.value, live.value
