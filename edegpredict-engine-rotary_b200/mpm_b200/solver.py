"""Python handle over the C ABI (used by the tests and the benchmark).

Solver mirrors the call sequence the engine makes on the reference's
MPMSolver (src/SimulationEngine.cpp:499-537): set the tool, step, sync the
metrics, read the particles.  Particle arrays are numpy arrays in the
reference's units, keyed by the field names of mpm_particles_soa.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

from . import _capi as A


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def soa_in(parts: Dict[str, np.ndarray], elem: int = 8):
    """mpm_particles_soa over host copies of `parts` (returned to keep alive)."""
    dt = np.float64 if elem == 8 else np.float32
    s = A.MpmParticlesSoa()
    s.elem = elem
    keep = []
    for name in A.PARTICLE_FIELDS:
        if name in parts and parts[name] is not None:
            a = np.ascontiguousarray(parts[name], dtype=dt)
            keep.append(a)
            setattr(s, name, a.ctypes.data)
    for name in ("status", "id"):
        if name in parts and parts[name] is not None:
            a = np.ascontiguousarray(parts[name], dtype=np.int32)
            keep.append(a)
            setattr(s, name, a.ctypes.data)
    return s, keep, len(parts["x"])


def soa_out(n: int, fields=None, elem: int = 8):
    """mpm_particles_soa over new host arrays for n particles."""
    dt = np.float64 if elem == 8 else np.float32
    s = A.MpmParticlesSoa()
    s.elem = elem
    out = {}
    for name, per in A.PARTICLE_FIELDS.items():
        if fields is None or name in fields:
            a = np.zeros((n, per) if per > 1 else (n,), dtype=dt)
            out[name] = a
            setattr(s, name, a.ctypes.data)
    for name in ("status", "id"):
        if fields is None or name in fields:
            a = np.zeros(n, dtype=np.int32)
            out[name] = a
            setattr(s, name, a.ctypes.data)
    return s, out


class Solver:
    def __init__(self, params: A.MpmParams, capacity: int, stream: int = 0):
        self._lib = A.lib()
        self.params = params
        h = C.c_void_p()
        A.check(self._lib.mpm_create(C.byref(params), int(capacity), C.c_void_p(stream or None), C.byref(h)))
        self.h = h
        self._keep = []

    def close(self) -> None:
        if self.h:
            self._lib.mpm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int) -> None:
        A.check(status, self.h)

    # ---------------------------------------------------------------- tool
    @staticmethod
    def tool_desc(tool: dict) -> A.MpmToolDesc:
        t = A.MpmToolDesc()
        t.mode = int(tool.get("mode", A.TOOL_NONE))
        t.shape = int(tool.get("shape", A.SHAPE_CYLINDER_Y))
        for k in range(3):
            t.position[k] = float(tool.get("position", (0, 0, 0))[k])
            t.velocity[k] = float(tool.get("velocity", (0, 0, 0))[k])
        t.radius = float(tool.get("radius", 0.0))
        t.rake = float(tool.get("rake", 0.0))
        t.clearance = float(tool.get("clearance", 0.0))
        t.tip_dz = float(tool.get("tip_dz", 0.0))
        s = tool.get("samples")
        if s is not None:
            s = np.ascontiguousarray(s, dtype=np.float64)
            cols = [np.ascontiguousarray(s[:, k]) for k in range(3)]
            t._cols = cols  # keep alive
            t.n_samples = len(s)
            t.sample_dx, t.sample_dy, t.sample_dz = (c.ctypes.data for c in cols)
        return t

    def set_tool(self, tool: dict) -> None:
        t = self.tool_desc(tool)
        self._check(self._lib.mpm_set_tool(self.h, C.byref(t)))

    @staticmethod
    def tool_sdf(sdf: Optional[dict]):
        """MpmToolSdf from {"v": float32 [nz, ny, nx], "origin": (x, y, z), "voxel": h, "angle": a}
        (the array is kept alive on the structure), or None."""
        if sdf is None:
            return None
        v = np.ascontiguousarray(sdf["v"], dtype=np.float32)
        s = A.MpmToolSdf()
        s.nz, s.ny, s.nx = v.shape
        s._v = v
        s.values = v.ctypes.data
        for i in range(3):
            s.origin[i] = float(sdf["origin"][i])
        s.voxel = float(sdf["voxel"])
        s.angle = float(sdf.get("angle", 0.0))
        return s

    def set_tool_sdf(self, sdf: Optional[dict]) -> None:
        """Voxel tool SDF for the particle-side contact (None: the analytic SDF)."""
        s = self.tool_sdf(sdf)
        self._check(self._lib.mpm_set_tool_sdf(self.h, C.byref(s) if s is not None else None))

    # ---------------------------------------------------------------- particles
    def init_box(self, c0, c1, ppc: int, seed: int, instance: int = 0, fixed_layers: int = 2, T0: float = 293.0,
                 tool: Optional[dict] = None) -> int:
        a0 = (C.c_int32 * 3)(*map(int, c0))
        a1 = (C.c_int32 * 3)(*map(int, c1))
        t = self.tool_desc(tool) if tool else None
        self._check(self._lib.mpm_init_box(self.h, a0, a1, int(ppc), C.c_uint64(seed), C.c_uint32(instance),
                                           int(fixed_layers), float(T0), C.byref(t) if t else None))
        return self.counts()[0]

    def upload(self, parts: Dict[str, np.ndarray], elem: int = 8) -> None:
        s, keep, n = soa_in(parts, elem)
        self._check(self._lib.mpm_upload(self.h, C.byref(s), n))

    def download(self, fields=None, elem: int = 8, strict: bool = True) -> Dict[str, np.ndarray]:
        """The particle state in upload order.  strict=False also returns the
        state of a workpiece whose error word is set (MPM_NUMERIC), for
        inspection."""
        s, out = soa_out(self.counts()[0], fields, elem)
        self._check_state(self._lib.mpm_download(self.h, C.byref(s)), strict)
        return out

    def status(self) -> int:
        """mpm_status of the workpiece from its device error word (instance 0
        of the handle): MPM_OK or MPM_NUMERIC."""
        st = (C.c_int32 * 1)()
        self._check(self._lib.mpm_batch_instance_status(self.h, st, 1))
        return int(st[0])

    def checkpoint(self, inst: int = 0) -> np.ndarray:
        """The workpiece's checkpoint (mpm_checkpoint_save) as a byte array;
        write it to a file with .tofile() or keep it in memory."""
        n = C.c_int64()
        self._check(self._lib.mpm_checkpoint_bytes(self.h, int(inst), C.byref(n)))
        buf = np.empty(n.value, dtype=np.uint8)
        self._check(self._lib.mpm_checkpoint_save(self.h, int(inst), buf.ctypes.data, buf.nbytes))
        return buf

    def restore(self, ckpt, inst: int = 0) -> None:
        """Loads a checkpoint (bytes or a uint8 array) into the workpiece."""
        buf = np.frombuffer(ckpt, dtype=np.uint8) if isinstance(ckpt, (bytes, bytearray)) else \
            np.ascontiguousarray(ckpt, dtype=np.uint8)
        self._check(self._lib.mpm_checkpoint_load(self.h, int(inst), buf.ctypes.data, buf.nbytes))

    def launch_config(self) -> dict:
        c = A.MpmLaunchConfig()
        self._check(self._lib.mpm_get_launch_config(self.h, C.byref(c)))
        return c.as_dict()

    def set_launch_config(self, ctas_per_sm: int = 4, sort_every: int = 16, use_graph: bool = False,
                          deterministic: bool = True, pass_size: int = 0) -> None:
        """Launch shape; deterministic=True (the default) gives the same
        results bit for bit on every run and launch shape, False sums node
        tiles with float atomics (mpm_launch_config.deterministic);
        pass_size: FP32 particles per pass of the step kernel (128, 256, 512;
        0: the default)."""
        c = A.MpmLaunchConfig(int(ctas_per_sm), int(sort_every), 1 if use_graph else 0, 1 if deterministic else 0,
                              int(pass_size))
        self._check(self._lib.mpm_set_launch_config(self.h, C.byref(c)))

    def _check_state(self, status: int, strict: bool) -> None:
        if strict or status != A.MPM_NUMERIC:
            self._check(status)

    def download_into(self, bufs: Dict[str, np.ndarray], elem: int = 8) -> None:
        """Download into caller-owned arrays (e.g. pinned host memory)."""
        s = A.MpmParticlesSoa()
        s.elem = elem
        for name, a in bufs.items():
            setattr(s, name, a.ctypes.data)
        self._check(self._lib.mpm_download(self.h, C.byref(s)))

    def export_aos(self) -> np.ndarray:
        n = self.counts()[0]
        buf = np.zeros(max(n, 1) * 504, dtype=np.uint8)
        self._check(self._lib.mpm_export_aos(self.h, buf.ctypes.data_as(C.c_void_p), buf.nbytes))
        return buf[: n * 504]

    def set_workpiece_semantics(self, ws: Optional[dict]) -> None:
        """mpm_set_workpiece_semantics: MPMWorkpieceSolver's step with its
        constants (failure_strain, critical_plastic_strain, thermal_chip_ratio,
        tool_contact_radius, contact_damping, max_contact_temp_rise,
        thermal_clamp); None returns to MPMSolver's."""
        if ws is None:
            self._check(self._lib.mpm_set_workpiece_semantics(self.h, None))
            return
        w = A.MpmWorkpieceParams()
        for k in ("failure_strain", "critical_plastic_strain", "thermal_chip_ratio", "tool_contact_radius",
                  "contact_damping", "max_contact_temp_rise"):
            setattr(w, k, float(ws[k]))
        w.thermal_clamp = int(ws.get("thermal_clamp", 1))
        self._check(self._lib.mpm_set_workpiece_semantics(self.h, C.byref(w)))

    def export_aos_device(self, ptr: int, nbytes: int) -> None:
        """mpm_export_aos into device memory at ptr (nbytes >= 504 per particle)."""
        self._check(self._lib.mpm_export_aos(self.h, C.c_void_p(ptr), int(nbytes)))

    def import_aos(self, src, fields: int = A.AOS_WRITABLE, nbytes: Optional[int] = None) -> None:
        """mpm_import_aos: reads `fields` (A.AOS_*) of MPMParticle records back
        into the workpiece.  src: a host uint8/record array, or an int device
        address with nbytes."""
        if isinstance(src, np.ndarray):
            buf = np.ascontiguousarray(src)
            self._check(self._lib.mpm_import_aos(self.h, buf.ctypes.data_as(C.c_void_p), buf.nbytes, int(fields)))
        else:
            self._check(self._lib.mpm_import_aos(self.h, C.c_void_p(int(src)), int(nbytes), int(fields)))

    # ---------------------------------------------------------------- stepping
    def step(self, dt: float, nsteps: int = 1) -> None:
        self._check(self._lib.mpm_step(self.h, float(dt), int(nsteps)))

    def stable_dt(self, cfl: float) -> float:
        d = C.c_double()
        self._check(self._lib.mpm_stable_dt(self.h, float(cfl), C.byref(d)))
        return d.value

    def metrics(self) -> dict:
        m = A.MpmMetrics()
        self._check(self._lib.mpm_sync_metrics(self.h, C.byref(m)))
        return m.as_dict()

    def set_mass_scaling(self, f: float) -> None:
        self._check(self._lib.mpm_set_mass_scaling(self.h, float(f)))

    def apply_external_force(self, center, radius, force) -> None:
        c = (C.c_double * 3)(*center)
        f = (C.c_double * 3)(*force)
        self._check(self._lib.mpm_apply_external_force(self.h, c, float(radius), f))

    def set_temperatures(self, T: np.ndarray) -> None:
        T = np.ascontiguousarray(T, dtype=np.float64)
        self._check(self._lib.mpm_set_temperatures(self.h, T.ctypes.data_as(C.POINTER(C.c_double)), len(T)))

    def counts(self):
        n, k, t = C.c_int64(), C.c_int64(), C.c_double()
        self._check(self._lib.mpm_get_counts(self.h, C.byref(n), C.byref(k), C.byref(t)))
        return n.value, k.value, t.value

    def profile(self, enable: bool = True) -> None:
        self._check(self._lib.mpm_profile_enable(self.h, 1 if enable else 0))

    def profile_read(self):
        ms, n = C.c_double(), C.c_int64()
        self._check(self._lib.mpm_profile_read(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def launches(self) -> int:
        c = C.c_int64()
        self._check(self._lib.mpm_launch_count(self.h, C.byref(c)))
        return c.value

    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self._lib.mpm_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def reset_clock(self) -> None:
        self._check(self._lib.mpm_reset_clock(self.h))


def metrics_aos_noalloc(params: A.MpmParams, d_particles: int, n: int, stream: int = 0) -> dict:
    """mpm_metrics_aos_noalloc: metrics of n MPMParticle records (504 bytes
    each) at device address d_particles, without a handle or any allocation.
    Calls on one device must not overlap."""
    m = A.MpmMetrics()
    A.check(A.lib().mpm_metrics_aos_noalloc(C.byref(params), C.c_void_p(d_particles or None), int(n),
                                            C.c_void_p(stream or None), C.byref(m)))
    return m.as_dict()


def tool_sdf_build(verts: np.ndarray, tris: np.ndarray, normals: Optional[np.ndarray] = None, padding: float = 0.002,
                   voxels_per_axis: int = 128) -> dict:
    """The voxel SDF of a closed tool mesh (mpm_tool_sdf_build) as the dict that
    Solver.set_tool_sdf takes: {"v": float32 [nz, ny, nx], "origin", "voxel", "angle": 0}."""
    L = A.lib()
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    nrm = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
    d = A.MpmToolSdf()
    args = (v.ctypes.data, len(v), t.ctypes.data, len(t), None if nrm is None else nrm.ctypes.data, float(padding),
            int(voxels_per_axis))
    A.check(L.mpm_tool_sdf_build(*args, C.byref(d), None))
    out = np.zeros((d.nz, d.ny, d.nx), np.float32)
    A.check(L.mpm_tool_sdf_build(*args, C.byref(d), out.ctypes.data))
    return {"v": out, "origin": tuple(d.origin), "voxel": float(d.voxel), "angle": 0.0}


class Batch(Solver):
    """Many independent workpieces in one handle (mpm_batch_*): every step of
    all of them is one persistent launch over the bins of all instances.
    Solver's own methods act on instance 0."""

    def __init__(self, params, capacities, stream: int = 0):
        self._lib = A.lib()
        n = len(params)
        arr = (A.MpmParams * n)(*params)
        caps = (C.c_int64 * n)(*map(int, capacities))
        h = C.c_void_p()
        A.check(self._lib.mpm_batch_create(arr, caps, n, C.c_void_p(stream or None), C.byref(h)))
        self.h = h
        self.params = list(params)
        self._keep = []

    def count(self) -> int:
        c = C.c_int32()
        self._check(self._lib.mpm_batch_count(self.h, C.byref(c)))
        return c.value

    def init_box_i(self, i: int, c0, c1, ppc: int, seed: int, instance_key: int = 0, fixed_layers: int = 2,
                   T0: float = 293.0, tool: Optional[dict] = None) -> int:
        a0 = (C.c_int32 * 3)(*map(int, c0))
        a1 = (C.c_int32 * 3)(*map(int, c1))
        t = self.tool_desc(tool) if tool else None
        self._check(self._lib.mpm_batch_init_box(self.h, int(i), a0, a1, int(ppc), C.c_uint64(seed),
                                                 C.c_uint32(instance_key), int(fixed_layers), float(T0),
                                                 C.byref(t) if t else None))
        return self.counts_i(i)[0]

    def set_tool_i(self, i: int, tool: dict) -> None:
        t = self.tool_desc(tool)
        self._check(self._lib.mpm_batch_set_tool(self.h, int(i), C.byref(t)))

    def set_tool_sdf_i(self, i: int, sdf: Optional[dict]) -> None:
        s = self.tool_sdf(sdf)
        self._check(self._lib.mpm_batch_set_tool_sdf(self.h, int(i), C.byref(s) if s is not None else None))

    def upload_i(self, i: int, parts: Dict[str, np.ndarray], elem: int = 8) -> None:
        s, keep, n = soa_in(parts, elem)
        self._check(self._lib.mpm_batch_upload(self.h, int(i), C.byref(s), n))

    def download_i(self, i: int, fields=None, elem: int = 8, strict: bool = True) -> Dict[str, np.ndarray]:
        s, out = soa_out(self.counts_i(i)[0], fields, elem)
        self._check_state(self._lib.mpm_batch_download(self.h, int(i), C.byref(s)), strict)
        return out

    def step_all(self, dts, nsteps: int = 1) -> None:
        d = np.ascontiguousarray(dts, dtype=np.float64)
        self._check(self._lib.mpm_batch_step(self.h, d.ctypes.data_as(C.POINTER(C.c_double)), int(nsteps)))

    def metrics_i(self, i: int) -> dict:
        m = A.MpmMetrics()
        self._check(self._lib.mpm_batch_sync_metrics(self.h, int(i), C.byref(m)))
        return m.as_dict()

    def instance_status(self) -> list:
        """mpm_status of every instance from its device error word (MPM_OK or
        MPM_NUMERIC; MPM_TIMEOUT for all after a bounded wait gave up)."""
        n = self.count()
        st = (C.c_int32 * max(n, 1))()
        self._check(self._lib.mpm_batch_instance_status(self.h, st, n))
        return list(st[:n])

    def counts_i(self, i: int):
        n, k, t = C.c_int64(), C.c_int64(), C.c_double()
        self._check(self._lib.mpm_batch_get_counts(self.h, int(i), C.byref(n), C.byref(k), C.byref(t)))
        return n.value, k.value, t.value

    def change(self, add_params=(), add_caps=(), remove=()) -> int:
        na, nr = len(add_params), len(remove)
        arr = (A.MpmParams * max(na, 1))(*add_params)
        caps = (C.c_int64 * max(na, 1))(*map(int, add_caps))
        rem = (C.c_int32 * max(nr, 1))(*map(int, remove))
        first = C.c_int32()
        self._check(self._lib.mpm_batch_change(self.h, arr, caps, na, rem, nr, C.byref(first)))
        self.params = [p for k, p in enumerate(self.params) if k not in set(remove)] + list(add_params)
        return first.value


    def autotune(self, dts) -> dict:
        d = np.ascontiguousarray(dts, dtype=np.float64)
        c = A.MpmLaunchConfig()
        self._check(self._lib.mpm_autotune(self.h, d.ctypes.data_as(C.POINTER(C.c_double)), C.byref(c)))
        return c.as_dict()


def make_request(case: dict, nsteps: int, precision: int = A.PREC_F32, dt: Optional[float] = None) -> A.MpmRequest:
    """mpm_request of a workpiece case (workpiece.make_case layout)."""
    from . import workpiece as W
    r = A.MpmRequest()
    r.params = W.to_mpm_params(case, precision=precision)
    r.tool = Solver.tool_desc(case["tool"])
    b = case["box"]
    for k in range(3):
        r.c0[k] = int(b["c0"][k])
        r.c1[k] = int(b["c1"][k])
    r.ppc = int(b["ppc"])
    r.fixed_layers = int(b["fixed_layers"])
    r.seed = int(b["seed"])
    r.instance_key = int(b["instance"])
    r.nsteps = int(nsteps)
    r.dt = float(dt if dt is not None else case["dt"])
    r.T0 = float(b["T0"])
    return r


class Server:
    """The serving loop (mpm_server_*): submit requests at any time, call
    tick() to admit, step and retire; poll() for results."""

    def __init__(self, precision: int = A.PREC_F32, hbm_budget_bytes: int = 8 << 30, max_chunk: int = 50,
                 max_resident: int = 0, use_graph: bool = True, backstress: bool = False, stream: int = 0,
                 max_resident_particles: int = 0, deterministic: bool = False):
        self._lib = A.lib()
        self.precision = precision
        self.cfg = A.MpmServerConfig(int(precision), int(max_chunk), int(hbm_budget_bytes), int(max_resident),
                                     1 if use_graph else 0, 1 if backstress else 0, 1 if deterministic else 0,
                                     int(max_resident_particles))
        h = C.c_void_p()
        A.check(self._lib.mpm_server_create(C.byref(self.cfg), C.c_void_p(stream or None), C.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            self._lib.mpm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, case: dict, nsteps: int, dt: Optional[float] = None) -> int:
        return self.submit_request(make_request(case, nsteps, self.precision, dt))

    def submit_request(self, r: A.MpmRequest) -> int:
        i = C.c_int64()
        A.check(self._lib.mpm_server_submit(self.h, C.byref(r), C.byref(i)))
        return i.value

    def cancel(self, rid: int) -> None:
        """Cancels a queued request at once, a running one at the next tick."""
        A.check(self._lib.mpm_server_cancel(self.h, int(rid)))

    def preempt(self, rid: int) -> None:
        """Saves a running request's workpiece at the next tick and queues it
        again; it resumes where it stopped when it is admitted again."""
        A.check(self._lib.mpm_server_preempt(self.h, int(rid)))

    def tick(self) -> int:
        n = C.c_int32()
        A.check(self._lib.mpm_server_tick(self.h, C.byref(n)))
        return n.value

    def poll(self, rid: int) -> dict:
        r = A.MpmResult()
        A.check(self._lib.mpm_server_poll(self.h, int(rid), C.byref(r)))
        return r.as_dict()

    def stats(self) -> dict:
        s = A.MpmServerStats()
        A.check(self._lib.mpm_server_stats_get(self.h, C.byref(s)))
        return s.as_dict()

    def footprint(self, case: dict, nsteps: int = 1) -> int:
        r = make_request(case, nsteps, self.precision)
        b = C.c_int64()
        A.check(self._lib.mpm_server_footprint(C.byref(self.cfg), C.byref(r), C.byref(b)))
        return b.value

