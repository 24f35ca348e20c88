"""ctypes view of the drop-in adapter's C driver (adapter/adapter_driver.cpp,
built by build.py --adapter into adapter/_build/libmpm_adapter.so against the
reference's headers).

The driver exposes MPMSolverB200 -- the class that replaces the reference's
MPMSolver behind IPhysicsSolver / IMetricsProvider (include/MPMSolver.h:34) --
through plain C calls, so that Python can drive it in SimulationEngine's call
pattern (src/SimulationEngine.cpp:495-536): setToolPosition,
beginInterpolatedToolMotion, interpolateToolForSubStep + step per sub-step,
endInterpolatedToolMotion, syncMetrics.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _capi as A

DRIVER = Path(__file__).resolve().parent.parent / "adapter" / "_build" / "libmpm_adapter.so"


def available() -> bool:
    return DRIVER.exists()


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not DRIVER.exists():
            raise RuntimeError(f"adapter driver not built: {DRIVER} (build.py --adapter with MPM_REFERENCE_SRC "
                               "naming the reference source tree)")
        L = C.CDLL(str(DRIVER))
        P = C.POINTER
        d, vp, i32 = C.c_double, C.c_void_p, C.c_int32
        for name, res, args in (
                ("mad_create", vp, [C.c_int]), ("mad_destroy", None, [vp]), ("mad_status", C.c_int, [vp]),
                ("mad_error", C.c_char_p, [vp]), ("mad_initialize_params", C.c_int, [vp, P(A.MpmParams)]),
                ("mad_init_seeded_box", C.c_int, [vp, P(i32), P(i32), C.c_int, C.c_uint64, C.c_int, d, vp]),
                ("mad_particle_count", C.c_int, [vp]), ("mad_set_tool_position", None, [vp, P(d)]),
                ("mad_begin_interp", None, [vp, vp, C.c_int]), ("mad_interp_substep", None, [vp, vp, d]),
                ("mad_end_interp", None, [vp, vp]), ("mad_step", None, [vp, d]), ("mad_pending", C.c_int, [vp]),
                ("mad_flush", None, [vp]), ("mad_sync_metrics", None, [vp, P(d), P(A.MpmMetrics)]),
                ("mad_get_particles", C.c_int64, [vp, vp, C.c_int64]), ("mad_device_particles", vp, [vp]),
                ("mad_stream", vp, [vp]), ("mad_handle", vp, [vp]),
                ("mad_fem_node_layout", C.c_int, [P(i32), P(i32)])):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def fem_node_layout() -> tuple[int, list[int]]:
    """sizeof(FEMNodeGPU) and the byte offsets of x, y, z, vx, vy, vz."""
    size, off = C.c_int32(), (C.c_int32 * 6)()
    lib().mad_fem_node_layout(C.byref(size), off)
    return size.value, list(off)


def fem_node_records(points: np.ndarray, velocity) -> np.ndarray:
    """FEMNodeGPU records (as bytes) at the given positions, all moving with
    `velocity`; the other members zero."""
    size, off = fem_node_layout()
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    rec = np.zeros((len(pts), size // 8), np.float64)
    for a in range(3):
        rec[:, off[a] // 8] = pts[:, a]
        rec[:, off[3 + a] // 8] = velocity[a]
    return rec.view(np.uint8).ravel()


class Adapter:
    """One MPMSolverB200 instance through the C driver."""

    def __init__(self, max_particles: int):
        self.L = lib()
        self.a = self.L.mad_create(int(max_particles))

    def ok(self, rc=0):
        if rc != 0 or self.L.mad_status(self.a) != 0:
            raise RuntimeError(f"MPMSolverB200: {self.L.mad_error(self.a).decode()} (rc {rc}, status "
                               f"{self.L.mad_status(self.a)})")

    def initialize(self, params: A.MpmParams):
        self.ok(self.L.mad_initialize_params(self.a, C.byref(params)))

    def seeded_box(self, c0, c1, ppc, seed, fixed_layers, T0, tool: dict | None = None) -> int:
        from .solver import Solver
        desc = C.byref(Solver.tool_desc(tool)) if tool is not None else None
        self.ok(self.L.mad_init_seeded_box(self.a, (C.c_int32 * 3)(*c0), (C.c_int32 * 3)(*c1), int(ppc), int(seed),
                                           int(fixed_layers), float(T0), desc))
        return self.L.mad_particle_count(self.a)

    def set_tool_position(self, p):
        self.L.mad_set_tool_position(self.a, (C.c_double * 3)(*p))

    def begin_interp(self, d_nodes: int, n: int):
        self.L.mad_begin_interp(self.a, C.c_void_p(d_nodes), int(n))

    def interp_substep(self, d_nodes: int, alpha: float):
        self.L.mad_interp_substep(self.a, C.c_void_p(d_nodes), float(alpha))

    def end_interp(self, d_nodes: int):
        self.L.mad_end_interp(self.a, C.c_void_p(d_nodes))

    def step(self, dt: float):
        self.L.mad_step(self.a, float(dt))

    def pending(self) -> int:
        return self.L.mad_pending(self.a)

    def flush(self):
        self.L.mad_flush(self.a)

    def sync_metrics(self) -> tuple[list[float], A.MpmMetrics]:
        iface, full = (C.c_double * 4)(), A.MpmMetrics()
        self.L.mad_sync_metrics(self.a, iface, C.byref(full))
        return list(iface), full

    def launches(self) -> int:
        n = C.c_int64()
        A.check(A.lib().mpm_launch_count(C.c_void_p(self.L.mad_handle(self.a)), C.byref(n)))
        return n.value

    def handle(self) -> int:
        return self.L.mad_handle(self.a)

    def stream(self) -> int:
        return self.L.mad_stream(self.a) or 0

    def device_particles(self) -> int:
        return self.L.mad_device_particles(self.a)

    def count(self) -> int:
        return self.L.mad_particle_count(self.a)

    def particles(self) -> np.ndarray:
        n = self.count()
        buf = np.zeros(n * A.MPM_PARTICLE.itemsize, np.uint8)
        assert self.L.mad_get_particles(self.a, buf.ctypes.data, buf.nbytes) == n
        return buf.view(A.MPM_PARTICLE)

    def close(self):
        if self.a:
            self.L.mad_destroy(self.a)
            self.a = None
