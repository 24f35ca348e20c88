"""ctypes binding of include/mpm_capi.h (libmpm_b200.so).

Only plain C types cross the boundary.  Importing this module loads the
library that build.py placed next to it and fails loudly when it is missing:
there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

# MPM_B200_LIB selects another build of the library (the bounds-checked
# libmpm_b200_checked.so) before the first call of lib().
LIB_PATH = Path(os.environ.get("MPM_B200_LIB") or Path(__file__).resolve().parent / "libmpm_b200.so")

MPM_ABI_VERSION = 1
MPM_OK, MPM_INVALID_ARG, MPM_OOM, MPM_CUDA_ERROR, MPM_NUMERIC, MPM_OUT_OF_GRID, MPM_TIMEOUT, \
    MPM_NOT_SUPPORTED, MPM_CAPACITY, MPM_CANCELLED = range(10)
ACTIVE, INACTIVE, CHIP, BOUNDARY, FIXED = 0, 1, 2, 3, 4
PREC_F32, PREC_F64 = 0, 1
TOOL_NONE, TOOL_RASTER, TOOL_SDF_STICKY, TOOL_SDF_SLIP = 0, 1, 2, 3
SHAPE_CYLINDER_Y, SHAPE_WEDGE_Y = 0, 1
PLAST_EXPLICIT, PLAST_NEWTON = 0, 1
SCHED_SPLIT, SCHED_FUSED = 0, 1

# fields of mpm_import_aos
AOS_POSITION, AOS_VELOCITY, AOS_TEMPERATURE, AOS_STATUS, AOS_EXT_FORCE = 1, 2, 4, 8, 16
AOS_WRITABLE = 31

# MPMParticle (the reference's include/Types.h:199-266) as a numpy record, 504 bytes
MPM_PARTICLE = np.dtype([
    ("x", "f8"), ("y", "f8"), ("z", "f8"), ("vx", "f8"), ("vy", "f8"), ("vz", "f8"), ("fx", "f8"), ("fy", "f8"),
    ("fz", "f8"), ("ext_fx", "f8"), ("ext_fy", "f8"), ("ext_fz", "f8"), ("density", "f8"), ("pressure", "f8"),
    ("volume", "f8"), ("mass", "f8"), ("temperature", "f8"), ("F", "f8", 9), ("F_p", "f8", 9), ("C", "f8", 9),
    ("stress", "f8", 6), ("backstress", "f8", 6), ("plasticStrain", "f8"), ("strainRate", "f8"), ("damage", "f8"),
    ("residualStress", "f8"), ("id", "i4"), ("status", "i4"), ("cellHash", "i4"), ("lodZone", "i4"),
    ("lastUpdateStep", "i4"), ("asbCounter", "u1"), ("_pad", "u1", 3)])
assert MPM_PARTICLE.itemsize == 504

_d, _i32, _i64, _vp = C.c_double, C.c_int32, C.c_int64, C.c_void_p


class MpmParams(C.Structure):
    _fields_ = [
        ("abi_version", _i32), ("precision", _i32), ("nx", _i32), ("ny", _i32), ("nz", _i32), ("plasticity", _i32),
        ("dx", _d), ("origin", _d * 3), ("particle_mass", _d), ("particle_volume", _d),
        ("E", _d), ("nu", _d), ("rho_phys", _d), ("cp", _d), ("beta", _d), ("Tm", _d), ("Tamb", _d),
        ("jc_A", _d), ("jc_B", _d), ("jc_n", _d), ("jc_C", _d), ("jc_m", _d), ("edot0", _d), ("H_kin", _d),
        ("D1", _d), ("D2", _d), ("D3", _d), ("D4", _d), ("D5", _d), ("D_th", _d),
        ("fixture_thickness", _d), ("fixture_damping", _d), ("gravity_z", _d), ("mass_threshold", _d),
        ("apic_dinv_factor", _d), ("apic_decay", _d), ("deps_cap", _d), ("dT_cap", _d),
        ("lod_enabled", _i32), ("chip_every", _i32), ("lod_active_r", _d), ("lod_near_r", _d),
        ("newton_tol", _d), ("newton_maxit", _i32), ("schedule", _i32), ("sort_every", _i32),
        ("threads_per_block", _i32), ("contact_every", _i32), ("_pad_contact", _i32), ("contact_radius", _d),
        ("contact_friction", _d), ("contact_heat_partition", _d),
        ("asb_enabled", _i32), ("_pad_asb", _i32), ("asb_critical_rate", _d), ("asb_taylor_quinney", _d),
        ("asb_max_temp_ratio", _d), ("asb_touch_rise", _d),
        ("heat_conduction", _i32), ("_pad_heat", _i32), ("thermal_conductivity", _d),
    ]


class MpmToolSdf(C.Structure):
    _fields_ = [("nx", _i32), ("ny", _i32), ("nz", _i32), ("_pad", _i32), ("values", _vp),
                ("origin", C.c_float * 3), ("voxel", C.c_float), ("angle", C.c_float), ("_pad2", C.c_float)]


class MpmToolDesc(C.Structure):
    _fields_ = [
        ("mode", _i32), ("shape", _i32), ("position", _d * 3), ("velocity", _d * 3), ("radius", _d),
        ("rake", _d), ("clearance", _d), ("tip_dz", _d), ("n_samples", _i32), ("_pad", _i32),
        ("sample_dx", _vp), ("sample_dy", _vp), ("sample_dz", _vp),
    ]


class MpmToolNodes(C.Structure):
    """mpm_tool_nodes: the raster tool from FEM node records in device memory."""
    _fields_ = [("start", _vp), ("end", _vp), ("n", _i32), ("stride", _i32), ("off_pos", _i32 * 3),
                ("off_vel", _i32 * 3), ("alpha0", _d), ("dalpha", _d)]


class MpmWorkpieceParams(C.Structure):
    """mpm_workpiece_params: MPMWorkpieceSolver's own constants."""
    _fields_ = [("failure_strain", _d), ("critical_plastic_strain", _d), ("thermal_chip_ratio", _d),
                ("tool_contact_radius", _d), ("contact_damping", _d), ("max_contact_temp_rise", _d),
                ("thermal_clamp", _i32), ("_pad", _i32)]


class MpmParticlesSoa(C.Structure):
    _fields_ = [("elem", _i32), ("_pad", _i32)] + [
        (n, _vp) for n in ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "stress", "backstress",
                           "plastic_strain", "strain_rate", "temperature", "damage", "residual_stress", "status",
                           "id")
    ]


class MpmMetrics(C.Structure):
    _fields_ = [
        ("ref_max_stress", _d), ("ref_max_temperature", _d), ("ref_kinetic", _d), ("ref_internal", _d),
        ("mass", _d), ("momentum", _d * 3), ("kinetic", _d), ("internal_elastic", _d), ("thermal", _d),
        ("max_temperature", _d), ("max_von_mises", _d), ("max_plastic_strain", _d), ("mean_plastic_strain", _d),
        ("n_active", _i64), ("n_chip", _i64), ("n_fixed", _i64), ("n_inactive", _i64),
        ("bounds_min", _d * 3), ("bounds_max", _d * 3), ("n_escaped", _i64), ("n_sorts", _i64),
        ("n_yielded", _i64), ("n_contacts", _i64), ("contact_work", _d), ("contact_force", _d),
        ("n_asb_heated", _i64),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


PARTICLE_FIELDS = {  # name -> values per particle
    "x": 1, "y": 1, "z": 1, "vx": 1, "vy": 1, "vz": 1, "F": 9, "Fp": 9, "C": 9, "stress": 6, "backstress": 6,
    "plastic_strain": 1, "strain_rate": 1, "temperature": 1, "damage": 1, "residual_stress": 1,
}

REQ_UNKNOWN, REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = range(6)


class MpmRequest(C.Structure):
    _fields_ = [("params", MpmParams), ("tool", MpmToolDesc), ("c0", _i32 * 3), ("c1", _i32 * 3), ("ppc", _i32),
                ("fixed_layers", _i32), ("seed", C.c_uint64), ("instance_key", C.c_uint32), ("nsteps", _i32),
                ("dt", _d), ("T0", _d)]


class MpmResult(C.Structure):
    _fields_ = [("state", _i32), ("status", _i32), ("n_particles", _i64), ("steps_done", _i64),
                ("t_submit", _d), ("t_admit", _d), ("t_done", _d), ("metrics", MpmMetrics)]

    def as_dict(self) -> dict:
        return {"state": self.state, "status": self.status, "n_particles": self.n_particles,
                "steps_done": self.steps_done, "t_submit": self.t_submit, "t_admit": self.t_admit,
                "t_done": self.t_done, "metrics": self.metrics.as_dict()}


class MpmServerConfig(C.Structure):
    _fields_ = [("precision", _i32), ("max_chunk", _i32), ("hbm_budget_bytes", _i64), ("max_resident", _i32),
                ("use_graph", _i32), ("backstress", _i32), ("deterministic", _i32), ("max_resident_particles", _i64)]


class MpmServerStats(C.Structure):
    _fields_ = [("offered", _i64), ("admitted", _i64), ("completed", _i64), ("failed", _i64), ("queued", _i64),
                ("resident", _i64), ("particle_updates", _i64), ("resident_particles", _i64), ("ticks", _i64),
                ("busy_seconds", _d), ("cancelled", _i64), ("preempted", _i64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class MpmLaunchConfig(C.Structure):
    _fields_ = [("ctas_per_sm", C.c_int32), ("sort_every", C.c_int32), ("use_graph", C.c_int32),
                ("deterministic", C.c_int32), ("pass_size", C.c_int32)]

    def as_dict(self) -> dict:
        return {"ctas_per_sm": self.ctas_per_sm, "sort_every": self.sort_every, "use_graph": self.use_graph,
                "deterministic": self.deterministic, "pass_size": self.pass_size}


_lib = None


def lib() -> C.CDLL:
    """Load libmpm_b200.so (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run edegpredict-engine-rotary_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER
        sig = {
            "mpm_params_default": (_i32, [P(MpmParams)]),
            "mpm_create": (_i32, [P(MpmParams), _i64, _vp, P(_vp)]),
            "mpm_destroy": (_i32, [_vp]),
            "mpm_init_box": (_i32, [_vp, P(_i32), P(_i32), _i32, C.c_uint64, C.c_uint32, _i32, _d, P(MpmToolDesc)]),
            "mpm_upload": (_i32, [_vp, P(MpmParticlesSoa), _i64]),
            "mpm_download": (_i32, [_vp, P(MpmParticlesSoa)]),
            "mpm_export_aos": (_i32, [_vp, _vp, _i64]),
            "mpm_import_aos": (_i32, [_vp, _vp, _i64, C.c_uint32]),
            "mpm_set_tool_nodes": (_i32, [_vp, _vp]),
            "mpm_set_workpiece_semantics": (_i32, [_vp, _vp]),
            "mpm_batch_set_tool_nodes": (_i32, [_vp, _i32, _vp]),
            "mpm_batch_export_aos": (_i32, [_vp, _i32, _vp, _i64]),
            "mpm_batch_import_aos": (_i32, [_vp, _i32, _vp, _i64, C.c_uint32]),
            "mpm_set_tool": (_i32, [_vp, P(MpmToolDesc)]),
            "mpm_set_tool_sdf": (_i32, [_vp, P(MpmToolSdf)]),
            "mpm_batch_set_tool_sdf": (_i32, [_vp, _i32, P(MpmToolSdf)]),
            "mpm_tool_sdf_build": (_i32, [_vp, _i32, _vp, _i32, _vp, _d, _i32, P(MpmToolSdf), _vp]),
            "mpm_step": (_i32, [_vp, _d, _i32]),
            "mpm_stable_dt": (_i32, [_vp, _d, P(_d)]),
            "mpm_sync_metrics": (_i32, [_vp, P(MpmMetrics)]),
            "mpm_metrics_aos_noalloc": (_i32, [P(MpmParams), _vp, _i64, _vp, P(MpmMetrics)]),
            "mpm_batch_create": (_i32, [P(MpmParams), P(_i64), _i32, _vp, P(_vp)]),
            "mpm_batch_count": (_i32, [_vp, P(_i32)]),
            "mpm_batch_init_box": (_i32, [_vp, _i32, P(_i32), P(_i32), _i32, C.c_uint64, C.c_uint32, _i32, _d,
                                          P(MpmToolDesc)]),
            "mpm_batch_upload": (_i32, [_vp, _i32, P(MpmParticlesSoa), _i64]),
            "mpm_batch_download": (_i32, [_vp, _i32, P(MpmParticlesSoa)]),
            "mpm_batch_set_tool": (_i32, [_vp, _i32, P(MpmToolDesc)]),
            "mpm_batch_step": (_i32, [_vp, P(_d), _i32]),
            "mpm_batch_sync_metrics": (_i32, [_vp, _i32, P(MpmMetrics)]),
            "mpm_batch_get_counts": (_i32, [_vp, _i32, P(_i64), P(_i64), P(_d)]),
            "mpm_batch_instance_status": (_i32, [_vp, P(_i32), _i32]),
            "mpm_checkpoint_bytes": (_i32, [_vp, _i32, P(_i64)]),
            "mpm_checkpoint_save": (_i32, [_vp, _i32, _vp, _i64]),
            "mpm_checkpoint_load": (_i32, [_vp, _i32, _vp, _i64]),
            "mpm_batch_change": (_i32, [_vp, P(MpmParams), P(_i64), _i32, P(_i32), _i32, P(_i32)]),
            "mpm_server_create": (_i32, [P(MpmServerConfig), _vp, P(_vp)]),
            "mpm_server_destroy": (_i32, [_vp]),
            "mpm_server_submit": (_i32, [_vp, P(MpmRequest), P(_i64)]),
            "mpm_server_tick": (_i32, [_vp, P(_i32)]),
            "mpm_server_poll": (_i32, [_vp, _i64, P(MpmResult)]),
            "mpm_server_cancel": (_i32, [_vp, _i64]),
            "mpm_server_preempt": (_i32, [_vp, _i64]),
            "mpm_check_report": (_i32, [P(_i64), P(_i32), P(_i64), _i32]),
            "mpm_server_stats_get": (_i32, [_vp, P(MpmServerStats)]),
            "mpm_server_footprint": (_i32, [P(MpmServerConfig), P(MpmRequest), P(_i64)]),
            "mpm_get_launch_config": (_i32, [_vp, P(MpmLaunchConfig)]),
            "mpm_set_launch_config": (_i32, [_vp, P(MpmLaunchConfig)]),
            "mpm_autotune": (_i32, [_vp, P(_d), P(MpmLaunchConfig)]),
            "mpm_selftest_bounded_wait": (_i32, [_i64, _vp]),
            "mpm_set_mass_scaling": (_i32, [_vp, _d]),
            "mpm_apply_external_force": (_i32, [_vp, P(_d), _d, P(_d)]),
            "mpm_set_temperatures": (_i32, [_vp, P(_d), _i64]),
            "mpm_get_counts": (_i32, [_vp, P(_i64), P(_i64), P(_d)]),
            "mpm_get_stream": (_i32, [_vp, P(_vp)]),
            "mpm_reset_clock": (_i32, [_vp]),
            "mpm_launch_count": (_i32, [_vp, P(_i64)]),
            "mpm_profile_enable": (_i32, [_vp, _i32]),
            "mpm_profile_read": (_i32, [_vp, P(_d), P(_i64)]),
            "mpm_last_error": (C.c_char_p, [_vp]),
            "mpm_status_string": (C.c_char_p, [_i32]),
        }
        # entry points a library built before them lacks: it still loads, and a
        # call of one of them raises AttributeError
        later = {"mpm_import_aos", "mpm_batch_export_aos", "mpm_batch_import_aos", "mpm_set_tool_nodes",
                 "mpm_batch_set_tool_nodes", "mpm_set_workpiece_semantics"}
        for name, (res, args) in sig.items():
            if name in later and not hasattr(L, name):
                continue
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class MpmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{lib().mpm_status_string(status).decode()}: {msg}")
        self.status = status


def check(status: int, handle=None) -> None:
    if status != MPM_OK:
        msg = lib().mpm_last_error(handle)
        raise MpmError(status, msg.decode() if msg else "")


def default_params() -> MpmParams:
    p = MpmParams()
    check(lib().mpm_params_default(C.byref(p)))
    return p
