"""B200 MPM workpiece step: Python access to libmpm_b200.so (C ABI in include/mpm_capi.h)."""
from . import _capi as capi  # noqa: F401
from .solver import Batch, Server, Solver, tool_sdf_build  # noqa: F401
from . import workpiece  # noqa: F401
