"""The bounds-checked build on the GPU: a child process loads
libmpm_b200_checked.so (MPM_B200_LIB) and runs the parity scenarios in FP64
through the fused and split schedules and the deterministic mode, a batch of
uneven workpieces, FP32 cutting with the particle-side contact and heat
conduction with the adiabatic shear model.  No index check may fail (every
index the step kernels derive from data is checked before it is used; a
failure is counted instead of trapped), and the FP64 results match the oracle
to 1e-9 of each field's scale, as the default library does."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

RUN = r"""
import json, sys
root = sys.argv[1]
sys.path[:0] = [root + "/edegpredict-engine-rotary_b200", root, root + "/tests", root + "/tests/golden"]
import ctypes as C
import numpy as np
from mpm_b200 import Batch, Solver, capi as A, workpiece as W
from scenarios import PARITY_SCENARIOS
from test_gpu_parity import field_errors
from oracle.oracle import Oracle

L = A.lib()
assert L._name.endswith("libmpm_b200_checked.so"), L._name
o = Oracle()
worst = {}

def run(case, st, n, prec, sched=A.SCHED_FUSED, det=False):
    s = Solver(W.to_mpm_params(case, precision=prec, schedule=sched), len(st["x"]) + 64)
    s.set_launch_config(deterministic=det)
    s.set_tool(case["tool"])
    if case["tool"].get("sdf") is not None:
        s.set_tool_sdf(case["tool"]["sdf"])
    s.upload(st)
    if "ext" in case:
        e = case["ext"]
        s.apply_external_force(e["center"], e["radius"], e["force"])
    s.step(case["dt"], n)
    out = s.download()
    s.close()
    return out

for name, make in PARITY_SCENARIOS.items():
    case, st, n, extf = make()
    ref, rc = o.step(case, st, n, extf=extf)
    modes = [("fused", A.SCHED_FUSED, False), ("split", A.SCHED_SPLIT, False)]
    p = case["params"]
    if not (p.get("asb_enabled") or p.get("heat_conduction") or case["tool"].get("sdf") is not None):
        modes.append(("det", A.SCHED_SPLIT, True))
    for label, sched, det in modes:
        out = run(case, st, n, A.PREC_F64, sched, det)
        err = field_errors(out, ref, case)
        worst[name + "/" + label] = max(err.values())
        assert (out["status"] == ref["status"]).all(), (name, label)

rng = np.random.default_rng(3)
cases = [W.config3_case(rng, i, cells_lo=8, cells_hi=20, steps=10) for i in range(4)]
caps = [int(np.prod(np.subtract(c["box"]["c1"], c["box"]["c0"]))) * c["box"]["ppc"] for c in cases]
bt = Batch([W.to_mpm_params(c) for c in cases], caps)
for i, c in enumerate(cases):
    b = c["box"]
    bt.init_box_i(i, b["c0"], b["c1"], b["ppc"], b["seed"], b["instance"], b["fixed_layers"], b["T0"], tool=c["tool"])
bt.step_all([c["dt"] for c in cases], 40)
bt.close()

case = W.config1(cells=(24, 12, 12), speed=20.0)
b = case["box"]
prm = W.to_mpm_params(case)
prm.contact_every = 1
s = Solver(prm, 24 * 12 * 12 * b["ppc"])
s.init_box(b["c0"], b["c1"], b["ppc"], b["seed"], 0, b["fixed_layers"], b["T0"], tool=case["tool"])
s.step(case["dt"], 60)
s.close()

v, site, idx = C.c_int64(), C.c_int32(), C.c_int64()
assert L.mpm_check_report(C.byref(v), C.byref(site), C.byref(idx), 1) == A.MPM_OK
print(json.dumps({"violations": v.value, "site": site.value, "index": idx.value, "worst": worst}))
"""


def test_checked_build_finds_no_violation():
    lib = ROOT / "edegpredict-engine-rotary_b200" / "mpm_b200" / "libmpm_b200_checked.so"
    assert lib.exists(), "build with edegpredict-engine-rotary_b200/build.py --checked"
    env = dict(os.environ, MPM_B200_LIB=str(lib))
    r = subprocess.run([sys.executable, "-c", RUN, str(ROOT)], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    rep = json.loads(r.stdout.strip().splitlines()[-1])
    assert rep["violations"] == 0, rep
    bad = {k: v for k, v in rep["worst"].items() if v > 1e-9}
    assert not bad, bad
