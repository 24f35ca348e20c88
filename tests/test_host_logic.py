"""Host-side logic: workpiece configurations, the chunked generator, tool
samples, and the benchmark's JSON helpers."""
from __future__ import annotations

import math

import numpy as np

from mpm_b200 import capi as A, workpiece as W


def test_config_shapes_match_the_named_workloads():
    c1, c2, c4 = W.config1(), W.config2(), W.config4()
    assert c1["cells"] == (64, 32, 32) and c1["box"]["ppc"] == 8 and c1["params"]["dx"] == 5e-5
    assert c2["cells"] == (256, 128, 128) and c2["params"]["dx"] == 2e-5
    assert c4["cells"] == (128, 64, 64)
    assert abs(c1["dt"] - 0.3 * 5e-5 / math.sqrt(205e9 / 7850)) < 1e-20
    assert c1["params"]["jc_A"] == 792e6 and c2["params"]["jc_n"] == 0.93
    # candidates: 64*32*32*8 = 524288, minus those inside the tool at t=0
    n = len(W.generate_box(c1)["x"])
    assert 500_000 < n < 524_288


def test_kill_zone_clear_of_the_workpiece():
    for case in (W.config1(), W.config2(), W.config4()):
        p, b = case["params"], case["box"]
        for a, nn in enumerate((p["nx"], p["ny"], p["nz"])):
            assert b["c0"][a] >= 1 and b["c1"][a] < nn - 2


def test_chunked_generator_equals_full():
    case = W.config1(cells=(16, 8, 8))
    x, y, z, st = W.generate_box_chunked(case, zchunk=3)
    full = W.generate_box(case)
    assert np.array_equal(x, full["x"]) and np.array_equal(z, full["z"]) and np.array_equal(st, full["status"])


def test_tool_samples_lie_on_the_surface():
    for case in (W.config1(), W.config2()):
        s = W.tool_samples(case)
        t = case["tool"]
        phi = W.tool_sdf(t, s[:, 0] + t["position"][0], s[:, 2] + t["position"][2], t["position"][0],
                         t["position"][2])
        assert np.abs(phi).max() < 1e-12


def test_generator_excludes_tool_and_fixes_bottom_layers():
    case = W.config1(cells=(24, 8, 8))
    g = W.generate_box(case)
    t = case["tool"]
    assert (W.tool_sdf(t, g["x"], g["z"], t["position"][0], t["position"][2]) > 0).all()
    zc = np.floor((g["z"] - case["params"]["origin"][2]) / case["params"]["dx"]) - case["box"]["c0"][2]
    assert ((zc < 2) == (g["status"] == A.FIXED)).all()
