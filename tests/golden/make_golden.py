"""Generates tests/golden/*.npz from the REFERENCE's own CUDA kernels.

    python tests/golden/make_golden.py [outdir]

Needs a GPU and oracle/_ref/libmpm_ref.so (the reference's src/MPMSolver.cu
built from its sources by oracle/Makefile).  For every scenario of
scenarios.py it stores the input state, the reference's state after n steps,
and the reference's own stats kernel (computeParticleStatsKernel) on it.
The reference kernels accumulate with FP64 atomics, so two runs differ in
the last bits; the run-to-run spread of the reference is stored too.
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
from scenarios import SCENARIOS  # noqa: E402

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "F", "Fp", "C", "stress", "backstress", "plastic_strain", "strain_rate",
          "temperature", "damage", "residual_stress", "status", "id")


def main(outdir: Path) -> None:
    rk = RefKern()
    outdir.mkdir(parents=True, exist_ok=True)
    for name, fn in SCENARIOS.items():
        case, st, n, extf = fn()
        st["lod"] = np.zeros(len(st["x"]), np.int32)
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
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE)
