"""Record the reference step and RHS counts of every instance of the 256-instance scan.

Test infrastructure (CPU baseline of bench.py). Runs the plain FP64 device integrator,
whose accepted-step sequence is the reference's (checked against this oracle in
tests/test_gpu_parity.py), over the seeded scan with Luna.run's settings (dz0 = 1e-4,
max_dz = zmax/2, 201 saves per instance) and writes oracle/scan256_nrhs.json.

    python oracle/make_scan256_nrhs.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import luna_b200_loader  # noqa: E402

luna_b200_loader.load()
from luna_b200 import plan as P, scan  # noqa: E402


def main():
    inst = scan.draw_instances(256)
    probs = [scan.build_problem(p) for p in inst]
    plans = [p.transform.plan() for p in probs]
    b = P.Batch(plans, 201, np.linspace(0, 1, 201), max_steps=200000)
    b.upload([p.linop for p in probs], [p.Eω for p in probs], [0.0] * 256, [1e-4] * 256,
             [p.grid.zmax for p in probs], [np.linspace(0, p.grid.zmax, 201) for p in probs],
             [p.grid.zmax / 2 for p in probs])
    ms = b.run()
    _, _, stats = b.download()
    out = {"source": "plain FP64 device integrator (reference step sequence), seed 20261203",
           "device_ms": ms,
           "steps": [int(s.steps) for s in stats], "nrhs": [int(s.nrhs) for s in stats],
           "status": [int(s.status) for s in stats]}
    with open(os.path.join(ROOT, "oracle", "scan256_nrhs.json"), "w") as f:
        json.dump(out, f)
    print("instances", len(stats), "failed", sum(1 for s in stats if s.status), "device s", ms / 1e3)


if __name__ == "__main__":
    main()
