"""The benchmarked 256-instance scan at full length: a stratified subset of its instances
integrated by the benchmark's batched FP64 solver (long instances distributed over 8-CTA
clusters) against full FP64 solves of the C++ restatement of the reference algorithm
(``tests/golden/scan_subset.npz``, written by ``oracle/make_scan256_nrhs.py``: counts,
final states, |Eω|^2 at four saves and the step sequences).

Subset (scan indices): 93, the longest instance (H2 with Raman on the 32768-point grid,
~27,000 RK steps over 2.7 m); 90 (Ar, 32768 points), 73 (Ar, 16384 points) and 13 (H2,
16384 points), which the batch integrates on clusters; 97 (Ne) and 253 (He) on the
8192-point grid; 0 (Ar), which stops at its first step with the PPT "field exceeds
maximum" error in the oracle.

Instance 253 is not determined beyond rounding in FP64: a one-ulp change of its first step
(or a 1e-12 change of its input) moves its spectra by up to 0.5 (measured on a B200, like
22 other instances of the scan), so for it only the status and the step count are
compared (its free-running step count differs as well: 6210 against the oracle's 6321
on a B200). Bars for the others: on the oracle's step sequence the spectral intensity at
every compared save and at the end within 1e-6 (the saves are stored as FP32, the step
sequence as FP32 step sizes, whose rounding moves the solution by far less); free-running (the benchmark's setting) the same status and step
count within 0.1 %, and the metric's 1e-3 relative spectral L2 of |Eω|^2 at every compared
save.
"""
import os

import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import numpy as np
import pytest

from luna_b200 import _lib, scan
from luna_b200 import plan as P

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "scan_subset.npz")
SAVEN = 201
CHAOTIC = {253}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def runs():
    g = np.load(GOLD)
    subset = [int(i) for i in g["subset"]]
    inst = scan.draw_instances(256)
    probs = [scan.build_problem(inst[i], saveN=SAVEN) for i in subset]
    prios = [scan.schedule_priority(inst[i], p) for i, p in zip(subset, probs)]
    out = {}
    for mode in ("free", "replay"):
        plans = [P.Plan.from_transform(p.transform, _lib.PREC_FP64) for p in probs]
        b = P.Batch(plans, SAVEN, np.linspace(0.0, 1.0, SAVEN))
        if mode == "replay":
            for j, i in enumerate(subset):
                seq = g[f"seq_{i}"].astype(np.float64)
                b.set_replay(j, np.stack([np.abs(seq), (seq > 0).astype(np.float64)], axis=1).ravel())
        b.upload([p.linop for p in probs], [p.Eω for p in probs], [0.0] * len(probs),
                 [1e-4] * len(probs), [p.grid.zmax for p in probs],
                 [np.linspace(0.0, p.grid.zmax, SAVEN) for p in probs],
                 [p.grid.zmax / 2 for p in probs])
        b.set_priority(prios)
        info = b.info()
        b.run()
        out[mode] = (b.results(), info)
    return g, subset, out


def test_scan_subset_runs_distributed(runs):
    _, _, out = runs
    assert out["free"][1][1] >= 3  # 93, 90, 73 (and 13) on 8-CTA clusters


def test_scan_subset_fp64_on_the_oracle_step_sequence(runs):
    g, subset, out = runs
    res, _ = out["replay"]
    for i, r in zip(subset, res):
        assert r.status == int(g[f"status_{i}"]), i
        assert r.steps == int(g[f"steps_{i}"]), (i, r.steps)
        if r.status != 0 or i in CHAOTIC:
            continue
        # the final state sits at the first z beyond the fibre end, which the FP32 step
        # sizes move by ~1e-7 m: compare its spectral intensity (the saves are at fixed z)
        fin = np.abs(g[f"final_{i}"]) ** 2
        assert _rel(np.abs(r.y) ** 2, fin) < 1e-6, (i, _rel(np.abs(r.y) ** 2, fin))
        for k, spec in zip(g["save_idx"], g[f"spec_{i}"]):
            assert _rel(np.abs(r.Eω[k]) ** 2, spec.astype(np.float64)) < 1e-6, (i, k)


def test_scan_subset_fp64_free_running_within_the_metric_bar(runs):
    g, subset, out = runs
    res, _ = out["free"]
    for i, r in zip(subset, res):
        assert r.status == int(g[f"status_{i}"]), i
        if r.status != 0 or i in CHAOTIC:
            continue
        n = int(g[f"steps_{i}"])
        assert abs(r.steps - n) <= max(1, n // 1000), (i, r.steps, n)
        for k, spec in zip(g["save_idx"], g[f"spec_{i}"]):
            e = _rel(np.abs(r.Eω[k]) ** 2, spec.astype(np.float64))
            assert e <= 1e-3, (i, k, e)
        assert _rel(np.abs(r.y) ** 2, np.abs(g[f"final_{i}"]) ** 2) <= 1e-3, i
