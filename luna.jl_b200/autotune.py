"""Autotuner of a batch's CTA-per-instance shapes (the reference has no counterpart: its
scans run one ``prop_capillary`` after another, Scans.jl:275-353).

For every grid class of a batch (oversampled length No and whether a Raman response is
present) and the batch's precision it measures the device time of one RK step on one CTA,
on an 8-CTA cluster and (for the 32768-point grids) on a 16-CTA cluster (a batch of one
representative instance, the difference of two step budgets, CUDA events), once per device,
and caches the table in a JSON file (``$LUNA_B200_TUNE_CACHE``, default
``~/.cache/luna_b200/tune.json``). An instance's
predicted integration time on a shape is its class's time per step times its predicted
step count, ``scan.nonlinear_phase(p) ** 0.6`` up to a constant (the step model of
``scan.schedule_priority``; the constant cancels in every decision below).

The shapes follow from the table: an instance goes to a cluster when the cluster is faster
for its class and its single-CTA time is above the mean load of an SM (the total predicted
single-CTA time over the SMs), i.e. when it would otherwise set the makespan, and to a
cluster of 16 when that is faster still and its time on 8 would be at least twice the mean
load; the priority (processing order, longest first) is the predicted time on the chosen
shape.
"""
import json
import os
import time

import numpy as np

from . import _lib
from . import plan as P
from . import scan


def _cache_path():
    return os.environ.get("LUNA_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "luna_b200", "tune.json"))


def _device_key():
    import torch
    lib_t = os.path.getmtime(_lib.LIB_PATH)
    return f"{torch.cuda.get_device_name()}|{int(lib_t)}"


def grid_class(prob):
    raman = any(r.kind in ("raman_field", "raman_env") for r in prob.transform.resp)
    return f"No={prob.grid.No}{'+Raman' if raman else ''}"


def _step_ms(prob, precision, flags, steps, shape=None):
    """Device ms per RK step of one instance (difference of two step budgets) and whether
    it ran on a cluster; ``shape`` (2: 8 CTAs, 3: 16 CTAs) forces the cluster size."""
    t, on_cluster = [], False
    plan = P.Plan.from_transform(prob.transform, precision)
    for s in steps:
        b = P.Batch([plan], 2, np.array([0.0, prob.grid.zmax]), max_steps=s, flags=flags,
                    max_dt=prob.grid.zmax / 2)
        b.upload([prob.linop], [prob.Eω], [0.0], [1e-4], [prob.grid.zmax])
        if shape is not None:
            b.set_shapes([shape])
            b.set_priority([1.0])
        on_cluster = b.info()[1] > 0
        b.run()
        t.append(b.run())
        done = b.download()[2][0].steps
        if done < s:  # the instance ended (or failed) before the budget: no estimate
            return None, on_cluster
    return (t[1] - t[0]) / (steps[1] - steps[0]), on_cluster


def measure(probs, precision, steps=(20, 80), refresh=False, log=None, tries=8):
    """{class: {"single": ms/step, "cluster": ms/step or None}} for the classes of probs,
    from the cache where present."""
    path = _cache_path()
    try:
        with open(path) as f:
            cache = json.load(f)
    except Exception:
        cache = {}
    key = f"{_device_key()}|prec={precision}"
    table = cache.get(key, {}) if not refresh else {}
    members = {}
    for p in probs:
        members.setdefault(grid_class(p), []).append(p)
    t0 = time.perf_counter()
    for c, ps in members.items():
        if c in table and table[c].get("single"):
            continue
        # the first member of the class that runs the whole step budget (an instance that
        # stops early, e.g. at the PPT table limit, gives no timing)
        row = {"single": None, "cluster": None, "cluster16": None}
        for p in ps[:tries]:
            single, _ = _step_ms(p, precision, _lib.SOLVE_NO_DIST | _lib.SOLVE_NO_CLUSTERS, steps)
            if single is None:
                continue
            cl, on = _step_ms(p, precision, 0, steps, shape=2)
            row = {"single": single, "cluster": cl if on else None, "cluster16": None}
            if on and p.grid.No >= 32768:  # 16 CTAs need 1024 sample pairs each
                c16, on16 = _step_ms(p, precision, 0, steps, shape=3)
                row["cluster16"] = c16 if on16 else None
            break
        table[c] = row
        if log:
            log(f"autotune {c}: single {row['single']} ms/step, cluster {row['cluster']} ms/step")
    cache[key] = table
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1)
    except OSError:
        pass
    return table, time.perf_counter() - t0


def schedule(params, probs, table, nsm):
    """(shapes [n], priorities [n], predicted seconds on the chosen shapes [n]) for a
    batch: shapes 3 (cluster of 16), 2 (cluster of 8) or 1 (one CTA) as described in the
    module docstring."""
    n = len(probs)
    w = np.array([scan.nonlinear_phase(p) ** 0.6 for p in params])
    single = np.zeros(n)
    cluster = np.full(n, np.inf)
    cluster16 = np.full(n, np.inf)
    # a class without a timing (every tried member stopped early) falls back to the
    # transform-cost model of scan.schedule_priority, scaled like the measured classes
    measured = [(int(c.split("=")[1].split("+")[0]), r["single"]) for c, r in table.items() if r.get("single")]
    ref = np.mean([s / (No * np.log2(No)) for No, s in measured]) if measured else 1.0
    for i, p in enumerate(probs):
        row = table.get(grid_class(p), {})
        s = row.get("single")
        if not s:
            No = p.grid.No
            s = ref * No * np.log2(No) * (2.0 if "Raman" in grid_class(p) else 1.0)
        single[i] = w[i] * s
        if row.get("cluster"):
            cluster[i] = w[i] * row["cluster"]
        elif not row.get("single") and p.grid.No >= 16384:
            cluster[i] = single[i] / 2.0  # untimed long grid: assume the typical cluster gain
        if row.get("cluster16"):
            cluster16[i] = w[i] * row["cluster16"]
    mean_load = single.sum() / max(1, nsm)
    shapes = np.where((cluster < single) & (single >= mean_load), 2, 1)
    # 16 CTAs for a clustered instance that would still take twice the mean SM load on 8
    shapes = np.where((shapes == 2) & (cluster16 < cluster) & (cluster >= 2 * mean_load), 3, shapes)
    pred = np.where(shapes == 3, cluster16, np.where(shapes == 2, cluster, single))
    return shapes.astype(int), pred, pred
