"""Parameter scans over capillary instances and their split across GPUs.

Replaces the sequential ``Scans.runscan`` loop over ``prop_capillary`` calls
(Scans.jl:275-494) by one batched device launch per GPU. Instances are independent, so a
multi-GPU scan shards them by estimated cost with no collective on the data path.
"""
import math

import numpy as np

from .interface import prop_capillary_args

GASES = ("He", "Ne", "Ar", "H2")
RAMAN_GASES = ("N2", "H2", "D2", "N2O", "CH4", "SF6")
RADII = (75e-6, 100e-6, 125e-6, 150e-6)


def draw_instances(n=256, seed=20261203):
    """Seeded uniform draw of the capillary scan family (one dict of arguments each)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(dict(
            energy=float(rng.uniform(50e-6, 400e-6)),
            pressure=float(rng.uniform(0.5, 5.0)),
            gas=GASES[int(rng.integers(0, len(GASES)))],
            radius=RADII[int(rng.integers(0, len(RADII)))],
            τfwhm=float(rng.uniform(8e-15, 30e-15)),
            flength=float(rng.uniform(1.0, 3.0)),
            λmin=float(rng.uniform(120e-9, 200e-9)),
            λmax=float(rng.uniform(3e-6, 5e-6)),
            trange=float(rng.uniform(0.5e-12, 2e-12)),
        ))
    return out


def build_problem(p, λ0=800e-9, saveN=201):
    return prop_capillary_args(p["radius"], p["flength"], p["gas"], p["pressure"], λ0=λ0,
                               τfwhm=p["τfwhm"], energy=p["energy"],
                               λlims=(p["λmin"], p["λmax"]), trange=p["trange"], saveN=saveN)


def cost_estimate(prob):
    """Relative cost of one instance: transform work per RHS times the fibre length."""
    No = prob.grid.No
    return No * math.log2(No) * prob.grid.zmax


def nonlinear_phase(p):
    """Scale of the nonlinear phase of an instance, gamma3 * pressure * (energy/duration) *
    length / radius^2 (arbitrary units): the step count of the adaptive integrator grows
    with it, so it orders a batch's instances longest first."""
    from . import physdata as pd
    return (pd.gamma3_gas(p["gas"]) * p["pressure"] * p["energy"] / p["τfwhm"] * p["flength"]
            / p["radius"] ** 2)


def _work(No, raman, p):
    return No * math.log2(No) * (2.0 if raman else 1.0) * nonlinear_phase(p) ** 0.6


def schedule_priority(p, prob):
    """Estimated work of an instance: per-step transform cost times nonlinear phase^0.6."""
    raman = any(r.kind in ("raman_field", "raman_env") for r in prob.transform.resp)
    return _work(prob.grid.No, raman, p)


def shard_cost(p, λ0=800e-9):
    """``schedule_priority`` of an instance from its arguments alone (the grid, without the
    mode and response set-up), so that every rank of a multi-GPU scan computes the same
    costs for the whole draw cheaply and deterministically. Raman is on for the molecular
    gases, as in ``prop_capillary``'s default (Interface.jl:538-556)."""
    from .grid import RealGrid
    g = RealGrid(p["flength"], λ0, (p["λmin"], p["λmax"]), p["trange"])
    return _work(g.No, p["gas"] in RAMAN_GASES, p)


def partition(costs, nparts):
    """Longest-processing-time-first split of instance indices into ``nparts`` shards."""
    order = np.argsort(-np.asarray(costs, dtype=np.float64), kind="stable")
    loads = [0.0] * nparts
    shards = [[] for _ in range(nparts)]
    for i in order:
        j = int(np.argmin(loads))
        shards[j].append(int(i))
        loads[j] += float(costs[i])
    return [sorted(s) for s in shards]


def shard(costs, rank, world):
    """Indices this rank integrates (disjoint across ranks, covering all instances)."""
    return partition(costs, world)[rank]
