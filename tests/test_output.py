"""Resumable propagation (the HDF5Output cache of Output.jl:321-359, 473-488 and Luna.run's
resume, Luna.jl:374-379, with an .npz file): run on the C++ restatement of the integrator,
which has the device integrator's interface, so the host logic is checked without a GPU."""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import numpy as np
import pytest

from luna_b200 import output as O
from luna_b200.interface import prop_capillary_args
from oracle import cpu


def _problem():
    return prop_capillary_args(125e-6, 0.2, "Ar", 1.0, λ0=800e-9, τfwhm=10e-15, energy=120e-6,
                               λlims=(150e-9, 4e-6), trange=0.25e-12, saveN=11)


def _solver(p):
    cp = cpu.CpuPlan(p.transform)

    def solve(transform, linop, y, z0, dz0, zmax, zsave, max_dt):
        sv, yy, st = cp.solve(linop, y, z0, dz0, zmax, zsave=zsave, max_dt=max_dt)
        return sv, yy, st.z, st.dz, st.status
    return solve, cp


def test_segmented_run_matches_continuous(tmp_path):
    p = _problem()
    solve, cp = _solver(p)
    full, _, st = cp.solve(p.linop, p.Eω, 0.0, 1e-4, p.grid.zmax, saveN=11)
    o = O.run(p, O.CheckpointOutput(tmp_path / "a.npz", p.grid.zmax, 11), segments=4, solver=solve)
    assert len(o.Eω) == 11
    np.testing.assert_array_equal(o.data["z"], np.linspace(0, p.grid.zmax, 11))
    for a, b in zip(o.data["Eω"], full):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5  # the integrator's tolerance


def test_interrupted_run_resumes_from_the_cache(tmp_path):
    """An interrupted run resumed from its cache (check_cache) repeats the uninterrupted
    segmented run exactly."""
    p = _problem()
    solve, _ = _solver(p)
    ref = O.run(p, O.CheckpointOutput(tmp_path / "ref.npz", p.grid.zmax, 11), segments=5, solver=solve)
    path = tmp_path / "b.npz"
    seen = []

    def stop_after_two(z):
        seen.append(z)
        if len(seen) == 2:
            raise KeyboardInterrupt

    with pytest.raises(KeyboardInterrupt):
        O.run(p, O.CheckpointOutput(path, p.grid.zmax, 11), segments=5, solver=solve,
              on_segment=stop_after_two)
    out = O.CheckpointOutput(path, p.grid.zmax, 11)
    y, t, dt = out.check_cache(p.Eω, 0.0, 1e-4)
    assert t == seen[-1] and 0 < len(out.Eω) < 11
    out = O.run(p, out, segments=5, solver=solve)
    assert len(out.Eω) == 11
    for a, b in zip(out.data["Eω"], ref.data["Eω"]):
        np.testing.assert_array_equal(a, b)


def test_check_cache_ignores_missing_or_earlier_caches(tmp_path):
    p = _problem()
    out = O.CheckpointOutput(tmp_path / "none.npz", p.grid.zmax, 11)
    y, t, dt = out.check_cache(p.Eω, 0.0, 1e-4)
    assert t == 0.0 and dt == 1e-4 and y is p.Eω
    out.Eω = [p.Eω]
    out.write(p.Eω, 0.05, 2e-4)
    later = O.CheckpointOutput(tmp_path / "none.npz", p.grid.zmax, 11)
    assert later.check_cache(p.Eω, 0.1, 1e-4)[1] == 0.1  # the cache lies before t: not used
    other = O.CheckpointOutput(tmp_path / "none.npz", p.grid.zmax, 21)
    with pytest.raises(ValueError):
        other.check_cache(p.Eω, 0.0, 1e-4)


@pytest.mark.gpu
def test_device_resumable_run_matches_cpu_and_resumes_exactly(tmp_path):
    """output.run with the device integrator (its default solver): the segmented run agrees
    with the same segmented run on the C++ restatement, and an interrupted device run
    resumed from its cache repeats the uninterrupted device run exactly."""
    p = _problem()
    solve, _ = _solver(p)
    cpu_out = O.run(p, O.CheckpointOutput(tmp_path / "c.npz", p.grid.zmax, 11), segments=4, solver=solve)
    dev = O.run(p, O.CheckpointOutput(tmp_path / "d.npz", p.grid.zmax, 11), segments=4)
    assert len(dev.Eω) == 11
    for a, b in zip(dev.data["Eω"], cpu_out.data["Eω"]):
        # the same FP64 algorithm; the segments' step sequences follow rounding at this level
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5
    path = tmp_path / "e.npz"
    seen = []

    def stop_after_two(z):
        seen.append(z)
        if len(seen) == 2:
            raise KeyboardInterrupt

    with pytest.raises(KeyboardInterrupt):
        O.run(p, O.CheckpointOutput(path, p.grid.zmax, 11), segments=4, on_segment=stop_after_two)
    out = O.run(p, O.CheckpointOutput(path, p.grid.zmax, 11), segments=4)
    for a, b in zip(out.data["Eω"], dev.data["Eω"]):
        np.testing.assert_array_equal(a, b)
