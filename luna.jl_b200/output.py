"""Resumable propagation: the cache of Luna.jl's ``HDF5Output`` without HDF5.

``HDF5Output`` (Output.jl:321-359) appends the saved spectra to its file and, with
``cache=true``, rewrites ``meta/cache`` = (y, t, dt, saved) after every save; ``Luna.run``
(Luna.jl:374-379) asks ``check_cache`` (Output.jl:473-488) for that state and, when it lies
beyond z0, restarts ``RK45.solve_precon`` from it. No HDF5 library is available here, so
``CheckpointOutput`` keeps the same contents in an ``.npz`` file (written to a temporary file
and renamed, so an interrupted write leaves the previous cache). The integrator resumes from
any (y, z, dz): ``luna_b200_solve`` takes y, z0 and dz0 and reports the final z and dz.

``run`` integrates in segments: each segment runs the solver from the cached state to the
next mark on the fibre, saving on the whole fibre's save grid, and the cache is written after
every segment. Each segment starts the solver afresh, as the reference's resume does: the
first right-hand side is evaluated from the cached state and the step controller's memory
of the last error is reset, so a segmented run agrees with a continuous one to the
integrator's tolerance (1e-6 relative on a 20 cm argon case with rtol = 1e-6), while a run
that is interrupted and resumed from its cache repeats the uninterrupted segmented run
exactly.
"""
import os

import numpy as np


class CheckpointOutput:
    """Saved spectra on ``saveN`` points of [z0, zmax] plus the resume cache, in ``path``."""

    def __init__(self, path, zmax, saveN, z0=0.0):
        self.path = str(path)
        self.zgrid = np.linspace(z0, zmax, saveN)
        self.Eω = []
        self.cache = None

    def check_cache(self, y, t, dt):
        """``check_cache(o::HDF5Output, y, t, dt)`` (Output.jl:473-488): the cached (y, t, dt)
        if the file holds a cache at or beyond t, else the arguments. Restores the saved
        spectra."""
        if not os.path.exists(self.path):
            return y, t, dt
        with np.load(self.path) as d:
            tc = float(d["t"])
            if tc < t:
                return y, t, dt
            n = int(d["saved"])
            if n > len(self.zgrid) or not np.array_equal(d["zgrid"], self.zgrid):
                raise ValueError("the cache in the file belongs to a different save grid")
            self.Eω = list(d["Eω"][:n])
            self.cache = (d["y"].copy(), tc, float(d["dt"]))
        return self.cache

    def write(self, y, t, dt):
        tmp = self.path + ".tmp.npz"
        Ew = np.array(self.Eω) if self.Eω else np.zeros((0,) + np.shape(y), dtype=np.complex128)
        np.savez(tmp, y=y, t=t, dt=dt, saved=len(self.Eω), Eω=Ew, zgrid=self.zgrid)
        os.replace(tmp, self.path)
        self.cache = (y, t, dt)

    @property
    def data(self):
        n = len(self.Eω)
        return {"Eω": np.array(self.Eω), "z": self.zgrid[:n]}


def device_solver(precision=None, **kw):
    """The device integrator (``plan.solve_precon``) in the form ``run`` calls."""
    from . import _lib
    from .plan import solve_precon

    def solve(transform, linop, y, z0, dz0, zmax, zsave, max_dt):
        r = solve_precon(transform, linop, y, z0, dz0, zmax, zsave=zsave, max_dt=max_dt,
                         precision=_lib.PREC_FP64 if precision is None else precision,
                         raise_on_status=False, **kw)
        return r.Eω, r.y, r.zfinal, r.dzfinal, r.status
    return solve


def run(problem, output, segments=8, init_dz=1e-4, solver=None, on_segment=None):
    """``Luna.run(Eω, grid, linop, transform, FT, output)`` (Luna.jl:358-391) with a
    resumable output: resume from ``output.check_cache``, then integrate segment by segment
    (max_dz = zmax/2 as Luna.run sets it), writing the cache after each. ``solver(transform,
    linop, y, z0, dz0, zmax, zsave, max_dt)`` returns (saves, y, z, dz, status); the default
    is the device integrator. ``on_segment(z)`` is called after each cache write. Returns
    ``output``."""
    solver = device_solver() if solver is None else solver
    g = problem.grid
    zmax = g.zmax
    y, t, dt = output.check_cache(np.array(problem.Eω, dtype=np.complex128), 0.0, init_dz)
    marks = np.linspace(0.0, zmax, segments + 1)[1:]
    marks[-1] = zmax
    for zm in marks:
        if t > zmax:
            break
        if t > zm:
            continue
        zsave = np.ascontiguousarray(output.zgrid[len(output.Eω):])
        if len(zsave) == 0:  # every point saved (the last step ended exactly at zmax)
            break
        saves, y, t, dt, status = solver(problem.transform, problem.linop, y, t, dt, zm, zsave,
                                         zmax / 2)
        output.Eω.extend(list(saves))
        output.write(y, t, dt)
        if status != 0:
            raise RuntimeError(f"solver status {status} at z = {t}")
        if on_segment is not None:
            on_segment(t)
    return output
