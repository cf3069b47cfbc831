"""luna.jl_b200 — B200 (sm_100a) implementation of Luna.jl's UPPE hot path.

The per-step right-hand sides (``NonlinearRHS.TransModeAvg``, ``TransRadial`` and
``TransModal``) with Kerr, plasma (``PlasmaCumtrapz`` with PPT/ADK rates) and Raman
responses, and the adaptive interaction-picture RK45 integrator that drives them
(``RK45.solve_precon`` inside ``Luna.run``), run as CUDA kernels behind the C ABI of
``libluna_b200.so`` (``include/luna_b200.h``). The Python modules here build the same inputs
the reference builds on the host (grids, modes, linear operators, rate tables, Raman
responses, cubature rules), call the library and organise scans and resumable runs; they
never evaluate the hot path on the CPU.
"""
from . import physdata, maths, grid, ionisation, raman, modes, linops, fields, nonlinear
from . import nonlinearrhs, interface, modal, output, scans

__all__ = ["physdata", "maths", "grid", "ionisation", "raman", "modes", "linops", "fields",
           "nonlinear", "nonlinearrhs", "interface", "modal", "output", "scans"]
