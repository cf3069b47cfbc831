"""Mode-averaged UPPE transform, mirroring Luna.jl ``src/NonlinearRHS.jl``.

``TransModeAvg(grid, resp, densityfun, norm, aeff)`` (NonlinearRHS.jl:323-373) is a
callable ``t(nl, Eω, z)`` that fills ``nl`` with the nonlinear response of the field
``Eω``. Here the call runs the fused device right-hand side through the C-ABI library;
there is no host implementation behind it.

The normalisations ``norm_mode_average`` (NonlinearRHS.jl:375-387) and
``norm_mode_average_gnlse`` (NonlinearRHS.jl:389-399) are folded, together with the
frequency window on ``sidx``, into one complex factor per frequency bin that the device
applies after the forward transform. Bins outside ``sidx`` keep the raw transform
output, as in the reference.
"""
import math

import numpy as np

from . import physdata as pd

nlscale = math.sqrt(pd.eps_0 * pd.c / 2)


class _Norm:
    def __init__(self, pre, sidx):
        self.pre = pre  # complex prefactor on sidx bins (without sqrt(Aeff))
        self.sidx = sidx


def norm_mode_average(grid, βconst, shock=True):
    """``nl[i] *= pre[i]/β[i]*sqrt(Aeff)`` on sidx (NonlinearRHS.jl:375-387)."""
    ω = grid.ω
    shockterm = ω ** 2 if shock else ω * pd.wlfreq(grid.referenceλ)
    pre = -1j * shockterm / 4 / nlscale / pd.c
    return _Norm(pre / βconst, grid.sidx)


def norm_mode_average_gnlse(grid, shock=True):
    """``nl[i] *= pre[i]*sqrt(Aeff)`` on sidx (NonlinearRHS.jl:389-399)."""
    ω = grid.ω
    shockterm = ω ** 2 if shock else ω * pd.wlfreq(grid.referenceλ)
    with np.errstate(divide="ignore", invalid="ignore"):
        pre = -1j * shockterm / (2 * pd.c ** 1.5 * math.sqrt(2 * pd.eps_0)) / (ω / pd.c)
    pre = np.where(grid.sidx, pre, 0)
    return _Norm(pre, grid.sidx)


class TransModeAvg:
    """Mode-averaged transform E(ω) -> P_nl(ω) with constant density and effective area."""

    def __init__(self, grid, resp, density, norm, aeff):
        self.grid = grid
        self.resp = tuple(resp)
        self.density = float(density)
        self.norm = norm
        self.aeff = float(aeff)
        self._plan = None

    def output_factor(self):
        """Per-bin complex factor applied after the crop: norm * sqrt(Aeff) * ωwin on sidx."""
        g = self.grid
        f = np.ones(len(g.ω), dtype=np.complex128)
        s = g.sidx
        f[s] = self.norm.pre[s] * math.sqrt(self.aeff) * g.ωwin[s]
        return f

    def plan(self):
        if self._plan is None:
            from .plan import Plan
            self._plan = Plan.from_transform(self)
        return self._plan

    def __call__(self, nl, Eω, z):
        self.plan().rhs(nl, Eω, z)
