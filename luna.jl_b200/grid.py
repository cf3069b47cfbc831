"""Time/frequency grids (host setup).

Restates Luna.jl ``src/Grid.jl``: ``RealGrid`` (Grid.jl:38-81) for field-resolved
propagation with a 6x-oversampled nonlinear grid, and ``EnvGrid`` (Grid.jl:115-190) for
complex envelopes. The device consumes the arrays these produce (``omega``, ``sidx``,
``omega_win``, ``towin``, ``twin``) through the plan descriptor.
"""
import math

import numpy as np

from . import physdata as pd
from .maths import planck_taper


class RealGrid:
    """Field-resolved grid: coarse t/omega plus the oversampled nonlinear grid to/omega_o."""

    kind = "real"

    def __init__(self, zmax, referenceλ, λ_lims, trange, δt=1.0):
        f_lims = [pd.c / l for l in λ_lims]
        dto = min(1 / (6 * max(f_lims)), δt)
        samples = 2 ** int(math.ceil(math.log2(trange / dto)))
        trange_even = dto * samples
        dwo = 2 * math.pi / trange_even
        No = np.arange(samples, dtype=np.float64)
        to = (No - samples / 2) * dto
        wo = np.arange(samples // 2 + 1, dtype=np.float64) * dwo
        wmin = 2 * math.pi * min(f_lims)
        wmax = 2 * math.pi * max(f_lims)
        wmax_win = 1.1 * wmax
        cropidx = int(np.argmax(wo > wmax_win)) + 1  # 1-based findfirst
        cropidx = 2 ** int(math.ceil(math.log2(cropidx))) + 1
        w = wo[:cropidx]
        dt = math.pi / w.max()
        tsamples = (cropidx - 1) * 2
        Nt = np.arange(tsamples, dtype=np.float64)
        t = (Nt - tsamples / 2) * dt
        self.zmax = float(zmax)
        self.referenceλ = referenceλ
        self.t, self.ω, self.to, self.ωo = t, w, to, wo
        self.ωwin = planck_taper(w, wmin / 2, wmin, wmax, wmax_win)
        self.twin = planck_taper(t, t.min(), -trange / 2, trange / 2, t.max())
        self.towin = planck_taper(to, to.min(), -trange / 2, trange / 2, to.max())
        self.sidx = (w > wmin / 2) & (w < wmax_win)
        self.ω0 = None

    @property
    def N(self):
        return len(self.t)

    @property
    def No(self):
        return len(self.to)


class EnvGrid:
    """Complex-envelope grid (Grid.jl:115-190)."""

    kind = "env"

    def __init__(self, zmax, referenceλ, λ_lims, trange, δt=1.0, thg=False):
        fmin = pd.c / max(λ_lims)
        fmax = pd.c / min(λ_lims)
        fmax_win = 1.1 * fmax
        w0 = 2 * math.pi * pd.c / referenceλ
        if thg:
            ffac = 6
            f_lims = (fmin, fmax)
        else:
            ffac = 2
            f_lims = (fmin, fmax_win)
        rf = [f - pd.c / referenceλ for f in f_lims]
        dt_f = 1 / (ffac * max(rf))
        if dt_f <= δt:
            dto = dt_f
            oversampling = thg
        else:
            dto = δt
            oversampling = True
        samples = 2 ** int(math.ceil(math.log2(trange / dto)))
        trange_even = dto * samples
        dwo = 2 * math.pi / trange_even
        No = np.arange(samples, dtype=np.float64)
        to = (No - samples / 2) * dto
        vo = np.fft.fftshift((No - samples / 2) * dwo)
        wo = vo + w0
        wmin = 2 * math.pi * fmin
        wmax = 2 * math.pi * fmax
        wmax_win = 2 * math.pi * fmax_win
        if oversampling:
            cropidx = int(np.argmax(wo >= (wmax_win - dwo))) + 1
            cropidx = 2 ** int(math.ceil(math.log2(cropidx)))
            v = np.concatenate([vo[:cropidx], vo[-cropidx:]])
        else:
            v = vo
        dt = -math.pi / v.min()
        tsamples = len(v)
        Nt = np.arange(tsamples, dtype=np.float64)
        t = (Nt - tsamples / 2) * dt
        w = v + w0
        self.zmax = float(zmax)
        self.referenceλ = referenceλ
        self.ω0 = w0
        self.t, self.ω, self.to, self.ωo = t, w, to, wo
        self.sidx = (w > wmin / 2) & (w < wmax_win)
        self.ωwin = planck_taper(w, wmin / 2, wmin, wmax, wmax_win)
        self.twin = planck_taper(t, t.min(), -trange / 2, trange / 2, t.max())
        self.towin = planck_taper(to, to.min(), -trange / 2, trange / 2, to.max())

    @property
    def N(self):
        return len(self.t)

    @property
    def No(self):
        return len(self.to)
