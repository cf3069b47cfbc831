"""Modal (multimode) transform, mirroring Luna.jl's ``TransModal`` (NonlinearRHS.jl:148-302).

``TransModal(grid, ts, resp, density, norm)`` is a callable ``t(nl, Eω, z)`` for modal fields
``Eω`` of shape (Nω, nmodes). For each transverse point the reference builds the real-space
field from the modes (``Modes.to_space!``, Modes.jl:458-495), transforms it to time, applies
the responses (vector Kerr for two polarisation components), transforms back, windows and
normalises (``norm_modal``; NonlinearRHS.jl:273-282) and projects onto every mode;
``Cubature.pcubature_v`` integrates that over the core radius (``full=false``: a radial
integral with weight 2πr).

On the device the transforms and the mode projection commute with the sum over points (they
are linear), so one inverse transform per mode feeds every point, the point sums are taken
on time samples and one forward transform per mode and cubature level gives the integral;
see ``modal_plan``. The cubature rule is fixed here on the host: the nested Clenshaw-Curtis
levels of the p-adaptive rule, their nodes on (0, a) and weights.

On the device: Kerr, plasma and Raman for one polarisation component, Kerr and the vector
plasma response for two. Not available on the device: ``full=true`` (the 2-D h-adaptive
``hcubature_v``; the transform describes it and the oracle evaluates it), envelope grids,
vector Raman (not implemented in the reference either) and the no-THG response forms.
"""
import math

import numpy as np

from . import physdata as pd

MAX_MODES = 16
MAX_LEVELS = 9  # 2^9 + 1 = 513 points: more than the default mfcn of 512 allows


class ToSpace:
    """``Modes.ToSpace(ms; components)`` (Modes.jl:411-442): the modes and the polarisation
    components (``"xy"``, ``"x"`` or ``"y"``) the real-space field keeps."""

    def __init__(self, modes, components="xy"):
        if components == "xy":
            self.indices = (0, 1)
        elif components == "x":
            self.indices = (0,)
        elif components == "y":
            self.indices = (1,)
        else:
            raise ValueError(f"components {components} not recognised")
        self.ms = tuple(modes)
        self.nmodes = len(self.ms)
        self.npol = len(self.indices)

    def ems(self, r, θ=0.0):
        """(nmodes, npol) matrix of ``Exy(m, (r, θ))[indices]`` (Modes.jl:486-489)."""
        out = np.empty((self.nmodes, self.npol))
        for i, m in enumerate(self.ms):
            e = m.Exy(r, θ)
            out[i] = [e[k] for k in self.indices]
        return out


def norm_modal(grid, shock=True):
    """``norm_modal(grid; shock)`` (NonlinearRHS.jl:311-316): the factor ``-iω/4`` (or
    ``-iω0/4`` without shock) that multiplies the projected polarisation."""
    if shock:
        return -1j * np.asarray(grid.ω, dtype=np.float64) / 4
    ω0 = pd.wlfreq(grid.referenceλ)
    return np.full(len(grid.ω), -1j * ω0 / 4)


def make_const_linop_modes(grid, modes, λ0, ref_mode=1, thg=False):
    """``make_const_linop(grid, modes, λ0; ref_mode=1)`` (LinearOps.jl:401-435): one column
    per mode with β = 1 outside sidx and the frame velocity of mode ``ref_mode`` (1-based) at
    λ0; ``i(-β + ω β1) - α/2`` on a field-resolved grid (α on sidx), and on an envelope grid
    ``-i(β - (ω - ω0) β1 - βref) - α/2`` with βref = β(ω0) of the reference mode (0 with THG)
    and α over every bin. Unlike the single-mode operator, bins outside sidx are not
    zeroed."""
    ω0 = pd.wlfreq(λ0)
    β1 = modes[ref_mode - 1].dispersion(1, ω0)
    s = grid.sidx
    env = grid.kind == "env"
    βref = 0.0 if (not env or thg) else float(modes[ref_mode - 1].β(np.array([ω0]))[0])
    L = np.zeros((len(grid.ω), len(modes)), dtype=np.complex128)
    for i, m in enumerate(modes):
        β = np.ones(len(grid.ω))
        β[s] = m.β(grid.ω[s])
        α = np.zeros(len(grid.ω))
        if env:
            α = np.asarray(m.α(grid.ω), dtype=np.float64).copy()
        else:
            α[s] = m.α(grid.ω[s])
        α = np.clip(α, 0.0, 3000.0)
        if env:
            L[:, i] = -1j * (β - (grid.ω - grid.ω0) * β1 - βref) - α / 2
        else:
            L[:, i] = 1j * (-β + grid.ω * β1) - α / 2
    return L


def clenshaw_curtis(n):
    """Nodes cos(jπ/n) and weights of the (n+1)-point Clenshaw-Curtis rule on [-1, 1], n
    even: w_j = c_j/n (1 - sum_{k=1}^{n/2} b_k cos(2kjπ/n)/(4k² - 1)) with c_0 = c_n = 1,
    c_j = 2 otherwise, b_{n/2} = 1, b_k = 2 otherwise."""
    j = np.arange(n + 1)
    x = np.cos(j * math.pi / n)
    k = np.arange(1, n // 2 + 1)
    b = np.where(k == n // 2, 1.0, 2.0)
    s = (b / (4.0 * k * k - 1))[None, :] * np.cos(2.0 * np.outer(j, k) * math.pi / n)
    c = np.where((j == 0) | (j == n), 1.0, 2.0)
    return x, c / n * (1.0 - s.sum(axis=1))


def cubature_levels(mfcn):
    """Levels of the p-adaptive rule that fit in ``mfcn`` evaluations: level l has 2^(l+1)+1
    points, level 0 is always taken."""
    L = 0
    while L + 1 < MAX_LEVELS and (2 << (L + 1)) + 1 <= mfcn:
        L += 1
    return L + 1


def cubature_tables(a, nlevels, npre=True):
    """Interior nodes of the nested rules on (0, a) in evaluation order (slot 0: the centre,
    level 0; then the 2^l points each level l >= 1 adds) and the weight of every slot in
    every level's rule, 2πr included: ``(r[nslots], wts[nlevels, nslots], wlow)`` with wlow
    the weight of slot 0 in the midpoint rule that level 0's error estimate compares with.
    The two end points (r = 0 and r = a) contribute nothing (pointcalc!,
    NonlinearRHS.jl:234-271) and have no slot."""
    L = nlevels - 1
    nf = 2 << L  # intervals of the finest rule
    c, h = a / 2, a / 2
    idx = [nf // 2]
    for l in range(1, nlevels):
        s = 1 << (L - l)
        idx += list(range(s, nf, 2 * s))
    idx = np.array(idx)
    xf = np.cos(idx * math.pi / nf)
    r = c + h * xf
    pre = 2 * math.pi * r if npre else np.ones_like(r)
    wts = np.zeros((nlevels, len(idx)))
    for l in range(nlevels):
        s = 1 << (L - l)
        _, w = clenshaw_curtis(2 << l)
        on = idx % s == 0
        wts[l, on] = h * w[idx[on] // s] * pre[on]
    wlow = h * 2.0 * pre[0]
    return r, wts, wlow


class TransModal:
    """Modal transform E(ω) -> P_nl(ω) with constant density (NonlinearRHS.jl:148-302).

    ``rtol``, ``atol`` and ``mfcn`` are the pcubature tolerances and evaluation limit of the
    reference's constructor (NonlinearRHS.jl:203-216)."""

    kind = "modal"

    def __init__(self, grid, ts, resp, density, norm, rtol=1e-3, atol=0.0, mfcn=512, full=False):
        dl = [m.dimlimits() for m in ts.ms]
        if any(d[0] != "polar" for d in dl) or len({d[2][0] for d in dl}) != 1:
            raise NotImplementedError("modes must share polar limits (0, a)")
        self.grid, self.ts = grid, ts
        self.resp = tuple(resp)
        self.density = float(density)
        self.norm = np.asarray(norm, dtype=np.complex128)
        self.rtol, self.atol, self.mfcn = float(rtol), float(atol), int(mfcn)
        self.full = bool(full)  # full=true: described (the oracle evaluates it), not on the device
        self.a = dl[0][2][0]
        self._plan = None

    def output_factor(self):
        """ωwin then norm! on every bin (NonlinearRHS.jl:279-281)."""
        return self.grid.ωwin * self.norm

    def tables(self):
        """(ems[nslots, nmodes, npol], wts[nlevels, nslots], wlow) of the device rule."""
        nl = cubature_levels(self.mfcn)
        r, wts, wlow = cubature_tables(self.a, nl)
        ems = np.stack([self.ts.ems(ri) for ri in r])
        return ems, wts, wlow

    def plan(self):
        if self.full:
            raise NotImplementedError("the full 2-D modal integral (hcubature) is not available on "
                                      "the device; use full=False")
        if self._plan is None:
            from .modal_plan import ModalPlan
            self._plan = ModalPlan.from_transform(self)
        return self._plan

    def __call__(self, nl, Eω, z):
        self.plan().rhs(nl, Eω, z)


def doinput_mm(grid, inputs, nmodes):
    """``doinput_mm!`` (Luna.jl:154-171): a field or a tuple of fields goes into mode 1; a
    tuple of ``{"mode": i, "fields": (...)}`` (1-based ``i``) adds each field to its mode."""
    Eω = np.zeros((len(grid.ω), nmodes), dtype=np.complex128)
    if callable(inputs):
        inputs = ({"mode": 1, "fields": (inputs,)},)
    elif all(callable(f) for f in inputs):
        inputs = ({"mode": 1, "fields": tuple(inputs)},)
    for inp in inputs:
        for f in inp["fields"]:
            Eω[:, inp["mode"] - 1] += f(grid)
    return Eω


def setup_modal(grid, density, responses, inputs, modes, components, full=False, norm=None,
                rtol=1e-3, atol=0.0, mfcn=512):
    """``Luna.setup(grid, densityfun, responses, inputs, modes, components; full, norm!,
    rtol, atol, mfcn)`` (Luna.jl:173-227, field-resolved and envelope grids) with a constant
    density: (Eω, transform)."""
    ts = ToSpace(modes, components=components)
    norm = norm_modal(grid) if norm is None else norm
    t = TransModal(grid, ts, responses, density, norm, rtol=rtol, atol=atol, mfcn=mfcn, full=full)
    return doinput_mm(grid, inputs, len(modes)), t
