"""Pressure-gradient capillary fills, mirroring Luna.jl.

* ``Gradient`` — Capillary.gradient(gas, L, p0, p1) (Capillary.jl:306-315):
  p(z) = sqrt(p0^2 + z/L (p1^2 - p0^2)) inside [0, L], p0 before and p1 after, and the
  multi-point form gradient(gas, Z, P) (:317-337), the same law on each segment; the core
  index sqrt(1 + γ(λ) ρ(z)). The density is this package's closed form (ideal gas with a
  second virial coefficient, ``physdata.density``) where the reference interpolates a
  CoolProp spline.
* ``MarcatiliGradientMode`` — MarcatiliMode(a, coren) with that z-dependent core index:
  the waveguide term nwg(ω) (``neff_wg``, Capillary.jl:188-200) is fixed and
  neff(ω; z) = sqrt(coren(ω; z)^2 - nwg(ω)) (Capillary.jl:216-224, neff_β_grid :345-360).
* ``make_linop`` — LinearOps.make_linop for a field-resolved grid (LinearOps.jl:337-360):
  L(ω; z) = -i(ω/c conj_clamp(neff(ω; z)) - ω β1(z)) on sidx (conj_clamp, :254), and
  βfun(z) for the normalisation.
* ``TransModeAvgZ`` — TransModeAvg with densityfun(z) and norm_mode_average's βfun!(β, z)
  (NonlinearRHS.jl:362-387).
"""
import math

import numpy as np

from . import modes, physdata as pd
from .nonlinearrhs import TransModeAvg, nlscale


class Gradient:
    """Two-point fill ``Gradient(gas, L, p0, p1)`` (Capillary.jl:306-315) or multi-point fill
    ``Gradient(gas, Z, P)`` (Capillary.jl:317-337); pressures in bar."""

    def __init__(self, gas, L_or_Z, p0_or_P, p1=None, T=pd.roomtemp):
        self.gas, self.T = gas, T
        if p1 is not None:
            self.two_point = True
            self.Z = np.array([0.0, float(L_or_Z)])
            self.P = np.array([float(p0_or_P), float(p1)])
        else:
            self.two_point = False
            self.Z = np.asarray(L_or_Z, dtype=np.float64).copy()
            self.P = np.asarray(p0_or_P, dtype=np.float64).copy()
            if len(self.Z) != len(self.P) or len(self.Z) < 2 or np.any(np.diff(self.Z) <= 0):
                raise ValueError("Z must be increasing and match P in length")
        self.L = float(self.Z[-1])
        self.p0, self.p1 = float(self.P[0]), float(self.P[-1])
        self.gam = pd.sellmeier_gas(gas)
        # density(p) = a p / (1 + b p), p in bar (physdata.density written out)
        self.dens_a = pd.bar / (pd.k_B * T)
        self.dens_b = pd._B2.get(gas, 0.0) * pd.bar / (pd._R_GAS * T)

    def p(self, z):
        Z, P = self.Z, self.P
        if self.two_point:
            if z > Z[1]:
                return P[1]
            if z <= 0:
                return P[0]
            return math.sqrt(P[0] ** 2 + z / Z[1] * (P[1] ** 2 - P[0] ** 2))
        if z <= Z[0]:
            return P[0]
        if z >= Z[-1]:
            return P[-1]
        i = int(np.searchsorted(Z, z, side="left")) - 1  # last i with Z[i] < z
        return math.sqrt(P[i] ** 2 + (z - Z[i]) / (Z[i + 1] - Z[i]) * (P[i + 1] ** 2 - P[i] ** 2))

    def density(self, z):
        p = self.p(z)
        return self.dens_a * p / (1.0 + self.dens_b * p)

    def gamma(self, ω):
        """Sellmeier susceptibility per unit density at ω."""
        return np.asarray(self.gam(pd.wlfreq(np.asarray(ω, dtype=np.float64)) * 1e6), dtype=np.float64)

    def coren(self, ω, z):
        return np.sqrt(1 + (self.gamma(ω) * self.density(z)).astype(complex))


class MarcatiliGradientMode(modes.MarcatiliMode):
    def __init__(self, a, grad, n=1, m=1, kind="HE", model="full", loss=True):
        if model != "full":
            raise NotImplementedError("only the full Marcatili model")
        super().__init__(a, None, 1.0, n=n, m=m, kind=kind, model=model, loss=loss)
        self.grad = grad

    def nwg(self, ω):
        """Waveguide part (unm/(k a))^2 (1 - i vn/(k a))^2 (Capillary.jl:188-200)."""
        ω = np.asarray(ω, dtype=np.float64)
        εcl = pd.sio2_index(pd.wlfreq(ω)) ** 2
        vn = self._vn(εcl)
        k = ω / pd.c
        return (self.unm / (k * self.a)) ** 2 * (1 - 1j * vn / (k * self.a)) ** 2

    def neff_grid(self, ω, z):
        """neff(mode, coren^2, nwg) (Capillary.jl:216-224): no clamp."""
        εco = self.grad.coren(ω, z) ** 2
        n = np.sqrt(εco - self.nwg(ω))
        return n if self.loss else np.real(n) + 0j

    def neff_z(self, ω, z):
        """neff(m, ω; z) of the full model with its low-index rule (Capillary.jl:162-173)."""
        n = self.neff_grid(ω, z)
        re = np.where(np.real(n) < 1e-3, 1e-3, np.real(n))
        im = np.where(np.real(n) < 1e-3, np.clip(np.imag(n), 0, None), np.imag(n))
        return re + 1j * im

    def dispersion_z(self, ω0, z):
        """β1(z) = dβ/dω at ω0: the 4-point central difference of MarcatiliMode.dispersion."""
        h = ω0 * 1e-4
        f = lambda x: float(x / pd.c * np.real(self.neff_z(np.array([x]), z))[0])
        return (-f(ω0 + 2 * h) + 8 * f(ω0 + h) - 8 * f(ω0 - h) + f(ω0 - 2 * h)) / (12 * h)


def conj_clamp(n, ω):
    """LinearOps.conj_clamp (LinearOps.jl:254)."""
    return np.clip(np.real(n), 1e-3, None) - 1j * np.clip(np.imag(n), 0, 3000 * pd.c / ω)


def make_linop(grid, mode, λ0):
    """(linop(z), βfun(z)) for a field-resolved grid (LinearOps.jl:337-360)."""
    ω0 = pd.wlfreq(λ0)
    s = grid.sidx
    ω = grid.ω

    def linop(z):
        out = np.zeros(len(ω), dtype=np.complex128)
        β1 = mode.dispersion_z(ω0, z)
        nc = conj_clamp(mode.neff_grid(ω[s], z), ω[s])
        out[s] = -1j * (ω[s] / pd.c * nc - ω[s] * β1)
        return out

    def βfun(z):
        out = np.ones(len(ω))
        out[s] = ω[s] / pd.c * np.real(mode.neff_grid(ω[s], z))
        return out

    return linop, βfun


class TransModeAvgZ(TransModeAvg):
    """TransModeAvg with a z-dependent density and normalisation (pressure gradient)."""

    kind = "modeavg_z"

    def __init__(self, grid, resp, grad, mode, aeff, λ0, shock=True):
        self.grad, self.mode, self.λ0 = grad, mode, λ0
        ω = grid.ω
        shockterm = ω ** 2 if shock else ω * pd.wlfreq(grid.referenceλ)
        self.pre = -1j * shockterm / 4 / nlscale / pd.c
        _, self.βfun = make_linop(grid, mode, λ0)
        super().__init__(grid, resp, grad.density(0.0), None, aeff)

    def densityfun(self, z):
        return self.grad.density(z)

    def norm_factor(self, z):
        """pre/β(z) sqrt(Aeff) ωwin on sidx (NonlinearRHS.jl:375-387 and the ωwin loop)."""
        g = self.grid
        s = g.sidx
        f = np.ones(len(g.ω), dtype=np.complex128)
        β = self.βfun(z)
        f[s] = self.pre[s] / β[s] * math.sqrt(self.aeff) * g.ωwin[s]
        return f

    def output_factor(self):
        raise TypeError("the normalisation of a pressure gradient depends on z")
