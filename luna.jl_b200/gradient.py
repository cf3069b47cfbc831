"""Pressure-gradient fills and tapered capillaries, mirroring Luna.jl.

* ``Gradient`` — Capillary.gradient(gas, L, p0, p1) (Capillary.jl:306-315):
  p(z) = sqrt(p0^2 + z/L (p1^2 - p0^2)) inside [0, L], p0 before and p1 after, and the
  multi-point form gradient(gas, Z, P) (:317-337), the same law on each segment; the core
  index sqrt(1 + γ(λ) ρ(z)). The density is this package's closed form (ideal gas with a
  second virial coefficient, ``physdata.density``) where the reference interpolates a
  CoolProp spline.
* ``Taper`` — a core radius a(z) (MarcatiliMode(afun, ...), Capillary.jl:95-109, 236-242),
  given as piecewise-linear nodes: the reference takes any Julia function; a C ABI takes
  tables.
* ``MarcatiliGradientMode`` — MarcatiliMode(a, coren) with the z-dependent core index and,
  with a taper, radius: neff(ω; z) = sqrt(coren(ω; z)^2 - nwg(ω; a(z)))
  (Capillary.jl:153-224, neff_β_grid :345-360), Aeff(z) = a(z)^2 x the mode integral
  (Capillary.jl:295).
* ``make_linop`` — LinearOps.make_linop for a field-resolved grid (LinearOps.jl:330-360):
  L(ω; z) = -i(ω/c conj_clamp(neff(ω; z)) - ω β1(z)) on sidx (conj_clamp, :254), and
  βfun(z) for the normalisation (with the low-index rule of neff(m, ω; z) for a taper, whose
  make_linop goes through Modes.neff/Modes.β, LinearOps.jl:330-335).
* ``TransModeAvgZ`` — TransModeAvg with densityfun(z), aeff(z) and norm_mode_average's
  βfun!(β, z) (NonlinearRHS.jl:362-387).

Every z-dependent quantity is written out in IEEE-rounded real operations in the order the
device evaluates it: β1(z) is a finite difference with h = 1e-4 ω0 that turns an ulp of
neff into ~1e-12 of β1, so host and device must not differ in a single rounding.
"""
import math

import numpy as np

from . import modes, physdata as pd
from .nonlinearrhs import TransModeAvg, nlscale

MAXPTS = 16


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
        self.P2 = self.P * self.P
        self.L = float(self.Z[-1])
        self.p0, self.p1 = float(self.P[0]), float(self.P[-1])
        self.gam = pd.sellmeier_gas(gas)
        # density(p) = a p / (1 + b p), p in bar (physdata.density written out)
        self.dens_a = pd.bar / (pd.k_B * T)
        self.dens_b = pd._B2.get(gas, 0.0) * pd.bar / (pd._R_GAS * T)

    def p(self, z):
        Z, P, P2 = self.Z, self.P, self.P2
        if self.two_point:
            if z > Z[1]:
                return float(P[1])
            if z <= 0:
                return float(P[0])
            return math.sqrt(P2[0] + z / Z[1] * (P2[1] - P2[0]))
        if z <= Z[0]:
            return float(P[0])
        if z >= Z[-1]:
            return float(P[-1])
        i = int(np.searchsorted(Z, z, side="left")) - 1  # last i with Z[i] < z
        return math.sqrt(P2[i] + (z - Z[i]) / (Z[i + 1] - Z[i]) * (P2[i + 1] - P2[i]))

    def density(self, z):
        p = self.p(z)
        return self.dens_a * p / (1.0 + self.dens_b * p)

    def gamma(self, ω):
        """Sellmeier susceptibility per unit density at ω."""
        return np.asarray(self.gam(pd.wlfreq(np.asarray(ω, dtype=np.float64)) * 1e6), dtype=np.float64)

    def coren(self, ω, z):
        return np.sqrt(1 + self.gamma(ω) * self.density(z))


class Taper:
    """Core radius through nodes (Z, A): linear on each segment, A[0] for z <= Z[0] and A[-1]
    for z >= Z[-1]. One node is a constant radius."""

    def __init__(self, Z, A):
        self.Z = np.atleast_1d(np.asarray(Z, dtype=np.float64)).copy()
        self.A = np.atleast_1d(np.asarray(A, dtype=np.float64)).copy()
        if len(self.Z) != len(self.A) or not 1 <= len(self.Z) <= MAXPTS:
            raise ValueError(f"1 to {MAXPTS} radius nodes with one position each")
        if np.any(np.diff(self.Z) <= 0) or np.any(self.A <= 0):
            raise ValueError("taper nodes need increasing z and positive radii")

    @property
    def constant(self):
        return len(self.A) == 1

    def a(self, z):
        Z, A = self.Z, self.A
        if z <= Z[0]:
            return float(A[0])
        if z >= Z[-1]:
            return float(A[-1])
        i = int(np.searchsorted(Z, z, side="left")) - 1  # last i with Z[i] < z
        return float(A[i] + (z - Z[i]) / (Z[i + 1] - Z[i]) * (A[i + 1] - A[i]))


class MarcatiliGradientMode(modes.MarcatiliMode):
    """Full Marcatili model with a z-dependent fill (``Gradient``) and core radius
    (``Taper``; a number is a constant radius)."""

    def __init__(self, a, grad, n=1, m=1, kind="HE", model="full", loss=True):
        if model != "full":
            raise NotImplementedError("only the full Marcatili model")
        self.taper = a if isinstance(a, Taper) else Taper([0.0], [a])
        super().__init__(self.taper.a(0.0), None, 1.0, n=n, m=m, kind=kind, model=model, loss=loss)
        self.grad = grad

    @property
    def tapered(self):
        return not self.taper.constant

    def radius(self, z):
        return self.taper.a(z)

    def Aeff_z(self, z):
        """Modes.Aeff(m; z) = radius(m, z)^2 x the mode integral (Capillary.jl:295)."""
        r = self.radius(z)
        return r * r * self.aeff_intg

    def neff_parts(self, gam, kc, vn, rho, a):
        """(Re, Im) of sqrt(coren^2 - nwg) with coren = sqrt(1 + gam rho) and nwg at radius a
        (Capillary.jl:153-224), in the operation order the device uses."""
        nr, ni = modes.nwg_rn(kc, a, self.unm, vn)
        cr = np.sqrt(1 + gam * rho)
        re, im = modes.csqrt_rn(cr * cr - nr, -ni)
        if not self.loss:
            im = np.zeros_like(im)
        return re, im

    def neff_grid(self, ω, z):
        """sqrt(coren(ω; z)^2 - nwg(ω; a(z))) without the low-index rule."""
        ω = np.asarray(ω, dtype=np.float64)
        re, im = self.neff_parts(self.grad.gamma(ω), ω / pd.c, self.vn(ω), self.grad.density(z),
                                 self.radius(z))
        return re + 1j * im

    def neff_z(self, ω, z):
        """neff(m, ω; z) of the full model with its low-index rule (Capillary.jl:162-173)."""
        n = self.neff_grid(ω, z)
        re = np.where(np.real(n) < 1e-3, 1e-3, np.real(n))
        im = np.where(np.real(n) < 1e-3, np.clip(np.imag(n), 0, None), np.imag(n))
        return re + 1j * im

    def fd_tables(self, ω0):
        """The z-independent inputs of the group-delay finite difference at ω0 + 2h, ω0 + h,
        ω0 - h, ω0 - 2h (h = 1e-4 ω0): x/c, gam(x), vn(x), and 12h."""
        h = ω0 * 1e-4
        x = np.array([ω0 + 2 * h, ω0 + h, ω0 - h, ω0 - 2 * h])
        return x / pd.c, self.grad.gamma(x), self.vn(x), 12 * h

    def dispersion_z(self, ω0, z):
        """β1(z) = dβ/dω at ω0: the 4-point central difference of MarcatiliMode.dispersion,
        with β = x/c Re(neff) and the low-index rule."""
        xc, gam, vn, h12 = self.fd_tables(ω0)
        re, _ = self.neff_parts(gam, xc, vn, self.grad.density(z), self.radius(z))
        re = np.where(re < 1e-3, 1e-3, re)
        f = xc * re
        return float((-f[0] + 8 * f[1] - 8 * f[2] + f[3]) / h12)


def conj_clamp(n, ω):
    """LinearOps.conj_clamp (LinearOps.jl:254)."""
    return np.clip(np.real(n), 1e-3, None) - 1j * np.clip(np.imag(n), 0, 3000 * pd.c / ω)


def _om(grid):
    """The frequency factor of the group-delay term: ω, or ω - ω0 on an envelope grid."""
    return grid.ω - grid.ω0 if grid.kind == "env" else grid.ω


def make_linop(grid, mode, λ0, thg=False):
    """(linop(z), βfun(z)) (LinearOps.jl:330-388): on a field-resolved grid
    L = -i(ω/c conj_clamp(neff) - ω β1(z)), on an envelope grid
    L = -i(ω/c conj_clamp(neff) - (ω - ω0) β1(z)) + i β(ω0; z) (the last term without THG),
    on sidx, written out in real arithmetic (Re L = -ω/c Im nc,
    Im L = -(ω/c Re nc - ω' β1) [+ β(ω0; z)]), as the device evaluates it."""
    ω0 = pd.wlfreq(λ0)
    s = grid.sidx
    ω = grid.ω[s]
    om = _om(grid)[s]
    wc = ω / pd.c
    cap = 3000 * pd.c / ω
    gam = mode.grad.gamma(ω)
    vn = mode.vn(ω)
    env_ref = grid.kind == "env" and not thg

    def parts(z):
        return mode.neff_parts(gam, wc, vn, mode.grad.density(z), mode.radius(z))

    def βref(z):
        """Modes.β(mode, ω0; z) = ω0/c Re neff(ω0; z), the 1e-3 rule for a taper."""
        x = np.array([ω0])
        re, _ = mode.neff_parts(mode.grad.gamma(x), x / pd.c, mode.vn(x), mode.grad.density(z),
                                mode.radius(z))
        re = float(re[0])
        if mode.tapered and re < 1e-3:
            re = 1e-3
        return ω0 / pd.c * re

    def linop(z):
        out = np.zeros(len(grid.ω), dtype=np.complex128)
        β1 = mode.dispersion_z(ω0, z)
        re, im = parts(z)
        re = np.maximum(re, 1e-3)                   # conj_clamp (LinearOps.jl:254)
        im = np.minimum(np.maximum(im, 0.0), cap)
        out.real[s] = -(wc * im)
        out.imag[s] = -(wc * re - om * β1)
        if env_ref:                                 # out -= -im*βref (LinearOps.jl:380-382)
            out.imag[s] = out.imag[s] + βref(z)
        return out

    def βfun(z):
        out = np.ones(len(grid.ω))
        re, _ = parts(z)
        if mode.tapered:
            re = np.where(re < 1e-3, 1e-3, re)      # Modes.β through neff(m, ω; z)
        out[s] = wc * re
        return out

    return linop, βfun


class TransModeAvgZ(TransModeAvg):
    """TransModeAvg with a z-dependent density, effective area and normalisation
    (pressure gradient and/or taper)."""

    kind = "modeavg_z"

    def __init__(self, grid, resp, grad, mode, λ0, shock=True, thg=False):
        self.grad, self.mode, self.λ0, self.thg = grad, mode, λ0, thg
        ω = grid.ω
        shockterm = ω ** 2 if shock else ω * pd.wlfreq(grid.referenceλ)
        self.pre = -1j * shockterm / 4 / nlscale / pd.c
        _, self.βfun = make_linop(grid, mode, λ0, thg=thg)
        super().__init__(grid, resp, grad.density(0.0), None, mode.Aeff_z(0.0))

    def densityfun(self, z):
        return self.grad.density(z)

    def aefffun(self, z):
        return self.mode.Aeff_z(z)

    def norm_factor(self, z):
        """pre/β(z) sqrt(Aeff(z)) ωwin on sidx (NonlinearRHS.jl:375-387 and the ωwin loop)."""
        g = self.grid
        s = g.sidx
        f = np.ones(len(g.ω), dtype=np.complex128)
        β = self.βfun(z)
        f[s] = self.pre[s] / β[s] * math.sqrt(self.aefffun(z)) * g.ωwin[s]
        return f

    def output_factor(self):
        raise TypeError("the normalisation of a pressure gradient or taper depends on z")


def gradient_desc(t, crop, pad_No, keep):
    """luna_gradient_desc of a TransModeAvgZ for the C ABI (luna_b200_plan_set_gradient);
    ``crop`` is the plan's crop scale, ``pad_No`` its pad scale / No, ``keep`` collects the
    host arrays the descriptor points to."""
    from . import _lib
    grid, mode, grad = t.grid, t.mode, t.grad
    n, nta = len(grad.Z), len(mode.taper.Z)
    if n > _lib.GRAD_MAXPTS or nta > _lib.GRAD_MAXPTS:
        raise ValueError(f"at most {_lib.GRAD_MAXPTS} pressure or radius nodes")
    s = np.zeros(len(grid.ω), dtype=bool)
    s[grid.sidx] = True
    ω = grid.ω
    gam = np.zeros(len(ω))
    vn = np.zeros(len(ω), dtype=np.complex128)
    wc = np.zeros(len(ω))
    cap = np.zeros(len(ω))
    gam[s] = grad.gamma(ω[s])
    vn[s] = mode.vn(ω[s])
    wc[s] = ω[s] / pd.c
    cap[s] = 3000 * pd.c / ω[s]
    ofs = np.full(len(ω), crop, dtype=np.complex128)
    ofs[s] = crop * (t.pre[s] * grid.ωwin[s])
    om = np.ascontiguousarray(_om(grid), dtype=np.float64)
    arrs = [np.ascontiguousarray(a) for a in (gam, vn, wc, om, cap, ofs)]
    keep += arrs
    d = _lib.GradientDesc()
    d.npts, d.two_point, d.loss = n, int(grad.two_point), int(bool(mode.loss))
    for i in range(n):
        d.Z[i], d.P[i], d.P2[i] = grad.Z[i], grad.P[i], grad.P2[i]
    d.dens_a, d.dens_b = grad.dens_a, grad.dens_b
    d.nta = nta
    for i in range(nta):
        d.ZA[i], d.A[i] = mode.taper.Z[i], mode.taper.A[i]
    d.unm, d.aeff_intg = mode.unm, mode.aeff_intg
    d.in_base = pad_No / nlscale
    d.eps0c2 = pd.eps_0 * pd.c / 2
    d.gam, d.vn, d.wc, d.om, d.imcap, d.ofs = [_lib.dptr(a.view(np.float64)) for a in arrs]
    xc, fg, fv, h12 = mode.fd_tables(pd.wlfreq(t.λ0))
    for j in range(4):
        d.fd_xc[j], d.fd_gam[j] = xc[j], fg[j]
        d.fd_vn[2 * j], d.fd_vn[2 * j + 1] = fv[j].real, fv[j].imag
    d.fd_h12 = h12
    if grid.kind == "env":
        ω0 = pd.wlfreq(t.λ0)
        x = np.array([ω0])
        d.env_ref = int(not getattr(t, "thg", False))
        d.ref_xc = ω0 / pd.c
        d.ref_gam = float(grad.gamma(x)[0])
        v = complex(mode.vn(x)[0])
        d.ref_vn[0], d.ref_vn[1] = v.real, v.imag
    return d
