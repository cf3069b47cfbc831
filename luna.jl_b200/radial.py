"""Radially symmetric free-space propagation (host setup), mirroring Luna.jl.

* ``make_const_linop_radial`` — LinearOps.make_const_linop(grid, q::QDHT, nfun)
  (LinearOps.jl:130-166, 185-197, 213-226): L(ω, k) = -i(sqrt(k(ω)^2 - k_r^2) - β1 ω),
  evanescent components damped by min(sqrt|.|, 200); on an envelope grid without THG the
  reference propagation constant β(ω0) is taken out (+iβ(ω0)).
* ``const_norm_radial`` — NonlinearRHS.const_norm_radial / norm_radial
  (NonlinearRHS.jl:482-524): sqrt(k^2 - k_r^2)/(μ0 ω), 1 where that is not real or ω = 0.
* ``TransRadial`` — the transform description (NonlinearRHS.jl:406-474) that the device
  plan is built from.
* ``GaussGaussField`` — Fields.SpatioTemporalField with a Gaussian profile in time and
  radius, energy normalisation by ``energyfuncs(grid, q)`` and free-space propagation by
  ``propz`` (Fields.jl:343-411, 536-560); ``focal_length`` adds a thin-lens phase. On an
  envelope grid the field is sqrt(I) exp(i(ϕ + Δω t)) and the time transform a complex FFT
  (make_Etr for EnvGrid, Fields.jl:374-378).
"""
import math

import numpy as np

from . import physdata as pd
from .fields import analytic, simpson_even
from .grid import EnvGrid, RealGrid
from .hankel import QDHT
from .maths import gauss
from .nonlinear import (Kerr_env, Kerr_env_thg, Kerr_field, Kerr_field_nothg, PlasmaCumtrapz,
                        RamanPolarEnv, RamanPolarField, ionrate_fun_ADK)
from . import ionisation, raman as _raman


def _n_on_sidx(grid, nfun):
    n = np.zeros(len(grid.ω))
    s = grid.sidx
    n[s] = np.real(nfun(2 * math.pi * pd.c / grid.ω[s]))
    return n


def _beta1(nfun, λ0):
    """d/dω [ω/c Re n(ω)] at the reference wavelength (central difference)."""
    w0 = pd.wlfreq(λ0)
    f = lambda w: w / pd.c * float(np.real(nfun(np.array([pd.wlfreq(w)]))[0]))
    h = w0 * 1e-4
    return (-f(w0 + 2 * h) + 8 * f(w0 + h) - 8 * f(w0 - h) + f(w0 - 2 * h)) / (12 * h)


def make_const_linop_radial(grid, q, nfun, thg=False):
    n = _n_on_sidx(grid, nfun)
    β1 = _beta1(nfun, grid.referenceλ)
    k2 = (n * grid.ω / pd.c) ** 2
    kr2 = q.k ** 2
    βsq = k2[:, None] - kr2[None, :]
    w = grid.ω[:, None]
    L = np.where(βsq < 0,
                 -1j * (-β1 * w) - np.minimum(np.sqrt(np.abs(βsq)), 200.0),
                 -1j * (np.sqrt(np.maximum(βsq, 0.0)) - β1 * w))
    if grid.kind == "env" and not thg:
        # out -= -im*βref, βref = ω0/c n(λ0) (LinearOps.jl:146-156, 213-226)
        βref = grid.ω0 / pd.c * float(np.real(nfun(np.array([2 * math.pi * pd.c / grid.ω0]))[0]))
        L = L - (-1j * βref)
    return np.ascontiguousarray(L.astype(np.complex128)), β1


def const_norm_radial(grid, q, nfun):
    n = _n_on_sidx(grid, nfun)
    k2 = np.zeros(len(grid.ω))
    s = grid.sidx
    k2[s] = (n[s] * grid.ω[s] / pd.c) ** 2
    βsq = k2[:, None] - (q.k ** 2)[None, :]
    w = grid.ω[:, None] * np.ones((1, q.N))
    out = np.ones((len(grid.ω), q.N))
    ok = (w != 0) & (βsq > 0)
    out[ok] = np.sqrt(βsq[ok]) / (pd.mu_0 * w[ok])
    return out


class TransRadial:
    """Radial transform E(ω, k) -> P_nl(ω, k) with constant density."""

    kind = "radial"

    def __init__(self, grid, q, resp, density, normfun):
        self.grid, self.q = grid, q
        self.resp = tuple(resp)
        self.density = float(density)
        self.normfun = np.asarray(normfun, dtype=np.float64)
        self._plan = None

    def output_factor(self):
        """ωwin (-iω) / (2 normfun) over (ω, k) (NonlinearRHS.jl:473)."""
        g = self.grid
        return (g.ωwin * (-1j * g.ω))[:, None] / (2 * self.normfun)

    def plan(self):
        if self._plan is None:
            from .radial_plan import RadialPlan
            self._plan = RadialPlan.from_transform(self)
        return self._plan

    def __call__(self, nl, Eω, z):
        self.plan().rhs(nl, Eω, z)


def energy_t_radial(grid, q, Etr):
    """energyfuncs(grid, q)[1] (Fields.jl:536-554): Etr is (Nt, Nr); the analytic signal
    of a real field, the envelope itself on an envelope grid."""
    Eta = np.apply_along_axis(analytic, 0, Etr) if grid.kind == "real" else Etr
    tint = np.array([simpson_even(grid.t, np.abs(Eta[:, i]) ** 2) for i in range(Etr.shape[1])])
    return 2 * math.pi * pd.c * pd.eps_0 / 2 * q.integrateR(tint)


def GaussGaussField(grid, q, λ0, τfwhm, energy, w0, propz=0.0, focal_length=None, ϕ=0.0):
    t = grid.t
    ω0 = pd.wlfreq(λ0)
    shape = gauss(t, τfwhm)[:, None] * np.exp(-0.5 * (q.r / (w0 / 2)) ** 2)[None, :]
    if grid.kind == "real":
        Etr = np.sqrt(shape) * np.cos(ω0 * t + ϕ)[:, None]
    else:
        Etr = np.sqrt(shape) * np.exp(1j * (ϕ + (ω0 - grid.ω0) * t))[:, None]
    Etr = Etr * math.sqrt(energy) / math.sqrt(energy_t_radial(grid, q, Etr))
    Eωr = np.fft.rfft(Etr, axis=0) if grid.kind == "real" else np.fft.fft(Etr, axis=0)
    if focal_length is not None:
        # thin lens: exp(-i ω r^2 / (2 c f)) applied in (ω, r)
        Eωr = Eωr * np.exp(-1j * grid.ω[:, None] * (q.r ** 2)[None, :] / (2 * pd.c * focal_length))
    Eωk = q.forward(Eωr, axis=1)
    if propz != 0.0:
        kzsq = (grid.ω / pd.c)[:, None] ** 2 - (q.k ** 2)[None, :]
        kz = np.sqrt(np.maximum(kzsq, 0.0))
        Eωk = Eωk * np.exp(-1j * propz * (kz - (grid.ω / pd.c)[:, None]))
    return np.ascontiguousarray(Eωk)


# ------------------------------------------------------------------ gas fill gradient
def _sidx_mask(grid):
    m = np.zeros(len(grid.ω), dtype=bool)
    m[grid.sidx] = True
    return m


class RadialFill:
    """The z-dependent parts of radial propagation through a gas fill gradient: nfun(ω; z) =
    sqrt(1 + γ(ω) ρ(z)) with ρ(z) of ``gradient.Gradient``; make_linop(grid, q, nfun)
    (LinearOps.jl:174-226), norm_radial (NonlinearRHS.jl:494-524) and β1(z) as the 4-point
    central difference of x/c n(x; z) at ω0 (h = 1e-4 ω0), written out in IEEE-rounded
    operations in the order the device evaluates them (k2 as (n x ω/c)^2)."""

    def __init__(self, grid, q, grad, λ0, thg=False):
        self.grid, self.q, self.grad, self.λ0 = grid, q, grad, λ0
        s = _sidx_mask(grid)
        self.s = s
        ω = np.asarray(grid.ω, dtype=np.float64)
        self.om = ω
        self.wc = np.where(s, ω / pd.c, 0.0)
        self.gam = np.zeros(len(ω))
        self.gam[s] = grad.gamma(ω[s])
        self.kr2 = np.asarray(q.k, dtype=np.float64) ** 2
        self.mw = pd.mu_0 * ω
        ω0 = pd.wlfreq(λ0)
        h = ω0 * 1e-4
        x = np.array([ω0 + 2 * h, ω0 + h, ω0 - h, ω0 - 2 * h])
        self.fd_xc, self.fd_gam, self.fd_h12 = x / pd.c, grad.gamma(x), 12 * h
        self.env_ref = grid.kind == "env" and not thg
        self.ref_xc = ω0 / pd.c
        self.ref_gam = float(grad.gamma(np.array([ω0]))[0])

    def scalars(self, z):
        rho = self.grad.density(z)
        f = self.fd_xc * np.sqrt(1.0 + self.fd_gam * rho)
        b1 = (-f[0] + 8 * f[1] - 8 * f[2] + f[3]) / self.fd_h12
        br = self.ref_xc * math.sqrt(1.0 + self.ref_gam * rho) if self.env_ref else 0.0
        return rho, b1, br

    def _bsq(self, rho):
        nk = np.sqrt(1.0 + self.gam * rho) * self.wc
        k2 = np.where(self.s, nk * nk, 0.0)
        return k2[:, None] - self.kr2[None, :]

    def linop(self, z):
        rho, b1, br = self.scalars(z)
        bsq = self._bsq(rho)
        bw = (b1 * self.om)[:, None] * np.ones((1, len(self.kr2)))
        neg = bsq < 0
        re = np.where(neg, -np.minimum(np.sqrt(np.where(neg, -bsq, 0.0)), 200.0), 0.0)
        im = np.where(neg, bw, -(np.sqrt(np.where(neg, 0.0, bsq)) - bw))
        if self.env_ref:
            im = im + br
        return np.ascontiguousarray(re + 1j * im)

    def normfun(self, z):
        bsq = self._bsq(self.grad.density(z))
        ok = (self.om[:, None] != 0) & (bsq > 0)
        mw = np.where(self.om != 0, self.mw, 1.0)[:, None]
        return np.where(ok, np.sqrt(np.where(ok, bsq, 1.0)) / mw, 1.0)


class TransRadialZ(TransRadial):
    """TransRadial with densityfun(z) and normfun(z) of a gas fill gradient."""

    kind = "radial_z"

    def __init__(self, grid, q, resp, fill):
        self.fill = fill
        super().__init__(grid, q, resp, fill.grad.density(0.0), fill.normfun(0.0))

    def densityfun(self, z):
        return self.fill.grad.density(z)

    def output_factor_z(self, z):
        g = self.grid
        return (g.ωwin * (-1j * g.ω))[:, None] / (2 * self.fill.normfun(z))


class RadialProblem:
    def __init__(self, Eω, grid, linop, transform, q, saveN=201):
        self.Eω, self.grid, self.linop, self.transform, self.q = Eω, grid, linop, transform, q
        self.saveN = saveN


def prop_radial_args(gas, pressure, *, R, N, flength, λ0, λlims, trange, τfwhm, energy, w0,
                     propz=0.0, focal_length=None, plasma="PPT", kerr=True, saveN=201,
                     ppt_N=2 ** 16, envelope=False, thg=None, raman=False):
    """Low-level radial set-up as in test/test_radial.jl and the freespace/radial and
    radial_env examples. ``envelope`` builds an EnvGrid (Kerr_env, or Kerr_env_thg with
    ``thg``; no plasma); ``thg=False`` on a field-resolved grid selects Kerr_field_nothg;
    ``raman`` adds the gas's molecular Raman response (RamanPolarField / RamanPolarEnv,
    applied per radial column). ``pressure`` as a (p0, p1) pair or (Z, P) nodes gives a gas
    fill gradient (Capillary.gradient's law, Capillary.jl:306-337): make_linop(grid, q,
    nfun) with nfun(ω; z) = sqrt(1 + γ(ω) ρ(z)), densityfun(z) and norm_radial at z."""
    if thg is None:
        thg = not envelope
    grid = EnvGrid(flength, λ0, λlims, trange, thg=thg) if envelope else RealGrid(flength, λ0, λlims, trange)
    q = QDHT(R, N)
    grad = None
    if isinstance(pressure, (tuple, list)):
        from .gradient import Gradient
        if len(pressure) == 2 and all(np.ndim(x) == 0 for x in pressure):
            grad = Gradient(gas, flength, *pressure)
        else:
            grad = Gradient(gas, *pressure)
        pressure = grad.p0
    nfun = pd.ref_index_fun(gas, pressure)
    dens0 = pd.density(gas, pressure)
    resp = []
    γ3 = pd.gamma3_gas(gas)
    if kerr:
        if envelope:
            resp.append(Kerr_env_thg(γ3, grid.ω0, grid.to) if thg else Kerr_env(γ3))
        else:
            resp.append(Kerr_field(γ3) if thg else Kerr_field_nothg(γ3, len(grid.to)))
    if plasma and not envelope:
        ionpot = pd.ionisation_potential(gas)
        rate = ionrate_fun_ADK(gas) if plasma == "ADK" else ionisation.ionrate_PPTaccel(gas, λ0, N=ppt_N)
        resp.append(PlasmaCumtrapz(grid.to, grid.to, rate, ionpot))
    if raman:
        rr = _raman.raman_response(grid.to, gas)
        resp.append(RamanPolarEnv(grid.to, rr) if envelope else RamanPolarField(grid.to, rr, thg=thg))
    if grad is not None:
        fill = RadialFill(grid, q, grad, λ0, thg=thg)
        linop = fill.linop
        transform = TransRadialZ(grid, q, resp, fill)
    else:
        linop, _ = make_const_linop_radial(grid, q, nfun, thg=thg)
        norm = const_norm_radial(grid, q, nfun)
        transform = TransRadial(grid, q, resp, dens0, norm)
    Eω = GaussGaussField(grid, q, λ0, τfwhm, energy, w0, propz=propz, focal_length=focal_length)
    return RadialProblem(Eω, grid, linop, transform, q, saveN)
