"""User-facing entry points, mirroring Luna.jl ``src/Interface.jl``.

``prop_gnlse_args`` (Interface.jl:921-979) and ``prop_capillary_args``
(Interface.jl:360-401) build the grid, linear operator, responses, transform and
initial field exactly as the reference does, for the configurations this package
supports: single-mode mode-averaged propagation with a constant fill. ``prop_gnlse``
and ``prop_capillary`` then integrate on the GPU (``Luna.run``, Luna.jl:358-391).
"""
import math

import numpy as np

from . import fields, ionisation, modes, physdata as pd, raman
from .grid import EnvGrid, RealGrid
from .linops import make_const_linop
from .nonlinear import (Kerr_env, Kerr_field, Kerr_field_nothg, PlasmaCumtrapz, RamanPolarEnv,
                        RamanPolarField, ionrate_fun_ADK)
from .nonlinearrhs import TransModeAvg, norm_mode_average, norm_mode_average_gnlse


class Problem:
    """Everything ``Luna.run`` needs: Eω, grid, linop, transform (and save count)."""

    def __init__(self, Eω, grid, linop, transform, saveN=201):
        self.Eω, self.grid, self.linop, self.transform = Eω, grid, linop, transform
        self.saveN = saveN


def prop_gnlse_args(γ, flength, βs, *, λ0, λlims, trange, δt=1.0, τfwhm=None, τw=None,
                    power=None, energy=None, pulseshape="gauss", shotnoise=False,
                    shock=True, loss=0.0, raman=True, fr=0.18, ramanmodel="sdo",
                    τ1=12.2e-15, τ2=32e-15, saveN=201):
    """GNLSE set-up (Interface.jl:921-979)."""
    if shotnoise:
        raise NotImplementedError("shot noise uses a global RNG; pass shotnoise=False")
    grid = EnvGrid(flength, λ0, λlims, trange, δt=δt, thg=False)
    mode = modes.SimpleMode(pd.wlfreq(λ0), βs, loss=loss)
    aeff = 1.0
    density = 1.0
    linop, βconst, β1 = make_const_linop(grid, mode, λ0)
    k0 = 2 * math.pi / λ0
    n2 = γ / k0 * aeff
    χ3 = 4 / 3 * (1 - fr) * n2 * (pd.eps_0 * pd.c)
    resp = [Kerr_env(χ3)]
    if raman:
        if ramanmodel != "sdo":
            raise NotImplementedError("only ramanmodel='sdo' is supported")
        χ3R = 2 * fr * n2 * (pd.eps_0 * pd.c)
        rr = _raman.CombinedRamanResponse(
            grid.to, [_raman.RamanRespNormedSingleDampedOscillator(χ3R * pd.eps_0, 1 / τ1, τ2)])
        resp.append(RamanPolarEnv(grid.to, rr))
    if pulseshape == "gauss":
        fld = fields.GaussField(λ0, τfwhm, energy=energy, power=power)
    else:
        fld = fields.SechField(λ0, τfwhm=τfwhm, τw=τw, energy=energy, power=power)
    norm = norm_mode_average_gnlse(grid, shock=shock)
    transform = TransModeAvg(grid, resp, density, norm, aeff)
    Eω = fld(grid)
    return Problem(Eω, grid, linop, transform, saveN)


_raman = raman


def prop_capillary_args(radius, flength, gas, pressure, *, λlims, trange, λ0, τfwhm=None,
                        energy=None, power=None, pulseshape="gauss", shotnoise=False,
                        envelope=False, thg=None, δt=1.0, kerr=True, plasma=None,
                        raman=None, loss=True, model="full", saveN=201, ppt_N=2 ** 16):
    """Mode-averaged HE11 capillary set-up (Interface.jl:360-401). ``pressure`` is a number,
    a (p0, p1) gradient over the fibre or (Z, P) nodes (Capillary.gradient,
    Capillary.jl:306-337); ``radius`` is a number or (Z, A) nodes of a piecewise-linear taper
    (a z-dependent radius, Interface.jl:249-250)."""
    if shotnoise:
        raise NotImplementedError("shot noise uses a global RNG; pass shotnoise=False")
    if envelope:
        raise NotImplementedError("envelope capillary propagation is not supported")
    plasma = (not envelope) if plasma is None else plasma
    thg = (not envelope) if thg is None else thg
    grid = RealGrid(flength, λ0, λlims, trange, δt)
    grad = None
    tapered = isinstance(radius, (tuple, list)) or type(radius).__name__ == "Taper"
    if isinstance(pressure, (tuple, list)) or tapered:
        # pressure gradient (p0, p1) or (Z, P) (Interface.jl:495-504, 524-531) and/or a
        # z-dependent radius (Interface.jl:249-250), given here as nodes (Z, A)
        from .gradient import Gradient, MarcatiliGradientMode, Taper
        if not isinstance(pressure, (tuple, list)):
            grad = Gradient(gas, flength, pressure, pressure)
        elif len(pressure) == 2 and all(np.ndim(x) == 0 for x in pressure):
            grad = Gradient(gas, flength, *pressure)      # (p0, p1)
        else:
            grad = Gradient(gas, *pressure)               # (Z, P)
        if isinstance(radius, (tuple, list)):
            radius = Taper(*radius)
        mode = MarcatiliGradientMode(radius, grad, model=model, loss=loss)
        density = grad.density(0.0)
    else:
        mode = modes.MarcatiliMode(radius, gas, pressure, model=model, loss=loss)
        density = pd.density(gas, pressure)
    resp = []
    if kerr:
        # Interface.jl:534-541: without THG the Kerr term uses the analytic signal (the
        # oracle evaluates it; the device plan rejects it)
        resp.append(Kerr_field(pd.gamma3_gas(gas)) if thg else
                    Kerr_field_nothg(pd.gamma3_gas(gas), len(grid.to)))
    if plasma:
        ionpot = pd.ionisation_potential(gas)
        if gas in ("H2", "D2", "N2O", "CH4", "SF6"):
            rate = ionrate_fun_ADK(gas)
        else:
            rate = ionisation.ionrate_PPTaccel(gas, λ0, N=ppt_N)
        resp.append(PlasmaCumtrapz(grid.to, grid.to, rate, ionpot))
    if raman is None:
        raman = gas in ("N2", "H2", "D2", "N2O", "CH4", "SF6")
    if raman:
        rr = _raman.raman_response(grid.to, gas)
        resp.append(RamanPolarField(grid.to, rr, thg=thg))
    if grad is not None:
        # z-dependent linear operator and normalisation (LinearOps.make_linop,
        # LinearOps.jl:337-360; norm_mode_average with βfun!(β, z))
        from .gradient import TransModeAvgZ, make_linop
        if raman:
            raise NotImplementedError("Raman responses with a pressure gradient are not supported")
        linop, _ = make_linop(grid, mode, λ0)
        transform = TransModeAvgZ(grid, resp, grad, mode, λ0)
    else:
        aeff = mode.Aeff()
        linop, βconst, β1 = make_const_linop(grid, mode, λ0)
        norm = norm_mode_average(grid, βconst)
        transform = TransModeAvg(grid, resp, density, norm, aeff)
    if pulseshape == "gauss":
        fld = fields.GaussField(λ0, τfwhm, energy=energy, power=power)
    else:
        fld = fields.SechField(λ0, τfwhm=τfwhm, energy=energy, power=power)
    Eω = fld(grid)
    return Problem(Eω, grid, linop, transform, saveN)
