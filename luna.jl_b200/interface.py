"""User-facing entry points, mirroring Luna.jl ``src/Interface.jl``.

``prop_gnlse_args`` (Interface.jl:921-979) and ``prop_capillary_args``
(Interface.jl:360-401) build the grid, linear operator, responses, transform and
initial field exactly as the reference does, for the configurations this package
supports: mode-averaged propagation (constant fill, pressure gradients, tapers) and, with
``modes`` a number or a tuple of modes, multimode propagation with the modal transform
(constant fill). ``prop_gnlse`` and ``prop_capillary`` then integrate on the GPU
(``Luna.run``, Luna.jl:358-391).
"""
import math

import numpy as np

from . import fields, ionisation, modes, physdata as pd, raman
from .grid import EnvGrid, RealGrid
from .linops import make_const_linop
from .nonlinear import (Kerr_env, Kerr_env_thg, Kerr_field, Kerr_field_nothg, PlasmaCumtrapz, RamanPolarEnv,
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
                    τ1=12.2e-15, τ2=32e-15, saveN=201, rng=None, ϕ=()):
    """GNLSE set-up (Interface.jl:921-979); ``ϕ`` are the input pulse's spectral phases
    (CEP, group delay, GDD, ..., ``prop_taylor``). ``shotnoise=True`` adds one photon per mode
    (``fields.ShotNoise(rng)``, as ``shotnoise_maybe`` does, Interface.jl:773-776, 967);
    the default here is False, so that a set-up is reproducible unless noise is asked for."""
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
        # Interface.jl:945-961: the single damped oscillator, or fused silica's
        # intermediate-broadening model (ramanmodel "SiO2")
        χ3R = 2 * fr * n2 * (pd.eps_0 * pd.c)
        if ramanmodel == "SiO2":
            rr = _raman.raman_response(grid.to, "SiO2", χ3R * pd.eps_0)
        elif ramanmodel == "sdo":
            if τ1 is None or τ2 is None:
                raise ValueError("for :sdo ramanmodel you must specify τ1 and τ2")
            rr = _raman.CombinedRamanResponse(
                grid.to, [_raman.RamanRespNormedSingleDampedOscillator(χ3R * pd.eps_0, 1 / τ1, τ2)])
        else:
            raise ValueError("unrecognised value for ramanmodel")
        resp.append(RamanPolarEnv(grid.to, rr))
    fld = _pulse(pulseshape, λ0, τfwhm, τw, energy, power, ϕ)
    norm = norm_mode_average_gnlse(grid, shock=shock)
    transform = TransModeAvg(grid, resp, density, norm, aeff)
    Eω = fld(grid)
    if shotnoise:
        Eω = Eω + fields.ShotNoise(rng)(grid)
    return Problem(Eω, grid, linop, transform, saveN)


_raman = raman


def parse_mode(mode):
    """``parse_mode`` (Interface.jl:464-476): "HE11" -> {kind: "HE", n: 1, m: 1}."""
    if isinstance(mode, dict):
        return mode
    ms = str(mode).lstrip(":")
    if len(ms) > 4:
        raise ValueError(f"Ambiguous mode designation {mode}. Pass modes as dicts to disambiguate, "
                         "e.g. {'kind': 'HE', 'n': 1, 'm': 12}.")
    return {"kind": ms[:2], "n": int(ms[2]), "m": int(ms[3])}


def needpol_modes(modes_):
    """``needpol_modes`` (Interface.jl:439-446): two components unless only HE1m modes."""
    if isinstance(modes_, (str, int, dict)):
        return False
    return any(parse_mode(m)["kind"] != "HE" or parse_mode(m)["n"] > 1 for m in modes_)


def needpol(polarisation):
    """``needpol`` (Interface.jl:421-431): two field components unless linearly polarised."""
    if isinstance(polarisation, str):
        pol = polarisation.lstrip(":")
        if pol == "linear":
            return False
        if pol in ("circular", "x", "y"):
            return True
        raise ValueError(f"Polarisation must be :linear, :circular, :x/:y, or an ellipticity, not {polarisation}")
    return True


def ellfac(polarisation):
    """``ellfac`` (Interface.jl:744-749): the energy fractions (py, px) of the two components:
    one half each for circular polarisation, (1 - ε²/(1+ε²), ε²/(1+ε²)) for an ellipticity ε."""
    if isinstance(polarisation, str):
        return 0.5, 0.5
    ε = float(polarisation)
    if not -1 <= ε <= 1:
        raise ValueError("Ellipticity must be between -1 and 1.")
    return 1 - ε ** 2 / (1 + ε ** 2), ε ** 2 / (1 + ε ** 2)


def _addphase(ϕ, phase):
    """``addphase`` (Interface.jl:706-718): ``phase`` added to the constant spectral phase."""
    ϕ = [float(x) for x in np.atleast_1d(ϕ)] if ϕ is not None else []
    if phase == 0:
        return ϕ
    if not ϕ:
        return [phase]
    ϕ[0] += phase
    return ϕ


def findmode(ms, pulse):
    """``findmode`` (Interface.jl:638-656): the 1-based indices of the modes a pulse goes
    into: the lowest mode (both of its polarisations unless linear), or every mode of the
    named kind, n and m."""
    if pulse.mode == "lowest":
        return [1] if pulse.polarisation == "linear" else [1, 2]
    md = parse_mode(pulse.mode)
    return [i + 1 for i, m in enumerate(ms) if (m.kind, m.n, m.m) == (md["kind"], md["n"], md["m"])]


def makeinputs(ms, pulse):
    """``makeinputs`` for one pulse (Interface.jl:721-733, 751-761): linear or x polarisation
    into its first mode, y into the second, circular or elliptical split into (first mode,
    fraction py) and (second mode, fraction px, constant phase + π/2 sign(ε))."""
    idcs = findmode(ms, pulse)
    if not idcs:
        raise ValueError(f"Mode {pulse.mode} not found in mode list")
    pol = pulse.polarisation.lstrip(":") if isinstance(pulse.polarisation, str) else pulse.polarisation
    f = pulse.field
    if pol in ("linear", "x"):
        return ({"mode": idcs[0], "fields": (f,)},)
    if len(idcs) != 2:
        raise ValueError("Modes not set up for circular/elliptical polarisation")
    if pol == "y":
        return ({"mode": idcs[1], "fields": (f,)},)
    py, px = ellfac(pol)
    ε = 1.0 if isinstance(pol, str) else float(pol)
    nm = lambda x, k: None if x is None else x * k
    f1 = fields.PulseField(f.λ0, f.Itshape, nm(f.energy, py), nm(f.power, py), f.ϕ)
    f2 = fields.PulseField(f.λ0, f.Itshape, nm(f.energy, px), nm(f.power, px),
                           _addphase(f.ϕ, math.pi / 2 * float(np.sign(ε))))
    return ({"mode": idcs[0], "fields": (f1,)}, {"mode": idcs[1], "fields": (f2,)})


def makemode_s(modes_, radius, gas, pressure, T, model, loss, pol):
    """``makemode_s`` / ``makemodes_pol`` (Interface.jl:478-513) for a constant fill: a mode
    name gives one mode; a number n gives HE11..HE1n; a tuple gives each of its modes; with
    two components every HE1m mode comes twice (ϕ = 0 and π/2)."""
    def one(md):
        md = parse_mode(md)
        kw = dict(n=md["n"], m=md["m"], kind=md["kind"], T=T, model=model, loss=loss)
        if pol:
            if md["kind"] == "HE" and md["n"] == 1:
                return [modes.MarcatiliMode(radius, gas, pressure, ϕ=0.0, **kw),
                        modes.MarcatiliMode(radius, gas, pressure, ϕ=math.pi / 2, **kw)]
            return [modes.MarcatiliMode(radius, gas, pressure, ϕ=0.0, **kw)]
        return modes.MarcatiliMode(radius, gas, pressure, **kw)

    if isinstance(modes_, int):
        modes_ = tuple({"kind": "HE", "n": 1, "m": m} for m in range(1, modes_ + 1))
    if isinstance(modes_, (tuple, list)):
        out = []
        for md in modes_:
            r = one(md)
            out += r if isinstance(r, list) else [r]
        return out
    return one(modes_)


def needfull(ms):
    """``needfull`` (Interface.jl:801-803): the 2-D integral unless every mode is HE1m."""
    return not all(m.kind == "HE" and m.n == 1 for m in ms)


def _pulses(pulses, pulseshape, λ0, τfwhm, τw, energy, power, ϕ, polarisation):
    """The ``pulses`` list, or the one pulse the scalar arguments describe (Interface.jl:621-632)."""
    from .pulses import Pulse
    if pulses is not None:
        return list(pulses)
    return [Pulse(_pulse(pulseshape, λ0, τfwhm, τw, energy, power, ϕ), "lowest", polarisation)]


def _pulse(pulseshape, λ0, τfwhm, τw, energy, power, ϕ):
    """``makeinputs`` for a single pulse (Interface.jl:621-632): a Gaussian or sech² pulse
    with spectral phases ϕ."""
    if pulseshape == "gauss":
        return fields.GaussField(λ0, τfwhm, energy=energy, power=power, ϕ=ϕ)
    if pulseshape == "sech":
        return fields.SechField(λ0, τfwhm=τfwhm, τw=τw, energy=energy, power=power, ϕ=ϕ)
    raise ValueError("Valid pulse shapes are :gauss and :sech")


def _plasma(grid, gas, model, λ0, ppt_N, preionfrac):
    """``makeplasma!`` (Interface.jl:560-590): the ADK rate for molecular gases and the PPT
    rate otherwise (``model`` True), or the rate ``model`` names ("ADK" / "PPT")."""
    if model is True:
        model = "ADK" if gas in ("H2", "D2", "N2O", "CH4", "SF6") else "PPT"
    ionpot = pd.ionisation_potential(gas)
    if model == "ADK":
        rate = ionrate_fun_ADK(gas)
    elif model == "PPT":
        rate = ionisation.ionrate_PPTaccel(gas, λ0, N=ppt_N)
    else:
        raise ValueError(f"Unknown ionisation rate {model}.")
    return PlasmaCumtrapz(grid.to, grid.to, rate, ionpot, preionfrac=preionfrac)


def prop_capillary_args(radius, flength, gas, pressure, *, λlims, trange, λ0, τfwhm=None,
                        energy=None, power=None, pulseshape="gauss", shotnoise=False,
                        envelope=False, thg=None, δt=1.0, kerr=True, plasma=None,
                        raman=None, loss=True, model="full", saveN=201, ppt_N=2 ** 16,
                        modes="HE11", radial_integral_rtol=1e-3, temperature=pd.roomtemp,
                        rotation=True, vibration=True, rng=None, τw=None, ϕ=(), preionfrac=0.0,
                        polarisation="linear", pulses=None):
    """Capillary set-up (Interface.jl:360-401). ``pressure`` is a number, a (p0, p1) gradient
    over the fibre or (Z, P) nodes (Capillary.gradient, Capillary.jl:306-337); ``radius`` is
    a number or (Z, A) nodes of a piecewise-linear taper (a z-dependent radius,
    Interface.jl:249-250). ``modes`` (Interface.jl:478-513, 805-820): a mode name (e.g.
    "HE11", the default) gives mode-averaged propagation in that mode; a number n
    (HE11..HE1n) or a tuple of names gives multimode propagation with ``modal.TransModal``,
    linearly polarised input in the first mode, the radial integral when every mode is HE1m
    (the device runs it) and the full 2-D integral otherwise (described, evaluated by the
    oracle only); constant fill only. ``temperature`` sets the gas density, the core index
    and the Raman response's thermal populations; ``rotation``/``vibration`` select the Raman
    components (Interface.jl:360-374, 519-531, 534-560). ``plasma`` True selects ADK for
    molecular gases and PPT otherwise, "ADK" or "PPT" names the rate (makeplasma!,
    Interface.jl:560-590), ``preionfrac`` is the pre-ionised fraction; ``ϕ`` are the input
    pulse's spectral phases and ``τw`` the natural width of a sech² pulse (makeinputs,
    Interface.jl:621-632). ``polarisation`` ("linear", "x", "y", "circular" or an
    ellipticity -1 <= ε <= 1, Interface.jl:285-287) other than linear propagates two
    polarisation components: every HE1m mode twice (ϕ = 0 and π/2) in the multimode
    transform, as the reference's ``needpol`` does (Interface.jl:376, 421-431, 478-489).
    ``pulses`` (a list of ``pulses.GaussPulse`` / ``SechPulse``, each with its mode and
    polarisation) replaces the single pulse of the scalar arguments (Interface.jl:634-636,
    735-739). ``shotnoise=True`` adds one photon
    per mode to the input of every propagation mode (``fields.ShotNoise(rng)``, as
    ``shotnoise_maybe`` does, Interface.jl:389, 773-781); the default here is False, so that
    a set-up is reproducible unless noise is asked for."""
    modes_ = modes
    from . import modes
    plasma = (not envelope) if plasma is None else plasma
    thg = (not envelope) if thg is None else thg
    if envelope and plasma:  # makeresponse for EnvGrid (Interface.jl:593-594)
        raise ValueError("Plasma response for envelope fields has not been implemented yet.")
    # makegrid (Interface.jl:453-461)
    grid = EnvGrid(flength, λ0, λlims, trange, δt=δt, thg=thg) if envelope else \
        RealGrid(flength, λ0, λlims, trange, δt)
    pl = _pulses(pulses, pulseshape, λ0, τfwhm, τw, energy, power, ϕ, polarisation)
    if any(needpol(q.polarisation) for q in pl) and isinstance(modes_, str):
        modes_ = (modes_,)  # makemodes_pol: the mode in both polarisations
    if not isinstance(modes_, str) or parse_mode(modes_) != {"kind": "HE", "n": 1, "m": 1}:
        if isinstance(modes_, (int, tuple, list)):
            return _prop_capillary_modal(radius, flength, gas, pressure, grid, modes_, λ0, τfwhm,
                                         energy, power, pulseshape, thg, kerr, plasma, raman, loss,
                                         model, saveN, ppt_N, radial_integral_rtol, temperature,
                                         rotation, vibration, shotnoise, rng, preionfrac=preionfrac,
                                         ϕ=ϕ, τw=τw, polarisation=polarisation, pulses=pl)
    grad = None
    tapered = isinstance(radius, (tuple, list)) or type(radius).__name__ == "Taper"
    if isinstance(pressure, (tuple, list)) or tapered:
        # pressure gradient (p0, p1) or (Z, P) (Interface.jl:495-504, 524-531) and/or a
        # z-dependent radius (Interface.jl:249-250), given here as nodes (Z, A)
        if parse_mode(modes_) != {"kind": "HE", "n": 1, "m": 1}:
            raise NotImplementedError("pressure gradients and tapers are supported for HE11 only")
        from .gradient import Gradient, MarcatiliGradientMode, Taper
        if not isinstance(pressure, (tuple, list)):
            grad = Gradient(gas, flength, pressure, pressure, T=temperature)
        elif len(pressure) == 2 and all(np.ndim(x) == 0 for x in pressure):
            grad = Gradient(gas, flength, *pressure, T=temperature)      # (p0, p1)
        else:
            grad = Gradient(gas, *pressure, T=temperature)               # (Z, P)
        if isinstance(radius, (tuple, list)):
            radius = Taper(*radius)
        mode = MarcatiliGradientMode(radius, grad, model=model, loss=loss)
        density = grad.density(0.0)
    else:
        md = parse_mode(modes_)
        mode = modes.MarcatiliMode(radius, gas, pressure, n=md["n"], m=md["m"], kind=md["kind"],
                                   T=temperature, model=model, loss=loss)
        density = pd.density(gas, pressure, temperature)
    resp = []
    if kerr and envelope:
        # makeresponse for EnvGrid (Interface.jl:593-605)
        resp.append(Kerr_env_thg(pd.gamma3_gas(gas), pd.wlfreq(grid.referenceλ), grid.to) if thg else
                    Kerr_env(pd.gamma3_gas(gas)))
    elif kerr:
        # Interface.jl:534-541: without THG the Kerr term uses the analytic signal
        resp.append(Kerr_field(pd.gamma3_gas(gas)) if thg else
                    Kerr_field_nothg(pd.gamma3_gas(gas), len(grid.to)))
    if plasma:
        resp.append(_plasma(grid, gas, plasma, λ0, ppt_N, preionfrac))
    if raman is None:
        raman = gas in ("N2", "H2", "D2", "N2O", "CH4", "SF6")
    if raman:
        rr = _raman.raman_response(grid.to, gas, rotation=rotation, vibration=vibration, temp=temperature)
        resp.append(RamanPolarEnv(grid.to, rr) if envelope else RamanPolarField(grid.to, rr, thg=thg))
    if grad is not None:
        # z-dependent linear operator and normalisation (LinearOps.make_linop,
        # LinearOps.jl:337-388; norm_mode_average with βfun!(β, z))
        from .gradient import TransModeAvgZ, make_linop
        linop, _ = make_linop(grid, mode, λ0, thg=thg)
        transform = TransModeAvgZ(grid, resp, grad, mode, λ0, thg=thg)
    else:
        aeff = mode.Aeff()
        linop, βconst, β1 = make_const_linop(grid, mode, λ0, thg=thg)
        norm = norm_mode_average(grid, βconst)
        transform = TransModeAvg(grid, resp, density, norm, aeff)
    # doinput_sm (Luna.jl:94-113): every pulse goes into the one propagation mode
    md = parse_mode(modes_)
    for q in pl:
        if q.mode != "lowest" and parse_mode(q.mode) != md:
            raise ValueError("For mode-averaged propagation, all inputs must be in 1st mode.")
    Eω = pl[0].field(grid)
    for q in pl[1:]:
        Eω = Eω + q.field(grid)
    if shotnoise:
        Eω = Eω + fields.ShotNoise(rng)(grid)
    return Problem(Eω, grid, linop, transform, saveN)


def _prop_capillary_modal(radius, flength, gas, pressure, grid, modes_, λ0, τfwhm, energy, power,
                          pulseshape, thg, kerr, plasma, raman, loss, model, saveN, ppt_N, rtol,
                          temperature, rotation, vibration, shotnoise=False, rng=None, preionfrac=0.0,
                          ϕ=(), τw=None, polarisation="linear", pulses=None):
    """Multimode branch of ``prop_capillary_args``: ``setup(grid, modes, ...)`` with a constant
    linear operator (Interface.jl:805-812) and linearly polarised input in the first mode
    (``makeinputs``, Interface.jl:721-733); with ``shotnoise`` one photon per mode in every
    mode (``shotnoise_maybe``, Interface.jl:778-781)."""
    from . import modal
    if isinstance(pressure, (tuple, list)) or isinstance(radius, (tuple, list)):
        raise NotImplementedError("multimode propagation with a pressure gradient or a taper is not supported")
    pl = _pulses(pulses, pulseshape, λ0, τfwhm, τw, energy, power, ϕ, polarisation)
    pol = any(needpol(q.polarisation) for q in pl) or needpol_modes(modes_)
    ms = makemode_s(modes_, radius, gas, pressure, temperature, model, loss, pol)
    env = grid.kind == "env"
    thg = (not env) if thg is None else thg
    plasma = (not env) if plasma is None else plasma
    resp = []
    if kerr and env:  # makeresponse for EnvGrid (Interface.jl:592-605)
        resp.append(Kerr_env_thg(pd.gamma3_gas(gas), pd.wlfreq(grid.referenceλ), grid.to) if thg else
                    Kerr_env(pd.gamma3_gas(gas)))
    elif kerr:
        resp.append(Kerr_field(pd.gamma3_gas(gas)) if thg else
                    Kerr_field_nothg(pd.gamma3_gas(gas), len(grid.to)))
    if plasma:
        resp.append(_plasma(grid, gas, plasma, λ0, ppt_N, preionfrac))
    if raman is None:
        raman = gas in ("N2", "H2", "D2", "N2O", "CH4", "SF6")
    if raman:
        rr = _raman.raman_response(grid.to, gas, rotation=rotation, vibration=vibration, temp=temperature)
        resp.append(RamanPolarEnv(grid.to, rr) if env else RamanPolarField(grid.to, rr, thg=thg))
    inputs = tuple(x for q in pl for x in makeinputs(ms, q))
    Eω, t = modal.setup_modal(grid, pd.density(gas, pressure, temperature), resp, inputs, ms, "xy" if pol else "y",
                              full=needfull(ms), rtol=rtol)
    if shotnoise:
        noise = fields.ShotNoise(rng)
        Eω = np.array(Eω, dtype=np.complex128, copy=True)
        for m in range(Eω.shape[1]):
            Eω[:, m] += noise(grid)
    return Problem(Eω, grid, modal.make_const_linop_modes(grid, ms, λ0, thg=thg), t, saveN)


def prop_capillary(*args, precision=None, **kwargs):
    """``prop_capillary`` (Interface.jl:345-349): ``prop_capillary_args`` then ``Luna.run`` on
    the GPU (``plan.run``; a multimode set-up goes to the modal solver). Returns the solve
    result: the saved spectra ``Eω`` at ``z``, the final state and the step counts."""
    from . import _lib, plan
    p = prop_capillary_args(*args, **kwargs)
    return plan.run(p, precision=_lib.PREC_FP64 if precision is None else precision)


def prop_gnlse(*args, precision=None, **kwargs):
    """``prop_gnlse`` (Interface.jl:906-910): ``prop_gnlse_args`` then ``Luna.run`` on the GPU."""
    from . import _lib, plan
    p = prop_gnlse_args(*args, **kwargs)
    return plan.run(p, precision=_lib.PREC_FP64 if precision is None else precision)
