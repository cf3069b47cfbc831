"""Input pulses and energy functions (host setup of the initial state y0).

Restates Luna.jl ``src/Fields.jl``: ``PulseField`` with Gaussian / sech^2 shapes
(Fields.jl:40-145), the instantaneous power ``It`` (Fields.jl:503-504) and
``energyfuncs`` (Fields.jl:510-533). Simpson integration follows
NumericalIntegration.jl's ``SimpsonEven`` rule (composite 3/8-style end correction).
"""
import math

import numpy as np

from . import physdata as pd
from .maths import gauss


def simpson_even(x, y):
    """NumericalIntegration.jl ``integrate(x, y, SimpsonEven())`` for uniform x."""
    y = np.asarray(y)
    n = len(y)
    h = x[1] - x[0]
    retval = (17 * (y[0] + y[-1]) + 59 * (y[1] + y[-2]) + 43 * (y[2] + y[-3])
              + 49 * (y[3] + y[-4])) / 48
    retval = retval + np.sum(y[4:n - 4])
    return h * retval


def analytic(x):
    """Analytic signal (Maths.jl:560-569)."""
    xf = np.fft.fft(x)
    n = len(x)
    n1 = n // 2
    xf[1:n1] *= 2
    xf[n1:] = 0
    return np.fft.ifft(xf)


def It(Et, grid):
    if grid.kind == "real":
        return np.abs(analytic(Et)) ** 2
    return np.abs(Et) ** 2


def energy_t(grid, Et):
    return simpson_even(grid.t, It(Et, grid))


def to_freq_coarse(grid, Et):
    """Forward transform on the coarse grid: rfft (real) / fft (envelope), unnormalised."""
    return np.fft.rfft(Et) if grid.kind == "real" else np.fft.fft(Et)


def prop_taylor(Eω, ω, ϕs, λ0):
    """``prop_taylor`` (Fields.jl:618-636): Eω exp(-i sum_n ϕs[n] Δω^n / n!) with
    Δω = ω - ω(λ0) (ϕs = CEP, group delay, GDD, TOD, ...)."""
    Δω = np.asarray(ω) - pd.wlfreq(λ0)
    ϕ = np.zeros(len(Δω))
    for n, ϕi in enumerate(ϕs):
        ϕ = ϕ + Δω ** n / math.factorial(n) * ϕi
    return np.asarray(Eω) * np.exp(-1j * ϕ)


class PulseField:
    """``PulseField`` (Fields.jl:40-57, 112-145): the intensity shape on the grid's time axis
    (field-resolved or envelope), the spectral phases ``ϕ`` applied in the frequency domain
    (``prop_taylor``), then scaled to the energy or to the peak power after the phases."""

    def __init__(self, λ0, Itshape, energy=None, power=None, ϕ=()):
        if (energy is None) == (power is None):
            raise ValueError("exactly one of energy or power must be given")
        self.λ0, self.Itshape, self.energy, self.power = λ0, Itshape, energy, power
        self.ϕ = tuple(float(x) for x in np.atleast_1d(ϕ)) if ϕ is not None else ()

    def __call__(self, grid):
        t = grid.t
        ω0 = pd.wlfreq(self.λ0)
        if grid.kind == "real":
            Et = np.sqrt(self.Itshape(t)) * np.cos(ω0 * t)
        else:
            Δω = ω0 - grid.ω0
            Et = np.sqrt(self.Itshape(t)) * np.exp(1j * (Δω * t))
        if len(self.ϕ) >= 1:
            Eω = prop_taylor(to_freq_coarse(grid, Et), grid.ω, self.ϕ, self.λ0)
            Et = np.fft.irfft(Eω, len(t)) if grid.kind == "real" else np.fft.ifft(Eω)
        if self.energy is not None:
            Et = Et * (math.sqrt(self.energy) / math.sqrt(energy_t(grid, Et)))
        else:
            Et = Et * (math.sqrt(self.power) / math.sqrt(np.max(It(Et, grid))))
        return to_freq_coarse(grid, Et)


class ShotNoise:
    """One photon per mode quantum noise (``Fields.ShotNoise``, Fields.jl:284-321): on every
    frequency bin (envelope grids: the bins of the signal window, ``sidx``) the spectral
    amplitude sqrt(ħω/δω), scaled to the grid's transform (sqrt(2π)/(2δt) for the real one,
    sqrt(2π)/δt for the complex one), with a phase drawn uniformly from [0, 2π). ``rng`` is
    a numpy ``Generator`` (default: a fresh one); the reference draws from Julia's global
    RNG, so individual draws differ between the two while their distribution is the same."""

    def __init__(self, rng=None):
        self.rng = np.random.default_rng() if rng is None else rng

    def __call__(self, grid):
        ω = np.asarray(grid.ω)
        δω = ω[1] - ω[0]
        δt = grid.t[1] - grid.t[0]
        if grid.kind == "real":
            amp = np.sqrt(pd.hbar * ω / δω)
            famp = math.sqrt(2 * math.pi) / (2 * δt) * amp
        else:
            amp = np.zeros_like(ω)
            amp[grid.sidx] = np.sqrt(pd.hbar * ω[grid.sidx] / δω)
            famp = math.sqrt(2 * math.pi) / δt * amp
        φ = 2 * math.pi * self.rng.random(len(ω))
        return famp * np.exp(1j * φ)


def GaussField(λ0, τfwhm, energy=None, power=None, m=1, ϕ=()):
    return PulseField(λ0, lambda t: gauss(t, τfwhm, power=2 * m), energy, power, ϕ)


def SechField(λ0, τfwhm=None, τw=None, energy=None, power=None, ϕ=()):
    if τfwhm is not None and τw is not None:
        raise ValueError("only one of `τw` or `τfwhm` can be specified")
    if τw is None:
        if τfwhm is None:
            raise ValueError("one of `τw` or `τfwhm` must be specified")
        τw = τfwhm / (2 * math.log(1 + math.sqrt(2)))
    def shape(t):
        with np.errstate(over="ignore"):
            return 1 / np.cosh(t / τw) ** 2
    return PulseField(λ0, shape, energy, power, ϕ)
