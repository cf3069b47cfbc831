"""Nonlinear response descriptors, mirroring Luna.jl ``src/Nonlinear.jl``.

Each constructor keeps the reference's name and argument meaning, and returns a plain
description of the response that the device evaluates inside the fused right-hand side:

* ``Kerr_field(γ3)``       -> ``out += rho*eps0*γ3*E^3``           (Nonlinear.jl:8-34)
* ``Kerr_env(γ3)``         -> ``out += 3/4*rho*eps0*γ3*|E|^2*E``   (Nonlinear.jl:47-73)
* ``Kerr_field_nothg(γ3, n)`` -> ``out += 3/4*rho*eps0*γ3*|hilbert(E)|^2*E`` (Nonlinear.jl:36-45)
* ``Kerr_env_thg(γ3, ω0, t)`` -> ``out += rho*eps0*γ3/4*(3|E|^2 + exp(2iω0t) E^2)*E``
  (Nonlinear.jl:75-84)
* ``PlasmaCumtrapz(t, E, ratefunc, ionpot; preionfrac)``           (Nonlinear.jl:88-177)
* ``RamanPolarField(t, r; thg)`` / ``RamanPolarEnv(t, r)``          (Nonlinear.jl:183-333)

Responses accumulate into the polarisation in the order they are given, as
``Et_to_Pt!`` does (NonlinearRHS.jl:121-126). The device evaluates all of them in the
mode-averaged transform; the no-THG forms take the Hilbert transform H of the field from one
more inverse transform (|hilbert(E)|^2 = E^2 + H^2) and run on the single-CTA solvers.
The radial and modal transforms take Kerr_field and PlasmaCumtrapz.
"""
from . import physdata as pd
from .ionisation import PPTSpline, adk_params


class Kerr_field:
    kind = "kerr_field"

    def __init__(self, γ3):
        self.γ3 = float(γ3)


class Kerr_env:
    kind = "kerr_env"

    def __init__(self, γ3):
        self.γ3 = float(γ3)


class Kerr_field_nothg:
    """Kerr response of a real field without third-harmonic generation: the intensity of
    the analytic signal (``Maths.plan_hilbert``) times the field."""

    kind = "kerr_field_nothg"

    def __init__(self, γ3, n):
        self.γ3 = float(γ3)
        self.n = int(n)


class Kerr_env_thg:
    """Kerr response of an envelope with its third harmonic (Genty et al., Opt. Express 15,
    5382 (2007), Eq. 4) on the time grid ``t`` at the reference frequency ω0."""

    kind = "kerr_env_thg"

    def __init__(self, γ3, ω0, t):
        import numpy as np
        self.γ3 = float(γ3)
        self.ω0 = float(ω0)
        self.C = np.exp(2j * self.ω0 * np.asarray(t, dtype=np.float64))


class ADKRate:
    """ADK rate closure constants (Ionisation.jl:22-63)."""

    kind = "adk"

    def __init__(self, ionpot, threshold=True):
        self.ionpot = ionpot
        p = adk_params(ionpot, threshold)
        self.nstar, self.cn_sq = p["nstar"], p["cn_sq"]
        self.w_p, self.w_t_prefac, self.thr = p["w_p"], p["w_t_prefac"], p["thr"]


def ionrate_fun_ADK(gas_or_ip, threshold=True):
    ip = gas_or_ip if isinstance(gas_or_ip, float) else pd.ionisation_potential(gas_or_ip)
    return ADKRate(ip, threshold)


class PlasmaCumtrapz:
    kind = "plasma"

    def __init__(self, t, E, ratefunc, ionpot, preionfrac=0.0):
        if not (0.0 <= preionfrac <= 1.0):
            raise ValueError("preionfrac must be between 0 and 1")
        if not isinstance(ratefunc, (PPTSpline, ADKRate)):
            raise TypeError("ratefunc must be a PPT spline table or ADK rate")
        self.ratefunc = ratefunc
        self.ionpot = float(ionpot)
        self.δt = float(t[1] - t[0])
        self.preionfrac = float(preionfrac)


class RamanPolarField:
    kind = "raman_field"

    def __init__(self, t, r, thg=True):
        self.r = r
        self.thg = thg
        self.dt = float(t[1] - t[0])
        self.n = len(t)


class RamanPolarEnv:
    kind = "raman_env"

    def __init__(self, t, r):
        self.r = r
        self.dt = float(t[1] - t[0])
        self.n = len(t)
