"""Photoionisation rates (host setup of the device rate tables).

Restates Luna.jl ``src/Ionisation.jl``:

* ADK constants and threshold (Ionisation.jl:22-96). The per-sample closed form is
  evaluated on the device from the constants returned by :func:`adk_params`.
* The PPT rate (Ionisation.jl:317-429) with its series summed until the relative change
  falls below ``sum_tol`` (Maths.jl:721-736), the table of 2^16 fields between Emax/5000
  and 2*E_BSI (Ionisation.jl:185-212), and the log-rate cubic spline
  (Ionisation.jl:247-271). The device evaluates the spline per sample.

Special functions: Dawson's integral, Gamma and 1F1 come from scipy (the reference uses
SpecialFunctions.jl and HypergeometricFunctions.jl).
"""
import math

import numpy as np
from scipy import special

from . import physdata as pd
from .maths import cspline_slopes


# ---------------------------------------------------------------------------------- ADK
def _adk_rate(E, nstar, cn_sq, w_p, w_t_prefac, thr):
    aE = np.abs(np.asarray(E, dtype=np.float64))
    out = np.zeros_like(aE)
    m = aE >= thr
    if np.any(m):
        x = aE[m]
        out[m] = (w_p * cn_sq * (4 * w_p / (w_t_prefac * x)) ** (2 * nstar - 1)
                  * np.exp(-4 / 3 * w_p / (w_t_prefac * x)))
    return out


def adk_params(ionpot, threshold=True):
    """Constants of the ADK closure (Ionisation.jl:22-41) and its threshold field."""
    nstar = math.sqrt(0.5 / (ionpot / pd.au_energy))
    cn_sq = 2 ** (2 * nstar) / (nstar * math.gamma(nstar + 1) * math.gamma(nstar))
    w_p = ionpot / pd.hbar
    w_t_prefac = pd.electron / math.sqrt(2 * pd.m_e * ionpot)
    thr = 0.0
    if threshold:
        # ADK_threshold (Ionisation.jl:87-96): first field where the rate is non-zero
        E = 1e3
        while True:
            E *= 1.01
            if _adk_rate(np.array([E]), nstar, cn_sq, w_p, w_t_prefac, 0.0)[0] != 0:
                break
        thr = E
    return dict(nstar=nstar, cn_sq=cn_sq, w_p=w_p, w_t_prefac=w_t_prefac, thr=thr)


def ionrate_ADK(gas_or_ip, E, cycle_average=False):
    ip = gas_or_ip if isinstance(gas_or_ip, float) else pd.ionisation_potential(gas_or_ip)
    p = adk_params(ip)
    r = _adk_rate(E, p["nstar"], p["cn_sq"], p["w_p"], p["w_t_prefac"], p["thr"])
    if cycle_average:
        Ip_au = ip / pd.au_energy
        F0 = (2 * Ip_au) ** 1.5 * pd.au_Efield
        r = r * math.sqrt(3 / (math.pi * F0)) * np.sqrt(np.abs(E))
    return r


# ---------------------------------------------------------------------------------- PPT
def barrier_suppression(ionpot, Z):
    """Barrier-suppression field strength (Ionisation.jl:208-212)."""
    Ip_au = ionpot / pd.au_energy
    ns = Z / math.sqrt(2 * Ip_au)
    return Z ** 3 / (16 * ns ** 4) * pd.au_Efield


def _phi(m, x):
    """phi_m(x) of the PPT rate (Ionisation.jl:403-429), vectorised over x."""
    x = np.asarray(x, dtype=np.float64)
    if m == 0:
        return special.dawsn(x)
    mabs = abs(m)
    out = np.empty_like(x)
    small = x <= 26
    xs = x[small]
    out[small] = (np.exp(-xs ** 2) * math.sqrt(math.pi) * xs ** (2 * mabs + 1) * math.gamma(mabs + 1)
                  * special.hyp1f1(0.5, 1.5 + mabs, xs ** 2) / (2 * math.gamma(1.5 + mabs)))
    if np.any(~small):
        # exp(-x^2) * int_0^x (x^2-y^2)^|m| exp(y^2) dy, evaluated with the exponent
        # folded in so that it stays finite in double precision
        gx, gw = np.polynomial.legendre.leggauss(200)
        for j in np.nonzero(~small)[0]:
            xv = x[j]
            y = 0.5 * xv * (gx + 1)
            w = 0.5 * xv * gw
            out[j] = np.sum(w * (xv ** 2 - y ** 2) ** mabs * np.exp(y ** 2 - xv ** 2))
    return out


def ionrate_PPT(ionpot, λ0, Z, l, E, sum_tol=1e-6, cycle_average=False, Δα=0.0, α_ion=0.0,
                msum=True, occupancy=2):
    """PPT ionisation rate [1/s] for fields E (Ionisation.jl:317-390), vectorised over E.

    Every element's infinite sum is truncated by its own convergence test, exactly as
    the per-element ``converge_series`` call of the reference does.
    """
    E = np.atleast_1d(np.asarray(E, dtype=np.float64))
    Δα = 0.0 if Δα is None else Δα
    α_ion = 0.0 if α_ion is None else α_ion
    α_ion_au = α_ion / pd.au_polarisability
    Ip_au = (ionpot + Δα / 2 * E ** 2) / pd.au_energy
    ns = Z / np.sqrt(2 * Ip_au)
    ls = ns - 1
    Cnl2 = 2 ** (2 * ns) / (ns * special.gamma(ns + ls + 1) * special.gamma(ns - ls))
    w0 = 2 * math.pi * pd.c / λ0
    w0_au = pd.au_time * w0
    E0_au = (2 * Ip_au) ** 1.5
    E_au = np.abs(E) / pd.au_Efield
    g = w0_au * np.sqrt(2 * Ip_au) / E_au
    g2 = g * g
    beta = 2 * g / np.sqrt(1 + g2)
    alpha = 2 * (np.arcsinh(g) - g / np.sqrt(1 + g2))
    Up_au = E_au ** 2 / (4 * w0_au ** 2)
    v = (Ip_au + Up_au) / w0_au
    ret = np.zeros_like(E)
    mrange = range(-l, l + 1) if msum else (0,)
    for m in mrange:
        mabs = abs(m)
        flm = ((2 * l + 1) * math.factorial(l + mabs)
               / (2 ** mabs * math.factorial(mabs) * math.factorial(l - mabs)))
        lret = 4 * math.sqrt(2) / math.pi * Cnl2
        lret = lret * (2 * E0_au / (E_au * np.sqrt(1 + g2))) ** (2 * ns - mabs - 1.5)
        lret = lret * flm / math.factorial(mabs)
        lret = lret * np.exp(-2 * v * (np.arcsinh(g) - g * np.sqrt(1 + g2) / (1 + 2 * g2)))
        lret = lret * Ip_au * g2 / (1 + g2)
        if not cycle_average:
            lret = lret * np.sqrt(math.pi * E0_au / (3 * E_au))
        # converge_series(0, n0=ceil(v), rtol=sum_tol): x_{k+1} = x_k + term(n_k)
        n = np.ceil(v)
        s0 = np.zeros_like(E)
        done = np.zeros(E.shape, dtype=bool)
        s = np.zeros_like(E)
        while not np.all(done):
            act = ~done
            diff = n[act] - v[act]
            s1 = s0[act] + np.exp(-alpha[act] * diff) * _phi(m, np.sqrt(beta[act] * diff))
            with np.errstate(invalid="ignore", divide="ignore"):
                conv = 2 * np.abs(s1 - s0[act]) / np.abs(s1 + s0[act]) < sum_tol
            idx = np.nonzero(act)[0]
            s[idx] = s1
            s0[idx] = s1
            n[idx] += 1
            done[idx[conv]] = True
        lret = lret * s
        ret += occupancy * lret
    if α_ion_au != 0:
        ret = ret * np.exp(-2 * α_ion_au * E_au)
    return ret / pd.au_time


def ppt_gas_args(gas, stark_shift=True, dipole_corr=True):
    _, l, Z = pd.quantum_numbers(gas)
    Δα = pd.polarisability_difference(gas) if stark_shift else 0.0
    α_ion = pd.polarisability(gas, True) if dipole_corr else 0.0
    return pd.ionisation_potential(gas), Z, l, Δα, α_ion


def ionrate_PPT_gas(gas, λ0, E, stark_shift=True, dipole_corr=True, **kw):
    ip, Z, l, Δα, α_ion = ppt_gas_args(gas, stark_shift, dipole_corr)
    return ionrate_PPT(ip, λ0, Z, l, E, Δα=Δα, α_ion=α_ion, **kw)


class PPTSpline:
    """Log-rate cubic spline table on a uniform field axis (Ionisation.jl:247-271).

    ``x`` (fields), ``y`` (log rate) and ``D`` (Hermite slopes) are the device table.
    """

    kind = "ppt"

    def __init__(self, E, rate):
        keep = rate > 0
        self.x = np.ascontiguousarray(E[keep], dtype=np.float64)
        self.y = np.ascontiguousarray(np.log(rate[keep]), dtype=np.float64)
        self.D = cspline_slopes(self.y)
        dx = self.x[1] - self.x[0]
        if not np.allclose(np.diff(self.x), dx, rtol=1e-8, atol=0):
            raise ValueError("PPT table axis must be uniform")
        self.Emin = float(self.x[0])
        self.Emax = float(self.x[-1])


def makePPTcache(ionpot, λ0, Z, l, N=2 ** 16, Emax=None, **kw):
    """Tabulate the PPT rate on N fields from Emax/5000 to Emax (Ionisation.jl:185-200)."""
    Emax = 2 * barrier_suppression(ionpot, Z) if Emax is None else Emax
    Emin = Emax / 5000
    E = Emin + np.arange(N, dtype=np.float64) * ((Emax - Emin) / (N - 1))
    E[-1] = Emax
    return E, ionrate_PPT(ionpot, λ0, Z, l, E, **kw)


_PPT_CACHE = {}


def ionrate_PPTaccel(gas, λ0, N=2 ** 16, Emax=None, stark_shift=True, dipole_corr=True, **kw):
    """Build (and memoise per process) the PPT spline table for ``gas`` at ``λ0``."""
    key = (gas, float(λ0), N, Emax, stark_shift, dipole_corr, tuple(sorted(kw.items())))
    if key not in _PPT_CACHE:
        ip, Z, l, Δα, α_ion = ppt_gas_args(gas, stark_shift, dipole_corr)
        E, rate = makePPTcache(ip, λ0, Z, l, N=N, Emax=Emax, Δα=Δα, α_ion=α_ion, **kw)
        _PPT_CACHE[key] = PPTSpline(E, rate)
    return _PPT_CACHE[key]
