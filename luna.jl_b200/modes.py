"""Waveguide modes that feed the linear operator and normalisation (host setup).

* ``SimpleMode``: Taylor-expanded propagation constant for the GNLSE
  (SimpleFibre.jl:9-53).
* ``MarcatiliMode``: hollow-capillary HE/TE/TM modes with the complex effective index of
  Marcatili & Schmeltzer (Capillary.jl:29-186), effective area (Capillary.jl:284-300)
  and the group delay beta1 by a central finite difference (the reference uses
  FiniteDifferences.jl, Maths.jl:18-32); the transverse field, its normalisation and
  integration limits (Capillary.jl:267-287, Modes.jl:73) for the modal transform.
"""
import math

import numpy as np
from scipy import integrate, special

from . import physdata as pd


def csqrt_rn(a, b):
    """Principal square root of a + ib written out in IEEE-rounded real operations (no
    fused multiply-add): r = sqrt(a^2 + b^2); t = sqrt((r + |a|)/2); for a >= 0 the root is
    t + i b/(2t), else |b|/(2t) + i copysign(t, b). The device evaluates the same sequence,
    so effective indices, and the finite-difference group delay that amplifies an ulp of
    them about 10^4 times, agree bit for bit. Arguments are O(1) here: no scaling."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    r = np.sqrt(a * a + b * b)
    pos = a >= 0
    t = np.sqrt(np.where(pos, r + a, r - a) * 0.5)
    q = np.divide(b, 2 * t, out=np.zeros_like(t), where=t != 0)
    return np.where(pos, t, np.abs(q)), np.where(pos, q, np.copysign(t, b))


def nwg_rn(kc, a, unm, vn):
    """(Re, Im) of the Marcatili waveguide term (unm/(k a))^2 (1 - i vn/(k a))^2
    (Capillary.jl:188-200), in IEEE-rounded real operations: s = unm/(k a),
    p + iq = 1 - i vn/(k a) = (1 + Im vn/(k a)) - i Re vn/(k a), term = s^2 (p^2 - q^2, 2pq).
    The device evaluates the same sequence for a tapered core."""
    vn = np.asarray(vn)
    ka = kc * a
    s = unm / ka
    s2 = s * s
    p = 1 + np.imag(vn) / ka
    q = -(np.real(vn) / ka)
    return s2 * (p * p - q * q), s2 * (2 * (p * q))


class SimpleMode:
    def __init__(self, ωref, βs, Aeff=1.0, loss=0.0):
        self.ωref = ωref
        self.coef = [b / math.factorial(i) for i, b in enumerate(βs)]
        self._Aeff = Aeff
        self._α = math.log(10) / 10 * loss

    def β(self, ω):
        x = np.asarray(ω, dtype=np.float64) - self.ωref
        out = np.zeros_like(x)
        for cf in reversed(self.coef):  # Horner, as Polynomials.jl evaluates
            out = out * x + cf
        return out

    def α(self, ω):
        return np.full_like(np.asarray(ω, dtype=np.float64), self._α)

    def dispersion(self, order, ω):
        coef = list(self.coef)
        for _ in range(order):
            coef = [coef[i] * i for i in range(1, len(coef))]
        x = ω - self.ωref
        out = 0.0
        for cf in reversed(coef):
            out = out * x + cf
        return out

    def Aeff(self, z=0.0):
        return self._Aeff


def _unm(n, m, kind):
    if kind in ("TE", "TM"):
        return special.jn_zeros(1, m)[-1]
    return special.jn_zeros(n - 1, m)[-1]


class MarcatiliMode:
    """Hollow capillary mode filled with ``gas`` at pressure ``P`` (Capillary.jl:95-109)."""

    def __init__(self, a, gas, P, n=1, m=1, kind="HE", ϕ=0.0, T=pd.roomtemp, model="full", loss=True):
        self.a, self.n, self.m, self.kind, self.ϕ = a, n, m, kind, ϕ
        self.model, self.loss = model, loss
        self.unm = _unm(n, m, kind)
        self.coren = pd.ref_index_fun(gas, P, T) if gas is not None else (lambda lam: 1.0 + 0j)
        den, _ = integrate.quad(lambda r: r * special.jv(n - 1, self.unm * r) ** 4, 0, 1,
                                epsabs=0, epsrel=1e-12, limit=200)
        np1 = n if kind == "HE" else 2
        num = 0.25 * special.jv(np1, self.unm) ** 4
        self.aeff_intg = 2 * math.pi * num / den

    def _vn(self, εcl):
        εcl = np.asarray(εcl, dtype=complex)
        if self.kind == "HE":
            return (εcl + 1) / (2 * np.sqrt(εcl - 1))
        if self.kind == "TE":
            return 1 / np.sqrt(εcl - 1)
        return εcl / np.sqrt(εcl - 1)

    def vn(self, ω):
        """get_vn(εcl, kind) (Capillary.jl:88-93) with the silica cladding index at ω."""
        return np.ascontiguousarray(self._vn(pd.sio2_index(pd.wlfreq(np.asarray(ω, dtype=np.float64))) ** 2))

    def neff(self, ω):
        ω = np.asarray(ω, dtype=np.float64)
        lam = pd.wlfreq(ω)
        εco = np.real(self.coren(lam) ** 2)
        k = ω / pd.c
        nr, ni = nwg_rn(k, self.a, self.unm, self.vn(ω))
        re, im = csqrt_rn(εco - nr, -ni)
        nn = re + 1j * im
        if not self.loss:
            nn = np.real(nn) + 0j
        re = np.where(np.real(nn) < 1e-3, 1e-3, np.real(nn))
        im = np.where(np.real(nn) < 1e-3, np.clip(np.imag(nn), 0, None), np.imag(nn))
        return re + 1j * im

    def β(self, ω):
        return np.asarray(ω) / pd.c * np.real(self.neff(ω))

    def α(self, ω):
        return 2 * np.asarray(ω) / pd.c * np.imag(self.neff(ω))

    def dispersion(self, order, ω):
        if order != 1:
            raise NotImplementedError
        h = ω * 1e-4
        # 4th-order central difference for d(beta)/d(omega)
        f = lambda x: float(self.β(np.array([x]))[0])
        return (-f(ω + 2 * h) + 8 * f(ω + h) - 8 * f(ω - h) + f(ω - 2 * h)) / (12 * h)

    def Aeff(self, z=0.0):
        return self.a ** 2 * self.aeff_intg

    def dimlimits(self, z=0.0):
        """(:polar, (0, 0), (a, 2π)) (Capillary.jl:267)."""
        return ("polar", (0.0, 0.0), (self.a, 2 * math.pi))

    def field(self, r, θ=0.0):
        """Unnormalised (Ex, Ey) at polar (r, θ) (Capillary.jl:270-282)."""
        x = r * self.unm / self.a
        if self.kind == "HE":
            J = special.jv(self.n - 1, x)
            s, c = math.sin(self.n * (θ + self.ϕ)), math.cos(self.n * (θ + self.ϕ))
            return (J * (math.cos(θ) * s - math.sin(θ) * c), J * (math.sin(θ) * s + math.cos(θ) * c))
        J = special.jv(1, x)
        if self.kind == "TE":
            return (-J * math.sin(θ), J * math.cos(θ))
        return (J * math.cos(θ), J * math.sin(θ))

    def N(self, z=0.0):
        """Mode normalisation π/2 a² J_{n or 2}(unm)² sqrt(ε0/μ0) (Capillary.jl:284-287)."""
        np1 = self.n if self.kind == "HE" else 2
        return math.pi / 2 * self.a ** 2 * special.jv(np1, self.unm) ** 2 * math.sqrt(pd.eps_0 / pd.mu_0)

    def Exy(self, r, θ=0.0):
        """Normalised field field(m, xs)/sqrt(N(m)) (Modes.jl:73)."""
        s = 1.0 / math.sqrt(self.N())
        ex, ey = self.field(r, θ)
        return (ex * s, ey * s)
