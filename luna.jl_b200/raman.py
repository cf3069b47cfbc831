"""Raman response models (host setup of the device response tables).

Restates Luna.jl ``src/Raman.jl``: the normalised single damped oscillator
(Raman.jl:53-65), the molecular vibrational model (Raman.jl:142-157), the non-rigid rotor
sum over J (Raman.jl:196-240) and ``CombinedRamanResponse`` (Raman.jl:242-262).

A response is reduced to what the device needs to rebuild h(t; rho) on the Raman
grid: for each component its undamped response ``hpre_i(t)`` sampled on
``tt = (0..N-1)*dt``, its density-dependent dephasing time ``tau2_i(rho)`` and the
Planck-taper window ``w`` (Raman.jl:249-262). The device forms
``h = w * sum_i hpre_i * exp(-tt/tau2_i)`` and transforms it. The intermediate-broadening
model of fused silica (Raman.jl:66-113) fits the same form as one component with
``tau2 = inf`` and ``w = 1``.
"""
import math

import numpy as np

from . import physdata as pd
from .maths import planck_taper


class SDO:
    """Single damped oscillator K*sin(Omega t), t>0, with dephasing tau2(rho)."""

    def __init__(self, K, Omega, tau2fun):
        self.K, self.Omega, self.tau2fun = K, Omega, tau2fun

    def hrpre(self, t):
        t = np.asarray(t, dtype=np.float64)
        return np.where(t > 0.0, self.K * np.sin(self.Omega * t), 0.0)

    def hrdamp(self, rho):
        return self.tau2fun(rho)

    def __call__(self, t, rho):
        return self.hrpre(t) * np.exp(-np.asarray(t) / self.hrdamp(rho))


def RamanRespNormedSingleDampedOscillator(K, Omega, tau2):
    """SDO normalised to unit integral then scaled by K (Raman.jl:53-59)."""
    K = K * (Omega ** 2 + 1 / tau2 ** 2) / Omega
    return SDO(K, Omega, Dephasing(0, tau2=tau2))


class Dephasing:
    """Dephasing time tau2(rho) of a Raman component, in the three forms of Raman.jl and with
    the (model, A, B, C) row the C ABI takes (luna_resp_desc.tau2_rho):

    * model 0, constant: ``rho -> tau2`` (Raman.jl:53-59, 145-149, 223-227);
    * model 1, rotational with Brho (Raman.jl:229-235): 1/(pi (A/(rho/amg) + B rho/amg))
      for rho > 0, inf at rho = 0;
    * model 2, vibrational with Brho (Raman.jl:150-155): 1/(pi (C + A/(rho/amg) + B rho/amg)).
    """

    def __init__(self, model, tau2=math.nan, A=0.0, B=0.0, C=0.0):
        self.model, self.tau2, self.A, self.B, self.C = model, tau2, A, B, C

    def row(self):
        return [float(self.model), self.A, self.B, self.C]

    def __call__(self, rho):
        if self.model == 0:
            return self.tau2
        if self.model == 1:
            return (1 / (math.pi * (self.A / (rho / pd.amg) + self.B * rho / pd.amg))
                    if rho > 0 else math.inf)
        return 1 / (math.pi * (self.C + self.A / (rho / pd.amg) + self.B * rho / pd.amg))


def RamanRespVibrational(Omega_v, dadQ, mu, tau2=None, Brho=None, Arho=None, C=0.0):
    """Molecular vibrational Raman oscillator (Raman.jl:142-157)."""
    K = (4 * math.pi * pd.eps_0) ** 2 * dadQ ** 2 / (4 * mu * Omega_v)
    if Brho is None:
        if tau2 is None:
            raise ValueError("one of tau2 or Brho must be specified")
        f = Dephasing(0, tau2=tau2)
    else:
        f = Dephasing(2, A=Arho, B=Brho, C=C)
    return SDO(K, Omega_v, f)


class RotationalNonRigid:
    """Sum of SDOs over rotational J -> J+2 transitions (Raman.jl:196-240)."""

    def __init__(self, B, dalpha, qJodd, qJeven, D=0.0, minJ=0, maxJ=50, temp=pd.roomtemp,
                 tau2=None, Brho=None, Arho=None):
        J = np.arange(minJ, maxJ + 1)
        EJ = 2 * math.pi * pd.hbar * pd.c * (B * J * (J + 1) - D * (J * (J + 1)) ** 2)
        dE = np.diff(EJ)
        neg = np.nonzero(dE < 0)[0]
        if len(neg):
            mJ = neg[0] + 1  # 1-based index of the last monotonic level
            J = J[:mJ]
            EJ = EJ[:mJ]
        DJ = np.where(J % 2 == 1, qJodd, qJeven)
        rhoJ = DJ * (2 * J + 1) * np.exp(-EJ / (pd.k_B * temp))
        rhoJ = rhoJ / np.sum(rhoJ)
        Js = J[:-2]
        Om = (EJ[2:] - EJ[:-2]) / pd.hbar
        K = -(4 * math.pi * pd.eps_0) ** 2 * 2 / 15 * dalpha ** 2 / pd.hbar
        if Brho is None:
            if tau2 is None:
                raise ValueError("one of tau2 or Brho must be specified")
            self.tau2fun = Dephasing(0, tau2=tau2)
        else:
            self.tau2fun = Dephasing(1, A=Arho, B=Brho)
        self.Rs = [SDO(K * (Js[i] + 1) * (Js[i] + 2) / (2 * Js[i] + 3)
                       * (rhoJ[i + 2] / (2 * Js[i] + 5) - rhoJ[i] / (2 * Js[i] + 1)),
                       Om[i], self.tau2fun) for i in range(len(Js))]

    def hrpre(self, t):
        return sum(R.hrpre(t) for R in self.Rs)

    def hrdamp(self, rho):
        return self.tau2fun(rho)

    def __call__(self, t, rho):
        return self.hrpre(t) * np.exp(-np.asarray(t) / self.hrdamp(rho))


class CombinedRamanResponse:
    """Raman response on the grid ``t`` as the sum of several damped components."""

    def __init__(self, t, Rs):
        t = np.asarray(t, dtype=np.float64)
        self.Rs = list(Rs)
        self.dt = t[1] - t[0]
        self.tt = np.arange(len(t), dtype=np.float64) * self.dt
        self.hpres = [R.hrpre(self.tt) for R in self.Rs]
        te = self.tt[-1]
        self.w = planck_taper(self.tt, -te, -te * 0.7, te * 0.7, te)

    def tau2s(self, rho):
        return [R.hrdamp(rho) for R in self.Rs]

    def tau2_rows(self):
        """[ncomp, 4] (model, A, B, C) rows of the components' dephasing laws, or None when
        none depends on the density (luna_resp_desc.tau2_rho)."""
        rows = [R.tau2fun.row() for R in self.Rs]
        return np.array(rows, dtype=np.float64) if any(r[0] != 0 for r in rows) else None

    def h(self, rho):
        """h(t; rho) on tt (Raman.jl:256-262): sum of damped components times window."""
        ht = np.zeros_like(self.tt)
        for hp, R in zip(self.hpres, self.Rs):
            ht += hp * np.exp(-self.tt / R.hrdamp(rho))
        return ht * self.w


def molecular_raman_response(t, rp, rotation=True, vibration=True, minJ=0, maxJ=50,
                             temp=pd.roomtemp):
    """Rotational + vibrational response for a molecular gas (Raman.jl:279-307)."""
    Rs = []
    if rotation and rp.get("rotation") == "nonrigid":
        if "Brho_r" in rp:
            Rs.append(RotationalNonRigid(rp["B"], rp["dalpha"], rp["qJodd"], rp["qJeven"],
                                         D=rp["D"], minJ=minJ, maxJ=maxJ, temp=temp,
                                         Brho=rp["Brho_r"], Arho=rp["Arho_r"]))
        else:
            Rs.append(RotationalNonRigid(rp["B"], rp["dalpha"], rp["qJodd"], rp["qJeven"],
                                         D=rp["D"], minJ=minJ, maxJ=maxJ, temp=temp,
                                         tau2=rp["tau2_r"]))
    if vibration and rp.get("vibration") == "sdo":
        if "Brho_v" in rp:
            Rs.append(RamanRespVibrational(rp["Omega_v"], rp["dadQ"], rp["mu"],
                                           Brho=rp["Brho_v"], Arho=rp["Arho_v"],
                                           C=rp.get("Cv", 0.0)))
        else:
            Rs.append(RamanRespVibrational(rp["Omega_v"], rp["dadQ"], rp["mu"], tau2=rp["tau2_v"]))
    return CombinedRamanResponse(t, Rs)


class RamanRespIntermediateBroadening:
    """Intermediate-broadening model (Raman.jl:66-113, after Hollenbeck and Cantrell, J. Opt.
    Soc. Am. B 19, 2886 (2002)): h(t) = s sum_i A_i exp(-γ_i t) exp(-Γ_i² t²/4) sin(ω_i t)
    on tt = (0..N-1) dt, with s = scale / (integral of the unscaled sum over (0, 1 ns)).
    The reference integrates with Cubature's hquadrature at its default tolerance (relative
    sqrt(eps)); here adaptive Gauss-Kronrod quadrature runs to 1e-12 relative, so the two
    scales agree to the reference's tolerance. No window and no density dependence: for the
    device it is one component with tau2 = inf and w = 1 (``hpres``, ``tau2s``, ``w``)."""

    def __init__(self, t, omega_i, A_i, Gamma_i, gamma_i, scale):
        self.omega_i, self.A_i = np.asarray(omega_i, float), np.asarray(A_i, float)
        self.Gamma_i, self.gamma_i = np.asarray(Gamma_i, float), np.asarray(gamma_i, float)
        n = len(self.omega_i)
        if not (len(self.A_i) == len(self.Gamma_i) == len(self.gamma_i) == n):
            raise ValueError("all component vectors must have same length")
        from scipy.integrate import quad
        self.scale = 1.0
        # the response lives in the first picoseconds: integrate there to 1e-12 relative,
        # then the (vanishing) rest of (0, 1 ns) to an absolute bound below that
        edges = [0.0, 2e-14, 1e-13, 3e-13, 1e-12, 3e-12]
        head = sum(quad(self, a, b, limit=500, epsabs=0.0, epsrel=1e-12)[0] for a, b in zip(edges[:-1], edges[1:]))
        tail = quad(self, edges[-1], 1e-9, limit=500, epsabs=1e-14 * abs(head), epsrel=0.0)[0]
        self.scale = scale / (head + tail)
        t = np.asarray(t, dtype=np.float64)
        self.Rs = []
        self.dt = t[1] - t[0]
        self.tt = np.arange(len(t), dtype=np.float64) * self.dt
        self.hpres = [np.asarray(self(self.tt), dtype=np.float64)]
        self.w = np.ones_like(self.tt)

    def __call__(self, t):
        t = np.asarray(t, dtype=np.float64)
        h = np.zeros_like(t)
        for w, A, G, g in zip(self.omega_i, self.A_i, self.Gamma_i, self.gamma_i):
            h = h + self.scale * A * np.exp(-g * t) * np.exp(-G ** 2 * t ** 2 / 4) * np.sin(w * t)
        return h if h.ndim else float(h)

    def tau2s(self, rho):
        return [math.inf]

    def tau2_rows(self):
        return None

    def h(self, rho):
        """h(t) on tt (the response does not depend on the density)."""
        return self.hpres[0].copy()


def raman_response(t, material, scale=1.0, **kw):
    """``Raman.raman_response`` (Raman.jl:316-328): the molecular model of a gas, or the
    intermediate-broadening model of fused silica ("SiO2") scaled by ``scale``."""
    rp = pd.raman_parameters(material)
    if rp["kind"] == "intermediate":
        return RamanRespIntermediateBroadening(t, rp["omega_i"], rp["A_i"], rp["Gamma_i"], rp["gamma_i"], scale)
    return molecular_raman_response(t, rp, **kw)
