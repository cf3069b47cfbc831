"""Physical constants and gas data used to build the inputs of the UPPE hot path.

Restates the parts of Luna.jl ``src/PhysData.jl`` that the mode-averaged capillary,
GNLSE and radial transforms need on the host: CODATA2014 constants (PhysData.jl:14-48),
gas Sellmeier expansions (PhysData.jl:86-245), third-order susceptibility per molecule
``γ3_gas`` (PhysData.jl:588-657), ionisation potentials and PPT quantum numbers
(PhysData.jl:731-800), polarisabilities (PhysData.jl:815-846) and the molecular Raman
parameters (PhysData.jl:968-1100).

The reference computes gas number densities through CoolProp (PhysData.jl:695-698).
CoolProp is not available to this package; ``density`` uses the ideal-gas law with a
second-virial correction for the noble gases and H2. The hot path only ever sees the
resulting density as a number, so this affects physical fidelity, not kernel parity.
"""
import math

import numpy as np

# ---- CODATA2014 constants (PhysData.jl:14-48) --------------------------------------
c = 299792458.0
atm = 101325.0
bar = 100000.0
k_B = 1.38064852e-23
mu_0 = 4e-7 * math.pi
eps_0 = 1.0 / (mu_0 * c * c)
electron = 1.6021766208e-19
m_e = 9.10938356e-31
e_ratio = electron ** 2 / m_e
hbar = 6.626070040e-34 / (2 * math.pi)
_alpha_fs = 7.2973525664e-3
_a_0 = 0.52917721067e-10
au_energy = hbar * c * _alpha_fs / _a_0
au_time = hbar / au_energy
au_Efield = au_energy / (electron * _a_0)
roomtemp = 293.15
N_A = 6.022140857e23
amg = atm / (k_B * 273.15)
m_u = 1.660539040e-27
au_polarisability = electron ** 2 * _a_0 ** 2 / au_energy


def wlfreq(x):
    """Convert wavelength <-> angular frequency (PhysData.jl:77)."""
    return 2 * math.pi * c / x


# ---- densities -----------------------------------------------------------------------
# Second virial coefficients B(T) [m^3/mol] near room temperature (literature values);
# used as rho = P/(kT) / (1 + B*P/(R*T)) to first order.
_B2 = {"He": 11.8e-6, "Ne": 11.3e-6, "Ar": -16.0e-6, "H2": 14.1e-6, "N2": -4.5e-6,
       "Kr": -51.0e-6, "Xe": -130.0e-6}
_R_GAS = k_B * N_A


def density(gas, P=1.0, T=roomtemp):
    """Number density [1/m^3] of ``gas`` at pressure ``P`` [bar] and temperature ``T`` [K].

    Replaces the CoolProp call of PhysData.jl:695-698 by an ideal gas with a second
    virial correction.
    """
    if P == 0:
        return 0.0
    p = bar * P
    n_ideal = p / (k_B * T)
    B = _B2.get(gas, 0.0)
    return n_ideal / (1.0 + B * p / (_R_GAS * T))


def dens_1bar_0degC(gas):
    return density(gas, 1.0, 273.15)


def dens_1atm_0degC(gas):
    return density(gas, atm / bar, 273.15)


# ---- Sellmeier expansions (PhysData.jl:86-245) ----------------------------------------
def _borzsonyi(B1, C1, B2, C2):
    return lambda um: B1 * um ** 2 / (um ** 2 - C1) + B2 * um ** 2 / (um ** 2 - C2)


def _jct(B1, C1, B2, C2, B3, C3):
    return lambda um: (B1 * um ** 2 / (um ** 2 - C1) + B2 * um ** 2 / (um ** 2 - C2)
                       + B3 * um ** 2 / (um ** 2 - C3))


def _peck(B1, C1, B2, C2, dens):
    return lambda um: (((B1 / (C1 - 1 / um ** 2) + B2 / (C2 - 1 / um ** 2)) + 1) ** 2 - 1) / dens


def sellmeier_gas(gas):
    """Single-particle linear polarisability gamma(lambda[um]) (PhysData.jl:147-245)."""
    if gas in ("H2", "D2"):
        return _peck(14895.6e-6, 180.7, 4903.7e-6, 92.0, density(gas, atm / bar, 273.15))
    dens = dens_1bar_0degC(gas)
    if gas == "He":
        return _jct(2.16463842e-05 / dens, -6.80769781e-04, 2.10561127e-07 / dens,
                    5.13251289e-03, 4.75092720e-05 / dens, 3.18621354e-03)
    if gas == "Ne":
        return _borzsonyi(9154.48e-8 / dens, 656.97e-6, 4018.63e-8 / dens, 5.728e-3)
    if gas == "Ar":
        return _jct(0.00032323117217767093 / dens, 0.0045416501944977915,
                    0.00011557814904827939 / dens, 0.011120847461156543,
                    0.00010909808164540697 / dens, 0.0006827046691889898)
    if gas == "Kr":
        return _borzsonyi(26102.88e-8 / dens, 2.01e-6, 56946.82e-8 / dens, 10.043e-3)
    if gas == "Xe":
        return _borzsonyi(103701.61e-8 / dens, 12750e-6, 31228.61e-8 / dens, 0.561e-3)
    if gas == "N2":
        return _borzsonyi(39209.95e-8 / dens, 1146.24e-6, 18806.48e-8 / dens, 13.476e-3)
    raise ValueError(f"Unknown gas {gas}")


def ref_index_fun(gas, P=1.0, T=roomtemp):
    """Complex refractive index n(lambda [m]) of a gas fill (PhysData.jl:448-457)."""
    gam = sellmeier_gas(gas)
    dens = density(gas, P, T)
    return lambda lam: np.sqrt(1 + (gam(np.asarray(lam) * 1e6) * dens).astype(complex))


def sio2_index(lam):
    """Fused-silica refractive index from the three-term Malitson Sellmeier formula.

    The reference interpolates a tabulated SiO2 index (PhysData.jl:882-890); the
    cladding index only enters the capillary loss, so the analytic formula is used.
    """
    um2 = (np.asarray(lam) * 1e6) ** 2
    n2 = (1 + 0.6961663 * um2 / (um2 - 0.0684043 ** 2) + 0.4079426 * um2 / (um2 - 0.1162414 ** 2)
          + 0.8974794 * um2 / (um2 - 9.896161 ** 2))
    return np.sqrt(n2.astype(complex))


# ---- nonlinear and ionisation data ----------------------------------------------------
def gamma3_gas(gas):
    """Third-order susceptibility per particle (PhysData.jl:588-657, Lehmeier/Shelton)."""
    fac = {"He": 1.0, "Ne": 1.8, "Ar": 23.5, "Kr": 64.0, "Xe": 188.2, "N2": 21.1}
    if gas in fac:
        return 4 * fac[gas] * 3.43e-28 / dens_1atm_0degC(gas)
    if gas in ("H2", "D2"):
        return 15.77 * gamma3_gas("He")
    raise ValueError(f"no gamma3 for {gas}")


_IP_AU = {"He": 0.9036, "Ne": 0.7925, "Ar": 0.5792, "Kr": 0.5142, "Xe": 0.4458,
          "H": 0.5, "N2": 0.5726, "H2": 0.5669, "D2": 0.5684}


def ionisation_potential(gas, unit="SI"):
    """First ionisation potential (PhysData.jl:731-776)."""
    ip = _IP_AU[gas]
    if unit == "atomic":
        return ip
    if unit == "eV":
        return 27.21138602 * ip
    return 27.21138602 * electron * ip


def quantum_numbers(gas):
    """(n, l, Z) for the PPT rate (PhysData.jl:778-800)."""
    table = {"Ar": (3, 1, 1), "Ne": (2, 1, 1), "Kr": (4, 1, 1), "Xe": (5, 1, 1),
             "He": (1, 0, 1), "N2": (2, 0, 0.9)}
    return table[gas]


def polarisability(gas, ion=False):
    """Static dipole polarisability in SI units (PhysData.jl:815-835)."""
    table = {"He": (1.3207, 0.2811), "Ne": (2.376, 1.2417), "Ar": (10.762, 6.807)}
    if gas not in table:
        return None
    return table[gas][1 if ion else 0] * au_polarisability


def polarisability_difference(gas):
    a0 = polarisability(gas, False)
    if a0 is None:
        return None
    return a0 - polarisability(gas, True)


def raman_parameters(gas):
    """Raman parameters (PhysData.jl:968-1070) for the gases this package supports (and the
    intermediate-broadening model of fused silica used by ``prop_gnlse(ramanmodel="SiO2")``).
    Values are literature data and are kept identical to reproduce the physics."""
    if gas == "N2":
        return dict(kind="molecular", rotation="nonrigid", vibration="sdo", B=199.0, D=5.74e-4,
                    qJodd=1, qJeven=2, dalpha=6.7e-31, Brho_r=3.3e9, Arho_r=0.0,
                    dadQ=1.75e-20, Omega_v=2 * math.pi * 2330.0 * 100.0 * c,
                    mu=(m_u * 14.0067) ** 2 / (2 * m_u * 14.0067), tau2_v=6e-12)
    if gas == "H2":
        return dict(kind="molecular", rotation="nonrigid", vibration="sdo", B=5890.0, D=5.0,
                    qJodd=3, qJeven=1, dalpha=3e-31, Brho_r=114e6, Arho_r=6.15e6,
                    dadQ=1.3e-20, Omega_v=2 * math.pi * 124.5669e12,
                    mu=(m_u * 1.00784) ** 2 / (2 * m_u * 1.00784), Brho_v=52.2e6, Arho_v=309e6)
    if gas == "D2":
        return dict(kind="molecular", rotation="nonrigid", vibration="sdo", B=2930.0, D=2.1,
                    qJodd=1, qJeven=2, dalpha=3e-31, Brho_r=4e-3 * 100.0 * c, Arho_r=0.0,
                    dadQ=1.4e-20, Omega_v=2 * math.pi * 2987 * 100.0 * c,
                    mu=(m_u * 2.014) ** 2 / (2 * m_u * 2.014), Brho_v=120e6, Arho_v=101e6)
    if gas == "SiO2":
        # Hollenbeck and Cantrell, J. Opt. Soc. Am. B 19, 2886 (2002): line centres, amplitudes,
        # Gaussian and Lorentzian widths of the intermediate-broadening model
        return dict(kind="intermediate",
                    omega_i=[200 * math.pi * c * x for x in (56.25, 100.0, 231.25, 362.50, 463.00, 497.00, 611.50,
                                                            691.67, 793.67, 835.50, 930.0, 1080.00, 1215.00)],
                    A_i=[1.0, 11.40, 36.67, 67.67, 74.00, 4.50, 6.80, 4.60, 4.20, 4.50, 2.70, 3.10, 3.00],
                    Gamma_i=[100 * math.pi * c * x for x in (52.10, 110.42, 175.00, 162.50, 135.33, 24.50, 41.50,
                                                            155.0, 59.50, 64.30, 150.00, 91.00, 160.00)],
                    gamma_i=[100 * math.pi * c * x for x in (17.37, 38.81, 58.33, 54.17, 45.11, 8.17, 13.83,
                                                            51.67, 19.83, 21.43, 50.00, 30.33, 53.33)])
    raise ValueError(f"no Raman parameters for {gas}")
