"""Pin the CPU oracle (and the host set-up it consumes) to the reference's own known answers.

Each test cites the reference test it restates. These run without a GPU.
"""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import json
import math
import os

import numpy as np
import pytest

from luna_b200 import ionisation as I
from luna_b200 import maths, physdata as pd, raman
from luna_b200.grid import EnvGrid, RealGrid
from luna_b200.interface import prop_gnlse_args
from oracle import uppe

SQRT_EPS = math.sqrt(np.finfo(float).eps)

# the reference's own known answers, extracted from its test sources by golden/make_golden.py
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.json")) as _f:
    GOLDEN = json.load(_f)


def isapprox(a, b, rtol):
    a, b = np.asarray(a), np.asarray(b)
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


# ---------------------------------------------------------------- test_ionisation.jl:6-47
@pytest.mark.parametrize("gas,E,ref", [(g["gas"], g["E"], g["rate"]) for g in GOLDEN["adk"]])
def test_adk_known_answers(gas, E, ref):
    r = I.ionrate_ADK(gas, np.array([E]))[0]
    assert isapprox(r, ref, SQRT_EPS)


def test_adk_even_in_field():
    E = np.linspace(1e9, 1e11, 32)
    assert np.array_equal(I.ionrate_ADK("He", E), I.ionrate_ADK("He", -E))


@pytest.mark.parametrize("g", GOLDEN["ppt"], ids=lambda g: f"{g['gas']}-{g['E']:g}")
def test_ppt_known_answers(g):
    r = I.ionrate_PPT_gas(g["gas"], g["lambda0"], np.array([g["E"]]), dipole_corr=False)[0]
    assert isapprox(r, g["rate"], g["rtol"])


def test_cspline_uniform_index_matches_search():
    # test_ionisation.jl:18-34: an arithmetic index function and the brute-force
    # first-larger search give the same indices and the same spline values
    Emin, Emax, N = 1e9, 1e11, 2 ** 9
    E = np.linspace(Emin, Emax, N)
    rate = I.ionrate_PPT_gas("He", 800e-9, E)
    D = maths.cspline_slopes(rate)

    def ifun(x0):
        return 2 if x0 <= Emin else (N if x0 >= Emax else int(math.ceil((x0 - Emin) / (Emax - Emin) * N)) + 1)

    def ifun2(x0):
        return 2 if x0 <= E[0] else (len(E) if x0 >= E[-1] else int(np.argmax(E > x0)) + 1)

    def ev(i1, x0):
        i = i1 - 1
        if x0 == E[i]:
            return rate[i]
        if x0 == E[i - 1]:
            return rate[i - 1]
        t = (x0 - E[i - 1]) / (E[i] - E[i - 1])
        return (rate[i - 1] + D[i - 1] * t + (3 * (rate[i] - rate[i - 1]) - 2 * D[i - 1] - D[i]) * t ** 2
                + (2 * (rate[i - 1] - rate[i]) + D[i - 1] + D[i]) * t ** 3)

    for x0 in E:
        assert ifun(x0) == ifun2(x0)
        assert ev(ifun(x0), x0) == ev(ifun2(x0), x0)
        # the library's own index function (Maths.jl:772-774) evaluates to the same value
        assert maths.cspline_eval(E, rate, D, x0) == ev(ifun2(x0), x0)
    mid = 0.5 * (E[:-1] + E[1:])
    for x0 in mid:
        assert maths.cspline_eval(E, rate, D, x0) == ev(ifun2(x0), x0)


def test_ppt_spline_table_vs_direct():
    E = np.linspace(1e9, 1e11, 2 ** 9)
    direct = I.ionrate_PPT_gas("He", 800e-9, E)
    spl = I.ionrate_PPTaccel("He", 800e-9)
    acc = uppe.ppt_rate(spl, E)
    assert np.all(np.isclose(acc, direct, rtol=1e-2, atol=0))
    assert np.array_equal(acc, uppe.ppt_rate(spl, -E))


def test_ppt_above_table_raises():
    spl = I.ionrate_PPTaccel("He", 800e-9)
    with pytest.raises(ValueError):
        uppe.ppt_rate(spl, np.array([spl.Emax * 1.01]))


# ---------------------------------------------------------------- test_kerr.jl:5-30
def test_kerr_field_vs_envelope_low_frequencies():
    n = 2 ** 16
    t = (np.arange(n) - n / 2) * 3.430944979182369e-16 / 4
    E = np.exp(-0.5 * (t / 10e-15) ** 2) * np.cos(2 * np.pi * pd.c / 800e-9 * t)
    outf = np.zeros_like(E)
    uppe.kerr_field(outf, E, 1.0, 1.0 / pd.eps_0)
    xf = np.fft.fft(E)
    xf[1:n // 2] *= 2
    xf[n // 2:] = 0
    Eenv = np.fft.ifft(xf)
    oute = np.zeros_like(Eenv)
    uppe.kerr_env(oute, Eenv, 1.0, 1.0 / pd.eps_0)
    a = np.abs(np.fft.rfft(outf))[1799:2400]
    b = np.abs(np.fft.rfft(oute.real))[1799:2400]
    assert isapprox(b, a, 1e-15)
    # test_kerr.jl:13-16, 27: the no-THG form agrees with the full one there too
    outn = np.zeros_like(E)
    uppe.kerr_field_nothg(outn, E, 1.0, 1.0 / pd.eps_0)
    c = np.abs(np.fft.rfft(outn))[1799:2400]
    assert isapprox(c, a, 1e-15)


def test_kerr_env_thg_is_the_envelope_of_the_field_kerr_term():
    """Kerr_env_thg (Nonlinear.jl:75-84): for E = Re(A exp(iω0 t)), E³ has the envelope
    (3|A|²A + exp(2iω0t) A³)/4, so Re(P exp(iω0 t)) reproduces the field-resolved Kerr
    term exactly (Genty et al., Opt. Express 15, 5382 (2007), Eq. 4)."""
    from luna_b200.nonlinear import Kerr_env_thg
    n = 4096
    t = (np.arange(n) - n / 2) * 2e-16
    ω0 = 2 * np.pi * pd.c / 800e-9
    rng = np.random.default_rng(7)
    A = np.exp(-0.5 * (t / 12e-15) ** 2) * (1 + 0.3 * rng.standard_normal(n)) * np.exp(1j * 0.2 * rng.standard_normal(n))
    E = (A * np.exp(1j * ω0 * t)).real
    outf = np.zeros_like(E)
    uppe.kerr_field(outf, E, 1.0, 1.0 / pd.eps_0)
    r = Kerr_env_thg(1.0 / pd.eps_0, ω0, t)
    oute = np.zeros_like(A)
    uppe.kerr_env_thg(oute, A, 1.0, r)
    back = (oute * np.exp(1j * ω0 * t)).real
    assert np.max(np.abs(back - outf)) <= 1e-13 * np.max(np.abs(outf))


def test_raman_field_nothg_squares_the_analytic_signal():
    """sqr! without THG (Nonlinear.jl:267-274) uses 1/2 |hilbert(E)|²: E² minus its
    second-harmonic part 1/2 Re(hilbert(E)²)."""
    n = 2048
    t = (np.arange(n) - n / 2) * 2e-16
    E = np.exp(-0.5 * (t / 10e-15) ** 2) * np.cos(2 * np.pi * pd.c / 800e-9 * t)
    A = uppe.hilbert(E)
    np.testing.assert_allclose(A.real, E, atol=1e-15)
    np.testing.assert_allclose(0.5 * np.abs(A) ** 2, E ** 2 - 0.5 * (A ** 2).real, atol=1e-15)


def test_no_thg_responses_map_to_their_device_kinds():
    """prop_capillary(thg=false) (Interface.jl:534-555) builds Kerr_field_nothg and
    RamanPolarField(thg=false); the oracle evaluates them and the descriptors carry the
    no-THG kinds of the C ABI (the device evaluates them, tests/test_gpu_nothg.py)."""
    from luna_b200 import _lib
    from luna_b200.interface import prop_capillary_args
    from luna_b200.plan import resp_descs
    p = prop_capillary_args(125e-6, 0.1, "H2", 1.0, λ0=800e-9, τfwhm=10e-15, energy=50e-6,
                            λlims=(150e-9, 4e-6), trange=0.25e-12, thg=False, saveN=5)
    kinds = [(r.kind, getattr(r, "thg", None)) for r in p.transform.resp]
    assert ("kerr_field_nothg", None) in kinds and ("raman_field", False) in kinds
    nl = uppe.trans_mode_avg(p.transform, p.Eω, 0.0)
    assert np.all(np.isfinite(nl)) and np.linalg.norm(nl) > 0
    ds = resp_descs(p.transform.resp, 1.0, [])
    assert [d.kind for d in ds] == [_lib.RESP_KERR_FIELD_NOTHG, _lib.RESP_PLASMA_ADK, _lib.RESP_RAMAN_NOTHG]


# ---------------------------------------------------------------- test_raman.jl:9-70
def _raman_peak(grid, resp, rho, env):
    h = np.zeros(2 * len(grid.to))
    h[:len(grid.to)] = resp.h(rho)
    hw = np.fft.fft(h) if env else np.fft.rfft(h)
    n = len(grid.to)
    wR = 2 * np.pi * np.arange(n) / ((grid.to[1] - grid.to[0]) * n * 2)
    return wR[np.argmin(hw.imag[:n])]


def test_raman_response_causal_and_normalised():
    grid = RealGrid(1.0, 800e-9, (200e-9, 2000e-9), 40e-12)
    rho = pd.density("N2", 5.0)
    h = raman.raman_response(grid.to, "N2")
    T = np.linspace(-5e-12, 20e-12, 2 ** 16)
    for R in h.Rs:
        assert R(0.0, rho) == 0.0
        assert np.all(R(T[T <= 0], rho) == 0.0)
    hsdo = raman.RamanRespNormedSingleDampedOscillator(1.0, 2 * np.pi * 100e12, 100e-15)
    x = np.linspace(-1e-12, 2e-12, 2 ** 21 + 1)
    from scipy.integrate import simpson
    assert abs(simpson(hsdo(x, 1.0), x=x) - 1.0) < 1e-8


@pytest.mark.parametrize("env", [False, True])
def test_raman_n2_vibrational_peak(env):
    G = EnvGrid if env else RealGrid
    grid = G(1.0, 800e-9, (200e-9, 2000e-9), 40e-12)
    rho = pd.density("N2", 5.0)
    hv = raman.raman_response(grid.to, "N2", rotation=False)
    wpk = _raman_peak(grid, hv, rho, env)
    assert abs(wpk / pd.raman_parameters("N2")["Omega_v"] - 1) < 1e-4


def test_raman_h2_vibrational_and_rotational_peaks():
    grid = EnvGrid(1.0, 800e-9, (200e-9, 2000e-9), 40e-12)
    rho = pd.density("H2", 5.0)
    hv = raman.raman_response(grid.to, "H2", rotation=False)
    assert abs(_raman_peak(grid, hv, rho, True) / pd.raman_parameters("H2")["Omega_v"] - 1) < 1e-4
    hr = raman.raman_response(grid.to, "H2", vibration=False)
    assert abs(_raman_peak(grid, hr, rho, True) / (2 * np.pi * 17.45e12) - 1) < 1e-4


def test_raman_d2_vibrational_and_rotational_peaks():
    """D2 (PhysData.jl:1011-1026): the vibrational line at Ωv, and the rotational spectrum
    peaking on one of the S(J) lines of the non-rigid rotor (B and D in 1/m, Raman.jl:199-200)."""
    grid = EnvGrid(1.0, 800e-9, (200e-9, 2000e-9), 40e-12)
    rho = pd.density("D2", 5.0)
    hv = raman.raman_response(grid.to, "D2", rotation=False)
    assert abs(_raman_peak(grid, hv, rho, True) / pd.raman_parameters("D2")["Omega_v"] - 1) < 1e-4
    hr = raman.raman_response(grid.to, "D2", vibration=False)
    wr = _raman_peak(grid, hr, rho, True)
    B, D = 2930.0, 2.1
    E = lambda J: B * J * (J + 1) - D * (J * (J + 1)) ** 2
    lines = [2 * np.pi * pd.c * (E(J + 2) - E(J)) for J in range(6)]
    assert min(abs(wr / w - 1) for w in lines) < 1e-3


def test_raman_sio2_intermediate_broadening_response():
    """Raman.jl:66-113 with the fused-silica lines (PhysData.jl:1060-1068): the samples follow
    the formula, the response integrates to its scale over (0, 1 ns), and the device
    descriptor carries it as one component with tau2 = inf and no window."""
    from luna_b200.plan import resp_descs
    from luna_b200.nonlinear import RamanPolarEnv
    grid = EnvGrid(1.0, 835e-9, (500e-9, 2400e-9), 12.5e-12)
    r = raman.raman_response(grid.to, "SiO2", 2.5)
    rp = pd.raman_parameters("SiO2")
    tt = r.tt
    h = sum(r.scale * A * np.exp(-g * tt) * np.exp(-G ** 2 * tt ** 2 / 4) * np.sin(w * tt)
            for w, A, G, g in zip(rp["omega_i"], rp["A_i"], rp["Gamma_i"], rp["gamma_i"]))
    assert np.allclose(r.h(1.0), h, rtol=1e-13, atol=0)
    x = np.linspace(0.0, 3e-12, 3_000_001)
    assert abs(np.trapezoid(r(x), x) / 2.5 - 1) < 1e-6
    ds = resp_descs([RamanPolarEnv(grid.to, r)], 1.0, [])
    assert ds[0].ncomp == 1 and ds[0].tau2[0] == np.inf
    assert np.all(np.ctypeslib.as_array(ds[0].hwin, shape=(len(tt),)) == 1.0)


# ---------------------------------------------------------------- Maths.cumtrapz!
def test_cumtrapz_is_the_sequential_recurrence():
    rng = np.random.default_rng(0)
    y = rng.standard_normal(1000)
    out = np.zeros_like(y)
    for i in range(1, len(y)):
        out[i] = out[i - 1] + 0.5 * (y[i - 1] + y[i]) * 0.3
    assert np.array_equal(uppe.cumtrapz(y, 0.3), out)


# ---------------------------------------------------------------- test_rk45.jl:5-135
def _nlse_init():
    trange, wrange = 32, 160
    samples = 2 ** int(math.ceil(math.log2(trange * wrange / (2 * np.pi))))
    dt = trange / samples
    dw = 2 * np.pi / trange
    n = np.arange(samples)
    t = (n - samples / 2) * dt
    w = (n - samples / 2) * dw
    At = 5 / np.cosh(t)
    Aw = np.fft.fftshift(np.fft.fft(At))
    Lin = -1j / 2 * w ** 2

    def fnl(Aw, z):
        a = np.fft.ifft(Aw)
        return 1j * np.fft.fft(np.abs(a) ** 2 * a)

    return Aw, Lin, fnl


def test_rk45_precon_nlse_soliton_recovers():
    Aw, Lin, fnl = _nlse_init()
    zmax = np.pi / 2 * 2
    s = uppe.PreconStepper(fnl, Lin, Aw, 0.0, 1e-3, rtol=1e-8)
    while s.tn <= zmax:
        s.step()
    # the reference compares the dense output at zmax
    out = s.interpolate(zmax)
    assert isapprox(np.abs(Aw) ** 2, np.abs(out) ** 2, 1e-3)


# ---------------------------------------------------------------- test_gnlse.jl:33-56
@pytest.mark.slow
def test_soliton_shift_golden_values():
    """Soliton self-frequency shift: peak frequency and time checked against two
    independent GNLSE codes by the reference (rtol 1e-14)."""
    γ, β2, fr, τ0 = 0.1, -1e-26, 0.18, 10e-15
    P0 = abs(β2) / ((1 - fr) * γ * τ0 ** 2)
    flength = np.pi / 2 * τ0 ** 2 / abs(β2) * 90
    p = prop_gnlse_args(γ, flength, [0.0, 0.0, β2], λ0=835e-9, τfwhm=1.763 * τ0, power=P0,
                        pulseshape="sech", λlims=[450e-9, 8000e-9], trange=13e-12, raman=True,
                        shock=False, fr=fr)
    res = uppe.run(p.transform, p.grid, p.linop, p.Eω)
    Ew = res.Eω[-1]
    wpk = p.grid.ω[np.argmax(np.abs(Ew) ** 2)]
    ss = GOLDEN["soliton_shift"]
    assert abs(wpk / ss["omega_peak"] - 1) <= ss["rtol"]
    Et = np.fft.ifft(Ew) * np.exp(1j * p.grid.ω0 * p.grid.t)
    tpk = p.grid.t[np.argmax(np.abs(Et) ** 2)]
    assert abs(tpk / ss["t_peak"] - 1) <= ss["rtol"]


# ---------------------------------------------------------------- test_radial.jl:3-65
def test_radial_focus_matches_paraxial_gaussian_beam():
    """Radially symmetric propagation through a focus (TransRadial + QDHT + Kerr + PPT
    plasma at negligible energy): the fluence profile at ω0 after 0.6 m matches the
    paraxial Gaussian-beam width to 1.5e-4 (test_radial.jl:64)."""
    from luna_b200.radial import prop_radial_args
    w0, L = 40e-6, 0.6
    p = prop_radial_args("Ar", 1.2, R=4e-3, N=128, flength=L, λ0=800e-9,
                         λlims=(400e-9, 2000e-9), trange=0.2e-12, τfwhm=20e-15,
                         energy=1e-12, w0=w0, propz=-0.3)
    res = uppe.run(p.transform, p.grid, p.linop, p.Eω)
    g, q = p.grid, p.q
    Er = q.inverse(res.Eω[-1], axis=1)
    i0 = np.argmin(np.abs(g.ω - 2 * np.pi * pd.c / 800e-9))
    lam0 = 2 * np.pi * pd.c / g.ω[i0]
    w1 = w0 * np.sqrt(1 + (L / 2 * lam0 / (np.pi * w0 ** 2)) ** 2)
    Ia = np.exp(-0.5 * (q.r / (w1 / 2)) ** 2) * (w0 / w1) ** 2
    Ir = np.abs(Er[i0]) ** 2
    Ir, Ia = Ir / Ir.max(), Ia / Ia.max()
    assert np.max(np.abs(Ir - Ia)) / np.linalg.norm(Ir) < GOLDEN["radial_focus_bound"]


def test_radial_env_focus_matches_paraxial_gaussian_beam():
    """freespace/radial_env.jl's check on the envelope form of the oracle: a 2 nJ envelope
    (EnvGrid, Kerr_env, linop with β(ω0) taken out) through a focus at 0.3 m over 0.6 m;
    the fluence profile at ω0 matches the paraxial width to the same bound."""
    from luna_b200.radial import prop_radial_args
    w0, L = 40e-6, 0.6
    p = prop_radial_args("Ar", 1.2, R=4e-3, N=128, flength=L, λ0=800e-9,
                         λlims=(400e-9, 2000e-9), trange=0.2e-12, τfwhm=20e-15,
                         energy=2e-9, w0=w0, propz=-0.3, envelope=True)
    assert p.grid.kind == "env" and [r.kind for r in p.transform.resp] == ["kerr_env"]
    res = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=3)
    g, q = p.grid, p.q
    Er = q.inverse(res.Eω[-1], axis=1)
    i0 = np.argmin(np.abs(g.ω - 2 * np.pi * pd.c / 800e-9))
    lam0 = 2 * np.pi * pd.c / g.ω[i0]
    w1 = w0 * np.sqrt(1 + (L / 2 * lam0 / (np.pi * w0 ** 2)) ** 2)
    Ia = np.exp(-0.5 * (q.r / (w1 / 2)) ** 2) * (w0 / w1) ** 2
    Ir = np.abs(Er[i0]) ** 2
    Ir, Ia = Ir / Ir.max(), Ia / Ia.max()
    assert np.max(np.abs(Ir - Ia)) / np.linalg.norm(Ir) < GOLDEN["radial_focus_bound"]
    # the input carries the requested energy (energyfuncs(grid::EnvGrid, q), Fields.jl:550-560)
    from luna_b200.radial import energy_t_radial
    Et = np.fft.ifft(q.inverse(p.Eω, axis=1), axis=0)
    assert abs(energy_t_radial(g, q, Et) / 2e-9 - 1) < 1e-12


@pytest.mark.parametrize("envelope,thg", [(False, None), (True, False), (True, True)])
def test_radial_fill_gradient_at_equal_pressures_is_the_constant_fill(envelope, thg):
    """test_linops.jl "radial, field/env": make_linop(grid, q, nfun) with a z-independent
    fill equals make_const_linop(grid, q, nfun) at every z; here the fill is a gradient
    between equal pressures (LinearOps.jl:130-226), and norm_radial equals
    const_norm_radial."""
    from luna_b200.radial import prop_radial_args
    kw = dict(R=1e-3, N=64, flength=0.02, λ0=800e-9, λlims=(400e-9, 2000e-9), τfwhm=20e-15,
              energy=30e-6, w0=40e-6, plasma=False, envelope=envelope, thg=thg,
              trange=0.8e-12 if envelope else 0.2e-12)
    c = prop_radial_args("Ar", 1.2, **kw)
    p = prop_radial_args("Ar", (1.2, 1.2), **kw)
    assert p.transform.kind == "radial_z"
    for z in (0.0, 0.013, 0.02, 0.05):
        L = p.linop(z)
        assert np.max(np.abs(L - c.linop)) <= 1e-14 * np.max(np.abs(c.linop)), z
        assert np.max(np.abs(p.transform.fill.normfun(z) / c.transform.normfun - 1)) < 1e-14
        assert p.transform.densityfun(z) == pytest.approx(c.transform.density, rel=1e-15)


def test_radial_fill_gradient_propagation_at_equal_pressures():
    """The oracle's radial solve through an equal-pressure gradient takes the constant
    fill's steps; the saved fields agree to the rounding of β1 (a finite difference)."""
    from luna_b200.radial import prop_radial_args
    kw = dict(R=1e-3, N=64, flength=0.02, λ0=800e-9, λlims=(400e-9, 2000e-9), trange=0.2e-12,
              τfwhm=20e-15, energy=30e-6, w0=40e-6, plasma="PPT", saveN=5)
    c = prop_radial_args("Ar", 1.2, **kw)
    p = prop_radial_args("Ar", (1.2, 1.2), **kw)
    rc = uppe.run(c.transform, c.grid, c.linop, c.Eω, saveN=5)
    rp = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=5)
    assert rp.steps == rc.steps
    for a, b in zip(rp.Eω, rc.Eω):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-9


def test_qdht_roundtrip_and_gaussian_pair():
    from luna_b200.hankel import QDHT
    q = QDHT(4e-3, 128)
    assert np.abs(q.Mi @ q.Mf - np.eye(128)).max() < 1e-9
    w = 0.5e-3
    F = q.Mf @ np.exp(-q.r ** 2 / w ** 2)
    Fa = w ** 2 / 2 * np.exp(-q.k ** 2 * w ** 2 / 4)
    assert np.abs(F - Fa).max() / Fa.max() < 1e-12


# ---------------------------------------------------------------- test_maths.jl:121-137
def test_fwhm_linear_matches_reference_cases():
    x = np.linspace(-1, 1, 2048)
    g = lambda x, fw, x0=0.0: np.exp(-4 * math.log(2) * ((x - x0) / fw) ** 2)
    assert isapprox(uppe.fwhm_linear(x, g(x, 0.2), "min"), 0.2, 1e-4)
    fw, sep = 0.1, 0.5
    y = g(x, fw, -sep / 2) + g(x, fw, sep / 2)
    assert isapprox(uppe.fwhm_linear(x, y, "min"), fw, 1e-4)
    assert isapprox(uppe.fwhm_linear(x, y, "max"), fw + sep, 1e-4)


def test_stats_energy_of_input_pulse():
    """Stats.default's energy (energyfuncs' energy_ω, Fields.jl:510-520) of the input field
    equals the requested pulse energy, and the FWHM of the analytic power is the pulse's."""
    from luna_b200.interface import prop_capillary_args
    p = prop_capillary_args(125e-6, 0.3, "He", 1.0, λ0=800e-9, τfwhm=10e-15, energy=120e-6,
                            λlims=(150e-9, 4e-6), trange=0.25e-12)
    d = uppe.stats_default(p.transform, p.Eω, 0.0, 1e-4)
    assert isapprox(d["energy"], 120e-6, 1e-6)
    assert abs(d["fwhm_t_min"] - 10e-15) < 0.5e-15
    assert d["ω0"] > 0 and d["peakpower"] > 0 and d["electrondensity"] >= 0
