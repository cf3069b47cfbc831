"""Pressure-gradient fills: z-dependent density, linear operator and normalisation.

CPU cases mirror test/test_gradient.jl (the multi-point density law; a gradient with equal
end pressures reproduces the constant-pressure propagation) and test/test_linops.jl (the
z-dependent linop at equal pressures is the constant one). GPU cases compare the fused solver
with a gradient against the FP64 oracle.
"""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import math

import numpy as np
import pytest

from luna_b200 import physdata as pd
from luna_b200.gradient import Gradient, MarcatiliGradientMode, TransModeAvgZ, make_linop
from luna_b200.interface import prop_capillary_args
from luna_b200.linops import make_const_linop
from luna_b200.modes import MarcatiliMode
from luna_b200.nonlinearrhs import norm_mode_average
from oracle import uppe


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_multi_point_density_follows_segment_law():
    """test_gradient.jl:6-20: on each segment p(ζ) = sqrt(p0^2 + ζ/λ (p1^2 - p0^2))."""
    Z = [0, 0.25, 0.5, 1]
    P = [0, 1, 0.5, 0]
    g = Gradient("He", Z, P)
    for ii in range(3):
        lam = Z[ii + 1] - Z[ii]
        zeta = np.linspace(0, lam, 10)
        z = np.linspace(Z[ii], Z[ii + 1], 10)
        p0, p1 = P[ii], P[ii + 1]
        rho_zeta = [pd.density("He", math.sqrt(p0 ** 2 + s / lam * (p1 ** 2 - p0 ** 2))) for s in zeta]
        rho_z = [g.density(x) for x in z]
        np.testing.assert_allclose(rho_z, rho_zeta, rtol=1e-10, atol=0)


def test_two_point_gradient_ends_and_monotone():
    g = Gradient("Ar", 0.3, 2.0, 0.5)
    assert g.p(-1.0) == 2.0 and g.p(0.0) == 2.0 and g.p(0.31) == 0.5
    assert abs(g.p(0.3) - 0.5) < 1e-15
    z = np.linspace(0, 0.3, 31)
    rho = np.array([g.density(x) for x in z])
    assert np.all(np.diff(rho) < 0)
    assert abs(g.density(0.0) - pd.density("Ar", 2.0)) < 1e-12 * g.density(0.0)


@pytest.mark.parametrize("loss", [True, False])
def test_equal_pressure_linop_matches_constant(loss):
    """With p0 == p1 the z-dependent linop, β and normalisation are the constant ones at
    every z (make_linop vs make_const_linop, LinearOps.jl:254-360)."""
    p = prop_capillary_args(125e-6, 1.0, "Ar", 1.0, λ0=800e-9, τfwhm=10e-15, energy=50e-6,
                            λlims=(400e-9, 2000e-9), trange=0.5e-12, loss=loss)
    grid = p.grid
    g = Gradient("Ar", 1.0, 1.0, 1.0)
    m = MarcatiliGradientMode(125e-6, g, loss=loss)
    mc = MarcatiliMode(125e-6, "Ar", 1.0, loss=loss)
    lin, βfun = make_linop(grid, m, 800e-9)
    linc, βc, _ = make_const_linop(grid, mc, 800e-9)
    normc = norm_mode_average(grid, βc)
    t = TransModeAvgZ(grid, p.transform.resp, g, m, 800e-9)
    s = grid.sidx
    for z in np.linspace(0, 1.0, 10):
        assert _rel(lin(z), linc) < 1e-14
        assert _rel(βfun(z)[s], βc[s]) < 1e-15
        ref = normc.pre[s] * math.sqrt(m.Aeff()) * grid.ωwin[s]
        assert _rel(t.norm_factor(z)[s], ref) < 1e-14
        assert t.densityfun(z) == g.density(0.0)


def test_gradient_linop_tracks_local_pressure():
    """Away from equal pressures the linop at z equals the constant-pressure linop at the
    local pressure p(z) (same mode, same ω grid)."""
    p = prop_capillary_args(125e-6, 1.0, "Ar", (2.0, 0.2), λ0=800e-9, τfwhm=10e-15,
                            energy=50e-6, λlims=(400e-9, 2000e-9), trange=0.5e-12)
    g = p.transform.grad
    for z in (0.0, 0.37, 0.81, 1.0):
        pz = g.p(z)
        mc = MarcatiliMode(125e-6, "Ar", pz)
        linc, _, _ = make_const_linop(p.grid, mc, 800e-9)
        # the constant mode uses pd.density(p) itself, the gradient the same closed form
        assert _rel(p.linop(z), linc) < 1e-12, (z, _rel(p.linop(z), linc))


@pytest.mark.parametrize("thg", [False, True])
def test_envelope_equal_pressure_linop_matches_constant(thg):
    """make_linop for an EnvGrid (LinearOps.jl:363-388) at equal pressures is the constant
    envelope operator make_const_linop(grid::EnvGrid, mode, λ0; thg) (LinearOps.jl:266-300):
    -i(β - β1 (ω - ω0) - β(ω0)) without THG, -i(β - β1 (ω - ω0)) with it."""
    p = prop_capillary_args(125e-6, 0.5, "Ar", 1.0, λ0=800e-9, τfwhm=10e-15, energy=50e-6,
                            λlims=(200e-9, 2000e-9), trange=0.5e-12, envelope=True, thg=thg)
    c = p.grid
    assert c.kind == "env" and [r.kind for r in p.transform.resp] == (["kerr_env_thg"] if thg else ["kerr_env"])
    g = Gradient("Ar", 0.5, 1.0, 1.0)
    m = MarcatiliGradientMode(125e-6, g)
    lin, _ = make_linop(c, m, 800e-9, thg=thg)
    for z in (0.0, 0.2, 0.5):
        assert _rel(lin(z), p.linop) < 1e-13, (z, _rel(lin(z), p.linop))


def test_envelope_capillary_set_up_follows_the_interface():
    """prop_capillary(envelope=true) (Interface.jl:360-401, 453-461, 593-605): an EnvGrid
    without THG by default, Kerr_env, RamanPolarEnv for the molecular gases, and no plasma
    response for envelopes."""
    kw = dict(λ0=800e-9, τfwhm=10e-15, energy=50e-6, λlims=(200e-9, 2000e-9), trange=0.5e-12)
    p = prop_capillary_args(125e-6, 0.5, "H2", (2.0, 0.5), envelope=True, **kw)
    assert p.grid.kind == "env" and [r.kind for r in p.transform.resp] == ["kerr_env", "raman_env"]
    with pytest.raises(ValueError):
        prop_capillary_args(125e-6, 0.5, "Ar", 1.0, envelope=True, plasma=True, **kw)
    # the envelope and field-resolved set-ups carry the same pulse energy
    pe = prop_capillary_args(125e-6, 0.5, "Ar", 1.0, envelope=True, **kw)
    from luna_b200.fields import energy_t
    Et = np.fft.ifft(pe.Eω)
    assert abs(energy_t(pe.grid, Et) / 50e-6 - 1) < 1e-6


def test_envelope_equal_pressure_gradient_propagation_matches_constant():
    """test_gradient.jl's equal-pressure check on an envelope grid (oracle, FP64)."""
    kw = dict(λ0=800e-9, τfwhm=30e-15, energy=1e-6, λlims=(160e-9, 3000e-9), trange=1e-12,
              envelope=True, loss=False, saveN=11)
    c = prop_capillary_args(13e-6, 2e-2, "Ar", 5.0, **kw)
    rc = uppe.run(c.transform, c.grid, c.linop, c.Eω, saveN=11)
    p = prop_capillary_args(13e-6, 2e-2, "Ar", (5.0, 5.0), **kw)
    r = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=11)
    assert r.steps == rc.steps
    for a, b in zip(r.Eω, rc.Eω):
        assert _rel(a, b) < 1e-12


def _field_case(pressure):
    return prop_capillary_args(13e-6, 5e-2, "Ar", pressure, λ0=800e-9, τfwhm=30e-15,
                               energy=1e-6, λlims=(160e-9, 3000e-9), trange=0.5e-12,
                               plasma=False, loss=False, saveN=21)


def test_equal_pressure_gradient_propagation_matches_constant():
    """test_gradient.jl "field": a two-point and an array gradient at equal pressures give the
    constant-pressure fields (oracle, FP64)."""
    c = _field_case(5.0)
    rc = uppe.run(c.transform, c.grid, c.linop, c.Eω, saveN=21)
    s = c.grid.sidx
    for pr in ((5.0, 5.0), ([0, 5e-2], [5.0, 5.0])):
        p = _field_case(pr)
        r = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=21)
        assert r.steps == rc.steps
        for a, b in zip(r.Eω, rc.Eω):
            assert _rel(a[s], b[s]) < 1e-12


def test_raman_dephasing_laws_and_rows():
    """The dephasing laws of the molecular Raman models (Raman.jl:142-157, 229-238) and the
    (model, A, B, C) rows the C ABI takes: H2 has density-dependent rotational and vibrational
    linewidths, N2 a density-dependent rotational and a constant vibrational one."""
    from luna_b200 import raman
    from luna_b200.grid import RealGrid
    g = RealGrid(0.3, 800e-9, (150e-9, 4e-6), 0.25e-12)
    h2 = raman.raman_response(g.to, "H2")
    rows = h2.tau2_rows()
    assert rows.shape == (2, 4) and list(rows[:, 0]) == [1.0, 2.0]
    rp = pd.raman_parameters("H2")
    for rho in (0.3 * pd.amg, pd.amg, 4.5 * pd.amg):
        r = rho / pd.amg
        assert h2.tau2s(rho)[0] == 1 / (math.pi * (rp["Arho_r"] / r + rp["Brho_r"] * rho / pd.amg))
        assert h2.tau2s(rho)[1] == 1 / (math.pi * (rp.get("Cv", 0.0) + rp["Arho_v"] / r + rp["Brho_v"] * rho / pd.amg))
    assert h2.Rs[0].hrdamp(0.0) == math.inf
    n2 = raman.raman_response(g.to, "N2")
    rows = n2.tau2_rows()
    assert list(rows[:, 0]) == [1.0, 0.0]
    assert n2.tau2s(pd.amg)[1] == n2.tau2s(3 * pd.amg)[1]
    # the glass response of the GNLSE form does not depend on the density
    sio2 = raman.RamanRespNormedSingleDampedOscillator(1.0, 1e13, 32e-15)
    assert raman.CombinedRamanResponse(g.to, [sio2]).tau2_rows() is None


def test_gradient_with_raman_rebuilds_the_response_at_the_local_density():
    """prop_capillary with a pressure gradient in a Raman-active gas (Interface.jl:538-556):
    the transform's Raman response is h(t; ρ(z)) (Nonlinear.jl:306-307), so its spectrum at
    z equals the constant-fill one at the local pressure."""
    p = prop_capillary_args(125e-6, 0.3, "H2", (3.0, 0.5), λ0=800e-9, τfwhm=10e-15, energy=50e-6,
                            λlims=(150e-9, 4e-6), trange=0.25e-12)
    t = p.transform
    rr = [r for r in t.resp if r.kind == "raman_field"][0].r
    for z in (0.0, 0.13, 0.3):
        pz = t.grad.p(z)
        c = prop_capillary_args(125e-6, 0.3, "H2", pz, λ0=800e-9, τfwhm=10e-15, energy=50e-6,
                                λlims=(150e-9, 4e-6), trange=0.25e-12)
        rc = [r for r in c.transform.resp if r.kind == "raman_field"][0].r
        assert _rel(rr.h(t.densityfun(z)), rc.h(c.transform.density)) < 1e-12, z


def _taper_case(radius, pressure=5.0, flength=5e-2):
    return prop_capillary_args(radius, flength, "Ar", pressure, λ0=800e-9, τfwhm=30e-15,
                               energy=1e-6, λlims=(160e-9, 3000e-9), trange=0.5e-12,
                               plasma=False, loss=False, saveN=21)


def test_constant_taper_matches_constant_radius():
    """test_tapers.jl "const vs afun": a taper whose radius does not change reproduces the
    constant-radius linop and propagation."""
    a = 13e-6
    c = _taper_case(a)
    t = _taper_case(([0.0, 5e-2], [a, a]))
    for z in (0.0, 0.02, 0.05):
        assert np.array_equal(t.linop(z), c.linop)
        assert t.transform.aefffun(z) == pytest.approx(c.transform.aeff, rel=1e-15)
    rc = uppe.run(c.transform, c.grid, c.linop, c.Eω, saveN=21)
    rt = uppe.run(t.transform, t.grid, t.linop, t.Eω, saveN=21)
    assert rt.steps == rc.steps
    for x, y in zip(rt.Eω, rc.Eω):
        assert _rel(x, y) < 1e-12


def test_taper_linop_and_area_track_local_radius():
    """A linear taper a(z) = a0 + (aL - a0) z/L: at each z the linop is the constant-radius
    linop at a(z) and Aeff(z) = a(z)^2 x the mode integral (Capillary.jl:295)."""
    a0, aL, L = 13e-6, 0.75 * 13e-6, 0.1
    t = _taper_case(([0.0, L], [a0, aL]), flength=L)
    m = t.transform.mode
    for z in (0.0, 0.03, 0.07, L):
        az = a0 + (z / L) * (aL - a0)
        assert m.radius(z) == pytest.approx(az, rel=1e-15)
        c = _taper_case(m.radius(z), flength=L)
        assert _rel(t.linop(z), c.linop) < 1e-12, z
        assert t.transform.aefffun(z) == pytest.approx(m.radius(z) ** 2 * m.aeff_intg, rel=1e-15)
    # a narrower core has more waveguide dispersion and loss-free here: |L| grows along z
    assert np.linalg.norm(t.linop(L)) > np.linalg.norm(t.linop(0.0))


# ------------------------------------------------------------------ GPU
_CASES = {
    "Ar-falling": dict(radius=125e-6, flength=0.3, gas="Ar", pressure=(2.0, 0.2), λ0=800e-9,
                       τfwhm=10e-15, energy=150e-6, λlims=(150e-9, 4e-6), trange=0.25e-12),
    "He-rising": dict(radius=75e-6, flength=0.2, gas="He", pressure=(0.2, 3.0), λ0=800e-9,
                      τfwhm=10e-15, energy=120e-6, λlims=(120e-9, 4e-6), trange=0.25e-12),
    "Ne-multipoint": dict(radius=100e-6, flength=0.3, gas="Ne",
                          pressure=([0, 0.1, 0.2, 0.3], [0.5, 3.0, 3.0, 0.5]), λ0=800e-9,
                          τfwhm=10e-15, energy=150e-6, λlims=(150e-9, 4e-6), trange=0.25e-12),
    # test_tapers.jl's linear taper (13 µm to 3/4 of it over 10 cm, Ar 5 bar, Kerr, no loss)
    "Ar-taper": dict(radius=([0, 0.1], [13e-6, 9.75e-6]), flength=0.1, gas="Ar", pressure=5.0,
                     λ0=800e-9, τfwhm=30e-15, energy=600e-9, λlims=(160e-9, 3000e-9),
                     trange=0.5e-12, plasma=False, loss=False),
    "He-taper-gradient": dict(radius=([0, 0.2], [100e-6, 60e-6]), flength=0.2, gas="He",
                              pressure=(0.5, 3.0), λ0=800e-9, τfwhm=10e-15, energy=150e-6,
                              λlims=(120e-9, 4e-6), trange=0.25e-12),
    "Ne-taper-3node": dict(radius=([0, 0.05, 0.15], [120e-6, 80e-6, 80e-6]), flength=0.15,
                           gas="Ne", pressure=2.0, λ0=800e-9, τfwhm=10e-15, energy=200e-6,
                           λlims=(150e-9, 4e-6), trange=0.25e-12),
    # Raman-active fills: H2 (rotational and vibrational linewidths depend on the density,
    # ADK plasma) and N2 (density-dependent rotational, constant vibrational linewidth)
    "H2-falling": dict(radius=125e-6, flength=0.3, gas="H2", pressure=(3.0, 0.5), λ0=800e-9,
                       τfwhm=10e-15, energy=60e-6, λlims=(150e-9, 4e-6), trange=0.25e-12),
    "N2-rising": dict(radius=100e-6, flength=0.2, gas="N2", pressure=(0.3, 2.0), λ0=800e-9,
                      τfwhm=20e-15, energy=40e-6, λlims=(200e-9, 4e-6), trange=0.5e-12,
                      plasma=False),
    # envelope grids: gradients/gradient_modeAvg_env.jl (Ar 7.5 bar to vacuum over 15 cm in a
    # 13 µm core, Kerr_env, no loss), and H2 with its Raman response (RamanPolarEnv)
    "Ar-env-falling": dict(radius=13e-6, flength=0.15, gas="Ar", pressure=(7.5, 0.0), λ0=800e-9,
                           τfwhm=30e-15, energy=1e-6, λlims=(160e-9, 3000e-9), trange=1e-12,
                           envelope=True, loss=False),
    "H2-env-raman": dict(radius=125e-6, flength=0.3, gas="H2", pressure=(3.0, 0.5), λ0=800e-9,
                         τfwhm=10e-15, energy=60e-6, λlims=(150e-9, 4e-6), trange=0.5e-12,
                         envelope=True),
}


def _case(name, saveN=11, **kw):
    c = dict(_CASES[name])
    c.update(kw)
    return prop_capillary_args(c.pop("radius"), c.pop("flength"), c.pop("gas"), c.pop("pressure"),
                               saveN=saveN, **c)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(_CASES))
def test_device_linop_is_bit_identical_to_host(name):
    """linop!(out, z) on the device (luna_b200_plan_linop) equals the host restatement bit for
    bit at every z, including both ends and outside the fibre; the output factor agrees with
    ρ(z) x crop x norm_factor(z) to rounding."""
    from luna_b200 import _lib
    p = _case(name)
    t = p.transform
    plan = t.plan()
    g = p.grid
    crop = (len(g.ω) - 1) / (len(g.ωo) - 1)
    L = np.zeros(len(g.ω), dtype=np.complex128)
    of = np.zeros_like(L)
    for z in [-0.01, 0.0, 1e-9, 0.05, 0.1, 0.1 + 1e-12, 0.1234567, 0.2, 0.29999, g.zmax, g.zmax + 0.1]:
        _lib.check(_lib.load().luna_b200_plan_linop(plan.handle, z, _lib.dptr(L.view(np.float64)),
                                                   _lib.dptr(of.view(np.float64))))
        ref = p.linop(z)
        assert np.array_equal(L, ref), (z, _rel(L, ref))
        oref = crop * t.densityfun(z) * t.norm_factor(z)
        assert _rel(of, oref) < 1e-14, (z, _rel(of, oref))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["Ar-falling", "Ne-multipoint", "He-taper-gradient", "H2-falling",
                                  "N2-rising", "Ar-env-falling", "H2-env-raman"])
def test_gradient_rhs_matches_oracle(name):
    """(t::TransModeAvg)(nl, Eω, z) with densityfun(z) and βfun!(β, z) through the C ABI."""
    p = _case(name)
    rng = np.random.default_rng(7)
    Ew = p.Eω * np.exp(1j * 0.1 * rng.standard_normal(p.Eω.shape))
    for z in (0.0, 0.07, 0.15, 0.2, 0.3):
        nl = np.zeros_like(Ew)
        p.transform(nl, Ew, z)
        ref = uppe.trans_mode_avg(p.transform, Ew, z)
        # plasma: the three prefix sums are summed in a different order (as for constant fills)
        assert _rel(nl, ref) < 3e-11, (z, _rel(nl, ref))


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(_CASES))
def test_gradient_solve_fp64_replay_matches_oracle(name):
    """Luna.run with a pressure gradient on the oracle's step sequence (replay): the
    z-dependent linop is evaluated at every stage node, step end and save point (make_prop!,
    RK45.jl:284-297) and every saved field is within 1e-10."""
    from luna_b200 import plan as P
    p = _case(name)
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=11)
    replay = np.array(ores.steps_all, dtype=np.float64).ravel()
    r = P.run(p, replay=replay)
    assert r.status == 0 and r.nsaved == 11 and r.steps == ores.steps
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(_CASES))
def test_gradient_solve_fp64_free_running(name):
    """With each controller free, the device stays as close to the oracle as the oracle stays
    to itself when its first step is moved by one ulp. β1(z) is a finite difference whose
    rounding (~1e-12 relative) differs between nearby z: once two step sequences differ in
    the last bits their stage nodes meet different β1 rounding, which the error estimate
    resolves, and near kinks of a taper or where steps are rejected the sequences part
    (measured on a B200: oracle vs oracle 4e-9 to 1e-3 between cases, device vs oracle
    within the same range). The replay test above is the parity check of the arithmetic."""
    from luna_b200 import plan as P
    p = _case(name)
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=11)
    o2 = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=11, init_dz=1e-4 * (1 + 2.3e-16))
    spread = max(_rel(a, b) for a, b in zip(o2.Eω, ores.Eω))
    r = P.run(p)
    assert r.status == 0 and r.nsaved == 11
    assert abs(r.steps - ores.steps) <= max(3, 2 * abs(o2.steps - ores.steps)), (r.steps, ores.steps)
    err = max(_rel(a, b) for a, b in zip(r.Eω, ores.Eω))
    assert err < 10 * max(spread, 1e-7), (err, spread)


@pytest.mark.gpu
def test_equal_pressure_gradient_on_device_matches_constant():
    """test_gradient.jl "field" on the device: a gradient at equal pressures integrates like
    the constant fill (same steps; fields equal to rounding)."""
    from luna_b200 import plan as P
    c = _field_case(5.0)
    rc = P.run(c)
    for pr in ((5.0, 5.0), ([0, 5e-2], [5.0, 5.0])):
        p = _field_case(pr)
        r = P.run(p)
        assert r.steps == rc.steps
        for a, b in zip(r.Eω, rc.Eω):
            assert _rel(a, b) < 1e-12, _rel(a, b)


@pytest.mark.gpu
def test_gradient_solve_mixed_spectral_error():
    from luna_b200 import _lib
    from luna_b200 import plan as P
    p = _case("Ar-falling")
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=11)
    r = P.run(p, precision=_lib.PREC_MIXED)
    assert r.status == 0 and r.nsaved == 11
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-3, _rel(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["Ar-falling", "He-taper-gradient"])
def test_gradient_step_stats_use_local_density(name):
    """Stats.default with a gradient or taper on the oracle's step sequence (replay):
    electrondensity is the ionisation fraction x densityfun(z) (Stats.jl:228-257), peak
    intensity and the ionisation field scale use aeff(z); the other keys as for a constant
    fill."""
    from luna_b200 import _lib
    from luna_b200 import plan as P
    p = _case(name, saveN=5)
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=5, stats=True)
    replay = np.array(ores.steps_all, dtype=np.float64).ravel()
    r = P.solve_precon(p.transform, p.linop, p.Eω, 0.0, 1e-4, p.grid.zmax, saveN=5,
                       max_dt=p.grid.zmax / 2, replay=replay, stats_cap=4096)
    assert r.stats is not None and r.stats.shape == ores.stats.shape
    rho0 = p.transform.densityfun(0.0)
    for j, key in enumerate(_lib.STATS_KEYS):
        a, b = r.stats[:, j], ores.stats[:, j]
        assert np.array_equal(np.isnan(a), np.isnan(b)), key
        ok = ~np.isnan(b)
        if key == "electrondensity":
            assert np.all(np.abs(a[ok] - b[ok]) <= 1e-9 * np.abs(b[ok]) + 1e-15 * rho0), key
            continue
        if key == "dz":
            # after the last replayed step the device's own controller picks dz
            a, b, ok = a[:-1], b[:-1], ok[:-1]
        err = np.max(np.abs(a[ok] - b[ok]) / np.maximum(np.abs(b[ok]), 1e-300))
        assert err < 1e-9, (key, err)


@pytest.mark.gpu
def test_gradient_rejections():
    """A Raman plan whose gradient is removed again integrates as before it was attached (the
    spectrum rebuilt at ρ(z) goes back to the one at plan creation); the allocation-free
    entry point rejects gradient plans; a plan without a gradient has no device linop(z)."""
    from luna_b200 import _lib
    from luna_b200.gradient import gradient_desc
    from luna_b200.plan import Plan
    lib = _lib.load()
    p = _case("Ar-falling")
    t = p.transform
    g = t.grid
    crop = (len(g.ω) - 1) / (len(g.ωo) - 1)
    keep = []
    d = gradient_desc(t, crop, 1.0 / (len(g.ωo) - 1) / 2, keep)
    h2 = prop_capillary_args(125e-6, 0.3, "H2", 1.0, λ0=800e-9, τfwhm=10e-15, energy=50e-6,
                             λlims=(150e-9, 4e-6), trange=0.25e-12)
    rplan = Plan.from_transform(h2.transform)
    Ew = h2.Eω * np.exp(1j * 0.1 * np.random.default_rng(2).standard_normal(h2.Eω.shape))
    nl0 = rplan.rhs(np.zeros_like(Ew), Ew, 0.0)
    assert lib.luna_b200_plan_set_gradient(rplan.handle, _lib.ctypes.byref(d)) == 0
    rplan.rhs(np.zeros_like(Ew), Ew, 0.13)
    assert lib.luna_b200_plan_set_gradient(rplan.handle, None) == 0
    assert np.array_equal(rplan.rhs(np.zeros_like(Ew), Ew, 0.0), nl0)
    L = np.zeros(len(h2.grid.ω), dtype=np.complex128)
    assert lib.luna_b200_plan_linop(rplan.handle, 0.0, _lib.dptr(L.view(np.float64)),
                                    _lib.dptr(None)) == _lib.LUNA_ERR_BAD_ARG
    torch = pytest.importorskip("torch")
    gp = t.plan()
    dE = torch.zeros(2 * len(g.ω), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(dE)
    rc = lib.luna_b200_rhs_device_noalloc(gp.handle, _lib.ctypes.c_void_p(out.data_ptr()),
                                          _lib.ctypes.c_void_p(dE.data_ptr()), 0.0, None, None)
    assert rc == _lib.LUNA_ERR_UNSUPPORTED
