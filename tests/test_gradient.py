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
    t = TransModeAvgZ(grid, p.transform.resp, g, m, m.Aeff(), 800e-9)
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


def test_gradient_rejects_raman():
    with pytest.raises(NotImplementedError):
        prop_capillary_args(125e-6, 1.0, "H2", (2.0, 0.2), λ0=800e-9, τfwhm=10e-15,
                            energy=50e-6, λlims=(400e-9, 2000e-9), trange=0.5e-12)
