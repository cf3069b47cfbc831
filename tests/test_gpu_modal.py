"""Modal transform (TransModal, full=false) on the GPU against the FP64 oracle.

Cases follow test/test_multimode.jl: argon in a 13 µm capillary with HE11 alone (Kerr,
"Radial"), TM01 + HE21 on both polarisation components (Kerr; ϕ = 0 puts HE21 on y and TM01
on x along θ = 0, where the radial integral samples the cross-section, so the vector Kerr
term couples them; with the LP11 phase ϕ = -π/4 of "Full, LP11 vs TM01" and equal energies
the two cancel there), HE11 + HE12 in a 50 µm capillary with Kerr + PPT plasma at
20 µJ (the plasma term is comparable to Kerr and the cubature needs 129 points), TM01 + HE21
with the vector plasma response (PlasmaVector!) at 3 µJ (23 % of the response), and HE11 + HE12 in H2 with the
scalar Raman response.
"""
import math

import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import numpy as np
import pytest

from luna_b200 import _lib, fields, ionisation, modal, modal_plan, modes, raman
from luna_b200 import physdata as pd
from luna_b200.grid import EnvGrid, RealGrid
from luna_b200.linops import make_const_linop
from luna_b200.nonlinear import (Kerr_env, Kerr_env_thg, Kerr_field, Kerr_field_nothg, PlasmaCumtrapz,
                                 RamanPolarEnv, RamanPolarField)
from luna_b200.nonlinearrhs import TransModeAvg, norm_mode_average
from luna_b200.plan import solve_precon
from oracle import uppe

pytestmark = pytest.mark.gpu

LAM0 = 800e-9


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _case(name, flength=1e-2):
    if name.startswith("env_"):
        return _env_case(name, flength)
    if name == "he11":
        a, gas, pres, trange, energy = 13e-6, "Ar", 5.0, 1e-12, 1e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=1, m=1, kind="HE", ϕ=0.0, loss=False),)
        comps, inputs, plasma = "y", fields.GaussField(LAM0, 30e-15, energy=energy), False
    elif name == "vector":
        a, gas, pres, trange, energy = 13e-6, "Ar", 5.0, 0.4e-12, 1e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=0, m=1, kind="TM", ϕ=0.0, loss=False),
              modes.MarcatiliMode(a, gas, pres, n=2, m=1, kind="HE", ϕ=0.0, loss=False))
        f1 = fields.GaussField(LAM0, 30e-15, energy=energy / 2)
        f2 = fields.GaussField(LAM0, 30e-15, energy=energy / 5)
        comps, inputs, plasma = "xy", ({"mode": 1, "fields": (f1,)}, {"mode": 2, "fields": (f2,)}), False
    elif name == "vector_plasma":  # TM01 + HE21 with vector Kerr and PlasmaVector!
        a, gas, pres, trange, energy = 13e-6, "Ar", 5.0, 0.4e-12, 3e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=0, m=1, kind="TM", ϕ=0.0, loss=False),
              modes.MarcatiliMode(a, gas, pres, n=2, m=1, kind="HE", ϕ=0.0, loss=False))
        f1 = fields.GaussField(LAM0, 10e-15, energy=energy / 2)
        f2 = fields.GaussField(LAM0, 10e-15, energy=energy / 5)
        comps, inputs, plasma = "xy", ({"mode": 1, "fields": (f1,)}, {"mode": 2, "fields": (f2,)}), True
    elif name == "raman":  # HE11 + HE12 in H2 with Kerr and the scalar Raman response
        a, gas, pres, trange, energy = 50e-6, "H2", 2.0, 0.4e-12, 20e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=1, m=1, loss=False),
              modes.MarcatiliMode(a, gas, pres, n=1, m=2, loss=False))
        comps, inputs, plasma = "y", fields.GaussField(LAM0, 10e-15, energy=energy), False
    else:  # two HE modes with Kerr + PPT plasma
        a, gas, pres, trange, energy = 50e-6, "Ar", 1.0, 0.4e-12, 20e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=1, m=1, loss=False),
              modes.MarcatiliMode(a, gas, pres, n=1, m=2, loss=False))
        comps, inputs, plasma = "y", fields.GaussField(LAM0, 10e-15, energy=energy), True
    grid = RealGrid(flength, LAM0, (160e-9, 3000e-9), trange)
    resp = [Kerr_field(pd.gamma3_gas(gas))]
    if plasma:
        rate = ionisation.ionrate_PPTaccel(gas, LAM0, N=2 ** 12)
        resp.append(PlasmaCumtrapz(grid.to, grid.to, rate, pd.ionisation_potential(gas)))
    if name == "raman":
        resp.append(RamanPolarField(grid.to, raman.raman_response(grid.to, gas)))
    Eω, t = modal.setup_modal(grid, pd.density(gas, pres), resp, inputs, ms, comps)
    if name in ("plasma", "raman"):
        Eω[:, 1] = 0.3 * Eω[:, 0]  # some energy in HE12 as well
    return grid, Eω, t, modal.make_const_linop_modes(grid, ms, LAM0)


def _env_case(name, flength):
    """Envelope grids (basic_modal_env.jl): HE11 with Kerr_env; TM01 + HE21 on both
    components with KerrVectorEnv!; HE11 + HE12 in H2 with Kerr_env and RamanPolarEnv; HE11
    with Kerr_env_thg on a THG grid."""
    thg = name == "env_thg"
    grid = EnvGrid(flength, LAM0, (160e-9, 3000e-9), 1e-12, thg=thg)
    if name == "env_vector":
        a, gas, pres, energy = 13e-6, "Ar", 5.0, 1e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=0, m=1, kind="TM", ϕ=0.0, loss=False),
              modes.MarcatiliMode(a, gas, pres, n=2, m=1, kind="HE", ϕ=0.0, loss=False))
        f1 = fields.GaussField(LAM0, 30e-15, energy=energy / 2)
        f2 = fields.GaussField(LAM0, 30e-15, energy=energy / 5)
        comps, inputs = "xy", ({"mode": 1, "fields": (f1,)}, {"mode": 2, "fields": (f2,)})
    elif name == "env_raman":
        a, gas, pres, energy = 50e-6, "H2", 2.0, 20e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=1, m=1, loss=False),
              modes.MarcatiliMode(a, gas, pres, n=1, m=2, loss=False))
        comps, inputs = "y", fields.GaussField(LAM0, 10e-15, energy=energy)
    else:
        a, gas, pres, energy = 13e-6, "Ar", 5.0, 1e-6
        ms = (modes.MarcatiliMode(a, gas, pres, n=1, m=1, kind="HE", ϕ=0.0, loss=False),)
        comps, inputs = "y", fields.GaussField(LAM0, 30e-15, energy=energy)
    g3 = pd.gamma3_gas(gas)
    resp = [Kerr_env_thg(g3, grid.ω0, grid.to) if thg else Kerr_env(g3)]
    if name == "env_raman":
        resp.append(RamanPolarEnv(grid.to, raman.raman_response(grid.to, gas)))
    Eω, t = modal.setup_modal(grid, pd.density(gas, pres), resp, inputs, ms, comps)
    if name == "env_raman":
        Eω[:, 1] = 0.3 * Eω[:, 0]
    return grid, Eω, t, modal.make_const_linop_modes(grid, ms, LAM0, thg=thg)


_ENV = ["env_he11", "env_vector", "env_raman", "env_thg"]


@pytest.mark.parametrize("name", ["he11", "vector", "plasma", "vector_plasma", "raman"] + _ENV)
def test_modal_rhs_fp64_matches_oracle(name):
    """(t::TransModal)(nl, Eω, z) through the C ABI vs the oracle (NonlinearRHS.jl:284-302):
    the same number of cubature points and the integral within 1e-11. The device sums the
    points on time samples (the transforms and mode products are linear); the difference is
    rounding only."""
    grid, Eω, t, _ = _case(name)
    rng = np.random.default_rng(5)
    Ew = Eω * np.exp(1j * 0.1 * rng.standard_normal(Eω.shape))
    nl = np.zeros_like(Ew)
    t(nl, Ew, 0.0)
    ref = uppe.trans_modal(t, Ew, 0.0)
    assert t.plan().nevals == t.oracle_nevals
    tol = 1e-11 if name in ("plasma", "vector_plasma", "raman", "env_raman") else 1e-12
    assert _rel(nl, ref) < tol, _rel(nl, ref)
    # the device-pointer entry point gives the same numbers
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    Ec = np.ascontiguousarray(Ew.T)
    dE = torch.from_numpy(Ec.view(np.float64).copy()).cuda()
    out = torch.zeros_like(dE)
    s = torch.cuda.current_stream()
    _lib.check(lib.luna_b200_modal_rhs_device(t.plan().handle, _lib.ctypes.c_void_p(out.data_ptr()),
                                              _lib.ctypes.c_void_p(dE.data_ptr()), 0.0,
                                              _lib.ctypes.c_void_p(s.cuda_stream)))
    torch.cuda.synchronize()
    dev = out.cpu().numpy().view(np.complex128).reshape(Ec.shape).T
    assert np.array_equal(dev, nl)


@pytest.mark.parametrize("name", ["he11", "vector", "plasma", "vector_plasma", "raman"] + _ENV)
def test_modal_rhs_mixed_close_to_oracle(name):
    grid, Eω, t, _ = _case(name)
    plan = modal_plan.ModalPlan.from_transform(t, _lib.PREC_MIXED)
    nl = np.zeros_like(Eω)
    plan.rhs(nl, Eω, 0.0)
    ref = uppe.trans_modal(t, Eω, 0.0)
    assert _rel(nl, ref) < 1e-3, _rel(nl, ref)


@pytest.mark.parametrize("name,flength", [("he11", 5e-3), ("vector", 2e-3), ("plasma", 1e-3),
                                          ("vector_plasma", 1e-3), ("raman", 1e-3), ("env_he11", 5e-3),
                                          ("env_vector", 2e-3), ("env_raman", 1e-3)])
def test_modal_solve_replay_matches_oracle(name, flength):
    """Following the oracle's step sequence (replay), every saved field within 1e-10."""
    grid, Eω, t, L = _case(name, flength)
    ores = uppe.run(t, grid, L, Eω, saveN=5)
    replay = np.array(ores.steps_all, dtype=np.float64).ravel()
    r = modal_plan.run(Eω, grid, L, t, saveN=5, replay=replay)
    assert r.nsaved == 5
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)


def test_modal_solve_fp64_same_steps_as_oracle():
    grid, Eω, t, L = _case("he11", 5e-3)
    ores = uppe.run(t, grid, L, Eω, saveN=5)
    r = modal_plan.run(Eω, grid, L, t, saveN=5, steplog_cap=1000)
    assert r.status == 0 and r.nsaved == 5 and r.steps == ores.steps
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)


def test_modal_matches_mode_average_on_gpu():
    """test_multimode.jl:3-43 ("Radial") at full length on the device: HE11 with Kerr,
    mode-averaged vs modal spectra within 0.003; the mixed-precision modal solve stays
    within 1e-3 of the FP64 one."""
    grid, Eω, t, L = _case("he11", 5e-2)
    m = t.ts.ms[0]
    linop, βconst, _ = make_const_linop(grid, m, LAM0)
    t0 = TransModeAvg(grid, t.resp, t.density, norm_mode_average(grid, βconst), m.Aeff())
    r0 = solve_precon(t0, linop, np.ascontiguousarray(Eω[:, 0]), 0.0, 1e-4, grid.zmax, saveN=201,
                      max_dt=grid.zmax / 2)
    rm = modal_plan.run(Eω, grid, L, t, saveN=201)
    Iω = np.abs(r0.Eω) ** 2
    Iωr = np.abs(rm.Eω[:, :, 0]) ** 2
    assert np.linalg.norm(Iω - Iωr) / np.linalg.norm(Iω) < 0.003
    rx = modal_plan.run(Eω, grid, L, t, saveN=201, precision=_lib.PREC_MIXED)
    assert _rel(rx.Eω[-1], rm.Eω[-1]) < 1e-3


def test_modal_plan_rejects_unsupported_responses():
    """Vector Raman (an error in the reference too, Nonlinear.jl:288-292) and the no-THG
    response forms are refused."""
    grid, Eω, t, _ = _case("vector")
    rr = RamanPolarField(grid.to, raman.raman_response(grid.to, "N2"))
    for extra in (rr, Kerr_field_nothg(pd.gamma3_gas("Ar"), len(grid.to))):
        t2 = modal.TransModal(grid, t.ts, (t.resp[0], extra), t.density, t.norm)
        with pytest.raises(_lib.LunaError) as e:
            t2.plan()
        assert e.value.code == _lib.LUNA_ERR_UNSUPPORTED
