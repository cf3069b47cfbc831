"""The FP64 C++ restatement (oracle/uppe_cpu.cpp, the timed CPU baseline) against the numpy
restatement: the same right-hand sides to rounding, the same accepted steps and saved fields
in a solve. Both read the same transform; the C++ one through the device descriptors."""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import numpy as np
import pytest

from luna_b200.interface import prop_capillary_args, prop_gnlse_args
from oracle import cpu, uppe


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _case(gas, plasma, trange=0.5e-12, flength=0.05):
    return prop_capillary_args(125e-6, flength, gas, 1.0, λ0=800e-9, τfwhm=10e-15, energy=120e-6,
                               λlims=(150e-9, 4e-6), trange=trange, plasma=plasma, saveN=5)


@pytest.mark.parametrize("gas,plasma", [("He", False), ("Ar", None), ("H2", None), ("D2", None)])
def test_cpu_restatement_rhs_matches_numpy(gas, plasma):
    """Kerr only; Kerr + PPT plasma; Kerr + ADK plasma + Raman, for H2 and D2
    (NonlinearRHS.jl:362-373)."""
    p = _case(gas, plasma)
    cp = cpu.CpuPlan(p.transform)
    rng = np.random.default_rng(1)
    Ew = p.Eω * np.exp(1j * 0.1 * rng.standard_normal(p.Eω.shape))
    assert _rel(cp.rhs(Ew), uppe.trans_mode_avg(p.transform, Ew, 0.0)) < 1e-12


@pytest.mark.parametrize("gas,plasma,dz0", [("He", False, 1e-3), ("Ar", None, 1e-4), ("H2", None, 1e-4)])
def test_cpu_restatement_solve_matches_numpy(gas, plasma, dz0):
    """Luna.run with RK45.solve_precon (RK45.jl:27-89, Luna.jl:358-391): the same steps and
    saves within 1e-10 (He from dz0 = 1e-3: at 1e-4 its error estimates sit at the rounding
    level and any two implementations part ways)."""
    p = _case(gas, plasma)
    cp = cpu.CpuPlan(p.transform)
    sv, y, st = cp.solve(p.linop, p.Eω, 0.0, dz0, p.grid.zmax, saveN=5)
    o = uppe.run(p.transform, p.grid, p.linop, p.Eω, init_dz=dz0, saveN=5)
    assert st.status == 0 and st.nsaved == 5 and st.steps == o.steps and st.nrhs == o.nrhs
    for a, b in zip(sv, o.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)


def test_cpu_restatement_step_budget_and_field_limit():
    p = _case("Ar", None)
    cp = cpu.CpuPlan(p.transform)
    _, _, st = cp.solve(p.linop, p.Eω, 0.0, 1e-4, p.grid.zmax, saveN=5, max_steps=7)
    assert st.steps == 7 and st.status == 4  # LUNA_STEP_BUDGET
    strong = _case("Ar", None)
    with pytest.raises(Exception):
        cp.rhs(strong.Eω * 1e3)  # far above the PPT table: the reference errors


@pytest.mark.parametrize("ramanmodel", ["sdo", "SiO2"])
def test_cpu_restatement_envelope_rhs_matches_numpy(ramanmodel):
    """GNLSE on an envelope grid: Kerr_env + RamanPolarEnv (Nonlinear.jl:47-73, 276-333), with
    the single damped oscillator or fused silica's intermediate-broadening model
    (Interface.jl:945-961)."""
    p = prop_gnlse_args(0.11, 0.15, [0.0, 0.0, -11.83e-27, 8.1e-41], λ0=835e-9,
                        λlims=(500e-9, 2400e-9), trange=12.5e-12, τfwhm=50e-15, power=10e3, saveN=5,
                        ramanmodel=ramanmodel)
    cp = cpu.CpuPlan(p.transform)
    rng = np.random.default_rng(4)
    Ew = p.Eω * np.exp(1j * 0.1 * rng.standard_normal(p.Eω.shape))
    assert _rel(cp.rhs(Ew), uppe.trans_mode_avg(p.transform, Ew, 0.0)) < 1e-12


def test_cpu_restatement_soliton_shift_golden_values():
    """test_gnlse.jl:33-56: the soliton self-frequency shift's peak frequency and time
    (golden values of the reference, rtol 1e-14) from the C++ restatement as well."""
    γ, β2, fr, τ0 = 0.1, -1e-26, 0.18, 10e-15
    P0 = abs(β2) / ((1 - fr) * γ * τ0 ** 2)
    flength = np.pi / 2 * τ0 ** 2 / abs(β2) * 90
    p = prop_gnlse_args(γ, flength, [0.0, 0.0, β2], λ0=835e-9, τfwhm=1.763 * τ0, power=P0,
                        pulseshape="sech", λlims=[450e-9, 8000e-9], trange=13e-12, raman=True,
                        shock=False, fr=fr)
    sv, _, st = cpu.CpuPlan(p.transform).solve(p.linop, p.Eω, 0.0, 1e-4, p.grid.zmax, saveN=201)
    assert st.status == 0 and st.nsaved == 201
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.json")) as f:
        ss = json.load(f)["soliton_shift"]
    Ew = sv[-1]
    wpk = p.grid.ω[np.argmax(np.abs(Ew) ** 2)]
    assert abs(wpk / ss["omega_peak"] - 1) <= ss["rtol"]
    Et = np.fft.ifft(Ew) * np.exp(1j * p.grid.ω0 * p.grid.t)
    tpk = p.grid.t[np.argmax(np.abs(Et) ** 2)]
    assert abs(tpk / ss["t_peak"] - 1) <= ss["rtol"]


def test_scan_reference_rhs_counts_reproduced_by_the_cpu_restatement():
    """oracle/scan256_nrhs.json (the scan's reference RHS counts and statuses, recorded from
    the FP64 device integrator, used to extrapolate the CPU baseline) is reproduced exactly by
    full solves of the C++ restatement: a PPT failure at the first step, Ne with Kerr + PPT
    and H2 with ADK plasma and Raman (14 instances were checked the same way, He and Ar on
    every grid among them)."""
    import json
    import os
    from luna_b200 import scan
    ref = json.load(open(os.path.join(os.path.dirname(cpu.__file__), "scan256_nrhs.json")))
    inst = scan.draw_instances(256)
    for i in (206, 181, 162):
        p = scan.build_problem(inst[i], saveN=201)
        _, _, st = cpu.CpuPlan(p.transform).solve(p.linop, p.Eω, 0.0, 1e-4, p.grid.zmax, saveN=201)
        assert st.nrhs == ref["nrhs"][i] and st.status == ref["status"][i], i


def test_nan_in_the_field_ends_in_the_repeat_limit():
    """A NaN in y0 makes every error estimate non-finite: dz halves (RK45.jl:389-391) and
    after repeat_limit rejections the run stops with the reference's error (RK45.jl:72-76),
    in both restatements after the same 11 steps."""
    p = _case("Ar", None)
    y0 = p.Eω.copy()
    y0[len(y0) // 3] = np.nan
    _, _, st = cpu.CpuPlan(p.transform).solve(p.linop, y0, 0.0, 1e-4, p.grid.zmax, saveN=5)
    assert st.status == 2 and st.steps == 11 and st.accepted == 0  # LUNA_REPEAT_LIMIT
    with pytest.raises(RuntimeError, match="repetition"):
        uppe.run(p.transform, p.grid, p.linop, y0, saveN=5)


@pytest.mark.parametrize("gas,extra", [("He", {}), ("H2", {"kerr": False, "plasma": False})])
def test_temperature_changes_results(gas, extra):
    """test_interface.jl ("Temperature"): the same temperature gives identical spectra, a
    different one changes them (density and core index; for H2 with Kerr and plasma off,
    the Raman response's thermal populations), run on the C++ restatement."""
    kw = dict(λ0=800e-9, τfwhm=10e-15, energy=1e-12, trange=400e-15, λlims=(200e-9, 4e-6),
              saveN=5, **extra)

    def final(T):
        p = prop_capillary_args(100e-6, 0.1, gas, 1.0, temperature=T, **kw)
        sv, _, st = cpu.CpuPlan(p.transform).solve(p.linop, p.Eω, 0.0, 1e-4, p.grid.zmax, saveN=5)
        assert st.status == 0
        return sv[-1], p

    a, p300 = final(300.0)
    b, _ = final(300.0)
    c, p400 = final(400.0)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    if gas == "H2":
        r300, r400 = p300.transform.resp[0], p400.transform.resp[0]
        assert r300.kind == "raman_field"
        assert not np.array_equal(r300.r.h(p300.transform.density), r400.r.h(p400.transform.density))
