"""Radial transform (TransRadial + QDHT) on the GPU against the FP64 oracle.

Cases follow test/test_radial.jl: argon, a focused Gaussian beam, Kerr plus PPT or ADK
plasma, at energies where the plasma term is a visible part of the response (20 µJ: ~0.3%
with PPT; 50 µJ: ~6% with ADK, ~97% with PPT); and the other response forms per radial
column (Raman, the analytic-signal Kerr term) and envelope grids (freespace/radial_env.jl).
"""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import numpy as np
import pytest

from luna_b200 import _lib
from luna_b200 import physdata as pd
from luna_b200 import radial_plan
from luna_b200.radial import prop_radial_args
from oracle import uppe

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _problem(energy, plasma, flength=0.01, N=64, saveN=5):
    return prop_radial_args("Ar", 1.2, R=1e-3, N=N, flength=flength, λ0=800e-9,
                            λlims=(400e-9, 2000e-9), trange=0.2e-12, τfwhm=20e-15,
                            energy=energy, w0=40e-6, propz=0.0, plasma=plasma, saveN=saveN)


@pytest.mark.parametrize("energy,plasma", [(20e-6, "PPT"), (50e-6, "PPT"), (50e-6, "ADK"),
                                           (20e-6, False)])
def test_radial_rhs_fp64_matches_oracle(energy, plasma):
    """(t::TransRadial)(nl, Eω, z) through the C ABI vs the oracle (NonlinearRHS.jl:466-474).
    The device applies both QDHT products on the frequency side (they commute with the time
    transforms); the difference is rounding only."""
    p = _problem(energy, plasma)
    rng = np.random.default_rng(3)
    Ew = p.Eω * np.exp(1j * 0.1 * rng.standard_normal(p.Eω.shape))
    nl = np.zeros_like(Ew)
    p.transform(nl, Ew, 0.0)
    ref = uppe.trans_radial(p.transform, Ew, 0.0)
    tol = 1e-11 if plasma else 1e-12
    assert _rel(nl, ref) < tol, _rel(nl, ref)
    # the device-pointer entry point gives the same numbers
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    plan = p.transform.plan()
    Ec = np.ascontiguousarray(Ew.T)
    dE = torch.from_numpy(Ec.view(np.float64).copy()).cuda()
    out = torch.zeros_like(dE)
    s = torch.cuda.current_stream()
    _lib.check(lib.luna_b200_radial_rhs_device(plan.handle, _lib.ctypes.c_void_p(out.data_ptr()),
                                               _lib.ctypes.c_void_p(dE.data_ptr()), 0.0,
                                               _lib.ctypes.c_void_p(s.cuda_stream)))
    torch.cuda.synchronize()
    dev = out.cpu().numpy().view(np.complex128).reshape(Ec.shape).T
    assert np.array_equal(dev, nl)


@pytest.mark.parametrize("energy,plasma,flength", [(20e-6, "PPT", 0.03), (50e-6, "ADK", 0.01)])
def test_radial_solve_fp64_same_steps_as_oracle(energy, plasma, flength):
    """RK45.solve_precon + Luna.run on the radial problem: the same accepted-step sequence
    as the oracle and every saved field within 1e-10."""
    p = _problem(energy, plasma, flength=flength)
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=5)
    r = radial_plan.run(p, steplog_cap=1000)
    assert r.status == 0 and r.nsaved == 5
    assert r.steps == ores.steps
    acc = r.steplog[r.steplog[:, 3] == 1]
    oacc = np.array(ores.accepted)
    assert len(acc) == len(oacc)
    # the error estimate is a difference of nearly equal sums, so rounding moves the
    # controller's step sizes at the 1e-7 level (as for the capillary cases with plasma)
    np.testing.assert_allclose(acc[:, 1], oacc[:, 1], rtol=1e-6)
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)


def test_radial_solve_replay_matches_oracle():
    """Following the oracle's step sequence exactly (replay), the saved fields agree to
    1e-10 at every save point."""
    p = _problem(50e-6, "PPT", flength=0.01)
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=5)
    replay = np.array(ores.steps_all, dtype=np.float64).ravel()
    r = radial_plan.run(p, replay=replay)
    assert r.nsaved == 5
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)


def test_radial_focus_matches_paraxial_gaussian_beam_on_gpu():
    """test_radial.jl:3-65 on the device: after 0.6 m through a focus the fluence profile at
    ω0 matches the paraxial Gaussian-beam width to 1.5e-4."""
    w0, L = 40e-6, 0.6
    p = prop_radial_args("Ar", 1.2, R=4e-3, N=128, flength=L, λ0=800e-9,
                         λlims=(400e-9, 2000e-9), trange=0.2e-12, τfwhm=20e-15,
                         energy=1e-12, w0=w0, propz=-0.3)
    r = radial_plan.run(p)
    assert r.status == 0
    g, q = p.grid, p.q
    Er = q.inverse(r.Eω[-1], axis=1)
    i0 = np.argmin(np.abs(g.ω - 2 * np.pi * pd.c / 800e-9))
    lam0 = 2 * np.pi * pd.c / g.ω[i0]
    w1 = w0 * np.sqrt(1 + (L / 2 * lam0 / (np.pi * w0 ** 2)) ** 2)
    Ia = np.exp(-0.5 * (q.r / (w1 / 2)) ** 2) * (w0 / w1) ** 2
    Ir = np.abs(Er[i0]) ** 2
    Ir, Ia = Ir / Ir.max(), Ia / Ia.max()
    assert np.max(np.abs(Ir - Ia)) / np.linalg.norm(Ir) < 1.5e-4


# ------------------------------------------------------------------ every response form, envelopes
# TransRadial applies Et_to_Pt! column by column (NonlinearRHS.jl:137-141), so every
# response of the mode-averaged transform is available per radial column: Raman
# (RamanPolarField with and without THG), Kerr_field_nothg, and on an envelope grid
# (freespace/radial_env.jl) Kerr_env, Kerr_env_thg and RamanPolarEnv.
_FORMS = {
    "H2-raman": dict(gas="H2", pressure=1.0, plasma="ADK", raman=True, energy=30e-6),
    "H2-raman-nothg": dict(gas="H2", pressure=1.0, plasma=False, raman=True, thg=False, energy=30e-6),
    "Ar-kerr-nothg": dict(gas="Ar", pressure=1.2, plasma="PPT", thg=False, energy=30e-6),
    "Ar-env": dict(gas="Ar", pressure=1.2, envelope=True, energy=30e-6),
    "Ar-env-thg": dict(gas="Ar", pressure=1.2, envelope=True, thg=True, energy=30e-6),
    "N2-env-raman": dict(gas="N2", pressure=2.0, envelope=True, raman=True, energy=30e-6),
}


def _form(name, flength=0.01, N=64, saveN=5):
    """The envelope cases take 0.8 ps so that the oversampled grid has the 1024 samples the
    device's block transforms need at least (0.2 ps gives 256 on an envelope grid)."""
    c = dict(_FORMS[name])
    trange = 0.8e-12 if c.get("envelope") else 0.2e-12
    return prop_radial_args(c.pop("gas"), c.pop("pressure"), R=1e-3, N=N, flength=flength, λ0=800e-9,
                            λlims=(400e-9, 2000e-9), trange=trange, τfwhm=20e-15, w0=40e-6,
                            saveN=saveN, **c)


@pytest.mark.parametrize("name", list(_FORMS))
def test_radial_rhs_every_form_matches_oracle(name):
    p = _form(name)
    rng = np.random.default_rng(13)
    Ew = p.Eω * np.exp(1j * 0.1 * rng.standard_normal(p.Eω.shape))
    nl = np.zeros_like(Ew)
    p.transform(nl, Ew, 0.0)
    ref = uppe.trans_radial(p.transform, Ew, 0.0)
    assert _rel(nl, ref) < 1e-11, _rel(nl, ref)
    plan = radial_plan.RadialPlan.from_transform(p.transform, _lib.PREC_MIXED)
    nm = np.zeros_like(Ew)
    plan.rhs(nm, Ew, 0.0)
    assert _rel(nm, ref) < 2e-4, _rel(nm, ref)


@pytest.mark.parametrize("name", ["H2-raman", "Ar-env", "N2-env-raman"])
def test_radial_solve_every_form_replay_matches_oracle(name):
    """On the oracle's step sequence every saved field within 1e-10 (FP64); the mixed
    precision solve within 1e-3 spectral at every save."""
    p = _form(name, flength=0.02)
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=5)
    replay = np.array(ores.steps_all, dtype=np.float64).ravel()
    r = radial_plan.run(p, replay=replay)
    assert r.status == 0 and r.nsaved == 5 and r.steps == ores.steps
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)
    m = radial_plan.run(p, precision=_lib.PREC_MIXED)
    assert m.status == 0 and m.nsaved == 5
    for a, b in zip(m.Eω, ores.Eω):
        assert _rel(np.abs(a) ** 2, np.abs(b) ** 2) < 1e-3


def test_radial_env_focus_matches_paraxial_gaussian_beam_on_gpu():
    """freespace/radial_env.jl on the device: a 2 nJ envelope through a focus at 0.3 m over
    0.6 m; the fluence profile at ω0 matches the paraxial Gaussian-beam width (as the
    field-resolved test_radial.jl case). 0.8 ps for the device's 1024-sample minimum."""
    w0, L = 40e-6, 0.6
    p = prop_radial_args("Ar", 1.2, R=4e-3, N=128, flength=L, λ0=800e-9, λlims=(400e-9, 2000e-9),
                         trange=0.8e-12, τfwhm=20e-15, energy=2e-9, w0=w0, propz=-0.3,
                         envelope=True, plasma=False)
    r = radial_plan.run(p)
    assert r.status == 0
    g, q = p.grid, p.q
    Er = q.inverse(r.Eω[-1], axis=1)
    i0 = np.argmin(np.abs(g.ω - 2 * np.pi * pd.c / 800e-9))
    lam0 = 2 * np.pi * pd.c / g.ω[i0]
    w1 = w0 * np.sqrt(1 + (L / 2 * lam0 / (np.pi * w0 ** 2)) ** 2)
    Ia = np.exp(-0.5 * (q.r / (w1 / 2)) ** 2) * (w0 / w1) ** 2
    Ir = np.abs(Er[i0]) ** 2
    Ir, Ia = Ir / Ir.max(), Ia / Ia.max()
    assert np.max(np.abs(Ir - Ia)) / np.linalg.norm(Ir) < 1.5e-4


# ------------------------------------------------------------------ gas fill gradient
# make_linop(grid, q, nfun) with nfun(ω; z) from a pressure gradient (LinearOps.jl:174-226),
# densityfun(z) and norm_radial(z) (NonlinearRHS.jl:494-524), evaluated on the device at every
# stage node, step end and save point.
def _fill(name, flength=0.02, saveN=5):
    c = dict(R=1e-3, N=64, flength=flength, λ0=800e-9, λlims=(400e-9, 2000e-9), τfwhm=20e-15,
             w0=40e-6, saveN=saveN)
    if name == "Ar-falling":
        return prop_radial_args("Ar", (2.0, 0.3), trange=0.2e-12, energy=30e-6, plasma="PPT", **c)
    if name == "Ne-multipoint":
        return prop_radial_args("Ne", ([0, 0.005, 0.015, 0.02], [0.5, 3.0, 3.0, 1.0]), trange=0.2e-12,
                                energy=40e-6, plasma="PPT", **c)
    return prop_radial_args("Ar", (2.0, 0.3), trange=0.8e-12, energy=30e-6, plasma=False, envelope=True, **c)


@pytest.mark.parametrize("name", ["Ar-falling", "Ne-multipoint", "Ar-env-falling"])
def test_radial_fill_linop_is_bit_identical_to_host(name):
    p = _fill(name)
    plan = p.transform.plan()
    f = p.transform.fill
    crop = ((len(p.grid.ω) - 1) / (len(p.grid.ωo) - 1)) if p.grid.kind == "real" else len(p.grid.ω) / p.grid.No
    for z in (-0.01, 0.0, 0.004, 0.005, 0.0123, 0.02, 0.03):
        L, of = plan.linop(z)
        ref = f.linop(z)
        assert np.array_equal(L, ref), (z, _rel(L, ref))
        oref = crop * p.transform.densityfun(z) * p.transform.output_factor_z(z)
        assert _rel(of, oref) < 1e-14, (z, _rel(of, oref))


@pytest.mark.parametrize("name", ["Ar-falling", "Ne-multipoint", "Ar-env-falling"])
def test_radial_fill_rhs_and_replay_match_oracle(name):
    p = _fill(name)
    rng = np.random.default_rng(17)
    Ew = p.Eω * np.exp(1j * 0.1 * rng.standard_normal(p.Eω.shape))
    for z in (0.0, 0.0071, 0.02):
        nl = np.zeros_like(Ew)
        p.transform(nl, Ew, z)
        ref = uppe.trans_radial(p.transform, Ew, z)
        assert _rel(nl, ref) < 1e-11, (z, _rel(nl, ref))
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=5)
    replay = np.array(ores.steps_all, dtype=np.float64).ravel()
    r = radial_plan.run(p, replay=replay)
    assert r.status == 0 and r.nsaved == 5 and r.steps == ores.steps
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-10, _rel(a, b)
    m = radial_plan.run(p, precision=_lib.PREC_MIXED)
    assert m.status == 0 and m.nsaved == 5
    for a, b in zip(m.Eω, ores.Eω):
        assert _rel(np.abs(a) ** 2, np.abs(b) ** 2) < 1e-3


# ------------------------------------------------------------------ mixed precision
# FP32 transforms and responses, QDHT as 3xBF16 tensor-core products (tcgen05) with FP32
# accumulation; FP64 state, phase, controller and plasma prefix sums.

@pytest.mark.parametrize("energy,plasma", [(20e-6, "PPT"), (50e-6, "ADK"), (20e-6, False)])
def test_radial_rhs_mixed_close_to_oracle(energy, plasma):
    p = _problem(energy, plasma)
    rng = np.random.default_rng(5)
    Ew = p.Eω * np.exp(1j * 0.1 * rng.standard_normal(p.Eω.shape))
    plan = radial_plan.RadialPlan.from_transform(p.transform, _lib.PREC_MIXED)
    nl = np.zeros_like(Ew)
    plan.rhs(nl, Ew, 0.0)
    ref = uppe.trans_radial(p.transform, Ew, 0.0)
    assert _rel(nl, ref) < 2e-4, _rel(nl, ref)


def test_radial_solve_mixed_spectral_error():
    """The mixed-precision radial solve stays within 1e-3 relative spectral L2 error of the
    FP64 oracle at every save point."""
    p = _problem(20e-6, "PPT", flength=0.03)
    ores = uppe.run(p.transform, p.grid, p.linop, p.Eω, saveN=5)
    r = radial_plan.run(p, precision=_lib.PREC_MIXED)
    assert r.status == 0 and r.nsaved == 5
    for a, b in zip(r.Eω, ores.Eω):
        assert _rel(a, b) < 1e-3, _rel(a, b)


def test_radial_mixed_rejects_nr_not_multiple_of_64():
    p = prop_radial_args("Ar", 1.2, R=1e-3, N=48, flength=0.01, λ0=800e-9,
                         λlims=(400e-9, 2000e-9), trange=0.2e-12, τfwhm=20e-15,
                         energy=1e-6, w0=40e-6, plasma=False)
    with pytest.raises(_lib.LunaError) as e:
        radial_plan.RadialPlan.from_transform(p.transform, _lib.PREC_MIXED)
    assert e.value.code == _lib.LUNA_ERR_UNSUPPORTED


@pytest.mark.parametrize("prec,tol", [(_lib.PREC_FP64, 1e-13), (_lib.PREC_MIXED, 3e-5)])
@pytest.mark.parametrize("forward", [True, False])
@pytest.mark.parametrize("N", [128, 256])
def test_qdht_device_matches_matrix_product(prec, tol, forward, N):
    """luna_b200_qdht_device: the plan's Hankel transform along the radial index (mul!/ldiv!
    of Hankel.jl's QDHT), FP64 CUDA-core tiles or 3xBF16 tensor-core products (N = 128: two
    64-deep K chunks, fewer than the kernel's prefetch ring; N = 256: four, more than it)."""
    torch = pytest.importorskip("torch")
    p = prop_radial_args("Ar", 1.2, R=1e-3, N=N, flength=0.01, λ0=800e-9,
                         λlims=(400e-9, 2000e-9), trange=0.2e-12, τfwhm=20e-15,
                         energy=1e-6, w0=40e-6, plasma=False)
    plan = radial_plan.RadialPlan.from_transform(p.transform, prec)
    rng = np.random.default_rng(11)
    X = rng.standard_normal(p.Eω.shape) + 1j * rng.standard_normal(p.Eω.shape)
    ref = p.q.forward(X, axis=1) if forward else p.q.inverse(X, axis=1)
    ct = np.complex128 if prec == _lib.PREC_FP64 else np.complex64
    Xc = np.ascontiguousarray(X.T).astype(ct)
    rt = np.float64 if prec == _lib.PREC_FP64 else np.float32
    dX = torch.from_numpy(Xc.view(rt).copy()).cuda()
    dY = torch.full_like(dX, float("nan"))
    s = torch.cuda.current_stream()
    _lib.check(_lib.load().luna_b200_qdht_device(plan.handle, _lib.ctypes.c_void_p(dY.data_ptr()),
                                                 _lib.ctypes.c_void_p(dX.data_ptr()), int(forward),
                                                 _lib.ctypes.c_void_p(s.cuda_stream)))
    torch.cuda.synchronize()
    Y = dY.cpu().numpy().view(ct).reshape(Xc.shape).T.astype(np.complex128)
    assert _rel(Y, ref) < tol, _rel(Y, ref)


def test_qdht_device_rejects_unaligned_arrays():
    """The entry point checks the alignment of X and Y on the host, before any launch."""
    torch = pytest.importorskip("torch")
    p = prop_radial_args("Ar", 1.2, R=1e-3, N=64, flength=0.01, λ0=800e-9,
                         λlims=(400e-9, 2000e-9), trange=0.2e-12, τfwhm=20e-15,
                         energy=1e-6, w0=40e-6, plasma=False)
    plan = radial_plan.RadialPlan.from_transform(p.transform, _lib.PREC_MIXED)
    n = 2 * p.Eω.size
    dX = torch.zeros(n + 2, dtype=torch.float32, device="cuda")
    dY = torch.zeros(n + 2, dtype=torch.float32, device="cuda")
    s = _lib.ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.load().luna_b200_qdht_device(plan.handle, _lib.ctypes.c_void_p(dY.data_ptr()),
                                           _lib.ctypes.c_void_p(dX.data_ptr() + 4), 1, s)
    assert rc == _lib.LUNA_ERR_BAD_ARG
