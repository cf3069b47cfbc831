"""Host-side logic: grid sizes of the benchmark configurations, plan descriptors, the
scan generator, and the multi-rank split of a scan (gloo, world size 2, CPU only)."""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import os
import socket

import numpy as np
import pytest

from luna_b200 import scan
from luna_b200.grid import EnvGrid, RealGrid
from luna_b200.interface import prop_capillary_args, prop_gnlse_args


def test_capillary_readme_grid_sizes():
    # prop_capillary(125e-6, 3, :He, 1; λ0=800e-9, λlims=(150e-9, 4e-6), trange=1e-12)
    g = RealGrid(3.0, 800e-9, (150e-9, 4e-6), 1e-12)
    assert (g.N, len(g.ω), g.No, len(g.ωo)) == (8192, 4097, 16384, 8193)
    assert abs(g.to[1] - g.to[0] - 8.339e-17) < 1e-19


def test_gnlse_grid_sizes():
    g = EnvGrid(0.15, 835e-9, (500e-9, 2400e-9), 12.5e-12)
    assert g.N == g.No == 8192
    g = EnvGrid(1.0, 835e-9, (450e-9, 8000e-9), 13e-12)
    assert g.N == 16384


def test_linop_zero_outside_sidx_and_loss_clamped():
    p = prop_capillary_args(125e-6, 3.0, "He", 1.0, λ0=800e-9, τfwhm=10e-15, energy=120e-6,
                            λlims=(150e-9, 4e-6), trange=1e-12)
    g = p.grid
    assert np.all(p.linop[~g.sidx] == 0)
    assert np.all(-2 * p.linop.real <= 3000 + 1e-9)
    # the output factor is 1 outside sidx (raw transform output, NonlinearRHS.jl:368-372)
    f = p.transform.output_factor()
    assert np.all(f[~g.sidx] == 1)


def test_gnlse_input_peak_power():
    p = prop_gnlse_args(0.11, 0.15, [0.0, 0.0, -11.83e-27, 8.1e-41], λ0=835e-9, τfwhm=50e-15,
                        power=10e3, pulseshape="sech", λlims=(500e-9, 2400e-9), trange=12.5e-12)
    Et = np.fft.ifft(p.Eω)
    assert abs(np.max(np.abs(Et) ** 2) / 10e3 - 1) < 1e-12


def test_scan_draw_is_seeded_and_in_range():
    a = scan.draw_instances(256)
    b = scan.draw_instances(256)
    assert a == b
    for p in a:
        assert 50e-6 <= p["energy"] <= 400e-6 and 0.5 <= p["pressure"] <= 5
        assert p["gas"] in scan.GASES and p["radius"] in scan.RADII
        assert 8e-15 <= p["τfwhm"] <= 30e-15 and 1 <= p["flength"] <= 3
        assert 0.5e-12 <= p["trange"] <= 2e-12


def test_partition_covers_every_instance_once():
    costs = np.random.default_rng(3).uniform(1, 10, 257)
    for n in (1, 2, 3, 8):
        parts = scan.partition(costs, n)
        allidx = sorted(i for p in parts for i in p)
        assert allidx == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max() + 1e-9


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, costs, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    if costs is None:  # each rank prices the whole draw itself, as bench.py's ranks do
        costs = [scan.shard_cost(p) for p in scan.draw_instances(64)]
    mine = scan.shard(costs, rank, world)
    t = torch.zeros(len(costs), dtype=torch.int64)
    t[mine] = 1
    gathered = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(gathered, t)
    if rank == 0:
        q.put([g.tolist() for g in gathered])
    dist.destroy_process_group()


def test_shard_cost_is_the_schedule_priority():
    for p in scan.draw_instances(12):
        prob = scan.build_problem(p, saveN=2)
        assert scan.shard_cost(p) == pytest.approx(scan.schedule_priority(p, prob), rel=1e-12)


@pytest.mark.parametrize("costs", [np.random.default_rng(5).uniform(1, 10, 64).tolist(), None])
def test_multi_rank_scan_split_gloo(costs):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    masks = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    m = np.array(masks)
    assert np.all(m.sum(axis=0) == 1)  # every instance on exactly one rank
    assert m[0].sum() > 0 and m[1].sum() > 0


def test_accuracy_energy_weights_follow_energyfuncs():
    """energy_ω of Fields.energyfuncs (Fields.jl:510-532) as a weight vector: the input
    pulse carries its prescribed energy, and the weights reproduce SimpsonEven."""
    from luna_b200 import accuracy, fields
    from luna_b200.interface import prop_capillary_args
    p = prop_capillary_args(125e-6, 0.01, "He", 1.0, λ0=800e-9, τfwhm=10e-15, energy=120e-6,
                            λlims=(150e-9, 4e-6), trange=0.25e-12)
    w = accuracy.Weights(p.grid.ω, "real")
    assert abs(w.energy @ np.abs(p.Eω) ** 2 / 120e-6 - 1) < 1e-12
    y = np.random.default_rng(0).random(len(p.grid.ω))
    ref = 2 * np.pi / p.grid.ω[-1] ** 2 * fields.simpson_even(p.grid.ω, y)
    assert abs(w.energy @ y / ref - 1) < 1e-13
    # the drift of a scaled field: (1 + s)^2 - 1 in both energy and photon number
    c = accuracy.compare(np.stack([p.Eω * 1.001]), np.stack([p.Eω]), p.grid.ω)
    assert abs(c["energy"][0] - (1.001 ** 2 - 1)) < 1e-12
    assert abs(c["photons"][0] - (1.001 ** 2 - 1)) < 1e-12
    assert abs(c["spectral"][0] - (1.001 ** 2 - 1)) < 1e-12
    s = accuracy.summary([c, None, accuracy.compare(np.stack([p.Eω]), np.stack([p.Eω]), p.grid.ω)])
    assert s["instances"] == 2 and s["worst_instance"] == 0 and s["above_1e-3"] == [0]


def test_surrogate_cpu_gradients_match_finite_differences():
    """The CPU restatement that checks the device's training gradients is itself exact:
    in FP64 (no BF16 rounding) its gradients match central differences of its loss."""
    from luna_b200 import surrogate as S
    rng = np.random.default_rng(4)
    widths = (6, 5, 4, 3)
    W = [rng.standard_normal((n, k)) * 0.5 for k, n in zip(widths[:-1], widths[1:])]
    b = [rng.standard_normal(n) * 0.1 for n in widths[1:]]
    X = rng.standard_normal((7, widths[0]))
    T = rng.standard_normal((7, widths[-1]))
    loss, gW, gb = S.reference_gradients(X, W, b, T, rounding=False)
    h = 1e-6
    for l in range(len(W)):
        for (i, j) in ((0, 0), (W[l].shape[0] - 1, W[l].shape[1] - 1)):
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[l][i, j] += h
            Wm[l][i, j] -= h
            fd = (S.reference_gradients(X, Wp, b, T, rounding=False)[0] -
                  S.reference_gradients(X, Wm, b, T, rounding=False)[0]) / (2 * h)
            assert abs(fd - gW[l][i, j]) <= 1e-7 * max(1.0, abs(fd)), (l, i, j)
        bp = [v.copy() for v in b]
        bm = [v.copy() for v in b]
        bp[l][0] += h
        bm[l][0] -= h
        fd = (S.reference_gradients(X, W, bp, T, rounding=False)[0] -
              S.reference_gradients(X, W, bm, T, rounding=False)[0]) / (2 * h)
        assert abs(fd - gb[l][0]) <= 1e-7 * max(1.0, abs(fd)), l


def test_autotune_schedule_rule():
    """Clusters go to the instances whose predicted single-CTA time is above the mean SM
    load and whose grid class runs faster on a cluster; the priority is the predicted time
    on the chosen shape (longest first)."""
    from luna_b200 import autotune

    class G:
        def __init__(self, No):
            self.No = No

    class T:
        def __init__(self, raman):
            self.resp = [type("R", (), {"kind": "raman_field" if raman else "kerr_field"})()]

    class Pr:
        def __init__(self, No, raman=False):
            self.grid, self.transform = G(No), T(raman)

    inst = scan.draw_instances(6)
    probs = [Pr(32768, True), Pr(32768), Pr(16384), Pr(8192), Pr(16384), Pr(8192)]
    table = {"No=32768+Raman": {"single": 3.0, "cluster": 1.5, "cluster16": None},
             "No=32768": {"single": 1.6, "cluster": 0.7}, "No=16384": {"single": 0.8, "cluster": 0.9},
             "No=8192": {"single": 0.4, "cluster": None}}
    shapes, prio, pred = autotune.schedule(inst, probs, table, nsm=2)
    w = np.array([scan.nonlinear_phase(p) ** 0.6 for p in inst])
    single = w * np.array([3.0, 1.6, 0.8, 0.4, 0.8, 0.4])
    mean_load = single.sum() / 2
    for i in range(6):
        cl = {0: 1.5, 1: 0.7}.get(i)
        want = 2 if (cl is not None and single[i] >= mean_load) else 1
        assert shapes[i] == want, i
        assert prio[i] == pytest.approx(w[i] * cl if want == 2 else single[i])
    assert all(s == 1 for s in shapes[2:])  # the 16384 class is slower on a cluster here
    assert autotune.grid_class(probs[0]) == "No=32768+Raman"


def test_autotune_schedule_picks_sixteen_ctas_for_the_longest():
    """An instance whose 8-CTA time is at least twice the mean SM load goes to 16 CTAs when
    they are faster for its class."""
    from luna_b200 import autotune

    class Pr:
        def __init__(self, No):
            self.grid = type("G", (), {"No": No})()
            self.transform = type("T", (), {"resp": []})()

    inst = scan.draw_instances(40)
    probs = [Pr(32768)] + [Pr(8192)] * 39
    w = np.array([scan.nonlinear_phase(p) ** 0.6 for p in inst])
    # make instance 0 dominate: its class is slow on one CTA and fast on clusters
    table = {"No=32768": {"single": 1000.0 / w[0], "cluster": 300.0 / w[0], "cluster16": 200.0 / w[0]},
             "No=8192": {"single": 0.01, "cluster": None}}
    shapes, prio, _ = autotune.schedule(inst, probs, table, nsm=148)
    assert shapes[0] == 3 and prio[0] == pytest.approx(200.0)
    assert all(s == 1 for s in shapes[1:])


def test_shotnoise_is_one_photon_per_mode():
    """fields.ShotNoise (Fields.jl:304-321): amplitude sqrt(2π)/(2δt) sqrt(ħω/δω) on the
    real grid and sqrt(2π)/δt sqrt(ħω/δω) inside the envelope grid's signal window (zero
    outside), phases 2π times the generator's uniform draws; the energy weights of the
    reference's energy functions then count one photon per frequency bin (exactly on the
    envelope grid, within the SimpsonEven end weights on the real one)."""
    from luna_b200 import accuracy, fields
    from luna_b200 import physdata as pd
    g = RealGrid(0.1, 800e-9, (150e-9, 4e-6), 0.25e-12)
    n = fields.ShotNoise(np.random.default_rng(3))(g)
    δω, δt = g.ω[1] - g.ω[0], g.t[1] - g.t[0]
    amp = np.sqrt(2 * np.pi) / (2 * δt) * np.sqrt(pd.hbar * g.ω / δω)
    assert np.allclose(np.abs(n), amp, rtol=1e-13, atol=0)
    φ = 2 * np.pi * np.random.default_rng(3).random(len(g.ω))
    assert np.allclose(n, amp * np.exp(1j * φ), rtol=1e-13, atol=0)
    w = accuracy.Weights(g.ω, "real")
    photons = w.photons @ np.abs(n) ** 2 / pd.hbar
    assert abs(photons / np.count_nonzero(g.ω > 0) - 1) < 0.01
    e = EnvGrid(0.1, 800e-9, (150e-9, 4e-6), 0.25e-12)
    ne = fields.ShotNoise(np.random.default_rng(4))(e)
    assert np.all(ne[~e.sidx] == 0)
    δω, δt = e.ω[1] - e.ω[0], e.t[1] - e.t[0]
    amp = np.sqrt(2 * np.pi) / δt * np.sqrt(pd.hbar * e.ω[e.sidx] / δω)
    assert np.allclose(np.abs(ne[e.sidx]), amp, rtol=1e-13, atol=0)
    we = accuracy.Weights(e.ω, "env")
    photons = we.photons @ np.abs(ne) ** 2 / pd.hbar
    assert abs(photons / np.count_nonzero(e.sidx) - 1) < 1e-12


@pytest.mark.parametrize("kind", ["capillary", "gnlse", "multimode"])
def test_setup_shotnoise_adds_the_noise_to_every_mode(kind):
    """shotnoise=true (shotnoise_maybe, Interface.jl:773-781): the input spectrum of every
    propagation mode gains one ShotNoise draw; the rest of the set-up is unchanged."""
    from luna_b200 import fields
    if kind == "capillary":
        f = lambda **k: prop_capillary_args(125e-6, 0.01, "He", 1.0, λ0=800e-9, τfwhm=10e-15,
                                            energy=120e-6, λlims=(150e-9, 4e-6), trange=0.25e-12, **k)
    elif kind == "gnlse":
        f = lambda **k: prop_gnlse_args(0.11, 0.15, [0.0, 0.0, -11.83e-27, 8.1e-41], λ0=835e-9,
                                        τfwhm=50e-15, power=10e3, λlims=(450e-9, 8000e-9),
                                        trange=4e-12, **k)
    else:
        f = lambda **k: prop_capillary_args(13e-6, 1e-2, "Ar", 5.0, modes=2, envelope=True, λ0=800e-9,
                                            τfwhm=30e-15, energy=1e-6, λlims=(160e-9, 3000e-9),
                                            trange=1e-12, **k)
    p0 = f()
    p1 = f(shotnoise=True, rng=np.random.default_rng(11))
    noise = fields.ShotNoise(np.random.default_rng(11))
    d = np.asarray(p1.Eω) - np.asarray(p0.Eω)
    if d.ndim == 1:
        assert np.allclose(d, noise(p0.grid), rtol=0, atol=1e-12 * np.abs(p0.Eω).max())
    else:
        for m in range(d.shape[1]):
            assert np.allclose(d[:, m], noise(p0.grid), rtol=0, atol=1e-12 * np.abs(p0.Eω).max())
    assert np.array_equal(p1.linop, p0.linop)


def test_input_spectral_phase_follows_prop_taylor():
    """PulseField with ϕ (Fields.jl:131-145, prop_taylor Fields.jl:618-625): the spectrum of a
    pulse with GDD and TOD is the unchirped spectrum times exp(-i(ϕ2 Δω²/2 + ϕ3 Δω³/6)) (the
    energy is unchanged by a phase), and the Gaussian's duration grows as
    sqrt(1 + (4 ln2 ϕ2 / τ²)²)."""
    from luna_b200 import fields
    from luna_b200 import physdata as pd
    g = RealGrid(0.1, 800e-9, (150e-9, 4e-6), 1e-12)
    τ, ϕ2, ϕ3 = 10e-15, 50e-30, 20e-45
    E0 = fields.GaussField(800e-9, τ, energy=1e-6)(g)
    E1 = fields.GaussField(800e-9, τ, energy=1e-6, ϕ=[0.0, 0.0, ϕ2, ϕ3])(g)
    Δω = g.ω - pd.wlfreq(800e-9)
    ref = E0 * np.exp(-1j * (ϕ2 * Δω ** 2 / 2 + ϕ3 * Δω ** 3 / 6))
    big = np.abs(E0) > 1e-3 * np.abs(E0).max()
    assert np.allclose(E1[big], ref[big], rtol=1e-6, atol=1e-9 * np.abs(E0).max())
    E2 = fields.GaussField(800e-9, τ, energy=1e-6, ϕ=[0.0, 0.0, ϕ2])(g)
    It = np.abs(fields.analytic(np.fft.irfft(E2, len(g.t)))) ** 2
    above = g.t[It >= It.max() / 2]
    width = above.max() - above.min()
    assert abs(width / (τ * np.sqrt(1 + (4 * np.log(2) * ϕ2 / τ ** 2) ** 2)) - 1) < 0.02


def test_capillary_plasma_model_preionisation_and_sech_width():
    """makeplasma! (Interface.jl:560-590): plasma=true picks PPT for atoms and ADK for
    molecules, "ADK"/"PPT" name the rate, preionfrac reaches PlasmaCumtrapz; makeinputs'
    sech² pulse from its natural width τw equals the one from τfwhm = 2 ln(1+√2) τw."""
    from luna_b200.nonlinear import ADKRate, PPTSpline
    kw = dict(λ0=800e-9, energy=120e-6, λlims=(150e-9, 4e-6), trange=0.25e-12)
    plasma_of = lambda p: [r for r in p.transform.resp if r.kind == "plasma"][0]
    p = prop_capillary_args(125e-6, 0.01, "Ar", 1.0, τfwhm=10e-15, **kw)
    assert isinstance(plasma_of(p).ratefunc, PPTSpline) and plasma_of(p).preionfrac == 0.0
    p = prop_capillary_args(125e-6, 0.01, "Ar", 1.0, τfwhm=10e-15, plasma="ADK", preionfrac=0.1, **kw)
    assert isinstance(plasma_of(p).ratefunc, ADKRate) and plasma_of(p).preionfrac == 0.1
    with pytest.raises(ValueError):
        prop_capillary_args(125e-6, 0.01, "Ar", 1.0, τfwhm=10e-15, plasma="SFA", **kw)
    τw = 6e-15
    a = prop_capillary_args(125e-6, 0.01, "He", 1.0, pulseshape="sech", τw=τw, **kw)
    b = prop_capillary_args(125e-6, 0.01, "He", 1.0, pulseshape="sech",
                            τfwhm=2 * np.log(1 + np.sqrt(2)) * τw, **kw)
    assert np.allclose(a.Eω, b.Eω, rtol=1e-12, atol=1e-12 * np.abs(b.Eω).max())
