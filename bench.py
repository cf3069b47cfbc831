#!/usr/bin/env python
"""Benchmark of the batched capillary UPPE scan on B200.

Workload: the seeded 256-instance mode-averaged capillary scan (energy 50-400 uJ, 0.5-5 bar,
He/Ne/Ar/H2, core radius 75-150 um, 8-30 fs, 1-3 m, uneven grids No = 8192..32768),
integrated to completion in mixed precision by persistent launches: the long instances
distributed over 8-CTA clusters (one instance per cluster) and a single-CTA solver for the
rest, running concurrently. One bench step = one full scan. Metric: simulations
per hour per GPU (completed instances / step time).

  value   device time of the solver launches, inputs already resident in HBM (CUDA events)
  e2e     the same step through the C ABI with host buffers: H2D of every instance's
          linear operator and input field, the launch, D2H of all 201 saved spectra
  cpu_baseline / --impl reference: the FP64 C++ restatement of the reference algorithm
          (oracle/uppe_cpu.cpp, checked against the numpy one) timed per RK step on a
          bounded sample of the scan, extrapolated with the reference RHS counts of every
          instance

Multi-GPU (torchrun): each rank integrates a cost-balanced shard of a 256*N-instance scan
(weak scaling, no collective on the data path; the timing uses a max over ranks).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import luna_b200_loader  # noqa: E402

luna_b200_loader.load()

from luna_b200 import _lib, scan  # noqa: E402
from luna_b200 import plan as P  # noqa: E402

METRIC = "capillary UPPE sims/hour/GPU, mixed+batched vs plain FP64 at ≤1e-3 spec. err"
WORKLOAD = "scan256: 256 mode-averaged capillary instances (He/Ne/Ar/H2, PPT/ADK plasma, Raman for H2), mixed precision, persistent launches (long instances distributed over 8-CTA clusters + single-CTA solver)"
SAVEN = 201
STEPS_FILE = os.path.join(ROOT, "oracle", "scan256_nrhs.json")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_info():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        # start timing only once the sampler runs (its start-up must not overlap the
        # timed region)
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 15.0:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0 or self.p.poll() is not None:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        load = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def step_bytes(Nw, mixed):
    """Algorithmic HBM bytes of one RK step of one instance: each of the 6 stages reads y
    and the earlier stage derivatives and writes one; the final combine reads y and all 7
    and writes yn (y, yn FP64 complex; derivatives FP32 complex in mixed mode)."""
    ky = 16
    kk = 8 if mixed else 16
    stages = sum(ky + i * kk + kk for i in range(1, 7))
    return Nw * (stages + ky + 7 * kk + ky)


def build(world, rank, n_per_rank):
    inst = scan.draw_instances(n_per_rank * world)
    if world > 1:
        # cost-balanced shard of the whole draw (no collective on the data path)
        from luna_b200.grid import RealGrid
        costs = []
        for p in inst:
            g = RealGrid(p["flength"], 800e-9, (p["λmin"], p["λmax"]), p["trange"])
            costs.append(g.No * math.log2(g.No) * p["flength"] * (3 if p["gas"] == "H2" else 1))
        idx = scan.shard(costs, rank, world)
        inst = [inst[i] for i in idx]
    probs = [scan.build_problem(p, saveN=SAVEN) for p in inst]
    return inst, probs


# ----------------------------------------------------------------------------- CPU side
def _oracle_sample(args):
    """Time RK steps of one scan instance on one core with the FP64 C++ restatement of the
    reference algorithm (oracle/uppe_cpu.cpp, the same steps as the numpy restatement),
    or the numpy restatement when the C++ library is not there. Returns (instance, RHS
    evaluations, seconds, RK steps, which restatement)."""
    idx, budget = args
    import luna_b200_loader as L
    L.load()
    from luna_b200 import scan as S
    from oracle import uppe
    p = S.build_problem(S.draw_instances()[idx])
    try:
        from oracle import cpu
        cp = cpu.CpuPlan(p.transform)
    except Exception:
        cp = None
    if cp is not None:
        zmax = p.grid.zmax
        t0 = time.perf_counter()
        _, _, st = cp.solve(p.linop, p.Eω, 0.0, 1e-4, zmax, saveN=2, max_steps=5)
        per_step = (time.perf_counter() - t0) / max(st.steps, 1)
        nsteps = int(min(max(5, budget / per_step), 10 ** 6))
        t0 = time.perf_counter()
        _, _, st = cp.solve(p.linop, p.Eω, 0.0, 1e-4, zmax, saveN=2, max_steps=nsteps)
        return idx, st.nrhs, time.perf_counter() - t0, st.steps, "C++"
    f = lambda y, z: uppe.trans_mode_avg(p.transform, y, z)
    st = uppe.PreconStepper(f, p.linop, p.Eω, 0.0, 1e-4, max_dt=p.grid.zmax / 2)
    nrhs0 = st.nrhs
    t0 = time.perf_counter()
    done = 0
    try:
        while done < 3 or time.perf_counter() - t0 < budget:
            st.step()
            done += 1
    except ValueError:
        pass
    dt = time.perf_counter() - t0
    return idx, st.nrhs - nrhs0, dt, done, "numpy"


def cpu_estimate(sample_seconds=20.0, workers=1):
    """Oracle sims/hour for the 256-instance scan: time per RHS evaluation measured on a
    sample of instances (one per grid class), times each instance's reference RHS count."""
    with open(STEPS_FILE) as f:
        ref = json.load(f)
    nrhs = np.array(ref["nrhs"], dtype=np.float64)
    status = np.array(ref["status"])
    inst = scan.draw_instances(len(nrhs))
    from luna_b200.grid import RealGrid
    cls = []
    for p in inst:
        g = RealGrid(p["flength"], 800e-9, (p["λmin"], p["λmax"]), p["trange"])
        cls.append((g.No, p["gas"] == "H2"))
    classes = sorted(set(cls))
    # one completed (status 0) instance represents each grid class
    reps = [next(i for i in range(len(cls)) if cls[i] == c and status[i] == 0) for c in classes]
    # about sample_seconds of CPU work in total: RK steps per class until the class's
    # share of the time is used (at least 3)
    jobs = [(i, sample_seconds / len(reps)) for i in reps]
    try:  # compile the C++ restatement once, before any worker loads it
        from oracle import cpu
        cpu.build()
    except Exception:
        pass
    t0 = time.perf_counter()
    if workers > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            res = pool.map(_oracle_sample, jobs)
    else:
        res = [_oracle_sample(j) for j in jobs]
    wall = time.perf_counter() - t0
    per_rhs = {}
    for i, nr, dt, done, _ in res:
        per_rhs[cls[i]] = dt / max(nr, 1)
    total = sum(per_rhs[cls[i]] * nrhs[i] for i in range(len(nrhs)))
    ok = int(np.sum(status == 0))
    sims_per_hour_core = 3600.0 * ok / total
    return sims_per_hour_core, {"classes": len(classes), "rk_steps_each": [r[3] for r in res],
                                "impl": "FP64 C++" if all(r[4] == "C++" for r in res) else "FP64 numpy",
                                "sample_wall_s": round(wall, 1),
                                "per_rhs_ms": {f"No={k[0]}{'+Raman' if k[1] else ''}": round(v * 1e3, 2)
                                               for k, v in per_rhs.items()}}


def plain_fp64_estimate(inst):
    """Plain FP64 drop-in on this GPU: one instance per solve (one CTA, as the Julia shim
    calls luna_b200_solve for each prop_capillary). Device time per RK step is measured on
    one instance of each grid class (difference of a 250-step and a 50-step run) and scaled
    by every instance's FP64 step count (oracle/scan256_nrhs.json)."""
    with open(STEPS_FILE) as f:
        ref = json.load(f)
    steps = np.array(ref["steps"], dtype=np.float64)
    status = np.array(ref["status"])
    from luna_b200.grid import RealGrid
    cls = []
    for p in inst:
        g = RealGrid(p["flength"], 800e-9, (p["λmin"], p["λmax"]), p["trange"])
        cls.append((g.No, p["gas"] == "H2"))
    per_step = {}
    for c in sorted(set(cls)):
        i = next(j for j in range(len(cls)) if cls[j] == c and status[j] == 0)
        pr = scan.build_problem(inst[i], saveN=SAVEN)
        plan = P.Plan.from_transform(pr.transform, _lib.PREC_FP64)
        t = []
        for cap in (50, 250):
            b = P.Batch([plan], SAVEN, np.linspace(0.0, pr.grid.zmax, SAVEN), max_steps=cap,
                        max_dt=pr.grid.zmax / 2)
            b.upload([pr.linop], [pr.Eω], [0.0], [1e-4], [pr.grid.zmax])
            b.run()
            t.append(b.run())
        per_step[c] = (t[1] - t[0]) / 200.0 / 1e3
    total = sum(per_step[cls[i]] * steps[i] for i in range(len(steps)))
    ok = int(np.sum(status == 0))
    return 3600.0 * ok / total, {f"No={k[0]}{'+Raman' if k[1] else ''}": round(v * 1e3, 3)
                                 for k, v in per_step.items()}


def run_reference(args, world, rank):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    rates = []
    for _ in range(args.warmup):
        cpu_estimate(workers=cores)
    for _ in range(args.steps):
        r, info = cpu_estimate(workers=cores)
        rates.append(r)
    dt = time.perf_counter() - t0
    # each worker measures one core; the scan instances are independent, so the host
    # throughput is the per-core rate times the cores in use
    value = statistics.median(rates) * cores
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "sims/hour",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / max(args.steps + args.warmup, 1) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "instances": 256, "saveN": SAVEN},
            "cpu_baseline": {"value": value, "unit": "sims/hour", "cores": cores, "kind": "port",
                             "sample": f"{info['impl']} restatement of the reference algorithm, "
                                       f"{info['rk_steps_each']} RK steps per grid class "
                                       f"({info['classes']} classes) in parallel on {cores} cores, "
                                       "scaled by each instance's reference RHS count"},
            "e2e": {"value": value, "unit": "sims/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- radial
RADIAL_METRIC = "radial UPPE RHS evaluations/s (TransRadial, mixed precision, QDHT on tensor cores)"
RADIAL_WORKLOAD = ("radial: TransRadial Nr=256 (R=3 mm) x Nt=2048/No=4096 over 0.5 ps, Ar 1 bar, "
                   "w0=1 mm, 800 nm, 30 fs, 0.5 mJ, f=1 m focusing, 2 m, Kerr + PPT plasma")


def radial_problem():
    from luna_b200.radial import prop_radial_args
    return prop_radial_args("Ar", 1.0, R=3e-3, N=256, flength=2.0, λ0=800e-9,
                            λlims=(400e-9, 2000e-9), trange=0.5e-12, τfwhm=30e-15, energy=0.5e-3,
                            w0=1e-3, focal_length=1.0, plasma="PPT")


def radial_cpu_rate(p, seconds=10.0):
    """Oracle RHS evaluations per second on one core (bounded sample)."""
    from oracle import uppe
    n, t0 = 0, time.perf_counter()
    while n < 2 or time.perf_counter() - t0 < seconds:
        uppe.trans_radial(p.transform, p.Eω, 0.0)
        n += 1
    return n / (time.perf_counter() - t0), n


def run_radial(args, world, rank, local):
    """Per-RHS throughput of the radial transform (one bench step = one evaluation of
    (t::TransRadial)(nl, Eω, z) on the Nw x Nr field), replicas only across GPUs."""
    if args.impl == "reference":
        if rank == 0:
            p = radial_problem()
            rate, n = radial_cpu_rate(p)
            print(json.dumps({"impl": "reference", "metric": RADIAL_METRIC, "value": rate, "unit": "RHS/s",
                              "n_gpus": world, "steps": n, "warmup": 0, "ms_per_step": 1e3 / rate,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f64", "data": "synthetic", "config": {"workload": RADIAL_WORKLOAD},
                              "cpu_baseline": {"value": rate, "unit": "RHS/s", "cores": 1, "kind": "port",
                                               "sample": f"{n} oracle evaluations (numpy FP64)"},
                              "e2e": {"value": rate, "unit": "RHS/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    torch.cuda.set_device(local)
    from luna_b200 import radial_plan as RP
    p = radial_problem()
    lib = _lib.load()
    plan = RP.RadialPlan.from_transform(p.transform, _lib.PREC_MIXED)
    Nw, Nr = p.Eω.shape
    Ec = np.ascontiguousarray(p.Eω.T)
    dE = torch.from_numpy(Ec.view(np.float64).copy()).cuda()
    dN = torch.zeros_like(dE)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    s = torch.cuda.current_stream()
    vp = lambda t: _lib.ctypes.c_void_p(t.data_ptr())
    sp = _lib.ctypes.c_void_p(s.cuda_stream)

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        ts = []
        for _ in range(k):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return ts

    rhs = lambda: _lib.check(lib.luna_b200_radial_rhs_device(plan.handle, vp(dN), vp(dE), 0.0, sp))
    clk = Clocks(local)
    torch.cuda.synchronize()
    t_rhs = timed(rhs, args.steps, args.warmup)
    # the QDHT product alone (FP32 complex in and out, 3xBF16 tensor-core MMAs)
    X = torch.randn(2 * Nw * Nr, dtype=torch.float32, device="cuda")
    Y = torch.empty_like(X)
    qd = lambda: _lib.check(lib.luna_b200_qdht_device(plan.handle, vp(Y), vp(X), 1, sp))
    t_q = timed(qd, args.steps, args.warmup)
    clocks = clk.stop()
    # end to end through the host-buffer entry point (pinned host memory)
    Eh = torch.empty(Ec.shape, dtype=torch.complex128, pin_memory=True).numpy()
    Nh = torch.empty(Ec.shape, dtype=torch.complex128, pin_memory=True).numpy()
    Eh[:] = Ec
    for _ in range(args.warmup):
        lib.luna_b200_radial_rhs(plan.handle, _lib.dptr(Nh.view(np.float64)), _lib.dptr(Eh.view(np.float64)), 0.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _lib.check(lib.luna_b200_radial_rhs(plan.handle, _lib.dptr(Nh.view(np.float64)),
                                            _lib.dptr(Eh.view(np.float64)), 0.0))
    e2e_s = (time.perf_counter() - t0) / args.steps
    # one full propagation (22-28 RK steps, 201 saves of the Nw x Nr field)
    t0 = time.perf_counter()
    r = RP.run(p, precision=_lib.PREC_MIXED)
    solve_s = time.perf_counter() - t0
    ms = statistics.mean(t_rhs)
    q_ms = statistics.mean(t_q)
    flops = 3 * 2.0 * (2 * Nw) * Nr * Nr
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            tpk, pk_kind = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        tpk, pk_kind = 1590.0, "fallback"
    ach = flops / (q_ms / 1e3) / 1e12
    line = {"metric": RADIAL_METRIC, "value": 1e3 / ms, "unit": "RHS/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16x3", "data": "synthetic",
            "config": {"workload": RADIAL_WORKLOAD, "Nw": Nw, "Nr": Nr, "No": p.grid.No,
                       "l2": "256 MB buffer written between timed evaluations"},
            "e2e": {"value": 1.0 / e2e_s, "unit": "RHS/s", "h2d_bytes_per_step": Eh.nbytes,
                    "d2h_bytes_per_step": Nh.nbytes},
            "gpu_launches": 5 * args.steps,
            "roofline": {"bound": "tensor", "kernel": "tc_gemm_3xbf16 (QDHT r->k)", "achieved": ach,
                         "peak": tpk, "unit": "TFLOP/s", "frac": ach / tpk, "traffic": None,
                         "peak_kind": pk_kind, "qdht_ms": q_ms,
                         "note": "3 BF16 products x 2*(2Nw)*Nr^2 flops per launch; latency-bound at this size"},
            "solve": {"sims_per_hour_e2e": 3600.0 / solve_s, "rk_steps": int(r.steps), "status": int(r.status)},
            "clocks": clocks}
    if not args.no_cpu_baseline:
        rate, n = radial_cpu_rate(p)
        line["cpu_baseline"] = {"value": rate, "unit": "RHS/s", "cores": 1, "kind": "port",
                                "sample": f"{n} oracle evaluations of the same field (numpy FP64, one core)"}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- modal
MODAL_METRIC = "modal UPPE RHS evaluations/s (TransModal, radial integral, FP64)"
MODAL_WORKLOAD = ("modal: HE11 of a 13 µm capillary, Ar 5 bar, Nt=8192/No=16384 over 1 ps (160 nm - 3 µm), "
                  "800 nm, 30 fs, 1 µJ, 5 cm, Kerr; p-adaptive Clenshaw-Curtis radial integral, "
                  "reltol 1e-3, 512 evaluations at most")


def modal_problem():
    from luna_b200 import fields, modal, modes
    from luna_b200.grid import RealGrid
    from luna_b200.nonlinear import Kerr_field
    import luna_b200.physdata as pd
    grid = RealGrid(5e-2, 800e-9, (160e-9, 3000e-9), 1e-12)
    ms = (modes.MarcatiliMode(13e-6, "Ar", 5.0, n=1, m=1, kind="HE", loss=False),)
    Eω, t = modal.setup_modal(grid, pd.density("Ar", 5.0), (Kerr_field(pd.gamma3_gas("Ar")),),
                              fields.GaussField(800e-9, 30e-15, energy=1e-6), ms, "y")
    return grid, Eω, t, modal.make_const_linop_modes(grid, ms, 800e-9)


def modal_cpu_rate(t, Eω, seconds=10.0):
    """Oracle RHS evaluations per second on one core (bounded sample)."""
    from oracle import uppe
    n, t0 = 0, time.perf_counter()
    while n < 2 or time.perf_counter() - t0 < seconds:
        uppe.trans_modal(t, Eω, 0.0)
        n += 1
    return n / (time.perf_counter() - t0), n


def run_modal(args, world, rank, local):
    """Per-RHS throughput of the modal transform (one bench step = one evaluation of
    (t::TransModal)(nl, Eω, z) on the Nw x nmodes field), replicas only across GPUs."""
    grid, Eω, t, L = modal_problem()
    if args.impl == "reference":
        if rank == 0:
            rate, n = modal_cpu_rate(t, Eω)
            print(json.dumps({"impl": "reference", "metric": MODAL_METRIC, "value": rate, "unit": "RHS/s",
                              "n_gpus": world, "steps": n, "warmup": 0, "ms_per_step": 1e3 / rate,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f64", "data": "synthetic", "config": {"workload": MODAL_WORKLOAD},
                              "cpu_baseline": {"value": rate, "unit": "RHS/s", "cores": 1, "kind": "port",
                                               "sample": f"{n} oracle evaluations (numpy FP64)"},
                              "e2e": {"value": rate, "unit": "RHS/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    torch.cuda.set_device(local)
    from luna_b200 import modal_plan as MP
    lib = _lib.load()
    plan = t.plan()
    Nw, nm = Eω.shape
    Ec = np.ascontiguousarray(Eω.T)
    dE = torch.from_numpy(Ec.view(np.float64).copy()).cuda()
    dN = torch.zeros_like(dE)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    s = torch.cuda.current_stream()
    vp = lambda x: _lib.ctypes.c_void_p(x.data_ptr())
    sp = _lib.ctypes.c_void_p(s.cuda_stream)
    rhs = lambda: _lib.check(lib.luna_b200_modal_rhs_device(plan.handle, vp(dN), vp(dE), 0.0, sp))
    for _ in range(args.warmup):
        rhs()
    clk = Clocks(local)
    ts = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        rhs()
        e1.record(s)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    clocks = clk.stop()
    ms = statistics.mean(ts)
    # end to end through the host-buffer entry point (pinned host memory); it also reports
    # the number of cubature points the evaluation took
    Eh = torch.empty(Ec.shape, dtype=torch.complex128, pin_memory=True).numpy()
    Nh = torch.empty(Ec.shape, dtype=torch.complex128, pin_memory=True).numpy()
    Eh[:] = Ec
    nev = _lib.ctypes.c_int(0)
    call = lambda: _lib.check(lib.luna_b200_modal_rhs(plan.handle, _lib.dptr(Nh.view(np.float64)),
                                                      _lib.dptr(Eh.view(np.float64)), 0.0,
                                                      _lib.ctypes.byref(nev)))
    for _ in range(args.warmup):
        call()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        call()
    e2e_s = (time.perf_counter() - t0) / args.steps
    # one full propagation (Luna.run with 201 saves)
    t0 = time.perf_counter()
    r = MP.run(Eω, grid, L, t, saveN=201)
    solve_s = time.perf_counter() - t0
    # algorithmic bytes of one evaluation, per mode, in FP64 complex elements of 16 B: stage
    # and store kernels read and write Nw twice; the field kernel reads Nw and writes M = No/2
    # sample pairs; each interior node reads the M pairs and writes M; level l (up to the
    # last one taken, lv) reads the 2^(l+1)-1 node arrays (level 0 once more for its
    # midpoint comparison) and writes Nw
    M = grid.No // 2
    lv = int(round(np.log2(nev.value - 1))) - 1  # the last level has 2^(lv+1) + 1 points
    nodes = (2 << lv) - 1
    level_reads = 1 + sum((2 << l) - 1 for l in range(lv + 1))
    byts = 16 * nm * (4 * Nw + (Nw + M) + 2 * M * nodes + M * level_reads + Nw * (lv + 1))
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            hpk, pk_kind = float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        hpk, pk_kind = 6650.0, "fallback"
    ach = byts / (ms / 1e3) / 1e9
    line = {"metric": MODAL_METRIC, "value": 1e3 / ms, "unit": "RHS/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": MODAL_WORKLOAD, "Nw": Nw, "nmodes": nm, "No": grid.No,
                       "cubature_points": nev.value, "l2": "256 MB buffer written between timed evaluations"},
            "e2e": {"value": 1.0 / e2e_s, "unit": "RHS/s", "h2d_bytes_per_step": Eh.nbytes,
                    "d2h_bytes_per_step": Nh.nbytes},
            "gpu_launches": (3 + 2 * MP.cubature_levels(t.mfcn)) * args.steps,
            "roofline": {"bound": "hbm", "kernel": "modal RHS (time, node, level kernels)", "achieved": ach,
                         "peak": hpk, "unit": "GB/s", "frac": ach / hpk, "traffic": None, "peak_kind": pk_kind,
                         "note": "algorithmic bytes of the whole evaluation over its duration; launch-bound"},
            "solve": {"s": solve_s, "rk_steps": int(r.steps), "status": int(r.status)},
            "clocks": clocks}
    if not args.no_cpu_baseline:
        rate, n = modal_cpu_rate(t, Eω)
        line["cpu_baseline"] = {"value": rate, "unit": "RHS/s", "cores": 1, "kind": "port",
                                "sample": f"{n} oracle evaluations of the same field (numpy FP64, one core)"}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU side
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU and plain-FP64 baselines (timing experiments)")
    ap.add_argument("--max-rk-steps", type=int, default=200000,
                    help="per-instance step budget (profiling aid; the scan needs < 30000)")
    ap.add_argument("--no-dist", action="store_true",
                    help="integrate every instance on one CTA or a Raman cluster (no distributed instances)")
    ap.add_argument("--dist-min-no", type=int, default=0,
                    help="oversampled length from which an instance runs distributed (0: library default)")
    ap.add_argument("--no-clusters", action="store_true",
                    help="integrate every instance on one CTA (profiling aid)")
    ap.add_argument("--workload", default="scan256", choices=["scan256", "radial", "modal"],
                    help="scan256: the batched capillary scan (headline); radial: TransRadial RHS; "
                         "modal: TransModal RHS")
    args = ap.parse_args()
    world, rank, local = dist_info()
    if args.workload == "radial":
        return run_radial(args, world, rank, local)
    if args.workload == "modal":
        return run_modal(args, world, rank, local)
    if args.impl == "reference":
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo")
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    t_setup = time.perf_counter()
    inst, probs = build(world, rank, args.instances)
    n = len(probs)
    plans = [P.Plan.from_transform(p.transform, _lib.PREC_MIXED) for p in probs]
    # each instance saves on its own GridCondition range(0, zmax, 201) with max_dz = zmax/2
    batch = P.Batch(plans, SAVEN, np.linspace(0.0, 1.0, SAVEN), max_steps=args.max_rk_steps,
                    flags=(_lib.SOLVE_NO_CLUSTERS if args.no_clusters else 0) |
                    (_lib.SOLVE_NO_DIST if args.no_dist else 0),
                    dist_min_no=args.dist_min_no)
    zsaves = [np.linspace(0.0, p.grid.zmax, SAVEN) for p in probs]
    max_dts = [p.grid.zmax / 2 for p in probs]
    # pinned host buffers for the end-to-end path
    pin = lambda shape: torch.empty(shape, dtype=torch.complex128, pin_memory=True).numpy()
    Lh = [pin((len(p.linop),)) for p in probs]
    Yh = [pin((len(p.Eω),)) for p in probs]
    Sh = [pin((SAVEN, len(p.Eω))) for p in probs]
    Oh = [pin((len(p.Eω),)) for p in probs]
    for i, p in enumerate(probs):
        Lh[i][:] = p.linop
        Yh[i][:] = p.Eω
    z0 = [0.0] * n
    dz0 = [1e-4] * n
    zmax = [p.grid.zmax for p in probs]
    h2d = sum(Lh[i].nbytes + Yh[i].nbytes for i in range(n))
    d2h = sum(Sh[i].nbytes + Oh[i].nbytes for i in range(n))
    setup_s = time.perf_counter() - t_setup

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def maxr(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    batch.upload(Lh, Yh, z0, dz0, zmax, zsaves, max_dts)
    batch.set_priority([scan.schedule_priority(p, q) for p, q in zip(inst, probs)])
    kinfo = batch.info()
    for _ in range(args.warmup):
        batch.run()
    dev_ms, e2e_s, stats = [], [], None
    clk = Clocks(local)
    for _ in range(args.steps):
        barrier()
        t0 = time.perf_counter()
        batch.upload(Lh, Yh, z0, dz0, zmax, zsaves, max_dts)   # H2D from pinned host memory
        ms = batch.run()                              # device time of the solver launch
        _, _, stats = batch.download(Sh, Oh)          # D2H of all saved spectra
        barrier()
        e2e_s.append(time.perf_counter() - t0)
        dev_ms.append(ms)
    clocks = clk.stop()
    ms = maxr(max(dev_ms) if dev_ms else 0.0)
    e2e = maxr(max(e2e_s) if e2e_s else 0.0)
    ok = sum(1 for s in stats if s.status == 0)  # instances that reached zmax
    failed = n - ok
    total_ok = ok
    if dist is not None:
        t = torch.tensor([ok, failed], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        total_ok, failed = int(t[0].item()), int(t[1].item())
    value = total_ok / (ms / 1e3) * 3600.0
    e2e_value = total_ok / e2e * 3600.0
    steps_all = sum(s.steps for s in stats)
    nrhs_all = sum(s.nrhs for s in stats)
    alg_bytes = sum(s.steps * step_bytes(len(p.Eω), True) for s, p in zip(stats, probs))
    hbm, peak_kind = peaks()
    achieved = alg_bytes / (ms / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "solve_kernel_scan_traffic.json")
    if os.path.exists(tf):
        with open(tf) as f:
            tj = json.load(f)
        traffic = tj.get("dram_bytes_per_rk_step", 0) * steps_all
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "sims/hour", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64", "data": "synthetic (seeded scan draw, no noise)",
                "config": {"workload": WORKLOAD, "instances_per_gpu": n, "saveN": SAVEN,
                           "precision": "mixed: FP32 transforms/responses/stage derivatives, FP64 state/phase/controller/norms/plasma sums",
                           "l2": "per-instance state 0.1-1 MB x 256 instances > 126 MB L2 (no flush needed)",
                           "failed_instances": failed},
                "e2e": {"value": e2e_value, "unit": "sims/hour", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e * 1e3},
                "gpu_launches": args.steps * kinfo[0],
                "scheduling": {"kernels_per_step": kinfo[0], "cluster_instances": kinfo[1],
                               "clusters": kinfo[2]},
                "rk_steps_per_scan": steps_all, "rhs_evals_per_s": nrhs_all / (ms / 1e3),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": traffic,
                             "peak_kind": peak_kind,
                             "note": "algorithmic bytes = RK stage vectors per step (y/yn FP64, k FP32) x steps; kernel is latency/SMEM bound"},
                "clocks": clocks, "setup_s": round(setup_s, 1)}
        try:
            be, _ = batch.timeline()
            line["timeline"] = {"long_pole_s": float(np.max(be[:, 1] - be[:, 0])),
                                "p90_end_s": float(np.percentile(be[:, 1], 90)),
                                "busy_cta_s": float(np.sum(be[:, 1] - be[:, 0]))}
        except Exception as e:
            line["timeline"] = {"error": str(e)[:200]}
        if world == 1 and args.instances == 256 and not args.no_cpu_baseline:
            try:
                v0, per = plain_fp64_estimate(inst)
                line["plain_fp64"] = {"value": v0, "unit": "sims/hour", "ms_per_rk_step": per,
                                      "method": "FP64 single-instance solves (luna_b200_solve path), device time per RK step per grid class x FP64 step counts",
                                      "speedup_of_value": value / v0}
            except Exception as e:
                line["plain_fp64"] = {"value": None, "error": str(e)[:200]}
        if not args.no_cpu_baseline and world == 1:
            try:
                v1, info = cpu_estimate(workers=1)
                line["cpu_baseline"] = {"value": v1, "unit": "sims/hour", "cores": 1, "kind": "port",
                                        "sample": f"{info['impl']} restatement of the reference algorithm, {info['rk_steps_each']} RK steps of one instance per grid class ({info['classes']} classes, {info['sample_wall_s']} s), scaled by each instance's reference RHS count",
                                        "per_rhs_ms": info["per_rhs_ms"]}
            except Exception as e:  # report, do not hide
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
