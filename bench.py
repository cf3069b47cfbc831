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
  accuracy  after the timed region, the same scan integrated in plain FP64 (one batch,
          also timed: `fp64_batched`), every mixed save compared with the FP64 save at the
          same z: relative spectral L2 error of |Eω|^2, energy and photon-number drift
  plain_fp64  the plain FP64 drop-in measured: sequential single-instance solves (one
          luna_b200_solve each, as the Julia shim calls it per prop_capillary) of a
          stratified subset of the scan
  cpu_baseline / --impl reference: the FP64 C++ restatement of the reference algorithm
          (oracle/uppe_cpu.cpp, checked against the numpy one) timed per RHS evaluation
          on a bounded sample of the scan, one worker per host core all running at once,
          and scaled by every instance's RHS count from full solves of the same
          restatement (oracle/scan256_nrhs.json); the instances are spread over the cores
          longest first

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
WORKLOAD = ("scan256: 256 mode-averaged capillary instances (seed 20261203; He/Ne/Ar/H2, PPT/ADK "
            "plasma, Raman for H2; No 8192-32768), each integrated to its fibre length with 201 saves")
IMPL = {"fp64": ("FP64 batched: persistent launches, long instances distributed over 8-CTA clusters "
                 "(FP64 sub-transforms and responses), the rest on single CTAs"),
        "mixed": ("mixed precision (FP32 transforms/responses/stage derivatives, FP64 state/phase/controller/"
                  "norms/plasma sums), persistent launches: long instances distributed over 8-CTA clusters, "
                  "the rest on single CTAs")}
SAVEN = 201
# relative tolerance of the mixed-precision integrations (the plain FP64 path keeps the
# reference's 1e-6)
MIXED_RTOL = 1e-6
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


def fma_peaks():
    """FP32 and FP64 FMA throughput of this GPU in TFLOP/s, measured now by the project's
    microkernel (luna.jl_b200/csrc/peaks.cu, CUDA events, fastest of 5 launches)."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "luna.jl_b200", "libluna_peaks.so"))
    lib.luna_peaks_fma.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_float)]
    out = {}
    for name, fp64 in (("fp32", 0), ("fp64", 1)):
        tf, ms = ctypes.c_double(0), ctypes.c_float(0)
        if lib.luna_peaks_fma(fp64, 4096, ctypes.byref(tf), ctypes.byref(ms)) != 0:
            raise RuntimeError("FMA microbenchmark failed")
        out[name] = tf.value
    return out


def rhs_flops(No, raman):
    """Algorithmic flops of one mode-averaged RHS evaluation on an No-point oversampled real
    grid: two real transforms of No (2.5 No log2 No each), with Raman two more of 2 No (the
    response spectrum is computed once per plan), and per sample Kerr 4, plasma 30 (rate
    exp, three running integrals, ionisation fraction) and the PPT spline / ADK rate 15."""
    f = 2 * 2.5 * No * math.log2(No) + No * (4 + 30 + 15)
    if raman:
        f += 2 * 2.5 * (2 * No) * math.log2(2 * No) + 3 * No
    return f


def step_flops(No, N, raman):
    """Flops of one RK step: 6 RHS evaluations, the window filter's two transforms of the
    coarse grid (N real samples) and the stage combines (complex exp and axpys, ~60 per
    frequency bin and stage)."""
    Nw = N // 2 + 1
    return 6 * rhs_flops(No, raman) + 2 * 2.5 * N * math.log2(N) + 7 * 60 * Nw


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
        # cost-balanced shard of the whole draw by the scheduler's step model (no
        # collective on the data path; every rank computes the same costs)
        idx = scan.shard([scan.shard_cost(p) for p in inst], rank, world)
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


def _grid_classes(inst):
    from luna_b200.grid import RealGrid
    cls = []
    for p in inst:
        g = RealGrid(p["flength"], 800e-9, (p["λmin"], p["λmax"]), p["trange"])
        cls.append((g.No, p["gas"] == "H2"))
    return cls


def lpt_makespan(times, workers):
    """Makespan of independent jobs on ``workers`` cores, longest first to the least loaded."""
    loads = [0.0] * max(1, workers)
    for t in sorted(times, reverse=True):
        j = loads.index(min(loads))
        loads[j] += t
    return max(loads)


def julia_probe():
    """The reference itself is Julia: say whether this host could time it."""
    import shutil
    exe = shutil.which("julia")
    if exe is None:
        return "reference Julia timing: unavailable on this box (no julia executable; no network to install Luna.jl)"
    try:
        v = subprocess.run([exe, "--version"], capture_output=True, text=True, timeout=30).stdout.strip()
    except Exception as e:  # report, do not hide
        v = f"julia present but --version failed: {e}"
    return f"{v}; Luna.jl is not installed here (no network), so the reference Julia timing is unavailable"


def cpu_estimate(sample_seconds=20.0, workers=1, pool=None):
    """Host sims/hour of the 256-instance scan with the FP64 C++ restatement on ``workers``
    cores: ``workers`` samples run at once (one per core, cycling over the grid classes,
    each about ``sample_seconds`` of RK steps of a completed instance of its class), which
    gives the time per RHS evaluation of every class under full load; each instance's time
    is its RHS count (full C++ solves, oracle/scan256_nrhs.json) times its class's time,
    and the instances are spread over the cores longest first."""
    with open(STEPS_FILE) as f:
        ref = json.load(f)
    nrhs = np.array(ref["nrhs"], dtype=np.float64)
    status = np.array(ref["status"])
    inst = scan.draw_instances(len(nrhs))
    cls = _grid_classes(inst)
    classes = sorted(set(cls))
    # one completed (status 0) instance represents each grid class
    reps = [next(i for i in range(len(cls)) if cls[i] == c and status[i] == 0) for c in classes]
    jobs = [(reps[k % len(reps)], sample_seconds) for k in range(max(workers, len(reps)))]
    if workers == 1:
        # one core: the classes one after the other, sample_seconds in total
        jobs = [(i, sample_seconds / len(reps)) for i in reps]
    t0 = time.perf_counter()
    if pool is not None:
        res = pool.map(_oracle_sample, jobs, chunksize=1)
    else:
        res = [_oracle_sample(j) for j in jobs]
    wall = time.perf_counter() - t0
    tot = {}
    for i, nr, dt, done, _ in res:
        a = tot.setdefault(cls[i], [0.0, 0])
        a[0] += dt
        a[1] += nr
    per_rhs = {c: v[0] / max(v[1], 1) for c, v in tot.items()}
    t_inst = [per_rhs[cls[i]] * nrhs[i] for i in range(len(nrhs))]
    makespan = lpt_makespan(t_inst, workers)
    ok = int(np.sum(status == 0))
    return 3600.0 * ok / makespan, {
        "classes": len(classes), "samples": len(jobs), "rk_steps_each": [r[3] for r in res],
        "impl": "FP64 C++" if all(r[4] == "C++" for r in res) else "FP64 numpy",
        "sample_wall_s": round(wall, 1), "cpu_s_total": round(sum(t_inst), 1),
        "makespan_s": round(makespan, 1), "longest_instance_s": round(max(t_inst), 1),
        "per_rhs_ms": {f"No={k[0]}{'+Raman' if k[1] else ''}": round(v * 1e3, 3) for k, v in per_rhs.items()}}


def plain_fp64_measured(inst, probs, dur, status64, k=8):
    """The plain FP64 drop-in, measured: one single-instance FP64 solve after another (a
    batch of one, as luna_b200_solve runs it: on a cluster for the long grids, 16 CTAs for
    No = 32768 and 8 for No = 16384, on one CTA otherwise), device time with CUDA events, for
    a stratified subset of the completed instances: in each of the two strata (cluster,
    single CTA) k quantiles of their integration times in the single-CTA FP64 batch.
    Returns the subset's own
    sims/hour, the scan estimate (per stratum, the batch's per-instance times scaled by the
    subset's measured/batch ratio) and the per-instance record."""
    done = [i for i in range(len(probs)) if status64[i] == 0]
    strata = {True: [], False: []}
    for i in done:
        strata[probs[i].grid.No >= 16384].append(i)
    rows, t_all, n_all, scan_s = [], 0.0, 0, 0.0
    for big, members in strata.items():
        if not members:
            continue
        order = sorted(members, key=lambda i: dur[i])
        pick = sorted({order[min(len(order) - 1, int((j + 0.5) * len(order) / k))] for j in range(k)})
        t_sub, d_sub = 0.0, 0.0
        for i in pick:
            p = probs[i]
            plan = P.Plan.from_transform(p.transform, _lib.PREC_FP64)
            b = P.Batch([plan], SAVEN, np.linspace(0.0, p.grid.zmax, SAVEN), max_dt=p.grid.zmax / 2)
            b.upload([p.linop], [p.Eω], [0.0], [1e-4], [p.grid.zmax])
            clusters = b.info()[1]
            ms = b.run()
            st = b.download()[2][0]
            rows.append({"instance": i, "gas": inst[i]["gas"], "No": p.grid.No, "steps": int(st.steps),
                         "s": round(ms / 1e3, 3), "status": int(st.status), "cluster": bool(clusters)})
            t_sub += ms / 1e3
            d_sub += dur[i]
            del b, plan
        t_all += t_sub
        n_all += len(pick)
        scan_s += float(np.sum([dur[i] for i in members])) * (t_sub / max(d_sub, 1e-30))
    return 3600.0 * n_all / t_all, 3600.0 * len(done) / scan_s, rows


def run_reference(args, world, rank):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    import multiprocessing as mp
    try:  # compile the C++ restatement once, before any worker loads it
        from oracle import cpu
        cpu.build()
    except Exception:
        pass
    t0 = time.perf_counter()
    rates = []
    with mp.get_context("spawn").Pool(cores) as pool:
        for _ in range(args.warmup):
            cpu_estimate(sample_seconds=5.0, workers=cores, pool=pool)
        for _ in range(args.steps):
            r, info = cpu_estimate(sample_seconds=5.0, workers=cores, pool=pool)
            rates.append(r)
    dt = time.perf_counter() - t0
    value = statistics.median(rates)
    sample = (f"{info['impl']} restatement of the reference algorithm (oracle/uppe_cpu.cpp): "
              f"{info['samples']} samples of ~5 s of RK steps, one per core at once, over the "
              f"{info['classes']} grid classes; time per RHS evaluation under full load x each "
              f"instance's RHS count from full solves of the same restatement, instances spread "
              f"longest first over {cores} cores (makespan {info['makespan_s']} s, longest "
              f"instance {info['longest_instance_s']} s)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "sims/hour",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / max(args.steps + args.warmup, 1) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": scan_config(),
            "cpu_baseline": {"value": value, "unit": "sims/hour", "cores": cores, "kind": "port",
                             "sample": sample, "per_rhs_ms": info["per_rhs_ms"],
                             "julia": julia_probe()},
            "e2e": {"value": value, "unit": "sims/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def scan_config():
    """The workload of both arms (the same dict, so the two lines name one config)."""
    return {"workload": WORKLOAD, "instances_per_gpu": 256, "saveN": SAVEN,
            "l2": "per-instance state 0.1-1 MB x 256 instances > 126 MB L2 (no flush needed)"}


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


# ----------------------------------------------------------------------------- surrogate
SG_METRIC = "surrogate scan queries/s (capillary family, 4-member MLP ensemble) at held-out log-spectrum error"
SG_WORKLOAD = ("surrogate: (energy 50-400 uJ, 0.5-5 bar, He/Ne/Ar/H2, radius 75-150 um, 8-30 fs, z 0-3 m) -> "
               "log10 spectrum on 512 log-spaced bins 150 nm - 4 um + 256-sample envelope; 6x512 SiLU MLP, "
               "Fourier-feature input, 4 members, BF16 tensor-core training and inference, 10^6 queries per pass")


def run_surrogate(args, world, rank, local):
    """Data from the batched mixed-precision solver (args.sg_runs runs of 3 m, 201 saves),
    training of the ensemble, error on held-out runs against the solver and against the
    method without the network (the nearest training point), and the throughput of 10^6
    queries against the plain FP64 solver's time per query."""
    import torch
    from luna_b200 import surrogate as S
    torch.cuda.set_device(local)
    log = (lambda m: print(m, file=sys.stderr, flush=True)) if rank == 0 else None
    params = S.draw(args.sg_runs, seed=7 + rank)
    t0 = time.perf_counter()
    xr, T, runs, status, dev_s = S.generate(params, rtol=args.mixed_rtol, chunk=512, log=log)
    gen_wall = time.perf_counter() - t0
    ok_runs = sorted(set(runs.tolist()))
    nheld = max(1, len(ok_runs) // 10)
    held = set(ok_runs[-nheld:])
    tr = np.array([r not in held for r in runs])
    std = S.Standardise(xr[tr])
    x = torch.tensor(std(xr), dtype=torch.float32, device="cuda")
    trm = torch.from_numpy(tr).cuda()
    xt, Tt = x[trm].contiguous(), T[trm].contiguous()
    model = S.Ensemble(members=4, seed=11, batch=4096)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = S.train(model, xt, Tt, epochs=args.sg_epochs, lr=(args.sg_lr, 1e-5), log=log)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    steps = args.sg_epochs * (xt.shape[0] // model.batch)
    # held-out error (every save of the held-out runs) and the method without the network
    xq, Tq = x[~trm].contiguous(), T[~trm].contiguous()
    mean, spread = S.predict(model, xq)
    e = S.spectral_error(mean, Tq)
    # the same over the bins within 3 decades of the run's input peak (the informative part)
    inf = Tq[:, :S.NSPEC] > -3.0
    e3 = (((mean[:, :S.NSPEC] - Tq[:, :S.NSPEC]) ** 2 * inf).sum(dim=1) / inf.sum(dim=1).clamp(min=1)).sqrt()
    e_env = ((mean[:, S.NSPEC:] - Tq[:, S.NSPEC:]) ** 2).mean(dim=1).sqrt()
    e_nn = S.spectral_error(S.nearest_neighbour(xt, Tt, xq), Tq)
    flag = spread > args.sg_spread
    # 1 % audit of the held-out points against the solver's values
    g = torch.Generator(device="cuda").manual_seed(3)
    audit = torch.randperm(xq.shape[0], device="cuda", generator=g)[: max(1, xq.shape[0] // 100)]
    # 10^6 queries: parameter draws x random z (standardised like the training inputs)
    nq = 1_000_064
    rng = np.random.default_rng(17)
    qp = S.draw(nq // 64, seed=23)
    zq = rng.uniform(0.0, 3.0, nq)
    pick = np.repeat(np.arange(len(qp)), 64)
    xq_raw = S.raw_features([qp[i]["energy"] for i in pick], [qp[i]["pressure"] for i in pick],
                            [qp[i]["radius"] for i in pick], [qp[i]["τfwhm"] for i in pick], zq,
                            [qp[i]["gas"] for i in pick])
    xh = torch.tensor(std(xq_raw), dtype=torch.float32).pin_memory()
    xd = xh.cuda()
    for _ in range(args.warmup):
        S.predict(model, xd, chunk=nq)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tms = []
    for _ in range(args.steps):
        e0.record(st)
        mq, sq = S.predict(model, xd, chunk=nq)
        e1.record(st)
        e1.synchronize()
        tms.append(e0.elapsed_time(e1))
    ms = statistics.median(tms)
    # end to end: host inputs in, host means and spreads out
    mh = torch.empty(nq, S.NOUT, pin_memory=True)
    sh = torch.empty(nq, pin_memory=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m2, s2 = S.predict(model, xh.cuda(non_blocking=True), chunk=nq)
    mh.copy_(m2)
    sh.copy_(s2)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    qflag = float((sq > args.sg_spread).float().mean())
    # the plain FP64 solver's time per query point: single-instance solves of held-out
    # parameter sets (one luna_b200_solve per run), over the 201 points a run saves
    t_plain = []
    for i in sorted(held)[:3]:
        pr = S.problem(params[i])
        plan = P.Plan.from_transform(pr.transform, _lib.PREC_FP64)
        b = P.Batch([plan], 201, np.linspace(0.0, 3.0, 201), max_dt=1.5)
        b.upload([pr.linop], [pr.Eω], [0.0], [1e-4], [3.0])
        t_plain.append(b.run() / 1e3)
        del b, plan
    plain_q_s = statistics.mean(t_plain) / 201
    batched_q_s = dev_s / max(1, len(ok_runs)) / 201
    flops = 4 * 2.0 * sum(k * n for k, n in zip(S.WIDTHS[:-1], S.WIDTHS[1:])) * nq
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            tpk, pk_kind = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        tpk, pk_kind = 1590.0, "fallback"
    ach = flops / (ms / 1e3) / 1e12
    value = nq / (ms / 1e3)
    if rank == 0:
        line = {"metric": SG_METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16 (FP32 accumulate)", "data": "synthetic (batched-solver runs)",
                "config": {"workload": SG_WORKLOAD, "runs": args.sg_runs, "completed_runs": len(ok_runs),
                           "held_out_runs": nheld, "samples_train": int(xt.shape[0]), "epochs": args.sg_epochs,
                           "adam_steps": steps, "queries_per_step": nq,
                           "l2": "activations of 10^6 queries (GBs) exceed the 126 MB L2"},
                "e2e": {"value": nq / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": int(xh.numel() * 4),
                        "d2h_bytes_per_step": int(mh.numel() * 4 + sh.numel() * 4)},
                "gpu_launches": (1 + 6 + 1) * args.steps,
                "roofline": {"bound": "tensor", "kernel": "sg_gemm (forward, 4 members)", "achieved": ach, "peak": tpk,
                             "unit": "TFLOP/s", "frac": ach / tpk, "traffic": None, "peak_kind": pk_kind},
                "accuracy": {"heldout_points": int(xq.shape[0]),
                             "log_spectrum_rms_decades": {"mean": float(e.mean()), "median": float(e.median()),
                                                          "p90": float(torch.quantile(e, 0.9))},
                             "log_spectrum_rms_top3_decades": {"mean": float(e3.mean()), "median": float(e3.median())},
                             "envelope_rms": float(e_env.mean()),
                             "nearest_training_point": {"mean": float(e_nn.mean()), "median": float(e_nn.median())},
                             "audit_1pct": {"points": int(audit.numel()), "mean": float(e[audit].mean())},
                             "bar": 5e-2, "met_mean": bool(float(e.mean()) <= 5e-2),
                             "spread_limit_decades": args.sg_spread,
                             "flagged_heldout": float(flag.float().mean()),
                             "error_unflagged": float(e[~flag].mean()) if bool((~flag).any()) else None},
                "speed": {"plain_fp64_s_per_query": plain_q_s, "batched_mixed_s_per_query": batched_q_s,
                          "surrogate_s_per_query": ms / 1e3 / nq, "vs_plain": plain_q_s / (ms / 1e3 / nq),
                          "vs_batched": batched_q_s / (ms / 1e3 / nq), "flagged_queries": qflag},
                "training": {"s": train_s, "final_loss": hist[-1], "data_gen_s_device": dev_s,
                             "data_gen_s_wall": gen_wall}}
        print(json.dumps(line), flush=True)


def run_surrogate_forward(args, world, rank, local):
    """The surrogate's inference kernels alone (a randomly initialised ensemble of the
    trained architecture; no data generation or training): one forward of the 4 members and
    the ensemble statistics on args.sg_queries queries per step."""
    import torch
    from luna_b200 import surrogate as S
    torch.cuda.set_device(local)
    model = S.Ensemble(members=4, seed=11, batch=4096)
    nq = args.sg_queries
    x = torch.randn(nq, S.NFEAT, device="cuda")
    for _ in range(args.warmup):
        S.predict(model, x, chunk=nq)
    st = torch.cuda.current_stream()
    tms = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        S.predict(model, x, chunk=nq)
        e1.record(st)
        e1.synchronize()
        tms.append(e0.elapsed_time(e1))
    model.check_timeout()
    ms = statistics.median(tms)
    flops = 4 * 2.0 * sum(k * n for k, n in zip(S.WIDTHS[:-1], S.WIDTHS[1:])) * nq
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            tpk, pk_kind = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        tpk, pk_kind = 1590.0, "fallback"
    ach = flops / (ms / 1e3) / 1e12
    if rank == 0:
        print(json.dumps({"metric": "surrogate forward queries/s (4 members, random weights)", "value": nq / (ms / 1e3),
                          "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "bf16 (FP32 accumulate)", "data": "synthetic",
                          "config": {"workload": "surrogate_forward: " + SG_WORKLOAD, "queries": nq},
                          "gpu_launches": 8 * args.steps,
                          "roofline": {"bound": "tensor", "kernel": "sg_gemm (forward, 4 members)", "achieved": ach,
                                       "peak": tpk, "unit": "TFLOP/s", "frac": ach / tpk, "traffic": None,
                                       "peak_kind": pk_kind}}), flush=True)


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
    ap.add_argument("--accuracy", choices=["auto", "on", "off"], default="auto",
                    help="FP64 pass over the same scan after the timed region and the error of "
                         "every mixed save against it (auto: on at one GPU)")
    ap.add_argument("--sg-queries", type=int, default=1_000_064, help="surrogate_forward: queries per step")
    ap.add_argument("--workload", default="scan256",
                    choices=["scan256", "radial", "modal", "surrogate", "surrogate_forward"],
                    help="scan256: the batched capillary scan (headline); radial: TransRadial RHS; "
                         "modal: TransModal RHS; surrogate: the learned surrogate's queries")
    ap.add_argument("--mixed-rtol", type=float, default=MIXED_RTOL,
                    help="relative tolerance of the mixed-precision integrations")
    ap.add_argument("--no-autotune", action="store_true",
                    help="shapes from the fixed work-estimate rule instead of the measured autotuner")
    ap.add_argument("--cluster-shape", type=int, choices=[0, 2, 3], default=0,
                    help="profiling aid with --no-autotune: every instance that may run distributed "
                         "runs on a cluster of 8 (2) or 16 (3) CTAs; 0: the work-estimate rule")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="precision of the timed batched scan (the other one is run once and "
                         "reported beside it when the accuracy pass is on)")
    ap.add_argument("--sg-runs", type=int, default=2560, help="surrogate: solver runs of training data")
    ap.add_argument("--sg-epochs", type=int, default=400, help="surrogate: training epochs")
    ap.add_argument("--sg-lr", type=float, default=2e-3, help="surrogate: peak learning rate")
    ap.add_argument("--sg-spread", type=float, default=0.1,
                    help="surrogate: ensemble spread (decades) above which a query goes to the solver")
    args = ap.parse_args()
    world, rank, local = dist_info()
    if args.workload == "radial":
        return run_radial(args, world, rank, local)
    if args.workload == "modal":
        return run_modal(args, world, rank, local)
    if args.workload == "surrogate_forward":
        return run_surrogate_forward(args, world, rank, local)
    if args.workload == "surrogate":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no surrogate (it always integrates)"}))
            return
        return run_surrogate(args, world, rank, local)
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
    prec = _lib.PREC_FP64 if args.precision == "fp64" else _lib.PREC_MIXED
    rtol = 1e-6 if prec == _lib.PREC_FP64 else args.mixed_rtol
    plans = [P.Plan.from_transform(p.transform, prec) for p in probs]
    # each instance saves on its own GridCondition range(0, zmax, 201) with max_dz = zmax/2
    batch = P.Batch(plans, SAVEN, np.linspace(0.0, 1.0, SAVEN), max_steps=args.max_rk_steps, rtol=rtol,
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

    try:
        fpk, fpk_err = fma_peaks(), None
    except Exception as e:  # report, do not hide
        fpk, fpk_err = None, str(e)[:200]
    prios = [scan.schedule_priority(p, q) for p, q in zip(inst, probs)]
    batch.upload(Lh, Yh, z0, dz0, zmax, zsaves, max_dts)
    tune = None
    if not args.no_autotune and not (args.no_dist or args.no_clusters):
        # shapes and processing order from measured ms per RK step of each grid class
        from luna_b200 import autotune
        table, tune_s = autotune.measure(probs, prec)
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        shapes, tprios, _ = autotune.schedule(inst, probs, table, nsm)
        batch.set_shapes(shapes)
        batch.set_priority(tprios)
        tune = {"ms_per_rk_step": table, "tune_s": round(tune_s, 1), "cluster_shapes": int((shapes == 2).sum()),
                "rule": "cluster when faster for the class and the predicted single-CTA time is above the mean SM load"}
    else:
        if args.cluster_shape:
            batch.set_shapes(np.full(len(probs), args.cluster_shape, dtype=int))
        batch.set_priority(prios)
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
    alg_bytes = sum(s.steps * step_bytes(len(p.Eω), prec == _lib.PREC_MIXED) for s, p in zip(stats, probs))
    raman_of = [any(r.kind == "raman_field" for r in p.transform.resp) for p in probs]
    alg_flops = sum(s.steps * step_flops(p.grid.No, p.grid.N, rm) for s, p, rm in zip(stats, probs, raman_of))
    hbm, peak_kind = peaks()
    achieved = alg_bytes / (ms / 1e3) / 1e9
    traffic = None
    # DRAM bytes per RK step from an ncu capture of the same solver (profiles/)
    tf = os.path.join(ROOT, "profiles", "solve_kernel_scan_traffic.json" if prec == _lib.PREC_MIXED
                      else "solve_kernel_dist_fp64_traffic.json")
    if os.path.exists(tf):
        with open(tf) as f:
            tj = json.load(f)
        traffic = tj.get("dram_bytes_per_rk_step", 0) * steps_all
    timeline = None
    try:
        be, _ = batch.timeline()
        timeline = {"long_pole_s": float(np.max(be[:, 1] - be[:, 0])),
                    "p90_end_s": float(np.percentile(be[:, 1], 90)),
                    "busy_cta_s": float(np.sum(be[:, 1] - be[:, 0]))}
    except Exception as e:
        timeline = {"error": str(e)[:200]}
    del batch
    del plans
    # ------------------------------------------------ accuracy against the plain FP64 path
    acc, fp64b, plain, other = None, None, None, None
    if args.accuracy == "on" or (args.accuracy == "auto" and world == 1):
        from luna_b200 import accuracy as A
        t_acc = time.perf_counter()

        def scan_once(pr, flags=0, rt=1e-6):
            pl = [P.Plan.from_transform(p.transform, pr) for p in probs]
            bb = P.Batch(pl, SAVEN, np.linspace(0.0, 1.0, SAVEN), max_steps=args.max_rk_steps, rtol=rt, flags=flags)
            bb.upload(Lh, Yh, z0, dz0, zmax, zsaves, max_dts)
            bb.set_priority(prios)
            ms_ = bb.run()
            S_ = [np.zeros((SAVEN, len(p.Eω)), dtype=np.complex128) for p in probs]
            _, _, st_ = bb.download(S_, None)
            be_, _ = bb.timeline()
            return ms_, S_, st_, be_[:, 1] - be_[:, 0]

        def compare(S_, st_, Sref, stref):
            per = []
            for i, p in enumerate(probs):
                if st_[i].status != 0 or stref[i].status != 0:
                    per.append(None)
                    continue
                k = min(st_[i].nsaved, stref[i].nsaved)
                per.append(A.compare(S_[i][:k], Sref[i][:k], p.grid.ω))
            out = A.summary(per)
            out["status_agree"] = int(sum(1 for x, y in zip(st_, stref) if x.status == y.status))
            return out

        # the plain path's arithmetic: every instance on one CTA with the FP64 solver of
        # luna_b200_solve (no clusters)
        ms64, S64, st64, dur64 = scan_once(_lib.PREC_FP64, flags=_lib.SOLVE_NO_DIST | _lib.SOLVE_NO_CLUSTERS)
        ok64 = sum(1 for x in st64 if x.status == 0)
        acc = compare(Sh, stats, S64, st64)
        acc.update({"reference": "the same scan integrated by the plain FP64 path's solver (one CTA per "
                                 "instance, the arithmetic of luna_b200_solve), every save of every completed instance",
                    "bar": 1e-3, "met": bool(acc.get("spectral_max", 1.0) <= 1e-3),
                    "steps_timed": int(sum(x.steps for x in stats)),
                    "steps_reference": int(sum(x.steps for x in st64))})
        if prec == _lib.PREC_FP64:
            acc["note"] = ("both are FP64 with different summation orders: an instance above the bar is one whose "
                           "FP64 result is not determined beyond rounding (it diverges at this level under any "
                           "rounding-level change, e.g. a 1-ulp change of its first step)")
        fp64b = {"value": 3600.0 * ok64 / (ms64 / 1e3), "unit": "sims/hour", "ms": ms64, "completed": ok64,
                 "long_pole_s": float(np.max(dur64)),
                 "method": "the whole scan in plain FP64 as one batch on single CTAs, device time"}
        # the other precision, once
        oprec = _lib.PREC_MIXED if prec == _lib.PREC_FP64 else _lib.PREC_FP64
        mso, So, sto, _ = scan_once(oprec, rt=args.mixed_rtol if oprec == _lib.PREC_MIXED else 1e-6)
        oko = sum(1 for x in sto if x.status == 0)
        other = {"precision": "mixed" if oprec == _lib.PREC_MIXED else "fp64",
                 "value": 3600.0 * oko / (mso / 1e3), "unit": "sims/hour", "ms": mso,
                 "accuracy": compare(So, sto, S64, st64)}
        del So, S64
        if not args.no_cpu_baseline and args.instances == 256:
            try:
                v_sub, v_scan, rows = plain_fp64_measured(inst, probs, dur64, [x.status for x in st64])
                plain = {"value": v_scan, "unit": "sims/hour", "subset_value": v_sub,
                         "method": ("plain FP64 drop-in measured: one single-instance FP64 solve after another "
                                    f"(device time; clusters of 16 CTAs for No = 32768, of 8 for No = 16384) for {len(rows)} instances, "
                                    "8 quantiles of the single-CTA FP64 batch time in each of the two strata; value = "
                                    "the scan's sims/hour with each stratum's per-instance batch times scaled by its "
                                    "subset's measured/batch ratio, subset_value = the subset's own"),
                         "subset": rows, "speedup_of_value": value / v_scan}
            except Exception as e:  # report, do not hide
                plain = {"value": None, "error": str(e)[:200]}
        acc["seconds"] = round(time.perf_counter() - t_acc, 1)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "sims/hour", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if prec == _lib.PREC_FP64 else "f32+f64",
                "data": "synthetic (seeded scan draw, no noise)",
                "config": scan_config(), "implementation": IMPL[args.precision],
                "rtol": rtol,
                "instances_this_rank": n, "failed_instances": failed,
                "e2e": {"value": e2e_value, "unit": "sims/hour", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e * 1e3},
                "gpu_launches": args.steps * kinfo[0],
                "scheduling": {"kernels_per_step": kinfo[0], "cluster_instances": kinfo[1],
                               "clusters": kinfo[2], "autotune": tune},
                "rk_steps_per_scan": steps_all, "rhs_evals_per_s": nrhs_all / (ms / 1e3),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": traffic,
                             "peak_kind": peak_kind,
                             "note": "algorithmic bytes = RK stage vectors per step (y/yn FP64, k FP32) x steps; kernel is latency/SMEM bound"},
                "clocks": clocks, "setup_s": round(setup_s, 1), "timeline": timeline}
        if fpk is None:
            line["roofline_compute"] = {"error": fpk_err}
        else:
            ach_tf = alg_flops / (ms / 1e3) / 1e12
            pk = fpk["fp64"] if prec == _lib.PREC_FP64 else fpk["fp32"]
            line["roofline_compute"] = {
                "bound": "fp64" if prec == _lib.PREC_FP64 else "fp32", "achieved": ach_tf, "peak": pk,
                "unit": "TFLOP/s", "frac": ach_tf / pk, "peak_fp32": fpk["fp32"], "peak_fp64": fpk["fp64"],
                "peak_kind": "measured (FMA microkernel, this run)",
                "flops_per_scan": alg_flops,
                "note": "algorithmic flops of every RK step (transforms 2.5 N log2 N, pointwise responses, stage combines) over the step time"}
            if traffic:
                line["roofline"]["traffic_over_algorithmic"] = traffic / alg_bytes
        if acc is not None:
            line["accuracy"] = acc
            line["fp64_single_cta_batched"] = fp64b
            line["fp64_single_cta_batched"]["speedup_of_value"] = value / fp64b["value"]
            line["other_precision"] = other
        if plain is not None:
            line["plain_fp64"] = plain
        if not args.no_cpu_baseline and world == 1:
            try:
                v1, info = cpu_estimate(workers=1)
                line["cpu_baseline"] = {"value": v1, "unit": "sims/hour", "cores": 1, "kind": "port",
                                        "sample": (f"{info['impl']} restatement of the reference algorithm, "
                                                   f"{info['rk_steps_each']} RK steps of one instance per grid class "
                                                   f"({info['classes']} classes, {info['sample_wall_s']} s) on one core, "
                                                   "time per RHS x each instance's RHS count from full solves of "
                                                   "the same restatement"),
                                        "per_rhs_ms": info["per_rhs_ms"], "julia": julia_probe()}
            except Exception as e:  # report, do not hide
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
