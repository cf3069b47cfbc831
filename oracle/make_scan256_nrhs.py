"""Full-length FP64 solves of the 256-instance capillary scan with the C++ restatement of the
reference algorithm (test infrastructure and the CPU baseline's counts; nothing here runs on
a GPU).

Every instance of the seeded scan (``luna_b200.scan.draw_instances``, seed 20261203) is
integrated to its fibre length with Luna.run's settings (dz0 = 1e-4, max_dz = zmax/2, 201
GridCondition saves, rtol 1e-6, atol 1e-10) by ``oracle/uppe_cpu.cpp``, one instance per
process on all host cores. Writes

  oracle/scan256_nrhs.json     per instance: RK steps, accepted/rejected steps, RHS
                               evaluations, status, final z and the single-core wall time
                               of the solve (the CPU baseline scales per-RHS timings by
                               these counts);
  tests/golden/scan_subset.npz for a stratified subset (the longest instance, H2 on the
                               32768-point grid; instances that the device distributes
                               over CTA clusters; short, Raman and failing instances): the
                               counts, the final state (complex128), |Eω|^2 at four save
                               points (float32) and the step sequence (float32 step sizes,
                               negative for rejected steps), the references of the
                               full-length scan-subset GPU test.

    python oracle/make_scan256_nrhs.py [--workers N] [--subset-only]
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

SUBSET = (93, 90, 73, 13, 97, 253, 0)   # see the module docstring
SUBSET_SAVES = (50, 100, 150, 200)
SAVEN = 201


def solve_one(i):
    import luna_b200_loader
    luna_b200_loader.load()
    from luna_b200 import scan
    from oracle import cpu
    p = scan.build_problem(scan.draw_instances(256)[i], saveN=SAVEN)
    cp = cpu.CpuPlan(p.transform)
    zmax = p.grid.zmax
    t0 = time.perf_counter()
    if i in SUBSET:
        saves, y, st, log = cp.solve(p.linop, p.Eω, 0.0, 1e-4, zmax, saveN=SAVEN, max_dt=zmax / 2,
                                     steplog_cap=200000)
    else:
        saves, y, st = cp.solve(p.linop, p.Eω, 0.0, 1e-4, zmax, saveN=SAVEN, max_dt=zmax / 2)
    wall = time.perf_counter() - t0
    row = dict(i=i, steps=int(st.steps), accepted=int(st.accepted), rejected=int(st.rejected),
               nrhs=int(st.nrhs), status=int(st.status), z=float(st.z), nsaved=int(st.nsaved),
               wall_s=wall, Nw=len(p.Eω), No=int(p.grid.No))
    if i in SUBSET:
        idx = [k for k in SUBSET_SAVES if k < st.nsaved]
        row["final"] = y
        row["spec"] = np.abs(saves[idx]) ** 2 if idx else np.zeros((0, len(y)))
        row["save_idx"] = idx
        row["steps_seq"] = np.where(log[:, 3] != 0, log[:, 1], -log[:, 1]).astype(np.float32)
    return row


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--subset-only", action="store_true",
                    help="recompute only the subset fixture (tests/golden/scan_subset.npz)")
    args = ap.parse_args()
    from oracle import cpu
    cpu.build()
    import luna_b200_loader
    luna_b200_loader.load()
    from luna_b200 import scan
    n = 256
    # longest first, so the pool's tail is short (order from a cheap work estimate)
    inst = scan.draw_instances(n)
    order = sorted(range(n), key=lambda i: -scan.nonlinear_phase(inst[i]))
    if args.subset_only:
        order = [i for i in order if i in SUBSET]
    t0 = time.perf_counter()
    rows = {}
    with mp.get_context("spawn").Pool(args.workers) as pool:
        for r in pool.imap_unordered(solve_one, order):
            rows[r["i"]] = r
            print(f"{len(rows):3d}/{n} instance {r['i']:3d} steps {r['steps']:6d} status {r['status']} "
                  f"{r['wall_s']:7.1f} s", flush=True)
    wall = time.perf_counter() - t0
    if args.subset_only:
        write_subset(rows)
        return
    out = {"source": "FP64 C++ restatement of the reference algorithm (oracle/uppe_cpu.cpp), full "
                     "solves, seed 20261203, dz0 1e-4, max_dz zmax/2, 201 saves",
           "host": {"cores": args.workers, "wall_s": wall},
           **{k: [rows[i][k] for i in range(n)] for k in
              ("steps", "accepted", "rejected", "nrhs", "status", "z", "wall_s", "Nw", "No")}}
    with open(os.path.join(ROOT, "oracle", "scan256_nrhs.json"), "w") as f:
        json.dump(out, f)
    write_subset(rows)
    print("done", wall, "s; failed", sum(1 for s in out["status"] if s))


def write_subset(rows):
    sub = {"subset": np.array(SUBSET), "save_idx": np.array(SUBSET_SAVES)}
    for i in SUBSET:
        r = rows[i]
        for k in ("steps", "accepted", "rejected", "nrhs", "status", "nsaved"):
            sub[f"{k}_{i}"] = np.array(r[k])
        sub[f"z_{i}"] = np.array(r["z"])
        sub[f"final_{i}"] = r["final"].astype(np.complex128)
        sub[f"spec_{i}"] = r["spec"].astype(np.float32)
        sub[f"seq_{i}"] = r["steps_seq"]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "scan_subset.npz"), **sub)


if __name__ == "__main__":
    main()
