"""Parameter scans, mirroring Luna.jl's Scans module (Scans.jl) for the device integrator.

``Scan``, ``addvariable``, ``makefilename``, ``chunks``, ``getvalue`` and ``runscan`` keep the
reference's names, point order (the first variable varies fastest, Iterators.product) and
execution modes ``LocalExec``, ``RangeExec`` and ``BatchExec`` with their command-line forms
(``-l``, ``-r a:b``, ``-b n,i``; Scans.jl:199-241). ``runscan(f, scan)`` calls
``f(scanidx, *values)`` for the selected points as the reference does (Scans.jl:275-353).

``runscan_device(f, scan)`` is the replacement for the common case where each point runs
``prop_capillary``: ``f`` returns the set-up of the point (a ``Problem`` from
``interface.prop_capillary_args``) instead of running it, and all selected points are then
integrated together by one batch on the GPU (``luna_b200_batch_*``). Under torchrun each
rank takes ``BatchExec(world, rank + 1)``: the points are independent, no collective is needed.

Not mirrored: the file-based ``QueueExec`` and the cluster submitters (``SlurmExec``,
``CondorExec``, ``SSHExec``), which schedule processes rather than compute, and the HDF5
scan outputs (``@scansave``, ``ScanHDF5Output``), which need HDF5.
"""
import itertools
import logging
import math

import numpy as np

log = logging.getLogger("luna_b200.scans")


class LocalExec:
    """Run every point of the scan in this process (Scans.jl:20-24)."""


class RangeExec:
    """Run the points ``start:stop`` (1-based, inclusive, as a Julia UnitRange;
    Scans.jl:26-34)."""

    def __init__(self, start, stop):
        self.r = range(int(start), int(stop) + 1)


class BatchExec:
    """Split the scan into ``Nbatches`` chunks (``chunks``) and run chunk ``batch`` (1-based;
    Scans.jl:36-45)."""

    def __init__(self, Nbatches, batch):
        if not 1 <= batch <= Nbatches:
            raise ValueError("batch must be between 1 and Nbatches")
        self.Nbatches, self.batch = int(Nbatches), int(batch)


def makeexec(args):
    """Execution mode from command-line arguments (Scans.jl:199-241): none -> LocalExec,
    ``-l/--local``, ``-r/--range a:b``, ``-b/--batch n,i``."""
    args = list(args)
    if not args:
        return LocalExec()
    opts = {}
    i = 0
    while i < len(args):
        a = args[i]
        if a in ("-l", "--local"):
            opts["local"] = True
        elif a in ("-q", "--queue", "-p", "--procs"):
            raise NotImplementedError("the file-based queue execution mode is not available")
        elif a in ("-r", "--range", "-b", "--batch"):
            if i + 1 >= len(args):
                raise ValueError(f"{a} needs a value")
            opts[a.lstrip("-")[0]] = args[i + 1]
            i += 1
        else:
            raise ValueError(f"unknown argument {a!r}")
        i += 1
    if opts.get("local"):
        return LocalExec()
    if "r" in opts:
        a, b = opts["r"].split(":")
        return RangeExec(int(a), int(b))
    if "b" in opts:
        n, k = opts["b"].split(",")
        return BatchExec(int(n), int(k))
    raise ValueError("Command-line arguments do not define a valid execution mode.")


class Scan:
    """``Scan(name; kwargs...)`` / ``Scan(name, ex; kwargs...)`` (Scans.jl:121-160): named
    scan variables in the order given. Command-line ``args``, when given and not empty,
    override ``exec`` as the reference's ARGS do."""

    def __init__(self, name, exec=None, args=None, **variables):
        self.name = name
        self.exec = makeexec(args) if args else (exec if exec is not None else LocalExec())
        self.variables = []
        self.arrays = []
        for var, arr in variables.items():
            addvariable(self, var, arr)

    def __len__(self):
        return 0 if not self.arrays else int(np.prod([len(a) for a in self.arrays]))

    def size(self):
        return (0,) if not self.arrays else tuple(len(a) for a in self.arrays)


def addvariable(scan, variable=None, array=None, **kwargs):
    """``addvariable!(scan, variable, array)`` / ``addvariable!(scan; kwargs...)``
    (Scans.jl:162-179)."""
    if variable is not None:
        scan.variables.append(variable)
        scan.arrays.append(list(array))
    for var, arr in kwargs.items():
        scan.variables.append(var)
        scan.arrays.append(list(arr))


def makefilename(scan, scanidx):
    """Output file name of a scan point (Scans.jl:181-197)."""
    name = scan.name if isinstance(scan, Scan) else scan
    return "%s_%05d.h5" % (name, scanidx)


def chunks(a, n):
    """Split ``a`` into ``n`` chunks, dealing the entries out in turn (Scans.jl:308-332)."""
    out = [[] for _ in range(n)]
    for done, x in enumerate(a):
        out[done % n].append(x)
    return out


def combos(scan):
    """All points in linear order: the first variable varies fastest (Iterators.product)."""
    if not scan.arrays:
        return []
    return [tuple(reversed(c)) for c in itertools.product(*reversed(scan.arrays))]


def getvalue(scan, variable, scanidx):
    """Value of ``variable`` at the 1-based ``scanidx`` (Scans.jl:251-255)."""
    return combos(scan)[scanidx - 1][scan.variables.index(variable)]


def selection(scan):
    """(scanidx, values) of the points this process runs, in order, with the reference's
    numbering: LocalExec enumerates all points, RangeExec enumerates its sub-range from 1
    (Scans.jl:291-306), BatchExec keeps the linear indices of its chunk (Scans.jl:334-352)."""
    cs = combos(scan)
    ex = scan.exec
    if isinstance(ex, LocalExec):
        return [(i + 1, c) for i, c in enumerate(cs)]
    if isinstance(ex, RangeExec):
        sub = [cs[j - 1] for j in ex.r if 1 <= j <= len(cs)]
        return [(i + 1, c) for i, c in enumerate(sub)]
    if isinstance(ex, BatchExec):
        idx = chunks(list(range(1, len(cs) + 1)), ex.Nbatches)[ex.batch - 1]
        return [(i, cs[i - 1]) for i in idx]
    raise TypeError(f"unsupported execution mode {type(ex).__name__}")


def _logiter(scan, scanidx, values):
    msg = "Running scan: %s (%d points)\nIndex: %05d\nVariables:\n" % (scan.name, len(scan), scanidx)
    for var, v in zip(scan.variables, values):
        msg += "\t%s: %g\n" % (var, v)
    log.info(msg)


def runscan(f, scan):
    """``runscan(f, scan)`` (Scans.jl:257-353): ``f(scanidx, *values)`` for every selected
    point; an exception is logged as a warning and the scan goes on. Returns the outputs for
    LocalExec and RangeExec, nothing for BatchExec, as the reference does."""
    out = []
    for scanidx, values in selection(scan):
        _logiter(scan, scanidx, values)
        try:
            out.append(f(scanidx, *values))
        except Exception as e:  # the reference logs and continues
            log.warning("Error at scanidx %d:\n%r", scanidx, e)
    return None if isinstance(scan.exec, BatchExec) else out


def problem_priority(prob):
    """Estimated work of a point: per-RHS transform cost x fibre length, doubled with a
    Raman response (orders a batch longest first)."""
    No = prob.grid.No
    raman = any(getattr(r, "kind", "") in ("raman_field", "raman_env") for r in prob.transform.resp)
    return No * math.log2(No) * prob.grid.zmax * (2.0 if raman else 1.0)


def runscan_device(f, scan, precision=None, init_dz=1e-4, **opts):
    """Batched ``runscan`` for propagation scans: ``f(scanidx, *values)`` returns the
    ``Problem`` of each selected point (``interface.prop_capillary_args``); the points are
    then integrated together on the GPU as ``Luna.run`` would integrate each (saves on
    range(0, zmax, saveN), max_dz = zmax/2). Returns {scanidx: SolveResult}. A point whose
    set-up raises is logged and skipped; a point that ends with a non-zero status is logged
    and returned with that status."""
    from . import _lib
    from . import plan as P
    precision = _lib.PREC_MIXED if precision is None else precision
    probs, idx = [], []
    for scanidx, values in selection(scan):
        _logiter(scan, scanidx, values)
        try:
            probs.append(f(scanidx, *values))
            idx.append(scanidx)
        except Exception as e:
            log.warning("Error at scanidx %d:\n%r", scanidx, e)
    if not probs:
        return {}
    saveN = probs[0].saveN
    if any(p.saveN != saveN for p in probs):
        raise ValueError("every point of a device scan must save the same number of points")
    plans = [P.Plan.from_transform(p.transform, precision) for p in probs]
    batch = P.Batch(plans, saveN, np.linspace(0.0, 1.0, saveN), **opts)
    batch.upload([p.linop for p in probs], [p.Eω for p in probs], [0.0] * len(probs),
                 [init_dz] * len(probs), [p.grid.zmax for p in probs],
                 [np.linspace(0.0, p.grid.zmax, saveN) for p in probs],
                 [p.grid.zmax / 2 for p in probs])
    batch.set_priority([problem_priority(p) for p in probs])
    batch.run()
    res = batch.results()
    for p, r in zip(probs, res):  # each point saves on its own range(0, zmax, saveN)
        r.z = np.linspace(0.0, p.grid.zmax, saveN)[: r.nsaved]
    for scanidx, r in zip(idx, res):
        if r.status != 0:
            log.warning("Error at scanidx %d: solver status %d", scanidx, r.status)
    return dict(zip(idx, res))
