"""Scans (Scans.jl) mirror: point order, execution modes, chunking and the batched device scan.

CPU cases follow test/test_scans.jl ("Chunking", "Scanning" with -l / -r / -b, command-line
arguments overriding an explicit mode); the GPU case integrates a small scan in one batch and
compares it with single-instance solves of the same points.
"""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import numpy as np
import pytest

from luna_b200 import scans
from luna_b200.scans import (BatchExec, LocalExec, RangeExec, Scan, addvariable, chunks,
                             getvalue, makefilename, runscan)


def test_chunks_contain_every_entry_once():
    """test_scans.jl:7-24."""
    for L in range(5, 897, 11):
        x = list(range(1, L + 1))
        for n in range(1, 25):
            ch = chunks(x, n)
            assert sorted(v for c in ch for v in c) == x
    assert chunks(list(range(1, 11)), 3) == [[1, 4, 7, 10], [2, 5, 8], [3, 6, 9]]


@pytest.mark.parametrize("args,exec_type", [(["-l"], LocalExec), (["-r", "1:6"], RangeExec),
                                            (["-b", "2,1"], BatchExec)])
def test_scanning_modes_pass_the_right_values(args, exec_type):
    """test_scans.jl:27-46: under every mode the value handed to f is v[scanidx]."""
    v = list(range(1, 11))
    scan = Scan("scantest_cmdlineargs", args=args, var=v)
    assert isinstance(scan.exec, exec_type)
    seen = []

    def f(scanidx, vi):
        assert vi == v[scanidx - 1]
        seen.append(scanidx)
        return vi

    out = runscan(f, scan)
    if exec_type is LocalExec:
        assert seen == list(range(1, 11)) and out == v
    elif exec_type is RangeExec:
        assert seen == list(range(1, 7))
    else:
        assert seen == [1, 3, 5, 7, 9] and out is None


def test_command_line_args_override_explicit_mode():
    """test_scans.jl:49-62."""
    scan = Scan("scantest_cmdlineargs_overwrite", LocalExec(), args=["--range", "1:4"],
                var=list(range(1, 11)))
    assert isinstance(scan.exec, RangeExec)
    assert runscan(lambda i, v: v, scan) == [1, 2, 3, 4]


def test_point_order_first_variable_fastest():
    """Iterators.product order: (x1, y1), (x2, y1), ...; getvalue and size as Scans.jl."""
    scan = Scan("order", LocalExec())
    addvariable(scan, "x", [1, 2, 3])
    addvariable(scan, y=[10, 20])
    assert len(scan) == 6 and scan.size() == (3, 2)
    pts = runscan(lambda i, x, y: (i, x, y), scan)
    assert pts == [(1, 1, 10), (2, 2, 10), (3, 3, 10), (4, 1, 20), (5, 2, 20), (6, 3, 20)]
    assert getvalue(scan, "y", 4) == 20 and getvalue(scan, "x", 5) == 2
    assert makefilename(scan, 7) == "order_00007.h5"


def test_errors_are_logged_and_the_scan_goes_on():
    def f(i, v):
        if v == 3:
            raise RuntimeError("bad point")
        return v
    assert runscan(f, Scan("errs", var=[1, 2, 3, 4])) == [1, 2, 4]


def test_unavailable_modes_refused():
    with pytest.raises(NotImplementedError):
        Scan("q", args=["-q"], var=[1])
    with pytest.raises(ValueError):
        Scan("bad", args=["--nope"], var=[1])


@pytest.mark.gpu
def test_runscan_device_matches_single_solves():
    """A 2 x 2 energy x pressure scan integrated in one batch gives, point by point, the
    fields of single-instance solves (the batch integrates each point by the same code)."""
    from luna_b200 import _lib
    from luna_b200 import plan as P
    from luna_b200.interface import prop_capillary_args

    def setup(scanidx, energy, pressure):
        return prop_capillary_args(125e-6, 0.1, "He", pressure, λ0=800e-9, τfwhm=10e-15,
                                   energy=energy, λlims=(150e-9, 4e-6), trange=0.25e-12,
                                   saveN=11)

    scan = Scan("device", energy=[60e-6, 120e-6], pressure=[0.8, 1.6])
    res = scans.runscan_device(setup, scan, precision=_lib.PREC_FP64)
    assert sorted(res) == [1, 2, 3, 4]
    for scanidx, r in res.items():
        e, p = getvalue(scan, "energy", scanidx), getvalue(scan, "pressure", scanidx)
        ref = P.run(setup(scanidx, e, p))
        assert r.status == 0 and r.steps == ref.steps
        np.testing.assert_allclose(r.z, np.linspace(0, 0.1, 11)[: r.nsaved])
        for a, b in zip(r.Eω, ref.Eω):
            assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)
