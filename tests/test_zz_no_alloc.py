"""The allocation-free right-hand side entry point.

luna_b200_rhs_device_noalloc serves callers that cannot allocate device memory while they
run (an allocator-managed runtime, or a caching pool that owns the device memory): its
scratch is a fixed 1 MiB buffer in the library's static device memory. This file is
collected last so that a failure here leaves every other test already run.

The test calls the entry point through the C ABI, twice in a row on a fresh plan, in FP64
and in mixed precision, and compares each result with the allocating entry point
luna_b200_rhs_device on the same input (the two run the same device code, so they agree to
rounding) and with the FP64 oracle, within the tolerances the RHS parity tests use.
"""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import ctypes

import numpy as np
import pytest

from luna_b200 import _lib
from luna_b200 import plan as P
from luna_b200.interface import prop_capillary_args, prop_gnlse_args

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _problems():
    cap = prop_capillary_args(125e-6, 0.3, "He", 1.0, λ0=800e-9, τfwhm=10e-15, energy=120e-6,
                              λlims=(150e-9, 4e-6), trange=0.25e-12)
    gn = prop_gnlse_args(0.11, 0.15, [0.0, 0.0, -11.83e-27, 8.1e-41], λ0=835e-9, τfwhm=50e-15,
                         power=10e3, pulseshape="sech", λlims=(500e-9, 2400e-9), trange=12.5e-12)
    return {"capillary_ppt": cap, "gnlse_raman": gn}


# bars: the allocating entry point runs the same device code (rounding-level agreement);
# the oracle bars are those of the RHS parity tests (FP64 1e-11 with plasma, 1e-12 without;
# mixed precision 1e-5)
_BARS = {_lib.PREC_FP64: (1e-12, 1e-11), _lib.PREC_MIXED: (1e-5, 1e-5)}


@pytest.mark.parametrize("prec", [_lib.PREC_FP64, _lib.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", ["capillary_ppt", "gnlse_raman"])
def test_noalloc_rhs_matches_allocating_entry_on_two_calls(name, prec):
    """The allocation-free call comes first on a freshly created plan (nothing the
    allocating entry point set up is reused), twice in a row on different inputs; the
    reference values are computed afterwards."""
    torch = pytest.importorskip("torch")
    from oracle import uppe
    lib = _lib.load()
    prob = _problems()[name]
    plan = P.Plan.from_transform(prob.transform, prec)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(7)
    inputs = [prob.Eω * np.exp(1j * 0.2 * rng.standard_normal(len(prob.Eω))) for _ in range(2)]
    dEs = [torch.from_numpy(Ew.view(np.float64).copy()).cuda() for Ew in inputs]
    outs = [torch.full_like(d, float("nan")) for d in dEs]
    status = torch.full((2,), -1, dtype=torch.int32, device="cuda")
    for call in range(2):
        _lib.check(lib.luna_b200_rhs_device_noalloc(plan.handle, ctypes.c_void_p(outs[call].data_ptr()),
                                                    ctypes.c_void_p(dEs[call].data_ptr()), 0.0,
                                                    ctypes.c_void_p(stream.cuda_stream),
                                                    ctypes.c_void_p(status.data_ptr() + 4 * call)))
    torch.cuda.synchronize()
    assert status.cpu().tolist() == [_lib.LUNA_OK, _lib.LUNA_OK]
    same, orc = _BARS[prec]
    for call in range(2):
        ref = torch.zeros_like(dEs[call])
        _lib.check(lib.luna_b200_rhs_device(plan.handle, ctypes.c_void_p(ref.data_ptr()),
                                            ctypes.c_void_p(dEs[call].data_ptr()), 0.0,
                                            ctypes.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()
        a = outs[call].cpu().numpy().view(np.complex128)
        b = ref.cpu().numpy().view(np.complex128)
        assert np.all(np.isfinite(a))
        assert _rel(a, b) <= same, (call, _rel(a, b))
        o = uppe.trans_mode_avg(prob.transform, inputs[call], 0.0)
        assert _rel(a, o) <= orc, (call, _rel(a, o))


def test_noalloc_repeat_call_allocates_no_device_memory():
    """Once the library's module is loaded (the first call), further calls leave the
    device's free memory unchanged."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    prob = _problems()["capillary_ppt"]
    plan = P.Plan.from_transform(prob.transform, _lib.PREC_MIXED)
    dE = torch.from_numpy(prob.Eω.view(np.float64).copy()).cuda()
    out = torch.zeros_like(dE)
    call = lambda: _lib.check(lib.luna_b200_rhs_device_noalloc(
        plan.handle, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(dE.data_ptr()), 0.0, None, None))
    call()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_plans_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    # a 32768-point FP64 envelope grid with the Raman convolution needs 1.5 MiB of scratch
    prob = prop_gnlse_args(0.11, 0.15, [0.0, 0.0, -11.83e-27], λ0=835e-9, τfwhm=50e-15,
                           power=10e3, pulseshape="sech", λlims=(450e-9, 8000e-9), trange=26e-12)
    assert prob.grid.N == 32768
    plan = P.Plan.from_transform(prob.transform, _lib.PREC_FP64)
    dE = torch.zeros(2 * prob.grid.N, dtype=torch.float64, device="cuda")
    out = torch.zeros_like(dE)
    rc = lib.luna_b200_rhs_device_noalloc(plan.handle, ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_void_p(dE.data_ptr()), 0.0, None, None)
    assert rc == _lib.LUNA_ERR_UNSUPPORTED
    assert b"LUNA_NOALLOC_SCRATCH_BYTES" in lib.luna_b200_last_error()
