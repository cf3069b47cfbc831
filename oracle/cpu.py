"""ctypes binding of the FP64 C++ restatement (``uppe_cpu.cpp``; test infrastructure and the
timed CPU baseline only).

The C++ code reads the same C-ABI descriptors as the device library (built by
``luna_b200.plan.transform_descs``); the tests check it against the numpy restatement
(``uppe.py``), which reads the transform object itself.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "uppe_cpu.cpp")
LIB = os.path.join(HERE, "libuppe_cpu.so")
HEADER = os.path.join(HERE, "..", "include", "luna_b200.h")
# x86-64-v2 (no AVX) so the library also runs on other hosts; no contraction into FMA, so the
# rounding follows the numpy restatement's operation order
FLAGS = ["-O3", "-march=x86-64-v2", "-ffp-contract=off", "-fcx-limited-range", "-std=c++17",
         "-fPIC", "-shared"]

_lib = None


def build(force=False):
    """Compile ``libuppe_cpu.so`` beside its source (g++)."""
    if not force and os.path.exists(LIB) and all(os.path.getmtime(f) <= os.path.getmtime(LIB)
                                                 for f in (SRC, HEADER)):
        return LIB
    subprocess.run([os.environ.get("CXX", "g++")] + FLAGS + ["-o", LIB, SRC], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()  # compiles only when the source or the descriptor header is newer
    from luna_b200 import _lib as L
    lib = ctypes.CDLL(LIB)
    P = ctypes.POINTER
    lib.uo_plan_create.argtypes = [P(L.GridDesc), P(L.RespDesc), ctypes.c_int, P(ctypes.c_void_p)]
    lib.uo_plan_destroy.argtypes = [ctypes.c_void_p]
    lib.uo_plan_destroy.restype = None
    lib.uo_rhs.argtypes = [ctypes.c_void_p, L.PD, L.PD]
    lib.uo_solve.argtypes = [ctypes.c_void_p, L.PD, L.PD, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, P(L.SolveOpts), L.PD, L.PD, P(L.SolveStats)]
    lib.uo_last_error.argtypes = [ctypes.c_void_p]
    lib.uo_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


class CpuPlan:
    """A mode-averaged transform on the host in C++: field-resolved grids (Kerr, PPT/ADK
    plasma, Raman with THG) and envelope grids (Kerr_env, RamanPolarEnv)."""

    def __init__(self, transform):
        from luna_b200 import _lib as L
        from luna_b200.plan import transform_descs
        lib = load()
        gd, rds, keep, Nw, zdep, _, _ = transform_descs(transform)
        if zdep:
            raise NotImplementedError("z-dependent transforms are not restated in C++")
        self._keep = (gd, rds, keep)
        self.Nw = Nw
        arr = (L.RespDesc * max(1, len(rds)))(*rds)
        h = ctypes.c_void_p()
        rc = lib.uo_plan_create(gd, arr, len(rds), ctypes.byref(h))
        if rc != 0:
            raise NotImplementedError(f"CPU restatement: plan creation returned {rc}")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            load().uo_plan_destroy(h)
            self._h = None

    def rhs(self, Eω):
        from luna_b200 import _lib as L
        Ew = np.ascontiguousarray(Eω, dtype=np.complex128)
        nl = np.zeros_like(Ew)
        rc = load().uo_rhs(self._h, L.dptr(nl.view(np.float64)), L.dptr(Ew.view(np.float64)))
        if rc != 0:
            raise L.LunaError(rc, load().uo_last_error(self._h).decode())
        return nl

    def solve(self, linop, Eω, z0, dz0, zmax, saveN=201, rtol=1e-6, atol=1e-10, safety=0.9,
              max_dt=None, min_dt=0.0, repeat_limit=10, max_steps=0, zsave=None, steplog_cap=0,
              replay=None):
        """Luna.run with RK45.solve_precon; saves at saveN points on [z0, zmax] or at
        ``zsave``; returns (saves[nsaved, Nw], y, stats), or with ``steplog_cap`` > 0
        (saves, y, stats, steplog[steps, 4]) with rows (z, dz, err, accepted) as the device
        solver logs them. ``replay`` (flat (dz, accepted) pairs) makes the integrator follow
        a recorded step sequence."""
        from luna_b200 import _lib as L
        from luna_b200.plan import make_opts
        zs = np.linspace(z0, zmax, saveN) if zsave is None else np.asarray(zsave, dtype=np.float64)
        saveN = len(zs)
        rp = None if replay is None else np.ascontiguousarray(replay, dtype=np.float64)
        o = make_opts(saveN, zs, rtol=rtol, atol=atol, safety=safety,
                      max_dt=(zmax / 2 if max_dt is None else max_dt), min_dt=min_dt,
                      repeat_limit=repeat_limit, max_steps=max_steps, steplog_cap=steplog_cap,
                      replay=rp)
        Lc = np.ascontiguousarray(linop, dtype=np.complex128)
        y = np.array(Eω, dtype=np.complex128, copy=True)
        saves = np.zeros((max(saveN, 1), self.Nw), dtype=np.complex128)
        log = np.zeros((max(steplog_cap, 1), 4))
        st = L.SolveStats()
        load().uo_solve(self._h, L.dptr(Lc.view(np.float64)), L.dptr(y.view(np.float64)), float(z0),
                        float(dz0), float(zmax), ctypes.byref(o), L.dptr(saves.view(np.float64)),
                        L.dptr(log) if steplog_cap else L.dptr(None), ctypes.byref(st))
        if steplog_cap:
            return saves[: st.nsaved], y, st, log[: min(st.steps, steplog_cap)]
        return saves[: st.nsaved], y, st
