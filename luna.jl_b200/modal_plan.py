"""Device plan and solve of the modal transform (``TransModal``, full=false) behind the C ABI.

Fields cross the boundary as column-major Nw x nmodes complex arrays (Julia's
``Matrix{ComplexF64}``): element (ω, mode) at mode*Nw + ω. The Python side holds
(Nw, nmodes) arrays and passes their transposes.
"""
import numpy as np

from . import _lib
from .modal import cubature_levels
from .plan import SolveResult, _STATUS_MSG, make_opts, resp_descs
from .radial_plan import _colmajor


class ModalPlan:
    """Owns one ``luna_modal_plan``: the point grid and responses, the cubature rule with the
    mode fields at its nodes, and the output factor."""

    def __init__(self, gd, rds, md, keep, precision, Nw, nmodes):
        lib = _lib.load()
        self._keep = keep
        self.precision = precision
        self.Nw, self.nmodes = Nw, nmodes
        self.nevals = 0
        arr = (_lib.RespDesc * max(1, len(rds)))(*rds)
        h = _lib.c_void_p()
        _lib.check(lib.luna_b200_modal_plan_create(gd, arr, len(rds), md, precision,
                                                   _lib.ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().luna_b200_modal_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    @classmethod
    def from_transform(cls, t, precision=_lib.PREC_FP64):
        """Descriptors of a ``TransModal`` (NonlinearRHS.jl:203-216, 284-302)."""
        if t.full:
            raise NotImplementedError("the full 2-D modal integral (hcubature) is not available on "
                                      "the device; use full=False")
        g, ts = t.grid, t.ts
        keep = []
        Nw, No, N = len(g.ω), g.No, g.N
        if g.kind == "real":
            Nwo = len(g.ωo)
            pad = (Nwo - 1) / (Nw - 1)
            crop = (Nw - 1) / (Nwo - 1)
        else:  # copy_scale_both! (NonlinearRHS.jl:16-53)
            pad = No / Nw
            crop = Nw / No
        wwin = np.ascontiguousarray(g.ωwin, dtype=np.float64)
        towin = np.ascontiguousarray(g.towin, dtype=np.float64)
        twin = np.ascontiguousarray(g.twin, dtype=np.float64)
        keep += [wwin, towin, twin]
        gd = _lib.GridDesc()
        gd.kind, gd.N, gd.Nw, gd.No = (0 if g.kind == "real" else 1), N, Nw, No
        gd.outfac = _lib.dptr(None)
        gd.wwin, gd.towin, gd.twin = _lib.dptr(wwin), _lib.dptr(towin), _lib.dptr(twin)
        gd.in_scale = pad / No
        rds = resp_descs(t.resp, t.density, keep)
        ems, wts, wlow = t.tables()
        ems = np.ascontiguousarray(ems, dtype=np.float64)
        wts = np.ascontiguousarray(wts, dtype=np.float64)
        of = _colmajor(np.repeat((crop * t.output_factor())[:, None], ts.nmodes, axis=1))
        keep += [ems, wts, of]
        md = _lib.ModalDesc()
        md.nmodes, md.npol, md.nlevels = ts.nmodes, ts.npol, cubature_levels(t.mfcn)
        md.ems, md.wts = _lib.dptr(ems), _lib.dptr(wts)
        md.wlow, md.rtol, md.atol = wlow, t.rtol, t.atol
        md.outfac = _lib.dptr(of.view(np.float64))
        return cls(gd, rds, md, keep, precision, Nw, ts.nmodes)

    def rhs(self, nl, Eω, z=0.0):
        """nl[:, :] = T(Eω) on the GPU; (Nw, nmodes) complex128 host arrays. The number of
        integrand evaluations of the cubature is left in ``self.nevals``."""
        Ec = _colmajor(Eω)
        out = np.zeros_like(Ec)
        nev = _lib.c_int(0)
        _lib.check(_lib.load().luna_b200_modal_rhs(self._h, _lib.dptr(out.view(np.float64)),
                                                   _lib.dptr(Ec.view(np.float64)), float(z),
                                                   _lib.ctypes.byref(nev)))
        self.nevals = nev.value
        nl[...] = out.T
        return nl

    def solve(self, linop, Eω, z0, dz0, zmax, saveN=201, steplog_cap=0, replay=None,
              raise_on_status=True, **opt):
        """RK45.solve_precon with Luna.run's stepfun and saves (RK45.jl:19-25,
        Luna.jl:358-391); saves come back as (nsaved, Nw, nmodes)."""
        zs = np.linspace(z0, zmax, saveN)
        if replay is not None:
            replay = np.ascontiguousarray(replay, dtype=np.float64).ravel()
        o = make_opts(saveN, zs, steplog_cap=steplog_cap, replay=replay, **opt)
        L = _colmajor(linop)
        y = _colmajor(Eω)
        saves = np.zeros((saveN, self.nmodes, self.Nw), dtype=np.complex128)
        log = np.zeros((max(steplog_cap, 1), 4))
        st = _lib.SolveStats()
        rc = _lib.load().luna_b200_modal_solve(
            self._h, _lib.dptr(L.view(np.float64)), _lib.dptr(y.view(np.float64)), float(z0),
            float(dz0), float(zmax), _lib.ctypes.byref(o), _lib.dptr(saves.view(np.float64)),
            _lib.dptr(log) if steplog_cap else _lib.dptr(None), _lib.ctypes.byref(st))
        if rc not in (_lib.LUNA_OK, _lib.LUNA_FIELD_ABOVE_EMAX, _lib.LUNA_REPEAT_LIMIT,
                      _lib.LUNA_STEP_BUDGET):
            _lib.check(rc)
        if raise_on_status and st.status != 0:
            raise _lib.LunaError(st.status, _STATUS_MSG.get(st.status, "solver error"))
        n = st.nsaved
        sv = np.ascontiguousarray(saves[:n].transpose(0, 2, 1))
        steplog = log[: min(st.steps, steplog_cap)] if steplog_cap else None
        return SolveResult(zs[:n], sv, np.ascontiguousarray(y.T), st, steplog)


def run(Eω, grid, linop, transform, saveN=201, precision=_lib.PREC_FP64, **kw):
    """Luna.run (Luna.jl:358-391) on the GPU for a modal transform (max_dz = zmax/2)."""
    kw.setdefault("max_dt", grid.zmax / 2)
    dz0 = kw.pop("dz0", 1e-4)
    plan = transform.plan() if precision == _lib.PREC_FP64 else \
        ModalPlan.from_transform(transform, precision)
    return plan.solve(linop, Eω, 0.0, dz0, grid.zmax, saveN=saveN, **kw)
