"""Device plan and solve of the radial transform (``TransRadial``) behind the C ABI.

Fields cross the boundary as column-major Nw x Nr complex arrays (Julia's
``Matrix{ComplexF64}``): element (ω, k) at k*Nw + ω. The Python side holds (Nw, Nr)
arrays and passes their transposes.
"""
import math

import numpy as np

from . import _lib
from .plan import SolveResult, _STATUS_MSG, make_opts, resp_descs


def _colmajor(a):
    """(Nw, Nr) complex -> a new C-contiguous (Nr, Nw) array, i.e. the column-major layout.
    Always a copy: a solve writes its final state into it, and for one column the
    transpose of a contiguous array is itself contiguous (a view of the caller's array)."""
    return np.array(np.asarray(a, dtype=np.complex128).T, order="C", copy=True)


class RadialPlan:
    """Owns one ``luna_radial_plan``: the column grid and responses, the QDHT matrices and
    the (ω, k) output factor."""

    def __init__(self, gd, rds, rd, keep, precision, Nw, Nr):
        lib = _lib.load()
        self._keep = keep
        self.precision = precision
        self.Nw, self.Nr = Nw, Nr
        arr = (_lib.RespDesc * max(1, len(rds)))(*rds)
        h = _lib.c_void_p()
        _lib.check(lib.luna_b200_radial_plan_create(gd, arr, len(rds), rd, precision,
                                                    _lib.ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().luna_b200_radial_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    @classmethod
    def from_transform(cls, t, precision=_lib.PREC_FP64):
        """Descriptors of a ``TransRadial`` (NonlinearRHS.jl:430-458, 466-474)."""
        g, q = t.grid, t.q
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
        zdep = getattr(t, "kind", "") == "radial_z"
        # a gas fill gradient scales the output by ρ(z) on the device: coefficients for ρ = 1
        rds = resp_descs(t.resp, 1.0 if zdep else t.density, keep,
                         rho_tau2=t.densityfun(0.0) if zdep else None)
        Mi = np.ascontiguousarray(q.Mi, dtype=np.float64)
        Mf = np.ascontiguousarray(q.Mf, dtype=np.float64)
        of = _colmajor(crop * t.output_factor())
        keep += [Mi, Mf, of]
        rd = _lib.RadialDesc()
        rd.Nr = q.N
        rd.Mi, rd.Mf = _lib.dptr(Mi), _lib.dptr(Mf)
        rd.outfac = _lib.dptr(of.view(np.float64))
        plan = cls(gd, rds, rd, keep, precision, Nw, q.N)
        if zdep:
            gdesc, kr2, mw = radial_gradient_desc(t, crop, plan._keep)
            plan._gdesc = gdesc
            _lib.check(_lib.load().luna_b200_radial_set_gradient(plan.handle, _lib.ctypes.byref(gdesc),
                                                                 _lib.dptr(kr2), _lib.dptr(mw)))
        return plan

    def linop(self, z):
        """The device's linop!(out, z) and output factor of a plan with a gas fill gradient,
        (Nw, Nr) complex each."""
        L = np.zeros((self.Nr, self.Nw), dtype=np.complex128)
        of = np.zeros_like(L)
        _lib.check(_lib.load().luna_b200_radial_linop(self._h, float(z), _lib.dptr(L.view(np.float64)),
                                                      _lib.dptr(of.view(np.float64))))
        return L.T, of.T

    def rhs(self, nl, Eω, z=0.0):
        """nl[:, :] = T(Eω) on the GPU; (Nw, Nr) complex128 host arrays."""
        Ec = _colmajor(Eω)
        out = np.zeros_like(Ec)
        _lib.check(_lib.load().luna_b200_radial_rhs(self._h, _lib.dptr(out.view(np.float64)),
                                                    _lib.dptr(Ec.view(np.float64)), float(z)))
        nl[...] = out.T
        return nl

    def solve(self, linop, Eω, z0, dz0, zmax, saveN=201, steplog_cap=0, replay=None,
              raise_on_status=True, **opt):
        if callable(linop):  # a gas fill gradient: L(z) is evaluated on the device
            linop = None
        """RK45.solve_precon with Luna.run's stepfun and saves (RK45.jl:19-25,
        Luna.jl:358-391); saves come back as (nsaved, Nw, Nr)."""
        zs = np.linspace(z0, zmax, saveN)
        if replay is not None:
            replay = np.ascontiguousarray(replay, dtype=np.float64).ravel()
        o = make_opts(saveN, zs, steplog_cap=steplog_cap, replay=replay, **opt)
        L = _colmajor(linop) if linop is not None else None
        y = _colmajor(Eω)
        saves = np.zeros((saveN, self.Nr, self.Nw), dtype=np.complex128)
        log = np.zeros((max(steplog_cap, 1), 4))
        st = _lib.SolveStats()
        rc = _lib.load().luna_b200_radial_solve(
            self._h, _lib.dptr(L.view(np.float64) if L is not None else None), _lib.dptr(y.view(np.float64)), float(z0),
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


def radial_gradient_desc(t, crop, keep):
    """luna_gradient_desc, kr2 and μ0 ω of a TransRadialZ for luna_b200_radial_set_gradient;
    the arrays are appended to ``keep``."""
    f, g = t.fill, t.grid
    grad = f.grad
    if len(grad.Z) > _lib.GRAD_MAXPTS:
        raise ValueError(f"at most {_lib.GRAD_MAXPTS} pressure nodes")
    ofs = np.ascontiguousarray(crop * (g.ωwin * (-1j * g.ω)) / 2, dtype=np.complex128)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (f.gam, f.wc, f.om, f.kr2, f.mw)]
    keep += arrs + [ofs]
    gam, wc, om, kr2, mw = arrs
    d = _lib.GradientDesc()
    d.npts, d.two_point = len(grad.Z), int(grad.two_point)
    for i in range(len(grad.Z)):
        d.Z[i], d.P[i], d.P2[i] = grad.Z[i], grad.P[i], grad.P2[i]
    d.dens_a, d.dens_b = grad.dens_a, grad.dens_b
    d.nta = 1
    d.gam, d.wc, d.om = _lib.dptr(gam), _lib.dptr(wc), _lib.dptr(om)
    d.ofs = _lib.dptr(ofs.view(np.float64))
    for j in range(4):
        d.fd_xc[j], d.fd_gam[j] = f.fd_xc[j], f.fd_gam[j]
    d.fd_h12 = f.fd_h12
    d.env_ref = int(f.env_ref)
    d.ref_xc, d.ref_gam = f.ref_xc, f.ref_gam
    return d, kr2, mw


def run(problem, precision=_lib.PREC_FP64, **kw):
    """Luna.run (Luna.jl:358-391) on the GPU for a ``RadialProblem``."""
    g = problem.grid
    kw.setdefault("max_dt", g.zmax / 2)
    dz0 = kw.pop("dz0", 1e-4)
    plan = problem.transform.plan() if precision == _lib.PREC_FP64 else \
        RadialPlan.from_transform(problem.transform, precision)
    return plan.solve(problem.linop, problem.Eω, 0.0, dz0, g.zmax, saveN=problem.saveN, **kw)
