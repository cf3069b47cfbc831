"""Device plans and solves behind the reference-facing Python API.

``Plan.from_transform`` turns a ``TransModeAvg`` description into the C-ABI descriptors
(``include/luna_b200.h``) and creates the device plan. ``solve_precon`` and ``Batch``
drive ``RK45.solve_precon`` / ``Luna.run`` on the device.
"""
import math

import numpy as np

from . import _lib
from . import physdata as pd
from .nonlinearrhs import nlscale


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def resp_descs(resp, rho, keep, rho_tau2=None):
    """C-ABI descriptors of the responses (Et_to_Pt! order) at density ``rho``; arrays the
    descriptors point to are appended to ``keep``. ``rho_tau2`` (default ``rho``) is the
    density of the Raman dephasing times at plan creation (a pressure gradient's plan has
    coefficients for rho = 1 and rebuilds the Raman spectrum at rho(z))."""
    rds = []
    for r in resp:
        d = _lib.RespDesc()
        if r.kind == "kerr_field":
            d.kind = _lib.RESP_KERR_FIELD
            d.coef = rho * pd.eps_0 * r.γ3
        elif r.kind == "kerr_field_nothg":
            d.kind = _lib.RESP_KERR_FIELD_NOTHG
            d.coef = rho * pd.eps_0 * r.γ3
        elif r.kind == "kerr_env":
            d.kind = _lib.RESP_KERR_ENV
            d.coef = rho * pd.eps_0 * r.γ3
        elif r.kind == "kerr_env_thg":
            d.kind = _lib.RESP_KERR_ENV_THG
            d.coef = rho * pd.eps_0 * r.γ3
            C = np.ascontiguousarray(r.C, dtype=np.complex128)
            keep.append(C)
            d.cthg = _lib.dptr(C.view(np.float64))
        elif r.kind == "plasma":
            d.coef = rho
            d.ionpot = r.ionpot
            d.dt = r.δt
            d.preionfrac = r.preionfrac
            d.eratio = pd.e_ratio
            rf = r.ratefunc
            if rf.kind == "adk":
                d.kind = _lib.RESP_PLASMA_ADK
                d.adk_pre = rf.w_p * rf.cn_sq
                d.adk_a = 4 * rf.w_p / rf.w_t_prefac
                d.adk_b = 4 / 3 * rf.w_p / rf.w_t_prefac
                d.adk_pw = 2 * rf.nstar - 1
                d.adk_thr = rf.thr
            else:
                d.kind = _lib.RESP_PLASMA_PPT
                x, y, D = _f64(rf.x), _f64(rf.y), _f64(rf.D)
                keep += [x, y, D]
                d.spl_x, d.spl_y, d.spl_D = _lib.dptr(x), _lib.dptr(y), _lib.dptr(D)
                d.spl_n = len(x)
        elif r.kind in ("raman_field", "raman_env"):
            d.kind = _lib.RESP_RAMAN if (r.kind == "raman_env" or r.thg) else _lib.RESP_RAMAN_NOTHG
            d.coef = rho
            resp = r.r
            hpre = _f64(np.stack(resp.hpres))
            tau2 = _f64(resp.tau2s(rho if rho_tau2 is None else rho_tau2))
            rows = resp.tau2_rows()
            if rows is not None:
                rows = _f64(rows.ravel())
                keep.append(rows)
                d.tau2_rho = _lib.dptr(rows)
                d.amg = pd.amg
            hwin, htt = _f64(resp.w), _f64(resp.tt)
            keep += [hpre, tau2, hwin, htt]
            d.ncomp = len(resp.hpres)
            d.hpre, d.tau2 = _lib.dptr(hpre), _lib.dptr(tau2)
            d.hwin, d.htt = _lib.dptr(hwin), _lib.dptr(htt)
            d.hdt = r.dt
        else:
            raise ValueError(f"unsupported response {r.kind}")
        rds.append(d)
    return rds


class Plan:
    """Owns one ``luna_plan`` (device copy of the grid, normalisation and responses)."""

    def __init__(self, grid_desc, resp_descs, keep, precision, Nw):
        lib = _lib.load()
        self._keep = keep
        self.precision = precision
        self.Nw = Nw
        arr = (_lib.RespDesc * max(1, len(resp_descs)))(*resp_descs)
        h = _lib.c_void_p()
        _lib.check(lib.luna_b200_plan_create(grid_desc, arr, len(resp_descs), precision,
                                             _lib.ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().luna_b200_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    @classmethod
    def from_transform(cls, t, precision=_lib.PREC_FP64):
        gd, rds, keep, Nw, zdep, crop, pad = transform_descs(t)
        plan = cls(gd, rds, keep, precision, Nw)
        if zdep:
            from .gradient import gradient_desc
            gdesc = gradient_desc(t, crop, pad / t.grid.No, plan._keep)
            plan._gdesc = gdesc
            _lib.check(_lib.load().luna_b200_plan_set_gradient(plan.handle, _lib.ctypes.byref(gdesc)))
        return plan

    def rhs(self, nl, Eω, z=0.0):
        """nl[:] = T(Eω) on the GPU (host arrays of complex128)."""
        Ew = _c128(Eω)
        if nl.dtype != np.complex128 or not nl.flags.c_contiguous:
            raise TypeError("nl must be a C-contiguous complex128 array")
        _lib.check(_lib.load().luna_b200_rhs(self._h, _lib.dptr(nl.view(np.float64)),
                                             _lib.dptr(Ew.view(np.float64)), float(z)))
        return nl


def transform_descs(t):
    """C-ABI descriptors of a mode-averaged transform (NonlinearRHS.jl:344-399): the grid
    descriptor, the response descriptors and the arrays they point to, plus (Nw, whether a
    pressure gradient makes the transform z-dependent, crop and pad scales)."""
    g = t.grid
    keep = []
    Nw = len(g.ω)
    N, No = g.N, g.No
    if g.kind == "real":
        Nwo = len(g.ωo)
        pad = (Nwo - 1) / (Nw - 1)
        crop = (Nw - 1) / (Nwo - 1)
        kind = 0
    else:
        pad = No / Nw
        crop = Nw / No
        kind = 1
    zdep = getattr(t, "kind", "") == "modeavg_z"
    # a pressure gradient scales the output by ρ(z) pre/β(z) on the device
    outfac = _c128(np.full(Nw, crop, dtype=np.complex128) if zdep else crop * t.output_factor())
    wwin, towin, twin = _f64(g.ωwin), _f64(g.towin), _f64(g.twin)
    keep += [outfac, wwin, towin, twin]
    gd = _lib.GridDesc()
    gd.kind, gd.N, gd.Nw, gd.No = kind, N, Nw, No
    gd.outfac = _lib.dptr(outfac.view(np.float64))
    gd.wwin, gd.towin, gd.twin = _lib.dptr(wwin), _lib.dptr(towin), _lib.dptr(twin)
    gd.in_scale = pad / No / (nlscale * math.sqrt(t.aeff))
    # per-step statistics (Stats.default): grid axes, Aeff and the field scale
    om, tt = _f64(g.ω), _f64(g.t)
    keep += [om, tt]
    gd.omega, gd.t = _lib.dptr(om), _lib.dptr(tt)
    gd.aeff = t.aeff
    gd.escale = 1.0 / math.sqrt(pd.eps_0 * pd.c * t.aeff / 2)
    rds = resp_descs(t.resp, 1.0 if zdep else t.density, keep,
                     rho_tau2=t.densityfun(0.0) if zdep else None)
    return gd, rds, keep, Nw, zdep, crop, pad


def make_opts(saveN, zsave, rtol=1e-6, atol=1e-10, safety=0.9, max_dt=math.inf, min_dt=0.0,
              repeat_limit=10, max_steps=200000, steplog_cap=0, replay=None, flags=0, stats_cap=0,
              dist_min_no=0):
    o = _lib.SolveOpts()
    o.flags = flags
    o.stats_cap = stats_cap
    o.dist_min_no = dist_min_no
    if replay is not None:
        o.replay = _lib.dptr(replay)
        o.nreplay = len(replay) // 2
    o.rtol, o.atol, o.safety = rtol, atol, safety
    o.max_dt, o.min_dt = max_dt, min_dt
    o.repeat_limit = repeat_limit
    o.max_steps = max_steps
    o.saveN = saveN
    o.zsave = _lib.dptr(zsave)
    o.steplog_cap = steplog_cap
    return o


class SolveResult:
    def __init__(self, z, Eω, y, stats, steplog=None, step_stats=None):
        self.z = z
        self.Eω = Eω
        self.y = y
        self.status = stats.status
        self.steps = stats.steps
        self.accepted = stats.accepted
        self.rejected = stats.rejected
        self.nrhs = stats.nrhs
        self.zfinal = stats.z
        self.dzfinal = stats.dz
        self.nsaved = stats.nsaved
        self.steplog = steplog
        # Stats.default rows of the accepted steps (columns _lib.STATS_KEYS), or None
        self.stats = step_stats


class Batch:
    """Independent instances integrated together by one persistent launch."""

    def __init__(self, plans, saveN, zsave, **opt):
        self.plans = list(plans)
        self.zsave = _f64(zsave)
        self.saveN = saveN
        self.steplog_cap = opt.get("steplog_cap", 0)
        self.stats_cap = opt.get("stats_cap", 0)
        if opt.get("replay") is not None:
            opt["replay"] = _f64(opt["replay"])
            self._replay = opt["replay"]
        self.opts = make_opts(saveN, self.zsave, **opt)
        arr = (_lib.c_void_p * len(plans))(*[p.handle for p in plans])
        h = _lib.c_void_p()
        _lib.check(_lib.load().luna_b200_batch_create(arr, len(plans), self.opts,
                                                     _lib.ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().luna_b200_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def upload(self, linops, y0s, z0s, dz0s, zmaxs, zsaves=None, max_dts=None):
        """Copy the inputs of every instance to the device. ``zsaves`` (per-instance save
        points) and ``max_dts`` (per-instance step limits) are optional."""
        n = len(self.plans)
        # a z-dependent linop (pressure gradient) is evaluated on the device: pass NULL
        self._L = [None if (L is None or callable(L)) else _c128(L) for L in linops]
        self._Y = [_c128(y) for y in y0s]
        Lp = (_lib.PD * n)(*[_lib.dptr(None if L is None else L.view(np.float64)) for L in self._L])
        Yp = (_lib.PD * n)(*[_lib.dptr(y.view(np.float64)) for y in self._Y])
        z0 = _f64(z0s)
        dz0 = _f64(dz0s)
        zm = _f64(zmaxs)
        Zp = None
        if zsaves is not None:
            self._Z = [_f64(z) for z in zsaves]
            Zp = (_lib.PD * n)(*[_lib.dptr(z) for z in self._Z])
        md = None
        if max_dts is not None:
            self._MD = _f64(max_dts)
            md = _lib.dptr(self._MD)
        _lib.check(_lib.load().luna_b200_batch_upload(self._h, Lp, Yp, _lib.dptr(z0),
                                                     _lib.dptr(dz0), _lib.dptr(zm), Zp,
                                                     md if md is not None else _lib.dptr(None)))

    def run(self):
        ms = _lib.c_float(0)
        _lib.check(_lib.load().luna_b200_batch_run(self._h, _lib.ctypes.byref(ms)))
        return ms.value

    def download(self, saves=None, ys=None):
        n = len(self.plans)
        if saves is None:
            saves = [np.zeros((self.saveN, p.Nw), dtype=np.complex128) for p in self.plans]
        if ys is None:
            ys = [np.zeros(p.Nw, dtype=np.complex128) for p in self.plans]
        Sp = (_lib.PD * n)(*[_lib.dptr(s.view(np.float64)) for s in saves])
        Yp = (_lib.PD * n)(*[_lib.dptr(y.view(np.float64)) for y in ys])
        stats = (_lib.SolveStats * n)()
        _lib.check(_lib.load().luna_b200_batch_download(self._h, Sp, Yp, stats))
        return saves, ys, list(stats)

    def info(self):
        """(kernel launches per run, instances on response clusters, clusters)."""
        k, ci, cl = _lib.c_int(), _lib.c_int(), _lib.c_int()
        _lib.check(_lib.load().luna_b200_batch_info(self._h, _lib.ctypes.byref(k), _lib.ctypes.byref(ci),
                                                    _lib.ctypes.byref(cl)))
        return k.value, ci.value, cl.value

    def set_priority(self, priority):
        """Start instances with a larger priority first (an estimate of their work)."""
        self._prio = _f64(priority)
        _lib.check(_lib.load().luna_b200_batch_set_priority(self._h, _lib.dptr(self._prio)))

    def set_shapes(self, shapes):
        """Per-instance shape for the next set_priority: 0 decided by the work estimates,
        1 one CTA, 2 a cluster of 8, 3 a cluster of 16 (when eligible); None restores 0 for
        all."""
        if shapes is None:
            _lib.check(_lib.load().luna_b200_batch_set_shapes(self._h, None))
            return
        arr = (_lib.c_int * len(self.plans))(*[int(x) for x in shapes])
        _lib.check(_lib.load().luna_b200_batch_set_shapes(self._h, arr))

    def set_replay(self, i, replay):
        """Make instance i follow a recorded step sequence (flat (dz, accepted) pairs, e.g.
        columns 1 and 3 of its step log) from the next upload on; None removes it."""
        if replay is None:
            _lib.check(_lib.load().luna_b200_batch_set_replay(self._h, i, _lib.dptr(None), 0))
            return
        r = _f64(replay)
        _lib.check(_lib.load().luna_b200_batch_set_replay(self._h, i, _lib.dptr(r), len(r) // 2))

    def timeline(self):
        """(begin, end) seconds of every instance's integration in the last run, and the SM
        that ran it."""
        n = len(self.plans)
        be = np.zeros((n, 2))
        sm = (_lib.c_int * n)()
        _lib.check(_lib.load().luna_b200_batch_timeline(self._h, _lib.dptr(be), sm))
        return be, np.array(list(sm))

    def stats(self, i):
        """Per-step statistics of instance i: (stats_cap, NSTATS) array."""
        out = np.zeros((self.stats_cap, _lib.NSTATS))
        _lib.check(_lib.load().luna_b200_batch_stats(self._h, i, _lib.dptr(out)))
        return out

    def steplog(self, i):
        out = np.zeros((self.steplog_cap, 4))
        _lib.check(_lib.load().luna_b200_batch_steplog(self._h, i, _lib.dptr(out)))
        return out

    def results(self):
        saves, ys, stats = self.download()
        res = []
        for i, (s, y, st) in enumerate(zip(saves, ys, stats)):
            log = None
            if self.steplog_cap:
                log = self.steplog(i)[: min(st.steps, self.steplog_cap)]
            sts = self.stats(i)[: st.nstats] if self.stats_cap else None
            res.append(SolveResult(self.zsave[: st.nsaved], s[: st.nsaved], y, st, log, sts))
        return res


_STATUS_MSG = {
    _lib.LUNA_FIELD_ABOVE_EMAX: "Field strength exceeds maximum for PPT ionisation rate.",
    _lib.LUNA_REPEAT_LIMIT: "Reached limit for step repetition",
    _lib.LUNA_STEP_BUDGET: "Step budget exhausted before zmax",
}


def solve_precon(transform, linop, Eω, z0, dz0, zmax, saveN=201, rtol=1e-6, atol=1e-10,
                 safety=0.9, max_dt=math.inf, min_dt=0.0, repeat_limit=10, max_steps=200000,
                 steplog_cap=0, precision=_lib.PREC_FP64, raise_on_status=True, replay=None,
                 stats_cap=0, zsave=None):
    """RK45.solve_precon (RK45.jl:19-25) with Luna.run's window filter and saves, on the GPU.

    Saves are taken at ``saveN`` points on [z0, zmax], or at the points ``zsave`` (a
    resumed propagation keeps the save grid of the whole fibre). ``replay`` (optional,
    flat (dz, accepted) pairs) makes the integrator follow a given step sequence instead of
    its controller's choices; it is a verification aid.
    """
    plan = transform.plan() if precision == _lib.PREC_FP64 else Plan.from_transform(transform, precision)
    zs = np.linspace(z0, zmax, saveN) if zsave is None else np.asarray(zsave, dtype=np.float64)
    saveN = len(zs)
    b = Batch([plan], saveN, zs, rtol=rtol, atol=atol, safety=safety, max_dt=max_dt,
              min_dt=min_dt, repeat_limit=repeat_limit, max_steps=max_steps,
              steplog_cap=steplog_cap, replay=replay, stats_cap=stats_cap)
    b.upload([linop], [Eω], [z0], [dz0], [zmax])
    b.run()
    r = b.results()[0]
    if raise_on_status and r.status != 0:
        raise _lib.LunaError(r.status, _STATUS_MSG.get(r.status, "solver error"))
    return r


def run(problem, precision=_lib.PREC_FP64, **kw):
    """Luna.run (Luna.jl:358-391) on the GPU for a ``Problem`` from the interface module
    (a multimode problem goes to the modal solver)."""
    g = problem.grid
    if getattr(problem.transform, "kind", "") == "modal":
        from . import modal_plan
        return modal_plan.run(problem.Eω, g, problem.linop, problem.transform, saveN=problem.saveN,
                              precision=precision, **kw)
    kw.setdefault("max_dt", g.zmax / 2)
    return solve_precon(problem.transform, problem.linop, problem.Eω, 0.0, 1e-4, g.zmax,
                        saveN=problem.saveN, precision=precision, **kw)
