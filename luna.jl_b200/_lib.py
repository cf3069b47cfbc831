"""ctypes bindings of ``libluna_b200.so`` (declarations in ``include/luna_b200.h``).

The library is built in-tree by ``build.py``. Loading fails loudly when it is missing:
there is no host implementation of the right-hand side or the integrator to fall back on.
"""
import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_longlong, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libluna_b200.so")

LUNA_OK = 0
LUNA_FIELD_ABOVE_EMAX = 1
LUNA_REPEAT_LIMIT = 2
LUNA_NONFINITE = 3
LUNA_STEP_BUDGET = 4
LUNA_WAIT_TIMEOUT = 5
LUNA_ERR_BAD_ARG = 16
LUNA_ERR_UNSUPPORTED = 17
LUNA_ERR_CUDA = 18
NOALLOC_SCRATCH_BYTES = 1 << 20
SOLVE_NO_CLUSTERS = 1
SOLVE_NO_DIST = 2
NSTATS = 10
STATS_KEYS = ("z", "dz", "ω0", "energy", "peakpower", "peakintensity", "fwhm_t_min",
              "fwhm_t_max", "electrondensity", "peak_ionisation_rate")

RESP_KERR_FIELD = 1
RESP_KERR_ENV = 2
RESP_PLASMA_PPT = 3
RESP_PLASMA_ADK = 4
RESP_RAMAN = 5
RESP_KERR_FIELD_NOTHG = 6
RESP_RAMAN_NOTHG = 7
RESP_KERR_ENV_THG = 8

PREC_FP64 = 0
PREC_MIXED = 1

PD = POINTER(c_double)


class GridDesc(ctypes.Structure):
    _fields_ = [("kind", c_int), ("N", c_int), ("Nw", c_int), ("No", c_int),
                ("outfac", PD), ("wwin", PD), ("towin", PD), ("twin", PD),
                ("in_scale", c_double), ("omega", PD), ("t", PD), ("aeff", c_double),
                ("escale", c_double)]


class RespDesc(ctypes.Structure):
    _fields_ = [("kind", c_int), ("coef", c_double),
                ("ionpot", c_double), ("dt", c_double), ("preionfrac", c_double),
                ("eratio", c_double),
                ("spl_x", PD), ("spl_y", PD), ("spl_D", PD), ("spl_n", c_int),
                ("adk_pre", c_double), ("adk_a", c_double), ("adk_b", c_double),
                ("adk_pw", c_double), ("adk_thr", c_double),
                ("ncomp", c_int), ("hpre", PD), ("tau2", PD), ("hwin", PD), ("htt", PD),
                ("hdt", c_double), ("cthg", PD), ("tau2_rho", PD), ("amg", c_double)]


class RadialDesc(ctypes.Structure):
    _fields_ = [("Nr", c_int), ("Mi", PD), ("Mf", PD), ("outfac", PD)]


class ModalDesc(ctypes.Structure):
    _fields_ = [("nmodes", c_int), ("npol", c_int), ("nlevels", c_int), ("ems", PD), ("wts", PD),
                ("wlow", c_double), ("rtol", c_double), ("atol", c_double), ("outfac", PD)]


GRAD_MAXPTS = 16


class GradientDesc(ctypes.Structure):
    _fields_ = [("npts", c_int), ("two_point", c_int),
                ("Z", c_double * GRAD_MAXPTS), ("P", c_double * GRAD_MAXPTS),
                ("P2", c_double * GRAD_MAXPTS), ("dens_a", c_double), ("dens_b", c_double),
                ("loss", c_int), ("nta", c_int), ("ZA", c_double * GRAD_MAXPTS),
                ("A", c_double * GRAD_MAXPTS), ("unm", c_double), ("aeff_intg", c_double),
                ("in_base", c_double), ("eps0c2", c_double),
                ("gam", PD), ("vn", PD), ("wc", PD), ("om", PD),
                ("imcap", PD), ("ofs", PD), ("fd_xc", c_double * 4), ("fd_gam", c_double * 4),
                ("fd_vn", c_double * 8), ("fd_h12", c_double), ("env_ref", c_int),
                ("ref_xc", c_double), ("ref_gam", c_double), ("ref_vn", c_double * 2)]


class SolveOpts(ctypes.Structure):
    _fields_ = [("rtol", c_double), ("atol", c_double), ("safety", c_double),
                ("max_dt", c_double), ("min_dt", c_double), ("repeat_limit", c_int),
                ("max_steps", c_longlong), ("saveN", c_int), ("zsave", PD),
                ("steplog_cap", c_longlong), ("replay", PD), ("nreplay", c_longlong),
                ("flags", c_int), ("stats_cap", c_longlong), ("dist_min_no", c_int)]


class SolveStats(ctypes.Structure):
    _fields_ = [("status", c_int), ("nsaved", c_int), ("steps", c_longlong),
                ("accepted", c_longlong), ("rejected", c_longlong), ("nrhs", c_longlong),
                ("z", c_double), ("dz", c_double), ("nstats", c_longlong)]


EXPORTS = [
    "luna_b200_plan_create", "luna_b200_plan_destroy", "luna_b200_rhs", "luna_b200_rhs_device",
    "luna_b200_solve", "luna_b200_batch_create", "luna_b200_batch_upload", "luna_b200_batch_run",
    "luna_b200_batch_download", "luna_b200_batch_steplog", "luna_b200_batch_destroy",
    "luna_b200_last_error", "luna_b200_version", "luna_b200_rhs_device_noalloc",
    "luna_b200_radial_plan_create", "luna_b200_radial_plan_destroy", "luna_b200_radial_rhs",
    "luna_b200_radial_rhs_device", "luna_b200_radial_solve", "luna_b200_qdht_device",
    "luna_b200_batch_timeline", "luna_b200_batch_set_priority",
    "luna_b200_batch_info", "luna_b200_batch_stats", "luna_b200_plan_set_gradient",
    "luna_b200_plan_linop", "luna_b200_modal_plan_create", "luna_b200_modal_plan_destroy",
    "luna_b200_modal_rhs", "luna_b200_modal_rhs_device", "luna_b200_modal_solve",
    "luna_b200_batch_set_replay", "luna_b200_batch_set_shapes", "luna_b200_radial_set_gradient",
    "luna_b200_radial_linop",
]

_lib = None


class LunaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libluna_b200 error {code}: {msg}")
        self.code = code


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with luna.jl_b200/build.py "
                          "(there is no CPU implementation of the UPPE hot path)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.luna_b200_plan_create.argtypes = [POINTER(GridDesc), POINTER(RespDesc), c_int, c_int,
                                          POINTER(c_void_p)]
    lib.luna_b200_plan_set_gradient.argtypes = [c_void_p, POINTER(GradientDesc)]
    lib.luna_b200_plan_linop.argtypes = [c_void_p, c_double, PD, PD]
    lib.luna_b200_plan_destroy.argtypes = [c_void_p]
    lib.luna_b200_plan_destroy.restype = None
    lib.luna_b200_rhs.argtypes = [c_void_p, PD, PD, c_double]
    lib.luna_b200_rhs_device.argtypes = [c_void_p, c_void_p, c_void_p, c_double, c_void_p]
    lib.luna_b200_solve.argtypes = [c_void_p, PD, PD, c_double, c_double, c_double,
                                    POINTER(SolveOpts), PD, PD, POINTER(SolveStats)]
    lib.luna_b200_batch_create.argtypes = [POINTER(c_void_p), c_int, POINTER(SolveOpts),
                                           POINTER(c_void_p)]
    lib.luna_b200_batch_upload.argtypes = [c_void_p, POINTER(PD), POINTER(PD), PD, PD, PD,
                                           POINTER(PD), PD]
    lib.luna_b200_batch_run.argtypes = [c_void_p, POINTER(c_float)]
    lib.luna_b200_batch_download.argtypes = [c_void_p, POINTER(PD), POINTER(PD), POINTER(SolveStats)]
    lib.luna_b200_batch_steplog.argtypes = [c_void_p, c_int, PD]
    lib.luna_b200_batch_stats.argtypes = [c_void_p, c_int, PD]
    lib.luna_b200_batch_destroy.argtypes = [c_void_p]
    lib.luna_b200_batch_destroy.restype = None
    lib.luna_b200_rhs_device_noalloc.argtypes = [c_void_p, c_void_p, c_void_p, c_double, c_void_p,
                                                 c_void_p]
    lib.luna_b200_radial_plan_create.argtypes = [POINTER(GridDesc), POINTER(RespDesc), c_int,
                                                 POINTER(RadialDesc), c_int, POINTER(c_void_p)]
    lib.luna_b200_radial_plan_destroy.argtypes = [c_void_p]
    lib.luna_b200_radial_plan_destroy.restype = None
    lib.luna_b200_radial_rhs.argtypes = [c_void_p, PD, PD, c_double]
    lib.luna_b200_radial_rhs_device.argtypes = [c_void_p, c_void_p, c_void_p, c_double, c_void_p]
    lib.luna_b200_radial_solve.argtypes = [c_void_p, PD, PD, c_double, c_double, c_double,
                                           POINTER(SolveOpts), PD, PD, POINTER(SolveStats)]
    lib.luna_b200_radial_set_gradient.argtypes = [c_void_p, POINTER(GradientDesc), PD, PD]
    lib.luna_b200_radial_linop.argtypes = [c_void_p, c_double, PD, PD]
    lib.luna_b200_modal_plan_create.argtypes = [POINTER(GridDesc), POINTER(RespDesc), c_int,
                                                POINTER(ModalDesc), c_int, POINTER(c_void_p)]
    lib.luna_b200_modal_plan_destroy.argtypes = [c_void_p]
    lib.luna_b200_modal_plan_destroy.restype = None
    lib.luna_b200_modal_rhs.argtypes = [c_void_p, PD, PD, c_double, POINTER(c_int)]
    lib.luna_b200_modal_rhs_device.argtypes = [c_void_p, c_void_p, c_void_p, c_double, c_void_p]
    lib.luna_b200_modal_solve.argtypes = [c_void_p, PD, PD, c_double, c_double, c_double,
                                          POINTER(SolveOpts), PD, PD, POINTER(SolveStats)]
    lib.luna_b200_batch_info.argtypes = [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int)]
    lib.luna_b200_batch_set_priority.argtypes = [c_void_p, PD]
    lib.luna_b200_batch_set_replay.argtypes = [c_void_p, c_int, PD, c_longlong]
    lib.luna_b200_batch_set_shapes.argtypes = [c_void_p, POINTER(c_int)]
    lib.luna_b200_batch_timeline.argtypes = [c_void_p, PD, POINTER(c_int)]
    lib.luna_b200_qdht_device.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p]
    lib.luna_b200_last_error.restype = ctypes.c_char_p
    lib.luna_b200_version.restype = c_int
    _lib = lib
    return lib


def check(rc):
    if rc != LUNA_OK:
        msg = load().luna_b200_last_error().decode(errors="replace")
        raise LunaError(rc, msg)
    return rc


def dptr(a):
    """double* pointing at a C-contiguous float64/complex128 numpy array (or NULL)."""
    if a is None:
        return ctypes.cast(None, PD)
    return a.ctypes.data_as(PD)
