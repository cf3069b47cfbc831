"""The C-ABI libraries load and export every entry point declared in include/luna_b200.h and
include/luna_surrogate.h, and the descriptor structs have the layout the ctypes (and the
documented Julia) bindings assume. No compute calls."""
import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import ctypes
import os
import pathlib
import re
import subprocess

import pytest

from luna_b200 import _lib

ROOT = pathlib.Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "luna_b200.h"


def declared_functions():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"\b(luna_b200_\w+)\s*\(", txt)))


def test_library_present_and_loads():
    assert os.path.exists(_lib.LIB_PATH), "build with luna.jl_b200/build.py"
    lib = _lib.load()
    assert lib.luna_b200_version() >= 1


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    assert set(names) == set(_lib.EXPORTS)


def test_surrogate_library_exports_its_header():
    """libluna_surrogate.so (the learned surrogate's kernels) exports every function that
    include/luna_surrogate.h declares, and the ctypes binding loads them all."""
    from luna_b200 import surrogate
    hdr = (ROOT / "include" / "luna_surrogate.h").read_text()
    names = sorted(set(re.findall(r"\b(luna_sg_\w+)\s*\(", hdr)))
    assert len(names) == 7
    out = subprocess.run(["nm", "-D", "--defined-only", surrogate.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    assert not [n for n in names if n not in exported]
    lib = surrogate.load()
    for n in names:
        assert getattr(lib, n).argtypes is not None, n


def test_plan_create_without_device_fails_loudly():
    # On a machine without a GPU the library must refuse, not compute on the host.
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = _lib.load()
    gd = _lib.GridDesc()
    h = _lib.c_void_p()
    rc = lib.luna_b200_plan_create(ctypes.byref(gd), None, 0, 0, ctypes.byref(h))
    assert rc != _lib.LUNA_OK
    assert lib.luna_b200_last_error()


C_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "luna_b200.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
    printf("luna_grid_desc %zu\nluna_resp_desc %zu\nluna_solve_opts %zu\nluna_solve_stats %zu\n",
           sizeof(luna_grid_desc), sizeof(luna_resp_desc), sizeof(luna_solve_opts), sizeof(luna_solve_stats));
    printf("luna_radial_desc %zu\n", sizeof(luna_radial_desc));
    P(luna_grid_desc, in_scale); P(luna_resp_desc, spl_n); P(luna_resp_desc, adk_thr);
    P(luna_resp_desc, hdt); P(luna_resp_desc, cthg); P(luna_resp_desc, tau2_rho); P(luna_resp_desc, amg);
    P(luna_solve_opts, zsave); P(luna_solve_opts, steplog_cap);
    P(luna_solve_opts, replay); P(luna_solve_opts, nreplay); P(luna_solve_opts, flags);
    P(luna_radial_desc, Mf); P(luna_radial_desc, outfac);
    P(luna_grid_desc, omega); P(luna_grid_desc, escale); P(luna_solve_opts, stats_cap);
    P(luna_solve_stats, nstats); P(luna_solve_opts, dist_min_no);
    P(luna_solve_stats, z); P(luna_solve_stats, dz);
    printf("luna_gradient_desc %zu\n", sizeof(luna_gradient_desc));
    P(luna_gradient_desc, Z); P(luna_gradient_desc, P2); P(luna_gradient_desc, dens_b);
    P(luna_gradient_desc, loss); P(luna_gradient_desc, gam); P(luna_gradient_desc, ofs);
    P(luna_gradient_desc, fd_xc); P(luna_gradient_desc, fd_vn); P(luna_gradient_desc, fd_h12);
    P(luna_gradient_desc, nta); P(luna_gradient_desc, ZA); P(luna_gradient_desc, eps0c2);
    P(luna_gradient_desc, vn); P(luna_gradient_desc, env_ref); P(luna_gradient_desc, ref_xc);
    P(luna_gradient_desc, ref_gam); P(luna_gradient_desc, ref_vn);
    printf("luna_modal_desc %zu\n", sizeof(luna_modal_desc));
    P(luna_modal_desc, ems); P(luna_modal_desc, wts); P(luna_modal_desc, wlow);
    P(luna_modal_desc, rtol); P(luna_modal_desc, atol); P(luna_modal_desc, outfac);
    return 0;
}
"""


def test_struct_layout_matches_ctypes(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(C_PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    assert int(out["luna_grid_desc"]) == ctypes.sizeof(_lib.GridDesc)
    assert int(out["luna_resp_desc"]) == ctypes.sizeof(_lib.RespDesc)
    assert int(out["luna_solve_opts"]) == ctypes.sizeof(_lib.SolveOpts)
    assert int(out["luna_solve_stats"]) == ctypes.sizeof(_lib.SolveStats)
    assert int(out["luna_grid_desc.in_scale"]) == _lib.GridDesc.in_scale.offset
    assert int(out["luna_resp_desc.spl_n"]) == _lib.RespDesc.spl_n.offset
    assert int(out["luna_resp_desc.adk_thr"]) == _lib.RespDesc.adk_thr.offset
    assert int(out["luna_resp_desc.hdt"]) == _lib.RespDesc.hdt.offset
    assert int(out["luna_resp_desc.cthg"]) == _lib.RespDesc.cthg.offset
    assert int(out["luna_resp_desc.tau2_rho"]) == _lib.RespDesc.tau2_rho.offset
    assert int(out["luna_resp_desc.amg"]) == _lib.RespDesc.amg.offset
    assert int(out["luna_solve_opts.zsave"]) == _lib.SolveOpts.zsave.offset
    assert int(out["luna_solve_opts.steplog_cap"]) == _lib.SolveOpts.steplog_cap.offset
    assert int(out["luna_radial_desc"]) == ctypes.sizeof(_lib.RadialDesc)
    for f in ("replay", "nreplay", "flags"):
        assert int(out[f"luna_solve_opts.{f}"]) == getattr(_lib.SolveOpts, f).offset
    assert int(out["luna_grid_desc.omega"]) == _lib.GridDesc.omega.offset
    assert int(out["luna_grid_desc.escale"]) == _lib.GridDesc.escale.offset
    assert int(out["luna_solve_opts.stats_cap"]) == _lib.SolveOpts.stats_cap.offset
    assert int(out["luna_solve_opts.dist_min_no"]) == _lib.SolveOpts.dist_min_no.offset
    assert int(out["luna_solve_stats.nstats"]) == _lib.SolveStats.nstats.offset
    for f in ("Mf", "outfac"):
        assert int(out[f"luna_radial_desc.{f}"]) == getattr(_lib.RadialDesc, f).offset
    assert int(out["luna_solve_stats.z"]) == _lib.SolveStats.z.offset
    assert int(out["luna_solve_stats.dz"]) == _lib.SolveStats.dz.offset
    assert int(out["luna_gradient_desc"]) == ctypes.sizeof(_lib.GradientDesc)
    for f in ("Z", "P2", "dens_b", "loss", "gam", "ofs", "fd_xc", "fd_vn", "fd_h12", "nta", "ZA",
              "eps0c2", "vn", "env_ref", "ref_xc", "ref_gam", "ref_vn"):
        assert int(out[f"luna_gradient_desc.{f}"]) == getattr(_lib.GradientDesc, f).offset
    assert int(out["luna_modal_desc"]) == ctypes.sizeof(_lib.ModalDesc)
    for f in ("ems", "wts", "wlow", "rtol", "atol", "outfac"):
        assert int(out[f"luna_modal_desc.{f}"]) == getattr(_lib.ModalDesc, f).offset


# ------------------------------------------------------------------ the Julia binding
_JL_TYPES = {"Cint": ctypes.c_int, "Float64": ctypes.c_double, "Clonglong": ctypes.c_longlong}


def _julia_blocks():
    import re
    text = (HEADER.parent.parent / "INTEGRATION.md").read_text()
    return "\n".join(re.findall(r"```julia\n(.*?)```", text, flags=re.S))


def _julia_structs():
    """Immutable `struct Name ... end` blocks of the Julia shim: {name: [(field, type)]}."""
    import re
    out = {}
    for m in re.finditer(r"^struct (\w+)\s*\n(.*?)^end", _julia_blocks(), flags=re.S | re.M):
        body = re.sub(r"#.*", "", m.group(2))
        out[m.group(1)] = re.findall(r"(\w+)::(\w+(?:\{[^}]*\})?)", body)
    return out


def _ctype_matches(jl, ct):
    import re
    if jl.startswith("Ptr{"):
        return ct is _lib.PD or ct is ctypes.c_void_p or issubclass(ct, ctypes._Pointer)
    m = re.fullmatch(r"NTuple\{(\d+),\s*(\w+)\}", jl)
    if m:
        return issubclass(ct, ctypes.Array) and ct._length_ == int(m.group(1)) \
            and ct._type_ is _JL_TYPES[m.group(2)]
    return ct is _JL_TYPES[jl]


@pytest.mark.parametrize("name", ["GridDesc", "RespDesc", "RadialDesc", "ModalDesc", "GradientDesc",
                                  "SolveOpts", "SolveStats"])
def test_julia_binding_structs_match_the_header(name):
    """INTEGRATION.md's Julia structs mirror the C structs field for field (names, order and
    types); the ctypes structures they are compared with are checked against the C
    compiler's layout above."""
    jl = _julia_structs()[name]
    ct = getattr(_lib, name)._fields_
    assert [f for f, _ in jl] == [f for f, _ in ct], name
    for (f, jt), (_, ctt) in zip(jl, ct):
        assert _ctype_matches(jt, ctt), (name, f, jt, ctt)


def test_julia_binding_solveopts_call_passes_every_field():
    import re
    calls = re.findall(r"SolveOpts\(([^()]*(?:\([^()]*\)[^()]*)*)\)", _julia_blocks())
    assert calls
    for c in calls:
        assert len([a for a in c.split(",") if a.strip()]) == len(_lib.SolveOpts._fields_), c
