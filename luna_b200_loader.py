"""Import helper: registers the ``luna.jl_b200`` directory as the ``luna_b200`` package."""
import importlib.util
import pathlib
import sys


def load():
    if "luna_b200" in sys.modules:
        return sys.modules["luna_b200"]
    pkg = pathlib.Path(__file__).resolve().parent / "luna.jl_b200"
    spec = importlib.util.spec_from_file_location("luna_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["luna_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
