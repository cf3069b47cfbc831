"""Extract the reference's own known answers for this path from its test sources into
``reference_golden.json`` (run where the reference sources are available; the tests read
only the JSON file).

Values (file:line of Luna.jl's test directory):
* ADK rates: test_ionisation.jl:6-10, ``ionrate_ADK(gas, E) ≈ value``;
* PPT rates: test_ionisation.jl:15-16, ``ionrate_PPT(gas, λ0, E; dipole_corr=false)`` against
  ``2*value``, rtol 1e-3;
* soliton self-frequency shift: test_gnlse.jl:51, 55, peak frequency and time, rtol 1e-14;
* radial focus: test_radial.jl:64, the bound on the fluence profile error.

Usage: python tests/golden/make_golden.py <path to the reference checkout>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"([-+]?\d+(?:\.\d*)?(?:e[-+]?\d+)?)"


def _read(root, name):
    with open(os.path.join(root, "test", name)) as f:
        return f.read()


def extract(root):
    ion = _read(root, "test_ionisation.jl")
    adk = [{"gas": g, "E": float(E), "rate": float(v)}
           for g, E, v in re.findall(r"ionrate_ADK\(:(\w+)\s*,\s*" + NUM + r"\)\s*≈\s*" + NUM, ion)
           if not g.endswith("B")]  # :HeB is an alias of :He
    ppt = [{"gas": g, "lambda0": float(l), "E": float(E), "rate": 2 * float(v), "rtol": float(rt)}
           for g, l, E, v, rt in re.findall(
               r"ionrate_PPT\(:(\w+),\s*" + NUM + r",\s*" + NUM + r"; dipole_corr=false\),\s*2\*" + NUM
               + r",\s*rtol=" + NUM + r"\)", ion)]
    gnlse = _read(root, "test_gnlse.jl")
    w = re.search(r"ω\[argmax\(abs2\.\(Eωout\)\)\],\s*" + NUM + r",\s*rtol=" + NUM, gnlse)
    t = re.search(r"T\[argmax\(abs2\.\(Etout\)\)\],\s*" + NUM + r",\s*rtol=" + NUM, gnlse)
    radial = _read(root, "test_radial.jl")
    r = re.search(r"@test\s+maximum\([^\n]*\)\s*<\s*" + NUM, radial)
    out = {
        "source": "Luna.jl test sources (test_ionisation.jl, test_gnlse.jl, test_radial.jl)",
        "adk": adk,
        "ppt": ppt,
        "soliton_shift": {"omega_peak": float(w.group(1)), "t_peak": float(t.group(1)),
                          "rtol": float(w.group(2))},
        "radial_focus_bound": float(r.group(1)) if r else None,
    }
    if len(adk) != 4 or len(ppt) != 2:
        raise RuntimeError(f"unexpected reference test contents: {len(adk)} ADK, {len(ppt)} PPT values")
    return out


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LUNA_REFERENCE", "")
    data = extract(root)
    with open(os.path.join(HERE, "reference_golden.json"), "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps(data, indent=1))
