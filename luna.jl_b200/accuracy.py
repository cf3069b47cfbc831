"""Error of a mixed-precision result against an FP64 one: relative spectral L2 error and
energy / photon-number drift.

The spectral error of one saved field is the relative L2 distance of the spectral
intensities, ||(|Eω|^2 - |Eω_ref|^2)|| / |||Eω_ref|^2||. Energy is ``energy_ω`` of
``Fields.energyfuncs`` (Fields.jl:510-519 for a RealGrid, 522-532 for an EnvGrid): SimpsonEven
over ω of |Eω|^2 times 2π/ω_max^2 (RealGrid) or 2πδω/Δω^2 (EnvGrid). The photon number is
the same integral of |Eω|^2/ω over ω > 0 (each spectral component carries |Eω|^2 dω/(ħω)
photons; the constant factors cancel in a drift). A drift is the relative difference of a
quantity between the result and the reference at the same z.
"""
import numpy as np


def simpson_even_weights(n, h):
    """Weights w with sum(w*y) = NumericalIntegration.jl integrate(x, y, SimpsonEven()) for
    uniform x of spacing h and n >= 8 points (the rule of ``fields.simpson_even``)."""
    w = np.ones(n)
    end = np.array([17.0, 59.0, 43.0, 49.0]) / 48
    w[:4] = end
    w[-4:] = end[::-1]
    return h * w


class Weights:
    """Energy and photon-number weights of one frequency grid (ω ascending, uniform)."""

    def __init__(self, omega, kind="real"):
        om = np.asarray(omega, dtype=np.float64)
        n = len(om)
        dw = om[1] - om[0]
        if kind == "real":
            self.energy = simpson_even_weights(n, dw) * (2 * np.pi / om[-1] ** 2)
        else:
            self.energy = np.full(n, 2 * np.pi * dw / (n * dw) ** 2)
        pos = om > 0
        self.photons = np.where(pos, self.energy / np.where(pos, om, 1.0), 0.0)


def spectral_error(E, Eref):
    """Relative spectral L2 error of |E|^2 against |Eref|^2, per row for 2-D inputs."""
    a = np.abs(np.asarray(E)) ** 2
    b = np.abs(np.asarray(Eref)) ** 2
    num = np.linalg.norm(a - b, axis=-1)
    den = np.linalg.norm(b, axis=-1)
    return num / np.maximum(den, 1e-300)


def drifts(E, Eref, w):
    """(energy drift, photon-number drift) of E against Eref (per row for 2-D inputs)."""
    a = np.abs(np.asarray(E)) ** 2
    b = np.abs(np.asarray(Eref)) ** 2
    en = (a @ w.energy) / np.maximum(b @ w.energy, 1e-300) - 1.0
    ph = (a @ w.photons) / np.maximum(b @ w.photons, 1e-300) - 1.0
    return en, ph


def compare(saves, saves_ref, omega, kind="real"):
    """Per-save spectral error and drifts of a result against its FP64 reference (saved
    fields of equal shape, one row per saved z): dict of arrays."""
    w = Weights(omega, kind)
    en, ph = drifts(saves, saves_ref, w)
    return {"spectral": spectral_error(saves, saves_ref), "energy": en, "photons": ph}


def summary(per_instance):
    """Batch summary from per-instance comparisons (lists of ``compare`` dicts; None for an
    instance that did not complete): the worst and median over instances of each instance's
    worst save, and the worst instance."""
    done = [(i, c) for i, c in enumerate(per_instance) if c is not None and len(c["spectral"])]
    if not done:
        return {"instances": 0}
    worst = np.array([float(np.max(c["spectral"])) for _, c in done])
    en = np.array([float(np.max(np.abs(c["energy"]))) for _, c in done])
    ph = np.array([float(np.max(np.abs(c["photons"]))) for _, c in done])
    k = int(np.argmax(worst))
    return {"instances": len(done),
            "spectral_max": float(worst[k]), "spectral_median": float(np.median(worst)),
            "worst_instance": int(done[k][0]),
            "above_1e-3": [int(done[j][0]) for j in np.nonzero(worst > 1e-3)[0]],
            "energy_drift_max": float(np.max(en)), "energy_drift_median": float(np.median(en)),
            "photon_drift_max": float(np.max(ph)), "photon_drift_median": float(np.median(ph))}
