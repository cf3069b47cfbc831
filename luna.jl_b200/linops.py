"""Linear operators of the interaction-picture integrator (host setup).

Restates the mode-averaged constant operators of Luna.jl ``src/LinearOps.jl``
(LinearOps.jl:237-319):

* real grid: ``L = -i(beta - beta1*omega) - alpha/2``
* envelope grid: ``L = -i(beta - beta1*(omega-omega0) - beta0) - alpha/2``

with alpha clamped to [0, 3000] and ``L = 0`` outside ``sidx``. Also returns the
``betaconst`` array used by the mode-averaged normalisation (``beta=1`` outside sidx).
"""
import numpy as np

from . import physdata as pd


def make_const_linop(grid, mode, λ0, thg=False):
    """Return (linop, betaconst, beta1) for ``mode`` on ``grid``."""
    ω0 = pd.wlfreq(λ0)
    β1 = mode.dispersion(1, ω0)
    sidx = grid.sidx
    β = np.ones(len(grid.ω))
    β[sidx] = mode.β(grid.ω[sidx])
    α = np.zeros(len(grid.ω))
    α[sidx] = mode.α(grid.ω[sidx])
    α = np.clip(α, 0.0, 3000.0)
    if grid.kind == "real":
        L = -1j * (β - β1 * grid.ω) - α / 2
    else:
        β0 = 0.0 if thg else float(mode.β(np.array([ω0]))[0])
        L = -1j * (β - β1 * (grid.ω - grid.ω0) - β0) - α / 2
    L = L.astype(np.complex128)
    L[~sidx] = 0
    return L, β, β1
