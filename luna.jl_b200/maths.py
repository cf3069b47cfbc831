"""Host-side numerical helpers (setup only).

Restates from Luna.jl ``src/Maths.jl``: the Planck taper window (Maths.jl:422-449), the
Gaussian helpers (Maths.jl:40-50), the series convergence loop (Maths.jl:721-736) and the
construction of ``CSpline`` slopes by a tridiagonal solve (Maths.jl:812-828). The spline
*evaluation* and ``cumtrapz!`` run on the device (see ``csrc/``).
"""
import math

import numpy as np


def planck_taper(x, left0, left1, right1, right0):
    """Planck-taper window that rises between left0..left1 and falls between right1..right0."""
    x = np.asarray(x, dtype=np.float64)
    x0 = (right0 + left0) / 2
    xc = x - x0
    X = right0 - left0
    eps_l = abs(left1 - left0) / X
    eps_r = abs(right0 - right1) / X
    x1 = -X / 2
    x2 = -X / 2 * (1 - 2 * eps_l)
    x3 = X / 2 * (1 - 2 * eps_r)
    x4 = X / 2
    out = np.zeros_like(xc)
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        m = (x1 < xc) & (xc < x2)
        z12 = (x2 - x1) / (xc[m] - x1) + (x2 - x1) / (xc[m] - x2)
        out[m] = 1 / (1 + np.exp(z12))
        out[(x2 <= xc) & (xc <= x3)] = 1.0
        m = (x3 < xc) & (xc < x4)
        z34 = (x3 - x4) / (xc[m] - x3) + (x3 - x4) / (xc[m] - x4)
        out[m] = 1 / (1 + np.exp(z34))
    return out


def fwhm_to_sigma(fwhm, power=2):
    return fwhm / (2 * (2 * math.log(2)) ** (1 / power))


def gauss(x, fwhm, x0=0.0, power=2):
    sigma = fwhm_to_sigma(fwhm, power)
    return np.exp(-0.5 * ((np.asarray(x) - x0) / sigma) ** power)


def converge_series(f, x0, n0=0, rtol=1e-6, maxiter=10000):
    """Sum a series until the relative change falls below rtol (Maths.jl:721-736)."""
    n = n0
    x1 = x0
    success = False
    while not success and n < maxiter:
        x1 = f(x0, n)
        if 2 * abs(x1 - x0) / abs(x1 + x0) < rtol:
            success = True
        n += 1
        x0 = x1
    return x1, success, n


def cspline_slopes(y):
    """Slopes D of the cubic Hermite spline through y (Maths.jl:812-828).

    Solves the tridiagonal system with diagonal (2, 4, ..., 4, 2), off-diagonals 1 and
    right-hand side 3*(central differences) by the Thomas algorithm.
    """
    y = np.asarray(y, dtype=np.float64)
    n = len(y)
    R = np.empty(n)
    R[0] = y[1] - y[0]
    R[1:-1] = y[2:] - y[:-2]
    R[-1] = y[-1] - y[-2]
    R *= 3
    d = np.full(n, 4.0)
    d[0] = 2.0
    d[-1] = 2.0
    # Thomas algorithm with unit off-diagonals
    cp = np.empty(n)
    dp = np.empty(n)
    cp[0] = 1.0 / d[0]
    dp[0] = R[0] / d[0]
    for i in range(1, n):
        m = d[i] - cp[i - 1]
        cp[i] = 1.0 / m
        dp[i] = (R[i] - dp[i - 1]) / m
    D = np.empty(n)
    D[-1] = dp[-1]
    for i in range(n - 2, -1, -1):
        D[i] = dp[i] - cp[i] * D[i + 1]
    return D


def cspline_uniform_index(x0, xmin, xmax, n):
    """1-based index of the first knot above x0 on a uniform axis (Maths.jl:772-774)."""
    if x0 <= xmin:
        return 2
    if x0 >= xmax:
        return n
    return int(math.ceil((x0 - xmin) / (xmax - xmin) * (n - 1))) + 1


def cspline_eval(x, y, D, x0):
    """Evaluate the cubic Hermite spline (Maths.jl:835-848) with the uniform index function."""
    i = cspline_uniform_index(x0, x[0], x[-1], len(x)) - 1
    if x0 == x[i]:
        return y[i]
    if x0 == x[i - 1]:
        return y[i - 1]
    t = (x0 - x[i - 1]) / (x[i] - x[i - 1])
    return (y[i - 1] + D[i - 1] * t + (3 * (y[i] - y[i - 1]) - 2 * D[i - 1] - D[i]) * t ** 2
            + (2 * (y[i - 1] - y[i]) + D[i - 1] + D[i]) * t ** 3)
