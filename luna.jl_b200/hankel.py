"""Quasi-discrete Hankel transform of order 0 (host setup of the radial transform).

Luna.jl uses Hankel.jl's ``QDHT(R, N, dim=2)`` (third-party, compat 0.5.5, not vendored
with the reference). This module restates the published algorithm (M. Guizar-Sicairos and
J. C. Gutiérrez-Vega, JOSA A 21, 53 (2004)) for order 0:

* j_n, n = 1..N+1: zeros of J0; S = j_{N+1}; aperture R, band limit K = S/R;
* r_n = j_n R/S, k_n = j_n/R;
* forward F(k) = int_0^inf f(r) J0(k r) r dr  ->  F(k_m) = sum_n (2/K^2) J0(j_m j_n/S)/J1(j_n)^2 f(r_n)
* inverse f(r) = int_0^inf F(k) J0(k r) k dk  ->  f(r_n) = sum_m (2/R^2) J0(j_n j_m/S)/J1(j_m)^2 F(k_m)
* integrateR(f) = int f r dr = sum_n (2/K^2)/J1(j_n)^2 f(r_n); integrateK likewise with 2/R^2.

The forward and inverse matrices are the device inputs of the radial transform.
"""
import numpy as np
from scipy import special


class QDHT:
    def __init__(self, R, N):
        zeros = special.jn_zeros(0, N + 1)
        roots = zeros[:N]
        S = zeros[N]
        self.R, self.N = float(R), int(N)
        self.K = S / R
        self.r = roots * R / S
        self.k = roots / R
        J1sq = special.j1(roots) ** 2
        J0 = special.j0(np.outer(roots, roots) / S)
        self.Mf = (2 / self.K ** 2) * J0 / J1sq[None, :]   # k-space from r-space
        self.Mi = (2 / self.R ** 2) * J0 / J1sq[None, :]   # r-space from k-space
        self.scaleR = 2 / self.K ** 2 / J1sq
        self.scaleK = 2 / self.R ** 2 / J1sq

    def forward(self, A, axis=1):
        """q * A: r-space -> k-space along ``axis``."""
        return np.moveaxis(np.tensordot(self.Mf, np.moveaxis(A, axis, 0), axes=(1, 0)), 0, axis)

    def inverse(self, A, axis=1):
        """q \\ A: k-space -> r-space along ``axis``."""
        return np.moveaxis(np.tensordot(self.Mi, np.moveaxis(A, axis, 0), axes=(1, 0)), 0, axis)

    def integrateR(self, A, axis=-1):
        return np.tensordot(A, self.scaleR, axes=([axis], [0]))

    def integrateK(self, A, axis=-1):
        return np.tensordot(A, self.scaleK, axes=([axis], [0]))
