"""Mie series for a homogeneous sphere (TEST INFRASTRUCTURE ONLY).

Independent physics check for the BEM path on spheres, written from the
textbook mathematics (Bohren & Huffman, "Absorption and Scattering of Light by
Small Particles", ch. 4: coefficients a_n, b_n from Riccati-Bessel functions
with the logarithmic derivative D_n(mx) by downward recurrence, eqs. 4.88-4.89,
angular functions pi_n, tau_n by upward recurrence, eq. 4.47).  The reference
repository contains no Mie code.
"""
from __future__ import annotations

import numpy as np


def mie_S12(x: float, m: complex, theta: np.ndarray):
    """Amplitude functions S1(theta), S2(theta) for size parameter x and
    relative refractive index m."""
    m = complex(m)
    mu = np.cos(np.asarray(theta, dtype=np.float64))
    nstop = int(x + 4.0 * x ** (1.0 / 3.0) + 2.0)
    nmx = int(max(nstop, abs(m * x))) + 15
    y = m * x
    D = np.zeros(nmx + 1, dtype=complex)
    for n in range(nmx, 0, -1):
        D[n - 1] = n / y - 1.0 / (D[n] + n / y)
    psi0, psi1 = np.cos(x), np.sin(x)
    chi0, chi1 = -np.sin(x), np.cos(x)
    xi1 = complex(psi1, -chi1)
    pi0 = np.zeros_like(mu)
    pi1 = np.ones_like(mu)
    S1 = np.zeros(mu.shape, dtype=complex)
    S2 = np.zeros(mu.shape, dtype=complex)
    for n in range(1, nstop + 1):
        fn = (2.0 * n + 1.0) / (n * (n + 1.0))
        psi = (2.0 * n - 1.0) * psi1 / x - psi0
        chi = (2.0 * n - 1.0) * chi1 / x - chi0
        xi = complex(psi, -chi)
        a = ((D[n] / m + n / x) * psi - psi1) / ((D[n] / m + n / x) * xi - xi1)
        b = ((m * D[n] + n / x) * psi - psi1) / ((m * D[n] + n / x) * xi - xi1)
        pi = pi1
        tau = n * mu * pi - (n + 1.0) * pi0
        S1 += fn * (a * pi + b * tau)
        S2 += fn * (a * tau + b * pi)
        psi0, psi1 = psi1, psi
        chi0, chi1 = chi1, chi
        xi1 = complex(psi1, -chi1)
        pi1 = ((2.0 * n + 1.0) * mu * pi - (n + 1.0) * pi0) / n
        pi0 = pi
    return S1, S2


def mie_M11(x, m, theta, k=None):
    """dsigma/dOmega for unpolarised light, M11 = (|S1|^2+|S2|^2)/(2 k^2); unit
    radius means k = x."""
    S1, S2 = mie_S12(x, m, theta)
    k = x if k is None else k
    return 0.5 * (np.abs(S1) ** 2 + np.abs(S2) ** 2) / k ** 2
