"""Discrete-ordinates solution of a grey plane-parallel slab with scattering:
an independent check of the Monte Carlo path with particle scattering.

Slab 0 <= x <= L between cold black walls, uniform temperature T0, absorption
coefficient kappa, scattering coefficient sigma_s and a phase function
p(cos Theta) normalised to (1/4 pi) int p dOmega = 1.  The radiative transfer
equation in slab geometry,
    mu dI/dx = -(kappa + sigma_s) I + kappa I_b + (sigma_s / 2) int_{-1}^{1} pbar(mu, mu') I(mu') dmu',
with pbar the azimuthal average of p, is solved by source iteration on a
fine uniform grid: double Gauss-Legendre directions (n per hemisphere),
exact integration across a cell for a constant source (step
characteristics), cell-average intensities in the source.  The result is
div q = kappa (4 pi I_b - G), G = 2 pi sum_m w_m I_m (Modest, Radiative Heat
Transfer, chapters on the method of discrete ordinates; the exponential
integral solution is the sigma_s = 0 limit, checked in the tests).

TEST INFRASTRUCTURE ONLY (numpy).
"""
from __future__ import annotations

import numpy as np

SIGMA = 5.670373e-08


def double_gauss(n):
    x, w = np.polynomial.legendre.leggauss(n)
    mu = 0.5 * (x + 1.0)
    return mu, 0.5 * w  # nodes on (0, 1), weights summing to 1


def phase_matrix(mu_all, phase, nphi=1024):
    """pbar(mu_i, mu_j) = (1/2pi) int_0^2pi p(cos Theta) dphi for every pair,
    rows renormalised so that (1/2) sum_j w_j pbar_ij = 1 (the discrete
    scattering conserves energy exactly)."""
    phi = (np.arange(nphi) + 0.5) * 2 * np.pi / nphi
    s = np.sqrt(np.clip(1 - mu_all ** 2, 0, None))
    ct = mu_all[:, None, None] * mu_all[None, :, None] + s[:, None, None] * s[None, :, None] * np.cos(phi)[None, None, :]
    return phase(np.clip(ct, -1, 1)).mean(axis=2)


def solve(L, kappa, sigma_s, T0, x_eval, phase=None, n=48, nx=4000, tol=1e-12, max_iter=5000):
    """div q at the points x_eval (W/m^3)."""
    beta = kappa + sigma_s
    mu, w = double_gauss(n)
    mu_all = np.concatenate([mu, -mu])
    w_all = np.concatenate([w, w])
    if phase is None:
        P = np.ones((2 * n, 2 * n))
    else:
        P = phase_matrix(mu_all, phase)
    P = P / (0.5 * (P * w_all[None, :]).sum(axis=1))[:, None]
    Ib = SIGMA * T0 ** 4 / np.pi
    dx = L / nx
    xc = (np.arange(nx) + 0.5) * dx
    tau = beta * dx / mu                       # per direction of one hemisphere
    e = np.exp(-tau)
    f = -np.expm1(-tau) / tau                 # (1 - e^-tau) / tau
    Ibar = np.zeros((2 * n, nx))
    for _ in range(max_iter):
        J = kappa * Ib + 0.5 * sigma_s * (P * w_all[None, :]) @ Ibar   # [2n, nx]
        S = J / beta
        new = np.empty_like(Ibar)
        # mu > 0: sweep from x = 0
        Iin = np.zeros(n)
        Sp = S[:n]
        for i in range(nx):
            s = Sp[:, i]
            new[:n, i] = s + (Iin - s) * f
            Iin = Iin * e + s * (1 - e)
        # mu < 0: sweep from x = L
        Iin = np.zeros(n)
        Sm = S[n:]
        for i in range(nx - 1, -1, -1):
            s = Sm[:, i]
            new[n:, i] = s + (Iin - s) * f
            Iin = Iin * e + s * (1 - e)
        d = np.max(np.abs(new - Ibar))
        Ibar = new
        if d < tol * Ib or sigma_s == 0.0:
            break
    G = 2 * np.pi * (w_all[:, None] * Ibar).sum(axis=0)
    q = kappa * (4 * np.pi * Ib - G)
    return np.interp(x_eval, xc, q)


def henyey_greenstein(g):
    return lambda c: (1 - g * g) / (1 + g * g - 2 * g * c) ** 1.5


def hg_cdf(g, theta):
    """P(Theta <= theta) of the Henyey-Greenstein distribution."""
    c = np.cos(theta)
    if g == 0.0:
        return 0.5 * (1 - c)
    return 1 - (1 - g * g) / (2 * g) * (1 / np.sqrt(1 + g * g - 2 * g * c) - 1 / (1 + g))
