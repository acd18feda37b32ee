"""ORACLE -- test infrastructure only.

Analytic solvation energy of point charges inside a dielectric sphere
(radius a, eps_in) in a linearised Poisson-Boltzmann solvent (eps_out,
inverse Debye length kappa), from the multipole series of Kirkwood (1934).

Derivation (units: e, Angstrom, potentials with the 1/(4 pi) of
beep_constants, energies converted by N_A e^2 / (eps0 A 1000) to kJ/mol as in
src/bem/constants.h:51).  For a charge q at r_i inside the sphere, the
reaction potential inside is

    phi_RF(r) = 1/(4 pi) sum_n A_n r^n r_i^n P_n(cos gamma),

and matching phi and eps dphi/dr at r = a with the outside solution
C_n k_n(kappa r) P_n gives

    A_n = q [(n + 1) + (eps_out/eps_in) g_n] / (a^(2n+1) (eps_in n - eps_out g_n)),
    g_n = x k_n'(x) / k_n(x),  x = kappa a,

with k_n the modified spherical Bessel function of the second kind
(k_n' = -k_(n-1) - (n+1)/x k_n, so g_n = -x k_(n-1)/k_n - (n+1); for
kappa = 0, g_n = -(n+1), the salt-free Kirkwood series).  The solvation
energy is  E = 1/2 sum_j q_j phi_RF(r_j).  The single-charge structure and
the Bessel recurrence agree with the reference's analytic script
tools/off-centre.py:27-98, and n = 0 with one central charge is the Born
energy of tools/born_ion.py:6-11.
"""
from __future__ import annotations

import numpy as np

CONVERT_KJ_PER_MOL = 6.02214179e23 * 1.60217646e-19 ** 2 / (8.85418782e-12 * 1.0e-10 * 1000.0)


def _g(nmax: int, x: float) -> np.ndarray:
    """g_n = x k_n'(x)/k_n(x), n = 0..nmax."""
    if x == 0.0:
        return -(np.arange(nmax + 1) + 1.0)
    # scaled k_n: khat_n = k_n(x) * x * exp(x) * (2/pi); ratios are unchanged
    kh = np.zeros(nmax + 2)
    kh[0] = 1.0                       # k_0 -> 1 (also k_-1)
    kh[1] = 1.0 + 1.0 / x
    for n in range(1, nmax + 1):
        kh[n + 1] = kh[n - 1] + (2 * n + 1) / x * kh[n]
    g = np.zeros(nmax + 1)
    g[0] = -x - 1.0
    for n in range(1, nmax + 1):
        g[n] = -x * kh[n - 1] / kh[n] - (n + 1)
    return g


def legendre(nmax: int, x: np.ndarray) -> np.ndarray:
    P = np.zeros((nmax + 1,) + np.shape(x))
    P[0] = 1.0
    if nmax >= 1:
        P[1] = x
    for n in range(1, nmax):
        P[n + 1] = ((2 * n + 1) * x * P[n] - n * P[n - 1]) / (n + 1)
    return P


def solvation_energy(charges, radius: float, eps_in: float, eps_out: float, kappa: float,
                     centre=(0.0, 0.0, 0.0), nmax: int = 80) -> float:
    """Reaction-field energy in kJ/mol of charges [n][4] (x y z q)."""
    ch = np.asarray(charges, float)
    pos = ch[:, :3] - np.asarray(centre, float)
    q = ch[:, 3]
    r = np.linalg.norm(pos, axis=1)
    if np.any(r >= radius):
        raise ValueError("all charges must lie inside the sphere")
    u = pos / np.where(r > 0, r, 1.0)[:, None]
    cosg = np.clip(u @ u.T, -1.0, 1.0)
    g = _g(nmax, kappa * radius)
    P = legendre(nmax, cosg)
    rr = np.outer(r, r)
    total = np.zeros_like(rr)
    for n in range(nmax + 1):
        An = ((n + 1) + (eps_out / eps_in) * g[n]) / (radius ** (2 * n + 1) * (eps_in * n - eps_out * g[n]))
        total += An * rr ** n * P[n]
    E = 0.5 * (q[:, None] * q[None, :] * total).sum() / (4 * np.pi)
    return float(E * CONVERT_KJ_PER_MOL)


def born_energy(q: float, radius: float, eps_in: float, eps_out: float) -> float:
    """Born ion (kJ/mol): q^2/(8 pi a) (1/eps_out - 1/eps_in)."""
    return float(q * q / (8 * np.pi * radius) * (1.0 / eps_out - 1.0 / eps_in) * CONVERT_KJ_PER_MOL)
