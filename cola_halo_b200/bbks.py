"""BBKS no-wiggle linear power spectrum table in the reference's input format.

The reference reads a two-column ``k P(k)`` table (h/Mpc, (Mpc/h)^3) and does
not rescale it; it aborts when the table's sigma_8 is more than 5 % off the
parameter (``power.c:62-118``).  This module writes such a table for the
Bardeen, Bond, Kaiser & Szalay (1986, ApJ 304, 15, eq. G3) transfer function

    T(q) = ln(1 + 2.34 q)/(2.34 q)
           * [1 + 3.89 q + (16.1 q)^2 + (5.46 q)^3 + (6.71 q)^4]^(-1/4),
    q = k / Gamma,  Gamma = Omega_m h   (k in h/Mpc; no baryon correction),

P(k) = A k^n_s T(k)^2, with A fixed so that the top-hat variance at
R = 8 Mpc/h, integrated as ``power.c:204-222`` does (0 < k < 500/R), equals
sigma_8^2 -- the same normalisation ``tools/rescale_power.c:167-181`` applies
to a CAMB table.
"""
import numpy as np


def bbks_transfer(k, omega_m, h):
    q = np.asarray(k, dtype=np.float64) / (omega_m * h)
    t = np.log1p(2.34 * q) / (2.34 * q)
    return t * (1.0 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3
                + (6.71 * q) ** 4) ** -0.25


def tophat_sigma2(k, pk, R):
    """sigma^2(R) = 1/(2 pi^2) int k^2 W(kR)^2 P(k) dk on a log-k grid."""
    x = k * R
    w = 3.0 * (np.sin(x) - x * np.cos(x)) / x ** 3
    f = k ** 3 * w * w * pk / (2.0 * np.pi ** 2)   # integrand in d ln k
    lnk = np.log(k)
    return float(np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(lnk)))


def bbks_table(omega_m=0.273, h=0.705, n_s=0.96, sigma8=0.81,
               kmin=1e-4, kmax=1e4, nk=1201):
    """Return (k, P) arrays of the sigma_8-normalised BBKS spectrum at z=0."""
    k = np.logspace(np.log10(kmin), np.log10(kmax), nk)
    R = 8.0
    kk = np.logspace(np.log10(kmin), np.log10(500.0 / R), 400001)
    shape = kk ** n_s * bbks_transfer(kk, omega_m, h) ** 2
    amp = sigma8 ** 2 / tophat_sigma2(kk, shape, R)
    pk = amp * k ** n_s * bbks_transfer(k, omega_m, h) ** 2
    return k, pk


def write_bbks_table(path, **kw):
    k, pk = bbks_table(**kw)
    with open(path, "w") as f:
        for a, b in zip(k, pk):
            f.write("%.9e %.9e\n" % (a, b))
    return path
