"""Condon-Shortley angular algebra for the two-electron channel tables (host setup).

Gaunt integrals come from exact Wigner 3j symbols (sympy, the same third-party
arithmetic the reference uses, python/angular.py:4).  Conventions follow the
reference so that the generated Hamiltonian tables are identical:

* ``C(bra, k, q, ket)`` = <l m | C^k_q | j n>  (python/angular.py:8-12);
* ``cartesian`` = dipole (x, y, z) components from the spherical ones
  (python/angular.py:14-16);
* ``coulomb`` = multipole-lambda coefficient of 1/r12 between product channels
  (python/angular.py:18-24);
* ``channels`` = product (l1 m1)(l2 m2) list with total M filter
  (python/angular.py:26-29);
* ``radial_hydrogen`` = hydrogenic P/r radial functions (python/angular.py:31-35).
"""
from functools import lru_cache

import numpy as np
from scipy.special import eval_genlaguerre, factorial
from sympy.physics.wigner import wigner_3j


@lru_cache(None)
def C(bra, k, q, ket):
    """Reduced-normalised Gaunt coefficient <l m|C^k_q|j n> (0 when forbidden)."""
    l, m = bra
    j, n = ket
    allowed = m == n + q and abs(q) <= k and abs(l - j) <= k <= l + j and (l + k + j) % 2 == 0
    if not allowed:
        return 0.0
    three = wigner_3j(l, k, j, 0, 0, 0) * wigner_3j(l, k, j, -m, q, n)
    return float((-1) ** m * np.sqrt((2 * l + 1) * (2 * j + 1)) * three)


def cartesian(bra, ket):
    """Cartesian components of <bra| r_hat |ket> (x, y, z) as a complex 3-vector."""
    lower = C(bra, 1, -1, ket)
    upper = C(bra, 1, 1, ket)
    return np.array([(lower - upper) / np.sqrt(2), 1j * (lower + upper) / np.sqrt(2),
                     C(bra, 1, 0, ket)], complex)


def coulomb(bra, ket, lam):
    """Angular factor of the lambda-th multipole of 1/r12 between product channels."""
    (l1, m1), (l2, m2) = bra
    (k1, n1), (k2, n2) = ket
    q = m1 - n1  # magnetic conservation leaves a single q in the Gaunt sum
    if abs(q) > lam or m2 - n2 != -q:
        return 0.0
    first = C((l1, m1), lam, q, (k1, n1))
    if not first:
        return 0.0
    return (-1.0) ** q * first * C((l2, m2), lam, -q, (k2, n2))


def channels(lmax, M=0):
    """Product channels ((l1,m1),(l2,m2)) with l<=lmax; M=None keeps every total M."""
    if lmax < 0:
        raise ValueError('lmax>=0')
    single = [(l, m) for l in range(lmax + 1) for m in range(-l, l + 1)]
    return [(a, b) for a in single for b in single if M is None or a[1] + b[1] == M]


def radial_hydrogen(n, l, r, Z=2.0):
    """Hydrogenic radial function R_nl(r) for nuclear charge Z (analytic on complex r)."""
    if n < 1 or l < 0 or l >= n:
        raise ValueError('requires 0<=l<n')
    x = 2 * Z * np.asarray(r) / n
    norm = (2 * Z / n) ** 1.5 * np.sqrt(factorial(n - l - 1) / (2 * n * factorial(n + l)))
    return norm * np.exp(-x / 2) * x ** l * eval_genlaguerre(n - l - 1, 2 * l + 1, x)
