"""Boys function F_n(t) — oracle restatement of ``dftax/energy/boys.py``.

Test infrastructure only (see the package docstring).

Scheme (``boys.py:33-36``, ``:81-176``): a table of F_0..F_24 on the grid
t_j = 0.1 j, j = 0..400, built in float64 by an ascending series at a high
order followed by the downward recursion; evaluation at t < 40 takes the
nearest node and a degree-6 Taylor expansion in dx = t_j - t whose
coefficients are the higher orders at that node; t >= 40 uses the asymptotic
Gamma(n+1/2) / (2 t^{n+1/2}); orders with n + 6 > 24 use the exact form (a
28-term series for t < 1, the regularized incomplete gamma otherwise).
"""

from __future__ import annotations

import math

import numpy as np
from scipy.special import gammainc, gammaln

ORDER = 6
DT = 0.1
TMAX = 40.0
TBL_NMAX = 24
NGRID = int(round(TMAX / DT)) + 1


def build_table() -> np.ndarray:
    """(NGRID, TBL_NMAX+1) float64 table of F_n(t_j)  (``boys.py:81-123``)."""
    t = np.arange(NGRID, dtype=np.float64) * DT
    two_t = 2.0 * t
    emt = np.exp(-t)
    top = max(TBL_NMAX, int(TMAX)) + 20
    # F_top(t) = e^{-t} sum_k (2t)^k / ((2top+1)(2top+3)...(2top+2k+1))
    term = np.full(NGRID, 1.0 / (2 * top + 1))
    acc = term.copy()
    for k in range(1, 500):
        term = term * two_t / (2 * top + 2 * k + 1)
        acc += term
        if np.max(term) <= 1e-18 * np.min(acc):
            break
    f = emt * acc
    cols = [None] * (TBL_NMAX + 1)
    for n in range(top, 0, -1):
        if n <= TBL_NMAX:
            cols[n] = f
        f = (two_t * f + emt) / (2 * n - 1)
    cols[0] = f
    return np.stack(cols, axis=1)


TABLE = build_table()


def boys_exact(n: int, t) -> np.ndarray:
    """Exact F_n(t) (``boys.py:39-78``)."""
    t = np.asarray(t, dtype=np.float64)
    a = n + 0.5
    safe = np.where(t < 1.0, 1.0, t)
    big = 0.5 * np.exp(gammaln(a) + np.log(np.maximum(gammainc(a, safe), np.finfo(float).tiny))
                       - a * np.log(safe))
    small = np.full_like(t, 1.0 / (2 * n + 1))
    for k in range(1, 28):
        small = small + (-t) ** k / (math.factorial(k) * (2 * n + 2 * k + 1))
    return np.where(t < 1.0, small, big)


def boys(n: int, t) -> np.ndarray:
    """Fast F_n(t) by the table scheme (``boys.py:130-176``)."""
    if n + ORDER > TBL_NMAX:
        return boys_exact(n, t)
    t = np.asarray(t, dtype=np.float64)
    tt = np.minimum(t, TMAX)
    j = np.clip(np.round(tt / DT).astype(np.int64), 0, NGRID - 1)
    dx = j.astype(np.float64) * DT - tt
    acc = TABLE[j, n + ORDER]
    for k in range(ORDER - 1, -1, -1):
        acc = TABLE[j, n + k] + acc * dx / (k + 1)
    a = n + 0.5
    ta = np.maximum(t, TMAX)
    asy = 0.5 * math.exp(math.lgamma(a)) * ta ** (-a)
    return np.where(t < TMAX, acc, asy)


def boys_all(nmax: int, t) -> np.ndarray:
    """Stack F_0..F_nmax at t: shape (nmax+1, *t.shape)."""
    return np.stack([boys(n, t) for n in range(nmax + 1)])
