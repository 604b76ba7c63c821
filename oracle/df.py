"""Metric, DF energy, J and K — oracle restatement.

Test infrastructure only (see the package docstring).

* ``metric_pinv``: ``dftax/ks/terms.py:155-192`` — V+ = U diag(1/w) U^T over
  the eigenvalues w > 1e-7 * w_max (others dropped).
* ``metric_factor``: L = U diag(w^-1/2) over the same kept eigenvalues, so that
  V+ = L L^T exactly. This is the factor the library's B = (ij|P) L uses; it
  equals ``_rik_cholesky`` (``terms.py:391-395``) up to an orthogonal rotation
  of the fitted index, which J and K do not see.
* ``df_energy``: ``DFCoulomb.energy`` (``terms.py:592-613``) with
  ``_exchange_quadratic`` (``terms.py:500-509``).
* ``df_jk``: the analytic P-gradients of that energy: J = int3c (V+ gamma),
  gamma = int3c^T D; K = einsum("mlP,PQ,nsQ,ls->mn") (``dftax/energy/hybrid.py:23-41``).
* ``jk_from_b``: the same J, K from B: J = B (B^T D), K = sum_x (B_x C)(B_x C)^T.
* ``occ_orbitals``: ``_rik_occ_orbitals`` (``terms.py:369-388``).
"""

from __future__ import annotations

import numpy as np

CUTOFF = 1e-7


def metric_pinv(V):
    w, U = np.linalg.eigh(V)
    inv = np.where(w > CUTOFF * w[-1], 1.0 / w, 0.0)
    return (U * inv) @ U.T


def metric_factor(V):
    w, U = np.linalg.eigh(V)
    keep = w > CUTOFF * w[-1]
    return U[:, keep] / np.sqrt(w[keep])


def rik_cholesky(vinv):
    w, U = np.linalg.eigh(vinv)
    return U * np.sqrt(np.clip(w, 0.0, None))


def exchange_quadratic(kfun, P, ax):
    if P.shape[0] == 1:
        return -0.25 * ax * np.sum(P[0] * kfun(P[0]))
    return -0.5 * ax * sum(np.sum(Ps * kfun(Ps)) for Ps in P)


def df_k(int3c, vinv, Q):
    return np.einsum("mlP,PQ,nsQ,ls->mn", int3c, vinv, int3c, Q, optimize=True)


def df_energy(int3c, vinv, P, hf_coeff, int3c_lr=None, vinv_lr=None, hf_coeff_lr=0.0):
    """E_J + a_x E_K (+ a_lr E_K[erf(omega r)/r]) for the spin-stacked density P
    (nspin, nao, nao): ``DFCoulomb.energy`` (terms.py:592-613)."""
    Ptot = P.sum(0)
    gamma = np.einsum("mnP,mn->P", int3c, Ptot)
    e = 0.5 * gamma @ (vinv @ gamma)
    if hf_coeff != 0.0:
        e = e + exchange_quadratic(lambda Q: df_k(int3c, vinv, Q), P, hf_coeff)
    if hf_coeff_lr != 0.0:
        e = e + exchange_quadratic(lambda Q: df_k(int3c_lr, vinv_lr, Q), P, hf_coeff_lr)
    return float(e)


def df_jk(int3c, vinv, D):
    gamma = np.einsum("mnP,mn->P", int3c, D)
    J = np.einsum("mnP,P->mn", int3c, vinv @ gamma)
    return J, df_k(int3c, vinv, D)


def jk_from_b(B, C):
    """J[D], K[D] for D = C C^T from B (nao, nao, nfit)."""
    D = C @ C.T
    g = np.einsum("mnx,mn->x", B, D)
    J = np.einsum("mnx,x->mn", B, g)
    X = np.einsum("mnx,ni->mix", B, C)
    K = np.einsum("mix,nix->mn", X, X)
    return J, K


def fock_2e(J, K, hf_coeff, nspin=1):
    """Two-electron part of the closed-shell Fock, dE/dP = J - (a_x/2) K with J, K of P."""
    return J - 0.5 * hf_coeff * K


def occ_orbitals(P, S, nocc, dscale=0.5):
    sv, U = np.linalg.eigh(S)
    sv = np.clip(sv, 1e-12, None)
    s_ih = (U / np.sqrt(sv)) @ U.T
    s_h = (U * np.sqrt(sv)) @ U.T
    _, ev = np.linalg.eigh(s_h @ (dscale * P) @ s_h)
    return s_ih @ ev[:, ev.shape[1] - nocc:]
