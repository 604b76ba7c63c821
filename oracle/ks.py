"""Kohn-Sham energy, Fock matrix and SCF around the DF Coulomb term — oracle
restatement. TEST INFRASTRUCTURE ONLY (see the package docstring).

* ``one_electron``: S, T (``dftax/integrals/eri3c_bucketed.py:577-694``,
  overlap and kinetic per shell pair; T = b (2 L_b + 3) S - 2 b^2 sum_x
  S(a, b + 2_x) - 1/2 sum_x b_x (b_x - 1) S(a, b - 2_x)) and V
  (``:486-574``, V = -sum_C Z_C K_AB 2 pi / p sum_tuv E_t E_u E_v R_tuv(p,
  P - C)), then C^T M C with the basis's cart2sph;
* ``nuclear_repulsion``: ``dftax/integrals/nuclear_repulsion.py``;
* ``becke_grid``: ``dftax/grid/grid.py:139-255`` and ``becke.py`` (Becke
  radial shells r = R (1+x)/(1-x) at second-kind Chebyshev nodes, R the Bragg
  radius (half of it except for H), NWChem angular pruning by r / R_Bragg,
  shells past r_max dropped, Lebedev angular rules (SciPy's), fuzzy-Voronoi
  cell functions with the Bragg-radius size adjustment), then the 1e-15
  weight cutoff of ``KS`` (``energy.py:229-256``);
* ``eval_ao``: ``dftax/energy/gto.py:371-412`` (values) and their analytic
  gradients;
* ``exc_pbe0``: ``xc.py:87-252`` and ``:584-601`` (PBE exchange and PW92 +
  PBE correlation, 0.75 exchange) integrated as ``grid.py:10-45`` does (points
  with rho <= 1e-10 masked). Written with torch (float64) so that its
  gradient, the XC Fock matrix, is the autodiff gradient of the same
  expression, as dftax's Fock is (``scf.py:42-46``);
* ``scf``: ``dftax/ks/scf.py:279-391`` for a closed shell: canonical
  orthonormalizer (``:73-90``), core-Hamiltonian guess (``guess.py:605-606``),
  Pulay DIIS over a circular buffer with the 1e-10 ridge (``:245-273``),
  convergence on |dE| < e_tol and the commutator norm < d_tol.
"""

from __future__ import annotations

import math

import numpy as np

from . import df as odf
from . import md as omd

# Bragg-Slater radii of H..Ne in Bohr, rounded to 8 decimals as dftax
# tabulates them (becke.py: BRAGG_BOHR; 0.35, 1.40, 1.45, 1.05, 0.85, 0.70,
# 0.65, 0.60, 0.50, 1.50 Angstrom): the radial scale and the partition use
# these rounded values, so the grid reproduces dftax's only with them.
_BRAGG_BOHR = {1: 0.66140414, 2: 2.64561657, 3: 2.74010288, 4: 1.98421243, 5: 1.60626721,
               6: 1.32280829, 7: 1.22832198, 8: 1.13383567, 9: 0.94486306, 10: 2.83458919}
ANG = 1.0 / 0.529177210903
Z_OF = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10}
LEBEDEV_LADDER = (6, 14, 26, 38, 50, 74, 86, 110, 146, 170, 194, 230, 266, 302, 350, 434, 590,
                  770)
_NWCHEM_ALPHAS = np.array(((0.25, 0.5, 1.0, 4.5), (0.1667, 0.5, 0.9, 3.5), (0.1, 0.4, 0.8, 2.5)))


def bragg_radius(Z: int) -> float:
    return _BRAGG_BOHR[Z]


# ---------------------------------------------------------------------------
# one-electron integrals
# ---------------------------------------------------------------------------

def _shell_list(basis):
    sh = omd.shells(basis)
    ex = np.asarray(basis.exponents)
    co = np.asarray(basis.coefficients)
    ang = np.asarray(basis.angular)
    out = []
    for (l, r0, nc, npr) in sh:
        out.append((l, r0, nc, np.asarray(basis.centers)[r0], ex[r0, :npr], co[r0:r0 + nc, :npr],
                    [tuple(a) for a in ang[r0:r0 + nc]]))
    return out


def one_electron(basis, coords, charges):
    """(S, T, V) spherical (or cartesian without cart2sph)."""
    sh = _shell_list(basis)
    n = np.asarray(basis.angular).shape[0]
    S = np.zeros((n, n))
    T = np.zeros((n, n))
    V = np.zeros((n, n))
    coords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    charges = np.asarray(charges, dtype=np.float64)
    for ia, (la, ra, nca, A, ea, ca, anga) in enumerate(sh):
        for ib in range(ia, len(sh)):
            lb, rb, ncb, B, eb, cb, angb = sh[ib]
            AB = A - B
            ab2 = float(AB @ AB)
            s_blk = np.zeros((nca, ncb))
            t_blk = np.zeros((nca, ncb))
            v_blk = np.zeros((nca, ncb))
            mt = la + lb + 3
            for pa in range(len(ea)):
                for pb in range(len(eb)):
                    a, b = ea[pa], eb[pb]
                    p = a + b
                    P = (a * A + b * B) / p
                    K = math.exp(-a * b / p * ab2)
                    E = [omd.e_table(la, lb + 2, np.array([a]), np.array([b]), np.array([AB[x]]),
                                     mt)[0] for x in range(3)]
                    pref = (math.pi / p) ** 1.5 * K
                    mtv = la + lb + 1
                    R = sum(-Z * omd.hermite_r(np.array([p]), (P - C)[None], max(mtv, 2))[0]
                            for C, Z in zip(coords, charges))
                    for i, (ax, ay, az) in enumerate(anga):
                        for j, (bx, by, bz) in enumerate(angb):
                            def s1(x, ai, bi):
                                return E[x][ai, bi, 0] if bi >= 0 else 0.0
                            sx, sy, sz = s1(0, ax, bx), s1(1, ay, by), s1(2, az, bz)
                            sval = sx * sy * sz
                            up = (s1(0, ax, bx + 2) * sy * sz + sx * s1(1, ay, by + 2) * sz
                                  + sx * sy * s1(2, az, bz + 2))
                            dn = (bx * (bx - 1) * s1(0, ax, bx - 2) * sy * sz
                                  + by * (by - 1) * sx * s1(1, ay, by - 2) * sz
                                  + bz * (bz - 1) * sx * sy * s1(2, az, bz - 2))
                            lbt = bx + by + bz
                            w = ca[i, pa] * cb[j, pb]
                            s_blk[i, j] += w * pref * sval
                            t_blk[i, j] += w * pref * (b * (2 * lbt + 3) * sval - 2.0 * b * b * up
                                                       - 0.5 * dn)
                            acc = 0.0
                            for t in range(ax + bx + 1):
                                for u in range(ay + by + 1):
                                    for v in range(az + bz + 1):
                                        acc += E[0][ax, bx, t] * E[1][ay, by, u] * E[2][az, bz, v] \
                                            * R[t, u, v]
                            v_blk[i, j] += w * K * 2.0 * math.pi / p * acc
            for M, blk in ((S, s_blk), (T, t_blk), (V, v_blk)):
                M[ra:ra + nca, rb:rb + ncb] = blk
                M[rb:rb + ncb, ra:ra + nca] = blk.T
    if basis.cart2sph is not None:
        C2 = np.asarray(basis.cart2sph)
        S, T, V = (C2.T @ M @ C2 for M in (S, T, V))
    return S, T, V


def nuclear_repulsion(coords, charges):
    coords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    e = 0.0
    for i in range(len(charges)):
        for j in range(i):
            e += charges[i] * charges[j] / np.linalg.norm(coords[i] - coords[j])
    return float(e)


# ---------------------------------------------------------------------------
# Becke grid
# ---------------------------------------------------------------------------

def becke_radial(n, scale):
    i = np.arange(1, n + 1)
    theta = i * np.pi / (n + 1)
    x = np.cos(theta)
    r = scale * (1.0 + x) / (1.0 - x)
    drdx = 2.0 * scale / (1.0 - x) ** 2
    w = (np.pi / (n + 1)) * np.sin(theta) * r ** 2 * drdx
    return r, w


def nwchem_orders(Z, r, n_ang):
    if n_ang < 50:
        return np.full(r.shape[0], n_ang, dtype=np.int64)
    ladder = np.asarray(LEBEDEV_LADDER[3:])
    if n_ang == 50:
        leb_l = np.array([1, 2, 2, 2, 1])
    else:
        idx = int(np.where(ladder == n_ang)[0][0])
        leb_l = np.array([1, 3, idx - 1, idx, idx - 1])
    row = 0 if Z <= 2 else (1 if Z <= 10 else 2)
    place = (r[:, None] / bragg_radius(Z) > _NWCHEM_ALPHAS[row]).sum(axis=1)
    return ladder[leb_l[place]]


def lebedev(npts):
    """Unit-sphere Lebedev points (n, 3) and weights summing to 4 pi (SciPy)."""
    from scipy.integrate import lebedev_rule

    order = {6: 3, 14: 5, 26: 7, 38: 9, 50: 11, 74: 13, 86: 15, 110: 17, 146: 19, 170: 21,
             194: 23, 230: 25, 266: 27, 302: 29, 350: 31, 434: 35, 590: 41, 770: 47}[int(npts)]
    x, w = lebedev_rule(order)
    return np.ascontiguousarray(x.T), np.asarray(w)


def becke_partition(points, coords, Zs):
    """Unnormalized cell functions P_A(point), (n, natom)."""
    coords = np.asarray(coords)
    nat = coords.shape[0]
    bragg = np.array([bragg_radius(z) for z in Zs])
    RAB = np.sqrt(np.sum((coords[:, None] - coords[None]) ** 2, axis=2) + np.eye(nat))
    chi = bragg[:, None] / bragg[None, :]
    u = (chi - 1.0) / (chi + 1.0)
    a = np.clip(u / (u * u - 1.0), -0.45, 0.45)
    out = np.empty((points.shape[0], nat))
    for s in range(0, points.shape[0], 4096):
        p = points[s:s + 4096]
        rA = np.sqrt(np.sum((p[:, None, :] - coords[None]) ** 2, axis=2) + 1e-30)
        mu = (rA[:, :, None] - rA[:, None, :]) / RAB
        nu = mu + a * (1.0 - mu * mu)
        f = nu
        for _ in range(3):
            f = 1.5 * f - 0.5 * f ** 3
        sv = 0.5 * (1.0 - f)
        sv[:, np.arange(nat), np.arange(nat)] = 1.0
        out[s:s + 4096] = np.prod(sv, axis=2)
    return out


def becke_grid(symbols, coords, n_radial=75, n_ang=302, prune="nwchem", r_max=45.0,
               cutoff=1e-15):
    coords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    Zs = [Z_OF[s] for s in symbols]
    pts_all, w_all = [], []
    for A, Z in enumerate(Zs):
        scale = bragg_radius(Z) if Z == 1 else 0.5 * bragg_radius(Z)
        r, wr = becke_radial(n_radial, scale)
        if r_max is not None:
            keep = r <= r_max
            r, wr = r[keep], wr[keep]
        orders = nwchem_orders(Z, r, n_ang) if prune == "nwchem" else np.full(len(r), n_ang)
        pts, raw = [], []
        for i in range(len(r)):
            u, w = lebedev(int(orders[i]))
            pts.append(coords[A] + r[i] * u)
            raw.append(wr[i] * w)
        pts = np.concatenate(pts)
        raw = np.concatenate(raw)
        P = becke_partition(pts, coords, Zs)
        pts_all.append(pts)
        w_all.append(raw * P[:, A] / P.sum(axis=1))
    pts = np.concatenate(pts_all)
    w = np.concatenate(w_all)
    if cutoff is not None:
        keep = np.abs(w) > cutoff
        pts, w = pts[keep], w[keep]
    return pts, w


# ---------------------------------------------------------------------------
# AO values and PBE0
# ---------------------------------------------------------------------------

def eval_ao(basis, pts):
    """(ng, nao) values and (ng, nao, 3) gradients at the points."""
    cen = np.asarray(basis.centers)
    ex = np.asarray(basis.exponents)
    co = np.asarray(basis.coefficients)
    ang = np.asarray(basis.angular)
    dr = pts[:, None, :] - cen[None]                       # (g, n, 3)
    r2 = np.sum(dr * dr, axis=2)
    e = np.exp(-ex[None] * r2[:, :, None])                 # (g, n, p)
    rad = np.sum(co[None] * e, axis=2)
    drad = np.sum(-2.0 * ex[None] * co[None] * e, axis=2)  # d rad / d(r2) * 2 -> per-axis x dr
    pw = [np.where(ang[None, :, x] > 0, dr[:, :, x] ** np.maximum(ang[None, :, x], 0), 1.0)
          for x in range(3)]
    angular = pw[0] * pw[1] * pw[2]
    val = angular * rad
    grad = np.zeros(val.shape + (3,))
    for x in range(3):
        lx = ang[None, :, x]
        dpow = np.where(lx > 0, lx * dr[:, :, x] ** np.maximum(lx - 1, 0), 0.0)
        others = np.prod([pw[y] for y in range(3) if y != x], axis=0)
        grad[:, :, x] = dpow * others * rad + angular * drad * dr[:, :, x]
    if basis.cart2sph is not None:
        C2 = np.asarray(basis.cart2sph)
        val = val @ C2
        grad = np.einsum("gnx,nm->gmx", grad, C2)
    return val, grad


def pbe0_eps(torch, rho, grad, xs=0.75, cs=1.0):
    """eps_xc per particle of xs PBE exchange + cs PBE correlation (PBE0 by
    default, as dftax's PBE0.__call__; PBE with xs = 1), unpolarized."""
    pi = math.pi
    kappa, mu = 0.804, 0.2195149727645171
    gnorm = torch.linalg.norm(grad + 1e-30, dim=-1)
    kF = (3 * pi ** 2 * rho + 1e-30) ** (1 / 3)
    s = gnorm / torch.clamp(2 * kF * rho, min=1e-30)
    ex = -3 * kF / (4 * pi) * (1 + kappa - kappa / (1 + mu * s ** 2 / kappa))
    # PBE correlation (PW92 paramagnetic channel; zeta = 0, phi = 1)
    gamma = (1.0 - math.log(2.0)) / (pi ** 2)
    beta = 0.06672455060314922
    A, a1, b1, b2, b3, b4 = 0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    rt = torch.clamp(rho, min=1e-20)
    rs = (3 / (4 * pi * rt) + 1e-20) ** (1 / 3)
    rss = torch.sqrt(rs)
    den = 2.0 * A * (b1 * rss + b2 * rs + b3 * rs * rss + b4 * rs ** 2)
    eps_pw = -2.0 * A * (1.0 + a1 * rs) * torch.log1p(1 / torch.clamp(den, min=1e-20))
    kf = (3 * pi ** 2 * rt + 1e-20) ** (1 / 3)
    ks = torch.sqrt(4 * kf / pi)
    gn = torch.sqrt(torch.sum(grad ** 2, dim=-1) + 1e-30)
    t = gn / torch.clamp(2 * ks * rt, min=1e-20)
    dA = gamma * torch.expm1(-eps_pw / gamma)
    Ac = beta / torch.clamp(dA, min=1e-20)
    f1 = t ** 2 + Ac * t ** 4
    frac = beta * f1 / torch.clamp(gamma * (1.0 + Ac * f1), min=1e-20)
    H = gamma * torch.log1p(frac)
    return xs * ex + cs * (eps_pw + H)


def exc_and_vxc(basis, pts, w, P, ao=None, xs=0.75, cs=1.0):
    """E_xc of PBE0 for the closed-shell density P and its P-gradient V_xc,
    symmetrized like dftax's Fock (scf.py:42-46)."""
    import torch

    if ao is None:
        ao = eval_ao(basis, pts)
    val, grad = ao
    t = torch
    phi = t.as_tensor(val)
    dphi = t.as_tensor(grad)
    Pt = t.as_tensor(np.asarray(P, dtype=np.float64)).clone().requires_grad_(True)
    rho = t.einsum("gm,mn,gn->g", phi, Pt, phi)
    grho = 2.0 * t.einsum("gm,mn,gnx->gx", phi, Pt, dphi)
    mask = rho > 1e-10
    safe_rho = t.where(mask, rho, t.ones_like(rho))
    safe_grad = t.where(mask[:, None], grho, t.zeros_like(grho))
    eps = pbe0_eps(t, safe_rho, safe_grad, xs, cs)
    wt = t.as_tensor(np.asarray(w, dtype=np.float64))
    e = t.sum(t.where(mask, wt * eps * rho, t.zeros_like(rho)))
    e.backward()
    g = Pt.grad.numpy()
    return float(e.detach()), 0.5 * (g + g.T)


# ---------------------------------------------------------------------------
# closed-shell SCF
# ---------------------------------------------------------------------------

def canonical_orthonormalizer(S, thresh=1e-7):
    s, U = np.linalg.eigh(S)
    keep = s > thresh
    return U[:, keep] / np.sqrt(s[keep])


def _diis(dF, dE, count, m):
    errs = dE.reshape(m, -1)
    B = errs @ errs.T
    valid = np.arange(m) < count
    vv = valid[:, None] & valid[None, :]
    B = np.where(vv, B, np.eye(m))
    B = B + 1e-10 * np.diag(valid.astype(float))
    A = np.zeros((m + 1, m + 1))
    A[:m, :m] = B
    border = np.where(valid, -1.0, 0.0)
    A[:m, m] = border
    A[m, :m] = border
    rhs = np.zeros(m + 1)
    rhs[m] = -1.0
    c = np.linalg.solve(A, rhs)[:m]
    return np.einsum("i,iab->ab", c, dF)


class KSEnergy:
    """E(P) and F(P) of a closed-shell DF-PBE0 Kohn-Sham model (nspin = 1)."""

    def __init__(self, orb, aux, coords, charges, pts, w, hf_coeff=0.25, I3=None, vinv=None,
                 xs=0.75, cs=1.0):
        self.S, T, V = one_electron(orb, coords, charges)
        self.hcore = T + V
        self.e_nn = nuclear_repulsion(coords, charges)
        self.I3 = omd.eri3c(orb, aux) if I3 is None else I3
        self.vinv = odf.metric_pinv(omd.eri2c(aux)) if vinv is None else vinv
        self.pts, self.w = pts, w
        self.ao = eval_ao(orb, pts)
        self.orb = orb
        self.hf = hf_coeff
        self.xs, self.cs = xs, cs

    def energy_fock(self, P):
        e1 = float(np.sum(P * self.hcore))
        e2 = odf.df_energy(self.I3, self.vinv, P[None], self.hf)
        J, _ = odf.df_jk(self.I3, self.vinv, P)
        K = odf.df_k(self.I3, self.vinv, P)
        if self.xs == 0.0 and self.cs == 0.0:
            exc, vxc = 0.0, np.zeros_like(P)
        else:
            exc, vxc = exc_and_vxc(self.orb, self.pts, self.w, P, self.ao, self.xs, self.cs)
        F = self.hcore + J - 0.5 * self.hf * K + vxc
        return e1 + e2 + exc + self.e_nn, 0.5 * (F + F.T)


def scf(ks: KSEnergy, nocc, max_iter=128, e_tol=1e-8, d_tol=1e-6, m=8, P0=None,
        level_shift=0.0):
    """(e_tot, P, eps, C, n_iter, converged) of the closed-shell SCF."""
    S = ks.S
    X = canonical_orthonormalizer(S)
    nao, nmo = X.shape

    def make_density(F):
        eps, Cp = np.linalg.eigh(X.T @ F @ X)
        C = X @ Cp
        Co = C[:, :nocc]
        return 2.0 * Co @ Co.T, C, eps

    P = make_density(ks.hcore)[0] if P0 is None else P0
    e_prev, F = ks.energy_fock(P)
    dF = np.zeros((m, nao, nao))
    dE = np.zeros((m, nmo, nmo))
    C = eps = None
    it, converged = 0, False
    while it < max_iter and not converged:
        err = X.T @ (F @ P @ S - S @ P @ F) @ X
        derr = float(np.linalg.norm(err))
        slot = it % m
        dF[slot] = F
        dE[slot] = err
        F_ext = _diis(dF, dE, min(it + 1, m), m)
        F_ls = F_ext + level_shift * (S - 0.5 * (S @ P @ S))
        P, C, eps = make_density(F_ls)
        e, F = ks.energy_fock(P)
        converged = abs(e - e_prev) < e_tol and derr < d_tol
        e_prev = e
        it += 1
    return e_prev, P, eps, C, it, converged


__all__ = ["one_electron", "nuclear_repulsion", "becke_grid", "lebedev", "eval_ao",
           "exc_and_vxc", "pbe0_eps", "KSEnergy", "scf", "canonical_orthonormalizer"]
