"""McMurchie-Davidson 3-center / 2-center integrals — oracle restatement.

Test infrastructure only (see the package docstring).

Follows ``dftax/integrals/eri3c_bucketed.py``:
  * shells from static metadata: a shell starts where the component sequence
    restarts at (l, 0, 0) (``:119-137``); spherical row starts (``:172-183``);
  * bra shell pairs ia <= ib times every auxiliary shell, bucketed by
    (la, lb, lc) (``plan_eri3c`` ``:221-283``), optionally restricted to the
    Schwarz-kept pairs (``_shell_pair_keep`` ``:140-169``);
  * two-center E tables by the MD recursion (``_bump``/``_E_table``
    ``:290-313``), single-center aux tables with X_PA = 0 (``_Ec_table``
    ``:316-323``) signed by (-1)^t (``:409``);
  * Hermite R^0_{tuv} by the descending m-ladder from
    R^m_000 = (-2 rho)^m F_m(rho |PC|^2) (``_hermite_table`` ``:326-369``);
  * (ab|c) = K_AB 2 pi^{5/2} / (g_ab g_c sqrt(g_ab + g_c))
    * sum_{srq} GX GY GZ R with G_x[i,j,k,s] = sum_{t+tau=s} E^{ab}_t E^c_tau
    (``_make_class_kernel`` ``:376-426``), contracted over primitives with the
    per-component coefficients;
  * cart -> sph per block with one (ncart, 2l+1) slice per l of the basis's
    own cart2sph, written to the (ab) block and its (ba) transpose
    (``eri3c_matrix_bucketed`` ``:782-854``);
  * (P|Q) = 2 pi^{5/2} / (a b sqrt(a+b)) sum F_x F_y F_z R(rho = ab/(a+b), A-B)
    with single-center tables on both sides, mirrored, then C^T V C
    (``_make_eri2c_kernel`` ``:697-734``, ``eri2c_matrix_bucketed`` ``:746-779``).

Everything is vectorized over the shell triples of one class with numpy, in
chunks that bound the intermediate size.
"""

from __future__ import annotations

import math
from collections import defaultdict

import numpy as np

from .boys import boys

TWO_PI_2_5 = 2.0 * math.pi ** 2.5


# ---------------------------------------------------------------------------
# Static shell metadata
# ---------------------------------------------------------------------------

def shells(basis):
    """[(l, row0, ncomp, nprim)] in row order (``eri3c_bucketed.py:119-137``)."""
    ang = np.asarray(basis.angular)
    ex = np.asarray(basis.exponents)
    lt = ang.sum(1)
    n = ang.shape[0]
    starts = [i for i in range(n) if ang[i, 0] == lt[i] and ang[i, 1] == 0 and ang[i, 2] == 0]
    if not starts or starts[0] != 0:
        raise ValueError("basis rows do not start shells at (l,0,0)")
    b = starts + [n]
    return [(int(lt[s]), s, e - s, max(1, int((ex[s] != 0).sum()))) for s, e in zip(b[:-1], b[1:])]


def sph_starts(sh, cart2sph):
    starts, acc = [], 0
    for (l, _r, nc, _p) in sh:
        starts.append(acc)
        acc += (2 * l + 1) if cart2sph is not None else nc
    return np.array(starts, dtype=np.int64), acc


def _block(cart2sph, row0, s0, l, nc):
    if cart2sph is None:
        return np.eye(nc)
    return np.asarray(cart2sph)[row0:row0 + nc, s0:s0 + 2 * l + 1]


# ---------------------------------------------------------------------------
# MD tables (vectorized over a leading batch axis)
# ---------------------------------------------------------------------------

def _bump(row, X, i2g):
    """One E-recursion step: new_t = X row_t + i2g row_{t-1} + (t+1) row_{t+1}."""
    mt = row.shape[-1]
    out = X[..., None] * row
    out[..., 1:] += i2g[..., None] * row[..., :-1]
    out[..., :-1] += np.arange(1, mt) * row[..., 1:]
    return out


def e_table(la, lb, a, b, xab, mt):
    """(T, la+1, lb+1, mt) two-center Hermite expansion coefficients."""
    g = a + b
    i2g = 0.5 / g
    xpa = -b * xab / g
    xpb = a * xab / g
    T = a.shape[0]
    E = np.zeros((T, la + 1, lb + 1, mt))
    E[:, 0, 0, 0] = 1.0
    for i in range(la):
        E[:, i + 1, 0] = _bump(E[:, i, 0], xpa, i2g)
    for j in range(lb):
        E[:, :, j + 1] = _bump(E[:, :, j], xpb[:, None], i2g[:, None])
    return E


def ec_table(lc, g, mt):
    """(T, lc+1, mt) single-center table (X_PA = 0)."""
    T = g.shape[0]
    i2g = 0.5 / g
    E = np.zeros((T, lc + 1, mt))
    E[:, 0, 0] = 1.0
    zero = np.zeros(T)
    for i in range(lc):
        E[:, i + 1] = _bump(E[:, i], zero, i2g)
    return E


def hermite_r(rho, pc, mt, omega=None):
    """(T, mt, mt, mt) R^0_{tuv} by the descending m-ladder.

    ``omega``: the long-range erf(omega r)/r operator, whose base values are
    s^(m+1/2) F_m(s T) with s = omega^2 / (omega^2 + rho)
    (``eri3c_bucketed.py:342-346``)."""
    T = rho.shape[0]
    targ = rho * np.einsum("ti,ti->t", pc, pc)
    m2r = -2.0 * rho
    if omega is None:
        base = [m2r ** m * boys(m, targ) for m in range(mt)]
    else:
        sat = omega * omega / (omega * omega + rho)
        base = [m2r ** m * sat ** (m + 0.5) * boys(m, sat * targ) for m in range(mt)]
    R = np.zeros((T, mt, mt, mt))
    R[:, 0, 0, 0] = base[mt - 1]
    idx = np.arange(mt - 1, dtype=np.float64)
    X, Y, Z = pc[:, 0], pc[:, 1], pc[:, 2]
    for m in range(mt - 2, -1, -1):
        Rn = np.zeros_like(R)
        Rn[:, 0, 0, 0] = base[m]
        # t direction (u = v = 0)
        prev = np.concatenate([np.zeros((T, 1)), R[:, :-2, 0, 0]], axis=1)
        Rn[:, 1:, 0, 0] = X[:, None] * R[:, :-1, 0, 0] + idx * prev
        # u direction (all t, v = 0)
        prev = np.concatenate([np.zeros((T, mt, 1)), R[:, :, :-2, 0]], axis=2)
        Rn[:, :, 1:, 0] = Y[:, None, None] * R[:, :, :-1, 0] + idx[None, :] * prev
        # v direction (all t, u)
        prev = np.concatenate([np.zeros((T, mt, mt, 1)), R[:, :, :, :-2]], axis=3)
        Rn[:, :, :, 1:] = Z[:, None, None, None] * R[:, :, :, :-1] + idx * prev
        R = Rn
    return R


def _conv(Eab, Ec, mt):
    """G[t_, i, j, k, s] = sum_{t + tau = s} Eab[i, j, t] Ec[k, tau] (-1)^tau."""
    sign = (-1.0) ** np.arange(mt)
    Ecs = Ec * sign
    T, ni, nj, _ = Eab.shape
    nk = Ec.shape[1]
    G = np.zeros((T, ni, nj, nk, mt))
    for t in range(mt):
        for tau in range(mt - t):
            G[..., t + tau] += Eab[:, :, :, t, None] * Ecs[:, None, None, :, tau]
    return G


# ---------------------------------------------------------------------------
# 3-center (ab|c) for one class, cartesian, over a batch of triples
# ---------------------------------------------------------------------------

def _class_cart(la, lb, lc, anga, angb, angc, A, B, C, ea, eb, ec, ca, cb, cc, omega=None):
    """(T, nca, ncb, ncc) contracted cartesian integrals of one class."""
    mt = max(la + lb + lc + 1, 2)
    T = A.shape[0]
    nca, ncb, ncc = len(anga), len(angb), len(angc)
    out = np.zeros((T, nca, ncb, ncc))
    AB = A - B
    ab2 = np.einsum("ti,ti->t", AB, AB)
    ia = [np.array([c[x] for c in anga]) for x in range(3)]
    jb = [np.array([c[x] for c in angb]) for x in range(3)]
    kc = [np.array([c[x] for c in angc]) for x in range(3)]
    for pa in range(ea.shape[1]):
        for pb in range(eb.shape[1]):
            al = ea[:, pa]
            be = eb[:, pb]
            g = al + be
            g = np.where(g == 0.0, 1.0, g)
            P = (al[:, None] * A + be[:, None] * B) / g[:, None]
            K = np.exp(-al * be / g * ab2)
            Et = [e_table(la, lb, np.where(al == 0, 0.5, al), np.where(be == 0, 0.5, be),
                          AB[:, x], mt) for x in range(3)]
            for pc in range(ec.shape[1]):
                gc = ec[:, pc]
                gc = np.where(gc == 0.0, 1.0, gc)
                rho = g * gc / (g + gc)
                pref = K * TWO_PI_2_5 / (g * gc * np.sqrt(g + gc))
                R = hermite_r(rho, P - C, mt, omega)
                Ec = ec_table(lc, gc, mt)
                G = [_conv(Et[x], Ec, mt) for x in range(3)]
                GX = G[0][:, ia[0][:, None, None], jb[0][None, :, None], kc[0][None, None, :], :]
                GY = G[1][:, ia[1][:, None, None], jb[1][None, :, None], kc[1][None, None, :], :]
                GZ = G[2][:, ia[2][:, None, None], jb[2][None, :, None], kc[2][None, None, :], :]
                tmp = np.einsum("tabcq,tsrq->tabcsr", GZ, R)
                v = np.einsum("tabcsr,tabcs,tabcr->tabc", tmp, GX, GY)
                w = (ca[:, :, pa][:, :, None, None] * cb[:, :, pb][:, None, :, None]
                     * cc[:, :, pc][:, None, None, :])
                out += pref[:, None, None, None] * v * w
    return out


def plan_eri3c(orb, aux, keep_pairs=None):
    """Class buckets {(la, lb, lc): (ia, ib, kc) int arrays} (``:221-283``)."""
    sb = shells(orb)
    sa = shells(aux)
    buckets = defaultdict(lambda: ([], [], []))
    lo = np.array([s[0] for s in sb])
    lx = np.array([s[0] for s in sa])
    ia, ib = np.triu_indices(len(sb))
    if keep_pairs is not None:
        keep = np.array([(int(a), int(b)) in keep_pairs for a, b in zip(ia, ib)], dtype=bool)
        ia, ib = ia[keep], ib[keep]
    out = {}
    for la in sorted(set(lo.tolist())):
        for lb in sorted(set(lo.tolist())):
            sel = (lo[ia] == la) & (lo[ib] == lb)
            if not sel.any():
                continue
            pa, pb = ia[sel], ib[sel]
            for lc in sorted(set(lx.tolist())):
                kc = np.nonzero(lx == lc)[0]
                A = np.repeat(pa, len(kc))
                B = np.repeat(pb, len(kc))
                Cc = np.tile(kc, len(pa))
                out[(la, lb, lc)] = (A, B, Cc)
    del buckets
    return out


def _gather(basis, sh, idx):
    """Per-triple shell data: centers, exponents (nprim), coefficients (ncomp, nprim)."""
    rows = np.array([sh[i][1] for i in idx], dtype=np.int64)
    npr = max(sh[i][3] for i in idx) if len(idx) else 1
    nc = sh[idx[0]][2]
    cen = np.asarray(basis.centers)[rows]
    ex = np.asarray(basis.exponents)[rows][:, :npr]
    co = np.stack([np.asarray(basis.coefficients)[rows + k][:, :npr] for k in range(nc)], axis=1)
    return cen, ex, co, rows


def eri3c(orb, aux, keep_pairs=None, chunk_elems=2_000_000, omega=None):
    """Dense (nao, nao, naux) spherical 3-center tensor (both bra triangles);
    ``omega`` selects the erf(omega r)/r operator."""
    sb, sa = shells(orb), shells(aux)
    _, nao = sph_starts(sb, orb.cart2sph)
    _, naux = sph_starts(sa, aux.cart2sph)
    out = np.zeros((nao, nao, naux))
    for ra, rb, rc, v in eri3c_blocks(orb, aux, keep_pairs, chunk_elems, omega):
        out[ra[:, :, None, None], rb[:, None, :, None], rc[:, None, None, :]] = v
        out[rb[:, None, :, None], ra[:, :, None, None], rc[:, None, None, :]] = v
    return out


def eri3c_blocks(orb, aux, keep_pairs=None, chunk_elems=2_000_000, omega=None):
    """Yield (rows_a, rows_b, cols, values) per chunk of shell triples of one
    class: values[t] is the spherical (na, nb, nc) block of triple t, written at
    rows_a[t] x rows_b[t] x cols[t] of the dense tensor."""
    sb, sa = shells(orb), shells(aux)
    sbs, _ = sph_starts(sb, orb.cart2sph)
    sas, _ = sph_starts(sa, aux.cart2sph)
    ang_o, ang_a = np.asarray(orb.angular), np.asarray(aux.angular)
    for (la, lb, lc), (IA, IB, KC) in plan_eri3c(orb, aux, keep_pairs).items():
        anga = [tuple(ang_o[sb[IA[0]][1] + i]) for i in range(sb[IA[0]][2])]
        angb = [tuple(ang_o[sb[IB[0]][1] + i]) for i in range(sb[IB[0]][2])]
        angc = [tuple(ang_a[sa[KC[0]][1] + i]) for i in range(sa[KC[0]][2])]
        mt = max(la + lb + lc + 1, 2)
        per = len(anga) * len(angb) * len(angc) * mt * mt * 2 + mt ** 3 * 4
        step = max(1, chunk_elems // per)
        Ta = _block(orb.cart2sph, sb[IA[0]][1], sbs[IA[0]], la, len(anga))
        Tb = _block(orb.cart2sph, sb[IB[0]][1], sbs[IB[0]], lb, len(angb))
        Tc = _block(aux.cart2sph, sa[KC[0]][1], sas[KC[0]], lc, len(angc))
        for s in range(0, len(IA), step):
            ia, ib, kc = IA[s:s + step], IB[s:s + step], KC[s:s + step]
            A, ea, ca, _ = _gather(orb, sb, ia)
            B, eb, cb, _ = _gather(orb, sb, ib)
            C, ec, cc, _ = _gather(aux, sa, kc)
            v = _class_cart(la, lb, lc, anga, angb, angc, A, B, C, ea, eb, ec, ca, cb, cc,
                            omega)
            v = np.einsum("tabc,ap,bq,cr->tpqr", v, Ta, Tb, Tc)
            na, nb, nc = v.shape[1:]
            ra = sbs[ia][:, None] + np.arange(na)
            rb = sbs[ib][:, None] + np.arange(nb)
            rc = sas[kc][:, None] + np.arange(nc)
            yield ra, rb, rc, v


# ---------------------------------------------------------------------------
# 2-center (P|Q)
# ---------------------------------------------------------------------------

def eri2c(aux, omega=None):
    """(naux, naux) spherical Coulomb metric (``eri3c_bucketed.py:697-779``);
    ``omega`` selects the erf(omega r)/r operator."""
    sa = shells(aux)
    ang = np.asarray(aux.angular)
    ncart = ang.shape[0]
    out = np.zeros((ncart, ncart))
    la_of = np.array([s[0] for s in sa])
    ia, ib = np.triu_indices(len(sa))
    for la in sorted(set(la_of.tolist())):
        for lb in sorted(set(la_of.tolist())):
            sel = (la_of[ia] == la) & (la_of[ib] == lb)
            if not sel.any():
                continue
            pa, pb = ia[sel], ib[sel]
            mt = max(la + lb + 1, 2)
            anga = [tuple(ang[sa[pa[0]][1] + i]) for i in range(sa[pa[0]][2])]
            angb = [tuple(ang[sa[pb[0]][1] + i]) for i in range(sa[pb[0]][2])]
            A, ea, ca, ra0 = _gather(aux, sa, pa)
            B, eb, cb, rb0 = _gather(aux, sa, pb)
            T = len(pa)
            val = np.zeros((T, len(anga), len(angb)))
            ix = [np.array([c[x] for c in anga]) for x in range(3)]
            jx = [np.array([c[x] for c in angb]) for x in range(3)]
            sign = (-1.0) ** np.arange(mt)
            for p1 in range(ea.shape[1]):
                for p2 in range(eb.shape[1]):
                    al = np.where(ea[:, p1] == 0, 1.0, ea[:, p1])
                    be = np.where(eb[:, p2] == 0, 1.0, eb[:, p2])
                    rho = al * be / (al + be)
                    pref = TWO_PI_2_5 / (al * be * np.sqrt(al + be))
                    Ea = ec_table(la, al, mt)
                    Eb = ec_table(lb, be, mt) * sign
                    R = hermite_r(rho, A - B, mt, omega)
                    G = np.zeros((T, la + 1, lb + 1, mt))
                    for t in range(mt):
                        for tau in range(mt - t):
                            G[..., t + tau] += Ea[:, :, None, t] * Eb[:, None, :, tau]
                    GX = G[:, ix[0][:, None], jx[0][None, :], :]
                    GY = G[:, ix[1][:, None], jx[1][None, :], :]
                    GZ = G[:, ix[2][:, None], jx[2][None, :], :]
                    tmp = np.einsum("tabq,tsrq->tabsr", GZ, R)
                    v = np.einsum("tabsr,tabs,tabr->tab", tmp, GX, GY)
                    w = ca[:, :, p1][:, :, None] * cb[:, :, p2][:, None, :]
                    val += pref[:, None, None] * v * w
            r1 = ra0[:, None] + np.arange(len(anga))
            r2 = rb0[:, None] + np.arange(len(angb))
            out[r1[:, :, None], r2[:, None, :]] = val
            out[r2[:, None, :], r1[:, :, None]] = val
    if aux.cart2sph is not None:
        C = np.asarray(aux.cart2sph)
        out = C.T @ out @ C
    return out


# ---------------------------------------------------------------------------
# Schwarz shell-pair screening (eri3c_bucketed.py:140-169 via eri4c.py:206-220)
# ---------------------------------------------------------------------------

def schwarz_diagonal(basis):
    """sqrt((ab|ab)) for every cartesian AO pair a >= b, in np.tril_indices order
    (``dftax/integrals/eri4c.py:206-220``)."""
    sh = shells(basis)
    n = basis.angular.shape[0]
    row_shell = np.empty(n, dtype=np.int64)
    for si, (_l, r0, nc, _p) in enumerate(sh):
        row_shell[r0:r0 + nc] = si
    ang = np.asarray(basis.angular)
    cen = np.asarray(basis.centers)
    ex = np.asarray(basis.exponents)
    co = np.asarray(basis.coefficients)
    pa, pb = np.tril_indices(n)
    out = np.zeros(len(pa))
    # group AO pairs by their (la, lb) cartesian powers to vectorize
    for k in range(len(pa)):
        a, b = pa[k], pb[k]
        out[k] = _diag_element(ang[a], ang[b], cen[a], cen[b], ex[a], ex[b], co[a], co[b])
    return np.sqrt(np.maximum(out, 0.0))


def _e1d(i, j, a, b, xab):
    """List of E^{ij}_t, t = 0..i+j (scalar primitives)."""
    g = a + b
    xpa, xpb, i2g = -b * xab / g, a * xab / g, 0.5 / g
    mt = i + j + 1
    E = np.zeros((i + 1, j + 1, mt + 1))
    E[0, 0, 0] = 1.0
    for ii in range(i):
        for t in range(mt):
            E[ii + 1, 0, t] = xpa * E[ii, 0, t] + (i2g * E[ii, 0, t - 1] if t else 0.0) + (t + 1) * E[ii, 0, t + 1]
    for jj in range(j):
        for ii in range(i + 1):
            for t in range(mt):
                E[ii, jj + 1, t] = xpb * E[ii, jj, t] + (i2g * E[ii, jj, t - 1] if t else 0.0) + (t + 1) * E[ii, jj, t + 1]
    return E[i, j, :mt]


def _diag_element(ga, gb, A, B, ea, eb, ca, cb):
    """(ab|ab) for one cartesian AO pair, contracted."""
    tot = 0.0
    L = int(sum(ga) + sum(gb))
    mt = 2 * L + 1
    for i1 in np.nonzero(ea)[0]:
        for j1 in np.nonzero(eb)[0]:
            p = ea[i1] + eb[j1]
            AB = A - B
            Kp = math.exp(-ea[i1] * eb[j1] / p * float(AB @ AB))
            E1 = [_e1d(ga[x], gb[x], ea[i1], eb[j1], AB[x]) for x in range(3)]
            P1 = (ea[i1] * A + eb[j1] * B) / p
            for i2 in np.nonzero(ea)[0]:
                for j2 in np.nonzero(eb)[0]:
                    q = ea[i2] + eb[j2]
                    Kq = math.exp(-ea[i2] * eb[j2] / q * float(AB @ AB))
                    E2 = [_e1d(ga[x], gb[x], ea[i2], eb[j2], AB[x]) for x in range(3)]
                    P2 = (ea[i2] * A + eb[j2] * B) / q
                    alpha = p * q / (p + q)
                    R = hermite_r(np.array([alpha]), (P1 - P2)[None], mt)[0]
                    s = 0.0
                    for t, et in enumerate(E1[0]):
                        for u, eu in enumerate(E1[1]):
                            for v, ev in enumerate(E1[2]):
                                for t2, ft in enumerate(E2[0]):
                                    for u2, fu in enumerate(E2[1]):
                                        for v2, fv in enumerate(E2[2]):
                                            s += (et * eu * ev * ft * fu * fv * (-1.0) ** (t2 + u2 + v2)
                                                  * R[t + t2, u + u2, v + v2])
                    tot += (ca[i1] * cb[j1] * ca[i2] * cb[j2] * Kp * Kq * TWO_PI_2_5
                            / (p * q * math.sqrt(p + q)) * s)
    return tot


def shell_pair_keep(basis, thresh):
    """Kept shell pairs {(ia, ib), ia <= ib} under the relative Schwarz cutoff
    (``eri3c_bucketed.py:140-169``): keep when the pair's largest component
    sqrt((ab|ab)) >= thresh * the global maximum."""
    sh = shells(basis)
    n = basis.angular.shape[0]
    row_shell = np.empty(n, dtype=np.int64)
    for si, (_l, r0, nc, _p) in enumerate(sh):
        row_shell[r0:r0 + nc] = si
    Q = schwarz_diagonal(basis)
    pa, pb = np.tril_indices(n)
    lo = np.minimum(row_shell[pa], row_shell[pb])
    hi = np.maximum(row_shell[pa], row_shell[pb])
    ns = len(sh)
    Qsh = np.zeros((ns, ns))
    np.maximum.at(Qsh, (hi, lo), Q)
    qmax = float(Qsh.max()) if Qsh.size else 0.0
    hi_i, lo_i = np.nonzero(Qsh >= thresh * qmax)
    return {(int(a), int(b)) for b, a in zip(hi_i, lo_i)}
