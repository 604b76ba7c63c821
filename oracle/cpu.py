"""Compiled CPU restatement of dftax's DF build — TEST INFRASTRUCTURE ONLY.

The timed CPU baseline of ``bench.py`` (its ``cpu_baseline`` leg and its
``--impl reference`` arm) and a second checker of the numpy oracle. The 3-center
and 2-center integrals run in ``cpu_df.cpp`` (C++, all host threads); the metric
pseudo-inverse, J and K follow ``dftax/ks/terms.py`` with numpy (OpenBLAS, all
host threads):

* ``_metric_pinv`` (``terms.py:155-192``): eigh of (P|Q), 1/w over the
  eigenvalues above 1e-7 w_max;
* ``DFCoulomb.energy`` (``terms.py:592-613``): gamma = (mn|P) D_mn, E_J =
  1/2 gamma^T V+ gamma, and J = (mn|P) (V+ gamma), its gradient;
* K(D)_mn = sum (ml|P) V+_PQ (ns|Q) D_ls, the einsum of ``terms.py:598-603``,
  contracted as dftax's einsum path does it: (ml|P) V+ (2 nao^2 naux^2 flops),
  D (ns|Q) (2 nao^3 naux) and the final contraction (2 nao^3 naux).

``build_lib()`` compiles ``cpu_df.cpp`` with g++ into ``oracle/libdfcpu.so``
(next to the source; a built file, kept out of the repository's history).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import time
from ctypes import c_double, c_int, c_int64, c_void_p

import numpy as np

from . import boys as oboys
from . import df as odf
from . import md as omd

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_df.cpp")
LIB = os.path.join(HERE, "libdfcpu.so")
# AVX2/FMA (x86-64-v3): the host that builds the library need not be the one that runs it
CXXFLAGS = ["-O3", "-mavx2", "-mfma", "-std=c++17", "-fPIC", "-shared", "-pthread"]

_lib = None


def build_lib(force: bool = False) -> str:
    """Compile cpu_df.cpp when the library is missing or older than its source."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        r = subprocess.run(["g++", *CXXFLAGS, SRC, "-o", LIB], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed for {SRC}:\n{r.stderr}")
    return LIB


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build_lib()
        lib = ctypes.CDLL(LIB)
        V, I, L = c_void_p, c_int, c_int64
        basis = [I, V, V, V, V, V, V, V, V, V, V, V, V]
        lib.cpu_eri3c_dense.argtypes = basis + basis + [L, V, V, V, I, L, L, I, V]
        lib.cpu_eri3c_dense.restype = c_int
        lib.cpu_eri2c.argtypes = basis + [V, I, L, I, V]
        lib.cpu_eri2c.restype = c_int
        _lib = lib
    return _lib


def threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:   # pragma: no cover - platform without affinity
        return os.cpu_count() or 1


class _Shells:
    """Per-shell tables of a BasisData in the layout cpu_df.cpp reads."""

    def __init__(self, basis):
        sh = omd.shells(basis)
        starts, self.nbf = omd.sph_starts(sh, basis.cart2sph)
        ex = np.asarray(basis.exponents)
        co = np.asarray(basis.coefficients)
        self.l = np.array([s[0] for s in sh], dtype=np.int32)
        self.cen = np.ascontiguousarray(np.asarray(basis.centers)[[s[1] for s in sh]], dtype=np.float64)
        self.nprim = np.array([s[3] for s in sh], dtype=np.int32)
        self.prim0 = np.concatenate([[0], np.cumsum(self.nprim)[:-1]]).astype(np.int32)
        pe, pc = [], []
        for (l, r0, nc, npr) in sh:
            if not np.array_equal(co[r0:r0 + nc, :npr], np.broadcast_to(co[r0, :npr], (nc, npr))):
                raise ValueError("coefficients differ between a shell's cartesian rows")
            pe.extend(ex[r0, :npr])
            pc.extend(co[r0, :npr])
        self.pexp = np.asarray(pe, dtype=np.float64)
        self.pcoef = np.asarray(pc, dtype=np.float64)
        self.ang = np.ascontiguousarray(np.asarray(basis.angular), dtype=np.int32)
        self.ang0 = np.array([s[1] for s in sh], dtype=np.int32)
        blocks, offs, nsph = [], [], []
        off = 0
        for (l, r0, nc, _), s0 in zip(sh, starts):
            b = omd._block(basis.cart2sph, r0, s0, l, nc)
            blocks.append(np.ascontiguousarray(b).ravel())
            offs.append(off)
            nsph.append(b.shape[1])
            off += b.size
        self.c2s = np.concatenate(blocks).astype(np.float64)
        self.c2s0 = np.asarray(offs, dtype=np.int64)
        self.nsph = np.asarray(nsph, dtype=np.int32)
        self.sph0 = np.asarray(starts, dtype=np.int64)
        self.n = len(sh)

    def args(self):
        p = lambda a: a.ctypes.data   # noqa: E731
        return [self.n, p(self.l), p(self.cen), p(self.nprim), p(self.prim0), p(self.pexp),
                p(self.pcoef), p(self.ang), p(self.ang0), p(self.c2s), p(self.c2s0), p(self.nsph),
                p(self.sph0)]


_TABLE = np.ascontiguousarray(oboys.TABLE)


def eri3c_dense(orb, aux, keep_pairs=None, nthreads: int | None = None) -> np.ndarray:
    """Dense (nao, nao, naux) spherical 3-center tensor, both bra triangles
    (``eri3c_matrix_bucketed`` output); pairs outside ``keep_pairs`` stay zero."""
    lib = _load()
    so, sa = _Shells(orb), _Shells(aux)
    ia, ib = np.triu_indices(so.n)
    if keep_pairs is not None:
        sel = np.array([(int(a), int(b)) in keep_pairs for a, b in zip(ia, ib)], dtype=bool)
        ia, ib = ia[sel], ib[sel]
    pa = np.ascontiguousarray(ia, dtype=np.int32)
    pb = np.ascontiguousarray(ib, dtype=np.int32)
    out = np.zeros((so.nbf, so.nbf, sa.nbf))
    st = lib.cpu_eri3c_dense(*so.args(), *sa.args(), len(pa), pa.ctypes.data, pb.ctypes.data,
                             _TABLE.ctypes.data, _TABLE.shape[0], so.nbf, sa.nbf,
                             nthreads or threads(), out.ctypes.data)
    if st != 0:
        raise ValueError("cpu_eri3c_dense: angular momentum beyond orbital f / auxiliary g")
    return out


def eri2c(aux, nthreads: int | None = None) -> np.ndarray:
    """(naux, naux) spherical metric (``eri2c_matrix_bucketed`` output)."""
    lib = _load()
    sa = _Shells(aux)
    out = np.zeros((sa.nbf, sa.nbf))
    st = lib.cpu_eri2c(*sa.args(), _TABLE.ctypes.data, _TABLE.shape[0], sa.nbf,
                       nthreads or threads(), out.ctypes.data)
    if st != 0:
        raise ValueError("cpu_eri2c: angular momentum beyond g")
    return out


def k_reference_path(I3, vinv, D):
    """K(D) = einsum("mlP,PQ,nsQ,ls->mn") as three GEMMs (dftax's einsum path)."""
    nao, _, naux = I3.shape
    Z = (I3.reshape(nao * nao, naux) @ vinv).reshape(nao, nao * naux)       # (ml|Q)
    Y = np.empty_like(I3)                                                   # Y[n, l, Q]
    for n in range(nao):
        Y[n] = D @ I3[n]            # sum_s D_ls (ns|Q)
    return Z @ Y.reshape(nao, nao * naux).T


def df_build_jk(orb, aux, C, hf_coeff: float = 0.25, nthreads: int | None = None) -> dict:
    """One complete DF J/K build as dftax's materialized path does it: the
    metric, its pseudo-inverse, the dense 3-center tensor, then J, K of D = C C^T
    and the energy of P = 2 D. Returns J, K, E and the seconds of each part."""
    t = {}
    t0 = time.perf_counter()
    V = eri2c(aux, nthreads)
    t["eri2c"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    vinv = odf.metric_pinv(V)
    t["metric"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    I3 = eri3c_dense(orb, aux, nthreads=nthreads)
    t["eri3c"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    D = C @ C.T
    nao, _, naux = I3.shape
    I2 = I3.reshape(nao * nao, naux)
    gamma = D.reshape(-1) @ I2
    J = (I2 @ (vinv @ gamma)).reshape(nao, nao)
    t["j"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    K = k_reference_path(I3, vinv, D)
    t["k"] = time.perf_counter() - t0
    # E = 1/2 gamma(P)^T V+ gamma(P) - 1/4 a_x Tr(P K(P)) with P = 2 D
    E = 0.5 * (2.0 * gamma) @ (vinv @ (2.0 * gamma)) - 0.25 * hf_coeff * np.sum(
        (2.0 * D) * (2.0 * K))
    return {"J": J, "K": K, "E": float(E), "seconds": t}




# ---------------------------------------------------------------------------
# Nuclear gradient of the DF energy at a fixed density
# ---------------------------------------------------------------------------

def _moved(basis, atom_xyz, atom: int, axis: int, h: float):
    """A copy of ``basis`` whose functions on ``atom`` are moved by h along axis."""
    import dataclasses

    cen = np.array(basis.centers, dtype=np.float64, copy=True)
    on = np.linalg.norm(cen - np.asarray(atom_xyz)[atom], axis=1) < 1e-8
    cen[on, axis] += h
    return dataclasses.replace(basis, centers=cen)


def df_energy_terms(orb, aux, P, hf_coeff: float, nthreads: int | None = None, vinv=None):
    """The DF energy of ``DFCoulomb.energy`` (``terms.py:592-613``) at a fixed
    density P (nspin, nao, nao) and the two weights its geometry derivative
    contracts with the integral derivatives:

        dE = sum_{mnP} G[m,n,P] d(mn|P) - 1/2 sum_{PQ} W[P,Q] d(P|Q)

    with gamma = V+ c, c_P = sum P_tot (mn|P), and for each spin channel s of
    exchange weight k_s (-a_x/4 closed shell, -a_x/2 per spin):
    G = gamma_P P_tot + sum_s 2 k_s P_s Z_P P_s, Z_P = sum_Q V+_PQ (..|Q), and
    W = gamma gamma^T + sum_s 2 k_s V+ M_s V+, M_s[P,Q] = tr(P_s T_P P_s T_Q).
    The metric enters through d(V+) = -V+ dV V+, the rule of dftax's
    ``_metric_pinv_jvp`` (``terms.py:196-204``). ``vinv`` replaces the
    oracle's own pseudo-inverse (to separate the conditioning of the metric
    from the rest when comparing)."""
    P = np.asarray(P, dtype=np.float64)
    if P.ndim == 2:
        P = P[None]
    if vinv is None:
        vinv = odf.metric_pinv(eri2c(aux, nthreads))
    I3 = eri3c_dense(orb, aux, nthreads=nthreads)
    nao, _, naux = I3.shape
    Ptot = P.sum(0)
    c = np.einsum("mn,mnP->P", Ptot, I3)
    gam = vinv @ c
    E = 0.5 * c @ gam
    G = Ptot[:, :, None] * gam[None, None, :]
    W = np.outer(gam, gam)
    ks = [-0.25 * hf_coeff] if P.shape[0] == 1 else [-0.5 * hf_coeff] * P.shape[0]
    if hf_coeff != 0.0:
        Z = (I3.reshape(nao * nao, naux) @ vinv).reshape(nao, nao, naux)
        for Ps, k in zip(P, ks):
            Y = np.einsum("ml,lsP,sn->mnP", Ps, I3, Ps, optimize=True)
            M = np.einsum("mnP,nmQ->PQ", Y, I3, optimize=True)
            E += k * np.einsum("PQ,PQ->", vinv, M)
            G += 2.0 * k * np.einsum("ml,lsP,sn->mnP", Ps, Z, Ps, optimize=True)
            W += 2.0 * k * (vinv @ M @ vinv)
    return float(E), G, W


def df_energy_grad(orb, aux, P, hf_coeff: float, atom_xyz, h: float = 1e-3,
                   nthreads: int | None = None, vinv=None):
    """dE/dR (natom, 3) of the DF energy at fixed P: G and W from
    ``df_energy_terms`` contracted with the derivatives of (mn|P) and (P|Q)
    with respect to each atom's position (the functions on the atom move
    together), taken by central differences at h and h/2 with one Richardson
    step (error O(h^4)). Returns (E, grad)."""
    E, G, W = df_energy_terms(orb, aux, P, hf_coeff, nthreads, vinv)
    atom_xyz = np.asarray(atom_xyz, dtype=np.float64)

    def phi(atom, axis, d):
        o, a = _moved(orb, atom_xyz, atom, axis, d), _moved(aux, atom_xyz, atom, axis, d)
        return (np.einsum("mnP,mnP->", G, eri3c_dense(o, a, nthreads=nthreads))
                - 0.5 * np.einsum("PQ,PQ->", W, eri2c(a, nthreads)))

    grad = np.zeros((len(atom_xyz), 3))
    for A in range(len(atom_xyz)):
        for x in range(3):
            d1 = (phi(A, x, h) - phi(A, x, -h)) / (2 * h)
            d2 = (phi(A, x, h / 2) - phi(A, x, -h / 2)) / h
            grad[A, x] = (4.0 * d2 - d1) / 3.0
    return E, grad


def df_energy(orb, aux, P, hf_coeff: float, nthreads: int | None = None) -> float:
    """The DF energy alone (``df_energy_terms``'s first value)."""
    return df_energy_terms(orb, aux, P, hf_coeff, nthreads)[0]


__all__ = ["build_lib", "eri3c_dense", "eri2c", "df_build_jk", "k_reference_path", "threads",
           "df_energy_terms", "df_energy_grad", "df_energy"]
