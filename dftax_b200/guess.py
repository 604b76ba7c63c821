"""Initial densities for the SCF, with dftax's names (``dftax/ks/guess.py``).

* ``core()``: the aufbau fill of the core-Hamiltonian eigenvectors
  (``guess.py:104-113``, ``:588-606``), the SCF's default here. dftax's own
  default is ``minao()``, which projects atomic occupations from a minimal
  basis fetched from the Basis Set Exchange; without that data dftax falls
  back to ``core()`` (``guess.py:628-652``), and ``minao()`` is not provided.
* ``sad()``: superposition of atomic densities (``guess.py:115-123``,
  ``:382-452``, ``:529-546``). Per unique element, a spherically averaged
  atomic Hartree-Fock with the ground-state configuration occupations
  (``:172-213``, ``:349-379``) is converged in the molecule's own basis, and
  the atomic blocks go on the block diagonal, scaled so that Tr(P S) is the
  electron count (``:602-613``). The atom's J and K come from this library's
  density-fitting plan of the atom's own orbital and fitting functions on the
  device (dftax contracts exact 4-center integrals there); the few-dozen
  function eigenproblems and the occupation bookkeeping run on the host, as
  in dftax. Atomic densities are cached per element and basis, so a stream of
  molecules solves each element once.
"""

from __future__ import annotations

import ctypes
from ctypes import byref
from dataclasses import dataclass

import numpy as np

from . import _lib
from .basis import BasisData
from .grid import ATOMIC_NUMBER

# ---------------------------------------------------------------------------
# specs
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class CoreSpec:
    """The core-Hamiltonian guess."""


@dataclass(frozen=True)
class SADSpec:
    """Superposition of atomic densities from solved atoms."""
    max_iter: int = 300
    tol: float = 1e-8
    mix: float = 0.5


def core() -> CoreSpec:
    return CoreSpec()


def sad() -> SADSpec:
    return SADSpec()


# ---------------------------------------------------------------------------
# ground-state configurations (Madelung filling with the Z <= 54 exceptions)
# ---------------------------------------------------------------------------

_FILL_ORDER = ((1, 0), (2, 0), (2, 1), (3, 0), (3, 1), (4, 0), (3, 2), (4, 1), (5, 0), (4, 2),
               (5, 1))
# s -> d promotions of the neutral ground states up to xenon
_PROMOTED = {24: {(4, 0): 1, (3, 2): 5}, 29: {(4, 0): 1, (3, 2): 10},
             41: {(5, 0): 1, (4, 2): 4}, 42: {(5, 0): 1, (4, 2): 5},
             44: {(5, 0): 1, (4, 2): 7}, 45: {(5, 0): 1, (4, 2): 8},
             46: {(5, 0): 0, (4, 2): 10}, 47: {(5, 0): 1, (4, 2): 10}}


def ground_state(Z: int) -> list[tuple[int, int, int]]:
    """(n, l, electrons) of the neutral atom's ground-state configuration."""
    if not 1 <= Z <= 54:
        raise ValueError(f"atomic guesses cover Z <= 54 (got {Z})")
    occ: dict[tuple[int, int], int] = {}
    left = Z
    for n, l in _FILL_ORDER:
        c = min(left, 2 * (2 * l + 1))
        occ[(n, l)] = c
        left -= c
        if left == 0:
            break
    occ.update(_PROMOTED.get(Z, {}))
    return [(n, l, c) for (n, l), c in occ.items() if c > 0]


def config_occupations(C, S, ao_l, Z) -> np.ndarray:
    """Occupation of each orbital (columns of C, ascending energy): each
    orbital is assigned to the l channel holding most of its Mulliken
    population, and each channel's (2l+1)-fold multiplets take the
    configuration's shells in energy order, count/(2l+1) per orbital. Fixing
    the occupations by configuration keeps near-degenerate shells from
    swapping between iterations."""
    per_l: dict[int, list[float]] = {}
    for _, l, c in ground_state(Z):
        per_l.setdefault(l, []).append(float(c))
    contrib = C * (S @ C)
    ao_l = np.asarray(ao_l)
    wl = np.zeros((int(ao_l.max()) + 1, C.shape[1]))
    for l in range(wl.shape[0]):
        wl[l] = contrib[ao_l == l].sum(axis=0)
    dom = wl.argmax(axis=0)
    occ = np.zeros(C.shape[1])
    for l, counts in per_l.items():
        mos = np.nonzero(dom == l)[0]
        deg = 2 * l + 1
        if len(mos) < len(counts) * deg:
            raise ValueError(f"the atomic basis holds too few l={l} functions for Z={Z}")
        for k, c in enumerate(counts):
            occ[mos[k * deg:(k + 1) * deg]] = c / deg
    return occ


# ---------------------------------------------------------------------------
# one atom's functions
# ---------------------------------------------------------------------------

def _shells(b: BasisData):
    """(first cartesian row, l) of every shell, in order."""
    lrow = np.asarray(b.angular).sum(axis=1)
    out, i = [], 0
    while i < lrow.shape[0]:
        l = int(lrow[i])
        out.append((i, l))
        i += (l + 1) * (l + 2) // 2
    return out


def atom_blocks(b: BasisData, atom_xyz, tol: float = 1e-10):
    """Per atom, (cartesian row slice, final function slice) of its shells
    (matched by center; an atom's shells must be contiguous)."""
    cen = np.asarray(b.centers, dtype=np.float64)
    xyz = np.asarray(atom_xyz, dtype=np.float64).reshape(-1, 3)
    sph = b.cart2sph is not None
    sh = _shells(b)
    start = np.array([st for st, _ in sh], dtype=np.int64)
    ls = np.array([l for _, l in sh], dtype=np.int64)
    # nearest atom of each shell center (the first of equals, as argmin)
    d = np.linalg.norm(cen[start][:, None, :] - xyz[None, :, :], axis=2)
    owner = d.argmin(axis=1)
    if (d[np.arange(len(sh)), owner] > tol).any():
        raise ValueError("a shell center is on no atom")
    ncart = (ls + 1) * (ls + 2) // 2
    c0 = np.concatenate([[0], np.cumsum(ncart)])
    f0 = np.concatenate([[0], np.cumsum(2 * ls + 1 if sph else ncart)])
    # each atom's first and last shell; contiguous when they span its count
    na, idx = len(xyz), np.arange(len(sh))
    cnt = np.bincount(owner, minlength=na)
    first = np.full(na, len(sh))
    last = np.full(na, -1)
    np.minimum.at(first, owner, idx)
    np.maximum.at(last, owner, idx)
    bad = np.nonzero((cnt == 0) | (last - first + 1 != cnt))[0]
    if len(bad):
        raise ValueError(f"atom {int(bad[0])}: no shells, or shells not contiguous")
    return [(slice(int(c0[first[a]]), int(c0[last[a] + 1])),
             slice(int(f0[first[a]]), int(f0[last[a] + 1]))) for a in range(na)]


def _sub_basis(b: BasisData, cs: slice, fs: slice) -> BasisData:
    """The functions of one atom, moved to the origin."""
    cen = np.asarray(b.centers[cs], dtype=np.float64)
    return BasisData(centers=cen - cen[0], exponents=np.asarray(b.exponents[cs]),
                     coefficients=np.asarray(b.coefficients[cs]),
                     angular=np.asarray(b.angular[cs]),
                     cart2sph=None if b.cart2sph is None else np.asarray(b.cart2sph[cs, fs]),
                     max_l=int(np.asarray(b.angular[cs]).sum(axis=1).max()))


def _key(b: BasisData):
    arrs = [b.exponents, b.coefficients, b.angular] + ([b.cart2sph] if b.cart2sph is not None else [])
    return tuple(np.ascontiguousarray(a).tobytes() for a in arrs)


_ATOM_CACHE: dict = {}


def _final_l(b: BasisData) -> list[int]:
    sph = b.cart2sph is not None
    out = []
    for _, l in _shells(b):
        out.extend([l] * (2 * l + 1 if sph else (l + 1) * (l + 2) // 2))
    return out


def atomic_density(symbol: str, orb: BasisData, aux: BasisData, spec: SADSpec = SADSpec(),
                   device: int = 0) -> np.ndarray:
    """Spherically averaged Hartree-Fock density of a neutral atom at the
    origin in its own functions ``orb`` (``guess.py:382-452``), with J and K
    fitted in ``aux`` on the device."""
    from .coulomb import Plan, _stream_ptr, _torch

    key = (symbol, _key(orb), _key(aux), spec)
    if key in _ATOM_CACHE:
        return _ATOM_CACHE[key]
    Z = ATOMIC_NUMBER[symbol]
    torch = _torch()
    plan = Plan(orb, aux, device=device).build()
    lib = plan.lib
    # S, T, V of the atom: an SCF handle with no grid (its occupation is unused)
    o = _lib.ScfOptions()
    lib.dfscf_default_options(byref(o))
    o.hf_coeff, o.x_scale, o.c_scale = 1.0, 0.0, 0.0
    xyz = np.zeros(3)
    charge = np.array([float(Z)])
    h = ctypes.c_void_p()
    _lib.check(lib.dfscf_create(plan.h, 1, xyz.ctypes.data, charge.ctypes.data, 0, None, None,
                                1, byref(o), byref(h), _stream_ptr(torch)), plan.ctx.h)
    try:
        n = plan.nao
        S, T, V = (torch.empty((n, n), dtype=torch.float64, device=plan.dev) for _ in range(3))
        _lib.check(lib.dfscf_one_electron(h, S.data_ptr(), T.data_ptr(), V.data_ptr(),
                                          _stream_ptr(torch)), plan.ctx.h)
        S, hcore = S.cpu().numpy(), (T + V).cpu().numpy()
    finally:
        lib.dfscf_destroy(h)
    s, U = np.linalg.eigh(S)
    keep = s > 1e-9
    X = U[:, keep] / np.sqrt(s[keep])[None, :]
    if Z == 1:                               # one electron: the lowest core orbital
        _, Cp = np.linalg.eigh(X.T @ hcore @ X)
        c = X @ Cp[:, 0]
        P = np.outer(c, c)
    else:
        ao_l = _final_l(orb)
        F, P = hcore, np.zeros_like(S)
        for it in range(spec.max_iter):
            _, Cp = np.linalg.eigh(X.T @ F @ X)
            C = X @ Cp
            occ = config_occupations(C, S, ao_l, Z)
            Pn = (C * occ[None, :]) @ C.T
            if it > 0:
                Pn = (1.0 - spec.mix) * Pn + spec.mix * P
            dP = np.abs(Pn - P).max()
            P = Pn
            _, G = plan.energy(P, 1.0)       # dE/dP = J - K/2 of the total density
            F = hcore + G[0].cpu().numpy()
            if it > 0 and dP < spec.tol:
                break
    plan.close()
    _ATOM_CACHE[key] = P
    return P


def sad_density(symbols, coords_bohr, orb: BasisData, aux: BasisData, spec: SADSpec = SADSpec(),
                device: int = 0) -> np.ndarray:
    """Block-diagonal superposition of the neutral atoms' densities
    (``guess.py:529-546``), (nao, nao); the caller scales it to the electron
    count."""
    ob, ab = atom_blocks(orb, coords_bohr), atom_blocks(aux, coords_bohr)
    nao = orb.cart2sph.shape[1] if orb.cart2sph is not None else orb.angular.shape[0]
    P = np.zeros((nao, nao))
    for sym, (cs, fs), (acs, afs) in zip(symbols, ob, ab):
        P[fs, fs] = atomic_density(sym, _sub_basis(orb, cs, fs), _sub_basis(aux, acs, afs), spec,
                                   device)
    return P


def initial_density(guess, symbols, coords_bohr, orb, aux, nelec: int, device: int = 0):
    """The SCF's starting density for ``guess`` (None or ``core()``: None,
    the library's core guess; ``sad()``: the superposition scaled to nelec
    electrons; an array: itself). Each atomic block holds Tr(P_A S_AA) = Z_A
    electrons and the superposition is block diagonal, so Tr(P S) = sum Z_A
    and the scale is nelec / sum Z_A (1 for a neutral molecule)."""
    if guess is None or isinstance(guess, CoreSpec) or (isinstance(guess, str) and guess == "core"):
        return None
    if isinstance(guess, str):
        if guess != "sad":
            raise ValueError(f"unknown guess {guess!r}")
        guess = SADSpec()
    if isinstance(guess, SADSpec):
        P = sad_density(symbols, coords_bohr, orb, aux, guess, device)
        return P * (nelec / float(sum(ATOMIC_NUMBER[s] for s in symbols)))
    return guess


__all__ = ["core", "sad", "CoreSpec", "SADSpec", "ground_state", "config_occupations",
           "atomic_density", "sad_density", "initial_density", "atom_blocks"]
