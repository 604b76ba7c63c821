"""Synthetic molecular systems and even-tempered basis sets of the DF workloads.

All inputs are seeded and fully synthetic (no public dataset is involved):

* water monomer: O (0, 0, 0), H (+-0.757, 0.587, 0) Angstrom;
* water clusters (H2O)_n: O atoms by seeded rejection sampling in a cube of
  liquid density 1.0 g/cm^3 with a minimum O-O distance of 2.6 Angstrom, each
  molecule rotated by a seeded uniformly random rotation about its O atom;
* linear alkanes C_nH_2n+2: all-trans zigzag backbone (C-C 1.54, C-H 1.09
  Angstrom, tetrahedral angles) with a seeded +-10 degree torsion jitter.

Orbital basis (uncontracted, one primitive per shell):
  O 4s (0.25*3^k) 3p (0.3*3^k) 1d (1.0); H 3s (0.2*3^k) 1p (0.8);
  C 5s (0.12*3^k) 4p (0.15*3^k) 3d (0.3*3^k) 1f (0.8).
Auxiliary basis (uncontracted, alpha = 0.1*2.5^k, k from 0 for every l):
  O 10s8p6d3f; H 6s4p2d; C 12s10p8d5f3g.
The carbon sets are this project's choice (the workload names only their
angular content: orbital up to f, auxiliary up to g).

Coordinates are returned in Bohr (``ANGSTROM_TO_BOHR`` of
``dftax/system/molecule.py:15``).
"""

from __future__ import annotations

import math

import numpy as np

from .basis import BasisData, build_basis_data

ANGSTROM_TO_BOHR = 1.0 / 0.529177210903
AVOGADRO = 6.02214076e23
WATER_MASS = 18.015


def _even_tempered(spec):
    """[(l, count, alpha0, ratio)] -> [(l, [alpha], [1.0])] one primitive per shell."""
    shells = []
    for l, count, a0, ratio in spec:
        for k in range(count):
            shells.append((l, [a0 * ratio ** k], [1.0]))
    return shells


ORBITAL_SETS = {
    "O": _even_tempered([(0, 4, 0.25, 3.0), (1, 3, 0.3, 3.0), (2, 1, 1.0, 3.0)]),
    "H": _even_tempered([(0, 3, 0.2, 3.0), (1, 1, 0.8, 3.0)]),
    "C": _even_tempered([(0, 5, 0.12, 3.0), (1, 4, 0.15, 3.0), (2, 3, 0.3, 3.0),
                         (3, 1, 0.8, 3.0)]),
}

AUX_SETS = {
    "O": _even_tempered([(0, 10, 0.1, 2.5), (1, 8, 0.1, 2.5), (2, 6, 0.1, 2.5),
                         (3, 3, 0.1, 2.5)]),
    "H": _even_tempered([(0, 6, 0.1, 2.5), (1, 4, 0.1, 2.5), (2, 2, 0.1, 2.5)]),
    "C": _even_tempered([(0, 12, 0.1, 2.5), (1, 10, 0.1, 2.5), (2, 8, 0.1, 2.5),
                         (3, 5, 0.1, 2.5), (4, 3, 0.1, 2.5)]),
}

NUCLEAR_CHARGE = {"H": 1, "C": 6, "O": 8}


def water_monomer():
    """(symbols, coords_bohr) of the single water molecule."""
    sym = ["O", "H", "H"]
    xyz = np.array([[0.0, 0.0, 0.0], [0.757, 0.587, 0.0], [-0.757, 0.587, 0.0]])
    return sym, xyz * ANGSTROM_TO_BOHR


def _random_rotation(rng):
    """Uniformly random proper rotation (QR of a Gaussian, sign-fixed)."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def water_cluster(n: int, seed: int = 0, density: float = 1.0, min_oo: float = 2.6):
    """(symbols, coords_bohr) of a seeded (H2O)_n cluster at the given density."""
    rng = np.random.default_rng(seed)
    side = (n * WATER_MASS / (AVOGADRO * density)) ** (1.0 / 3.0) * 1e8  # Angstrom
    oxy = []
    tries = 0
    while len(oxy) < n:
        tries += 1
        if tries > 1_000_000:
            raise RuntimeError("could not place the water cluster; lower the density")
        p = rng.uniform(0.0, side, size=3)
        if all(np.linalg.norm(p - q) >= min_oo for q in oxy):
            oxy.append(p)
    _, mono = water_monomer()
    mono = mono / ANGSTROM_TO_BOHR
    sym, xyz = [], []
    for o in oxy:
        rot = _random_rotation(rng)
        for s, r in zip(["O", "H", "H"], mono):
            sym.append(s)
            xyz.append(o + rot @ r)
    return sym, np.array(xyz) * ANGSTROM_TO_BOHR


def _place(a, b, c, bond, angle, torsion):
    """Position d with |cd| = bond, angle(b,c,d) = angle, dihedral(a,b,c,d) = torsion
    (natural-extension reference frame; angles in radians)."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * math.cos(angle), bond * math.sin(angle) * math.cos(torsion),
                   bond * math.sin(angle) * math.sin(torsion)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def alkane(n: int, seed: int = 0, jitter_deg: float = 10.0):
    """(symbols, coords_bohr) of C_nH_2n+2, all-trans with seeded torsion jitter."""
    if n < 1:
        raise ValueError("alkane needs n >= 1")
    rng = np.random.default_rng(seed)
    tet = math.acos(-1.0 / 3.0)
    cc, ch = 1.54, 1.09
    carbons = [np.zeros(3)]
    if n >= 2:
        carbons.append(np.array([cc, 0.0, 0.0]))
    if n >= 3:
        carbons.append(carbons[1] + cc * np.array([-math.cos(tet), math.sin(tet), 0.0]))
    for i in range(3, n):
        tors = math.pi + math.radians(rng.uniform(-jitter_deg, jitter_deg))
        carbons.append(_place(carbons[i - 3], carbons[i - 2], carbons[i - 1], cc, tet, tors))
    hyd = []
    if n == 1:
        c0 = carbons[0]
        for v in ([1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]):
            hyd.append(c0 + ch * np.array(v, float) / math.sqrt(3.0))
    else:
        for i, c in enumerate(carbons):
            nb = [carbons[j] for j in (i - 1, i + 1) if 0 <= j < n]
            if len(nb) == 2:
                u = (c - nb[0]) / np.linalg.norm(c - nb[0]) + (c - nb[1]) / np.linalg.norm(c - nb[1])
                u /= np.linalg.norm(u)
                w = np.cross(nb[0] - c, nb[1] - c)
                w /= np.linalg.norm(w)
                half = tet / 2.0
                for s in (1.0, -1.0):
                    hyd.append(c + ch * (math.cos(half) * u + s * math.sin(half) * w))
            else:
                # terminal carbon: three staggered hydrogens about the C-C bond
                j = 1 if i == 0 else n - 2
                k = 2 if i == 0 else n - 3
                ref = carbons[k] if 0 <= k < n and k != i else c + np.array([0.0, 0.0, 1.0])
                for tors in (math.pi / 3.0, math.pi, -math.pi / 3.0):
                    hyd.append(_place(ref, carbons[j], c, ch, tet, tors))
    sym = ["C"] * n + ["H"] * len(hyd)
    xyz = np.array(carbons + hyd)
    return sym, xyz * ANGSTROM_TO_BOHR


def basis_for(symbols, coords_bohr, *, spherical=True):
    """(orbital BasisData, auxiliary BasisData) of the even-tempered sets."""
    orb = build_basis_data(symbols, coords_bohr, ORBITAL_SETS, spherical=spherical)
    aux = build_basis_data(symbols, coords_bohr, AUX_SETS, spherical=spherical)
    return orb, aux


def n_electrons(symbols) -> int:
    return int(sum(NUCLEAR_CHARGE[s] for s in symbols))


def random_occupied(nao: int, nocc: int, seed: int = 0) -> np.ndarray:
    """Seeded Euclidean-orthonormal C_occ (nao x nocc): QR of a Gaussian."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((nao, nocc)))
    return np.ascontiguousarray(q)


def workload(name: str, seed: int = 0):
    """Named workloads: 'water', 'water<n>' (cluster), 'alkane<n>'.

    Returns ``(symbols, coords_bohr, orbital BasisData, aux BasisData, nocc)``;
    nocc is half the electron count (5 per water).
    """
    if name == "water":
        sym, xyz = water_monomer()
    elif name.startswith("water"):
        sym, xyz = water_cluster(int(name[5:]), seed=seed)
    elif name.startswith("alkane"):
        sym, xyz = alkane(int(name[6:]), seed=seed)
    else:
        raise ValueError(f"unknown workload {name!r}")
    orb, aux = basis_for(sym, xyz)
    return sym, xyz, orb, aux, n_electrons(sym) // 2


__all__ = ["BasisData", "water_monomer", "water_cluster", "alkane", "basis_for",
           "random_occupied", "workload", "ORBITAL_SETS", "AUX_SETS"]
