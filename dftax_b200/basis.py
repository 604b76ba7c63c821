"""Host-side Gaussian basis layout: the ``BasisData`` arrays the library reads.

One row per *cartesian* atomic orbital, exactly dftax's layout
(``dftax/energy/gto.py:132-156``): the row's center (3), zero-padded primitive
exponents and final coefficients (``max_prim``), its cartesian powers
``(lx, ly, lz)``, and a block-diagonal cartesian->spherical matrix
``cart2sph`` (``nao_cart x nao_sph``) or ``None`` for a cartesian basis.

Normalization follows ``dftax/basis/loader.py:85-160``: every primitive
coefficient is multiplied by the radial norm ``gto_norm(l, alpha)``
(``loader.py:52-64``); for l <= 1 each cartesian component additionally gets
its contracted self-overlap norm (``gto.py:104-125``), for l >= 2 it does not
(libcint's per-shell convention; the spherical transform carries the rest).

The cartesian component order is the lexicographic one of
``gto.py:32-66`` (lx descending, then ly descending). The per-l spherical
blocks are the real solid harmonics normalized on the unit sphere, ordered
m = -l..l, with identity blocks for l <= 1 (``scripts/gen_cart2sph.py`` in the
reference documents this convention; the coefficients are generated here from
the closed-form expansion, see :func:`cart2sph_block`).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from fractions import Fraction
from functools import lru_cache

import numpy as np

L_MAX = 6


def cart_components(l: int) -> list[tuple[int, int, int]]:
    """Cartesian powers of one shell in dftax/libcint order (``gto.py:32-66``)."""
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def gto_norm(l: int, alpha: float) -> float:
    """Radial primitive norm, ``N`` with ``N r^l exp(-alpha r^2)`` unit-normalized
    over the sphere-integrated radial measure (``loader.py:52-64``)."""
    f = (2 ** (2 * l + 3) * math.factorial(l + 1) * (2 * alpha) ** (l + 1.5)
         / (math.factorial(2 * l + 2) * math.sqrt(math.pi)))
    return math.sqrt(f)


def _double_factorial_odd(k: int) -> int:
    """(2k-1)!! with (-1)!! = 1."""
    r = 1
    for j in range(1, 2 * k, 2):
        r *= j
    return r


def contracted_norm(exps, c_prim, ang) -> float:
    """Norm of a contracted cartesian GTO with primitive coefficients ``c_prim``
    (``gto.py:73-125``): ``1/sqrt(sum_ij c_i c_j (pi/a)^{3/2} prod_k (2k-1)!!/(2a)^k)``
    with ``a = alpha_i + alpha_j``."""
    s = 0.0
    for ai, ci in zip(exps, c_prim):
        for aj, cj in zip(exps, c_prim):
            a = ai + aj
            f = 1.0
            for lk in ang:
                if lk:
                    f *= _double_factorial_odd(lk) / (2.0 * a) ** lk
            s += ci * cj * (math.pi / a) ** 1.5 * f
    return 1.0 / math.sqrt(s)


@lru_cache(maxsize=None)
def cart2sph_block(l: int) -> np.ndarray:
    """``(ncart(l), 2l+1)`` block mapping cartesian monomials to real solid
    harmonics ``r^l Y_lm`` (unit-sphere normalized, m = -l..l, no Condon-Shortley
    phase), identity for l <= 1.

    Built from the closed-form expansion of the real regular solid harmonics
    (Helgaker, Jorgensen & Olsen, *Molecular Electronic-Structure Theory*,
    eqs. 6.4.47-6.4.50), evaluated in exact rational arithmetic and scaled by
    ``sqrt((2l+1)/4pi)``.
    """
    if l <= 1:
        return np.eye(2 * l + 1)
    comps = cart_components(l)
    index = {c: i for i, c in enumerate(comps)}
    out = np.zeros((len(comps), 2 * l + 1))
    for col, m in enumerate(range(-l, l + 1)):
        am = abs(m)
        vm = Fraction(1, 2) if m < 0 else Fraction(0)
        # N_lm = 1/(2^|m| l!) * sqrt(2 (l+|m|)! (l-|m|)! / 2^{delta_m0})
        nrm = math.sqrt(2 * math.factorial(l + am) * math.factorial(l - am)
                        / (2.0 if m == 0 else 1.0)) / (2 ** am * math.factorial(l))
        coeffs: dict[tuple[int, int, int], Fraction] = {}
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                # v runs over vm, vm+1, ..., floor(|m|/2 - vm) + vm
                v = vm
                vmax = Fraction(math.floor(am / 2 - vm)) + vm
                while v <= vmax:
                    two_v = int(2 * v)
                    sign = -1 if int(t + v - vm) % 2 else 1
                    c = (sign * Fraction(1, 4 ** t) * math.comb(l, t)
                         * math.comb(l - t, am + t) * math.comb(t, u)
                         * math.comb(am, two_v))
                    # exponents: x^{2t+|m|-2(u+v)} y^{2(u+v)} z^{l-2t-|m|}
                    py = int(2 * (u + v))
                    px = int(2 * t + am - 2 * (u + v))
                    pz = l - 2 * t - am
                    key = (px, py, pz)
                    coeffs[key] = coeffs.get(key, Fraction(0)) + c
                    v += 1
        for key, c in coeffs.items():
            if c != 0:
                out[index[key], col] = float(c) * nrm
    return out * math.sqrt((2 * l + 1) / (4 * math.pi))


@dataclass
class BasisData:
    """dftax's basis layout (``gto.py:132-156``) as host numpy arrays."""

    centers: np.ndarray       # (nao_cart, 3) float64, Bohr
    exponents: np.ndarray     # (nao_cart, max_prim) float64, zero padded
    coefficients: np.ndarray  # (nao_cart, max_prim) float64, zero padded
    angular: np.ndarray       # (nao_cart, 3) int32
    cart2sph: np.ndarray | None  # (nao_cart, nao_sph) float64 or None
    max_l: int = 4

    @property
    def nao_cart(self) -> int:
        return int(self.angular.shape[0])

    @property
    def nao(self) -> int:
        return int(self.cart2sph.shape[1]) if self.cart2sph is not None else self.nao_cart


def _block_diag(blocks: list[np.ndarray]) -> np.ndarray:
    nr = sum(b.shape[0] for b in blocks)
    nc = sum(b.shape[1] for b in blocks)
    out = np.zeros((nr, nc))
    r = c = 0
    for b in blocks:
        out[r:r + b.shape[0], c:c + b.shape[1]] = b
        r += b.shape[0]
        c += b.shape[1]
    return out


def build_basis_data(symbols, coords_bohr, shells_by_element, *, spherical=True,
                     return_atom_index=False):
    """Assemble :class:`BasisData` for a molecule (``loader.py:85-160``).

    ``shells_by_element`` maps an element symbol to a list of contracted shells
    ``(l, exponents, coefficients)`` in emission order; each shell expands to its
    cartesian components with the normalization described in the module doc.
    """
    coords = np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3)
    raw = []
    for atom, (sym, center) in enumerate(zip(symbols, coords)):
        for l, exps, cs in shells_by_element[sym]:
            raw.append((int(l), np.asarray(exps, float), np.asarray(cs, float),
                        center, atom))
    if not raw:
        raise ValueError("empty basis")
    max_prim = max(len(e) for (_, e, _, _, _) in raw)
    centers, ex, co, ang, atom_index = [], [], [], [], []
    for l, exps, c_raw, center, atom in raw:
        if l > L_MAX:
            raise ValueError(f"angular momentum l={l} exceeds the supported l<={L_MAX}")
        c_prim = c_raw * np.array([gto_norm(l, a) for a in exps])
        for comp in cart_components(l):
            c_final = c_prim * contracted_norm(exps, c_prim, comp) if l <= 1 else c_prim.copy()
            pe = np.zeros(max_prim)
            pc = np.zeros(max_prim)
            pe[:len(exps)] = exps
            pc[:len(c_final)] = c_final
            centers.append(center)
            ex.append(pe)
            co.append(pc)
            ang.append(comp)
            atom_index.append(atom)
    c2s = _block_diag([cart2sph_block(l) for (l, *_rest) in raw]) if spherical else None
    basis = BasisData(
        centers=np.array(centers, dtype=np.float64),
        exponents=np.array(ex, dtype=np.float64),
        coefficients=np.array(co, dtype=np.float64),
        angular=np.array(ang, dtype=np.int32),
        cart2sph=c2s,
        max_l=int(max(l for (l, *_r) in raw)),
    )
    if return_atom_index:
        return basis, np.array(atom_index, dtype=np.int64)
    return basis
