"""Atom-centered Becke molecular grids for the XC quadrature.

The layout follows dftax's ``becke_grid`` (``dftax/grid/grid.py:139-255``,
``dftax/grid/becke.py``): per atom, second-kind Chebyshev radial nodes mapped
by r = R (1 + x) / (1 - x) with R the Bragg radius (half of it except for H),
shells past ``r_max`` dropped, a Lebedev angular rule per shell chosen by the
NWChem pruning regions of r / R_Bragg, and Becke's fuzzy-Voronoi partition
with the Bragg-radius size adjustment; points whose weight is at or below
``cutoff`` are then dropped, as dftax's ``KS`` does (``energy.py:229-256``).

The radial nodes, pruning and angular points are laid out on the host (numpy;
the Lebedev rules are SciPy's ``lebedev_rule``, the same published quadratures
dftax vendors); the partition, natom^2 work per point, runs on the device
(``dfjk_becke_partition``).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from functools import lru_cache

import numpy as np

from . import _lib

# Bragg-Slater radii of H..Ne in Bohr, rounded to 8 decimals as dftax
# tabulates them (0.35, 1.40, 1.45, 1.05, 0.85, 0.70, 0.65, 0.60, 0.50, 1.50
# Angstrom): the radial scale and the partition use these rounded values.
BRAGG_BOHR = {1: 0.66140414, 2: 2.64561657, 3: 2.74010288, 4: 1.98421243, 5: 1.60626721,
              6: 1.32280829, 7: 1.22832198, 8: 1.13383567, 9: 0.94486306, 10: 2.83458919}
ATOMIC_NUMBER = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9,
                 "Ne": 10}
LEBEDEV_LADDER = (6, 14, 26, 38, 50, 74, 86, 110, 146, 170, 194, 230, 266, 302, 350, 434, 590,
                  770)
_LEBEDEV_DEGREE = {6: 3, 14: 5, 26: 7, 38: 9, 50: 11, 74: 13, 86: 15, 110: 17, 146: 19, 170: 21,
                   194: 23, 230: 25, 266: 27, 302: 29, 350: 31, 434: 35, 590: 41, 770: 47}
# NWChem region boundaries on r / R_Bragg; rows H-He, Li-Ne, Na and up
_NWCHEM_ALPHAS = np.array(((0.25, 0.5, 1.0, 4.5), (0.1667, 0.5, 0.9, 3.5), (0.1, 0.4, 0.8, 2.5)))


@dataclass(frozen=True)
class Becke:
    """Becke grid spec (dftax ``becke()``): radial shells per atom, the largest
    Lebedev order, pruning scheme, radial cutoff and weight cutoff."""

    n_radial: int = 75
    lebedev: int = 302
    prune: str | None = "nwchem"
    r_max: float | None = 45.0
    cutoff: float | None = 1e-15


def becke(n_radial: int = 75, lebedev: int = 302, *, prune: str | None = "nwchem",
          r_max: float | None = 45.0, cutoff: float | None = 1e-15) -> Becke:
    if lebedev not in _LEBEDEV_DEGREE:
        raise ValueError(f"lebedev={lebedev} is not a Lebedev order; available: "
                         f"{list(LEBEDEV_LADDER)}")
    if prune not in ("nwchem", None):
        raise ValueError(f"unknown prune scheme {prune!r}; use 'nwchem' or None.")
    return Becke(n_radial, lebedev, prune, r_max, cutoff)


def bragg_radius(Z: int) -> float:
    if Z not in BRAGG_BOHR:
        raise ValueError(f"Becke grid radii are tabulated here for H..Ne; got Z={Z}")
    return BRAGG_BOHR[Z]


@lru_cache(maxsize=None)
def lebedev(npts: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit-sphere points (n, 3) and weights summing to 4 pi."""
    from scipy.integrate import lebedev_rule

    x, w = lebedev_rule(_LEBEDEV_DEGREE[int(npts)])
    return np.ascontiguousarray(x.T), np.ascontiguousarray(w)


def becke_radial(n: int, scale: float):
    i = np.arange(1, n + 1)
    theta = i * np.pi / (n + 1)
    x = np.cos(theta)
    r = scale * (1.0 + x) / (1.0 - x)
    drdx = 2.0 * scale / (1.0 - x) ** 2
    return r, (np.pi / (n + 1)) * np.sin(theta) * r ** 2 * drdx


def _nwchem_orders(Z: int, r: np.ndarray, n_ang: int) -> np.ndarray:
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


@lru_cache(maxsize=None)
def _atom_template(Z: int, n_radial: int, n_ang: int, prune, r_max):
    """Unit-free template of one atom: offsets (n, 3) and raw weights (n,)."""
    scale = bragg_radius(Z) if Z == 1 else 0.5 * bragg_radius(Z)
    r, wr = becke_radial(n_radial, scale)
    if r_max is not None:
        keep = r <= r_max
        r, wr = r[keep], wr[keep]
    orders = _nwchem_orders(Z, r, n_ang) if prune == "nwchem" else np.full(len(r), n_ang)
    offs, raw = [], []
    for i in range(len(r)):
        u, w = lebedev(int(orders[i]))
        offs.append(r[i] * u)
        raw.append(wr[i] * w)
    return np.concatenate(offs), np.concatenate(raw)


def becke_grid(symbols, coords_bohr, spec: Becke | None = None, *, device: int = 0):
    """(points (n, 3), weights (n,)) as host float64 arrays."""
    import torch

    from .coulomb import Context

    spec = spec or Becke()
    coords = np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3)
    Zs = [ATOMIC_NUMBER[s] for s in symbols]
    tmpl = [_atom_template(Z, spec.n_radial, spec.lebedev, spec.prune,
                           None if spec.r_max is None else float(spec.r_max)) for Z in Zs]
    counts = np.array([len(w) for _, w in tmpl], dtype=np.int64)
    n = int(counts.sum())
    pts = np.empty((n, 3))
    raw = np.empty(n)
    o = 0
    for a, (off, w) in enumerate(tmpl):
        np.add(off, coords[a], out=pts[o:o + len(w)])
        raw[o:o + len(w)] = w
        o += len(w)
    owner = np.repeat(np.arange(len(Zs), dtype=np.int32), counts)
    ctx = Context.get(device)
    dev = f"cuda:{ctx.device}"
    dp = torch.as_tensor(pts, device=dev)
    do = torch.as_tensor(owner, device=dev)
    dr = torch.as_tensor(raw, device=dev)
    dw = torch.empty_like(dr)
    bragg = np.array([bragg_radius(Z) for Z in Zs])
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(ctx.lib.dfjk_becke_partition(ctx.h, dp.data_ptr(), do.data_ptr(), dr.data_ptr(),
                                            len(raw), len(Zs), coords.ctypes.data,
                                            bragg.ctypes.data, dw.data_ptr(), stream), ctx.h)
    if spec.cutoff is not None:
        # the points of negligible weight are dropped on the device
        keep = dw.abs() > spec.cutoff
        return dp[keep].cpu().numpy(), dw[keep].cpu().numpy()
    return pts, dw.cpu().numpy()


__all__ = ["Becke", "becke", "becke_grid", "lebedev", "bragg_radius", "BRAGG_BOHR"]
