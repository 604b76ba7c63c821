"""Golden fixtures of the rest of the Kohn-Sham energy, made by dftax's own code.

Run from the repository root, in a checkout that has the reference sources:

    python tests/golden/make_golden_scf.py --ref PATH_TO_DFTAX_CHECKOUT

Like ``make_golden.py`` it runs the reference's unmodified functions through
``jax_numpy_shim`` (JAX is not installed). For the water monomer of
``water_ref.npz`` (same basis, same occupied C):

* ``dftax/integrals/eri3c_bucketed.py``: ``overlap_kinetic_bucketed`` and
  ``nuclear_attraction_bucketed`` (S, T, V);
* ``dftax/integrals/nuclear_repulsion.py``: ``nuclear_repulsion``;
* ``dftax/grid/grid.py``: ``becke_grid`` (Becke radial shells, NWChem
  pruning, Lebedev angular grids, Becke partition) for a reduced spec
  (``n_radial=40, lebedev=110``) and the default one (75, 302), with the
  1e-15 weight cutoff that ``KS`` applies;
* ``dftax/energy/gto.py``: ``eval_gto`` at a sample of grid points, and its
  gradient by complex-step differentiation of the same function (exact to
  rounding: every operation in it is analytic);
* ``dftax/energy/grid.py``: ``xc_energy`` with ``dftax/energy/xc.py``'s
  ``PBE0`` on the reduced grid for P = 2 C C^T, with rho and grad rho from
  ``GridXC.density``'s contractions of those AO values; and the directional
  derivative of that E_xc along seeded symmetric directions Q (central
  differences, Richardson-extrapolated), which a Fock matrix V_xc must
  reproduce as Tr(V_xc Q);
* ``PBE0`` itself at seeded (rho, grad rho) inputs: the energy density per
  particle and, by Richardson-extrapolated central differences, the
  derivatives of rho * eps_xc with respect to rho and to each component of
  grad rho.

Output: ``tests/golden/water_scf_ref.npz``. Nothing at run time needs the
reference.
"""

from __future__ import annotations

import argparse
import importlib
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import jax_numpy_shim as shim  # noqa: E402
import make_golden as mg  # noqa: E402

from dftax_b200 import systems  # noqa: E402


def _extend_shim():
    jnp = shim.jnp
    for name in ("expm1", "log1p", "exp", "log", "sqrt", "clip", "where", "sum", "abs",
                 "atleast_1d", "maximum", "minimum"):
        if not hasattr(jnp, name):
            setattr(jnp, name, shim._w(getattr(np, name)))
    # jnp.clip(x, lo) with one bound, as JAX allows
    jnp.clip = shim._w(lambda a, a_min=None, a_max=None, min=None, max=None: np.clip(
        a, a_min if a_min is not None else min, a_max if a_max is not None else max))
    import typing
    if not hasattr(shim.eqx, "AbstractClassVar"):
        shim.eqx.AbstractClassVar = typing.ClassVar   # annotation only: not a dataclass field
    if not hasattr(jnp, "unstack"):
        jnp.unstack = lambda a, axis=0: tuple(np.moveaxis(np.asarray(a), axis, 0))


def load(ref):
    R = mg.load_reference(ref)
    _extend_shim()
    pkg = os.path.join(ref, "dftax")
    mg._fake_package("dftax.grid", os.path.join(pkg, "grid"))
    mg._fake_package("dftax.system", os.path.join(pkg, "system"))
    utils = sys.modules["dftax.utils"]
    utils.vmap = lambda fun, in_axes=0, out_axes=0, chunk_size=None, **k: shim.vmap(fun, in_axes)
    lebedev = importlib.import_module("dftax.grid.lebedev")
    path = os.path.join(pkg, "grid", "data", "lebedev.npz")

    def _tables():
        with np.load(path) as z:
            return {k: np.asarray(z[k], dtype=np.float64) for k in z.files}
    lebedev._tables = _tables
    R.grid = importlib.import_module("dftax.grid.grid")
    R.nrep = importlib.import_module("dftax.integrals.nuclear_repulsion")
    R.xc = importlib.import_module("dftax.energy.xc")
    R.egrid = importlib.import_module("dftax.energy.grid")
    return R


def _ao(R, orb, pts):
    """eval_gto at the points and its gradient by complex step (h = 1e-30)."""
    h = 1e-30
    vals = np.stack([np.asarray(R.gto.eval_gto(orb, p)) for p in pts])
    grads = np.zeros(vals.shape + (3,))
    cb = types.SimpleNamespace(**{k: getattr(orb, k) for k in
                                  ("centers", "exponents", "coefficients", "angular", "cart2sph")})
    for x in range(3):
        step = np.zeros(3, dtype=complex)
        step[x] = 1j * h
        grads[:, :, x] = np.stack([np.imag(np.asarray(
            R.gto.eval_gto(cb, p.astype(complex) + step))) / h for p in pts])
    return vals, grads


def _richardson(f, h):
    """f'(0) from central differences at h and h/2 (error O(h^4))."""
    d1 = (f(h) - f(-h)) / (2 * h)
    d2 = (f(h / 2) - f(-h / 2)) / h
    return (4.0 * d2 - d1) / 3.0


def make(R, out):
    t0 = time.time()
    sym, xyz = systems.water_monomer()
    charges = np.array([8.0, 1.0, 1.0])
    orb = R.loader.build_basis_data(sym, xyz, "even-tempered-orbital", spherical=True)
    S, T = (np.asarray(x) for x in R.eb.overlap_kinetic_bucketed(orb))
    V = np.asarray(R.eb.nuclear_attraction_bucketed(orb, xyz, charges))
    e_nn = float(R.nrep.nuclear_repulsion(xyz, charges))
    print(f"one-electron {time.time() - t0:.1f}s", flush=True)

    grids = {}
    for tag, (nr, nl) in {"small": (40, 110), "default": (75, 302)}.items():
        gc, gw = R.grid.becke_grid(sym, xyz, n_radial=nr, lebedev=nl)
        gc, gw = np.asarray(gc), np.asarray(gw)
        keep = np.abs(gw) > 1e-15
        grids[tag] = (gc[keep], gw[keep])
        print(f"grid {tag}: {keep.sum()} points {time.time() - t0:.1f}s", flush=True)
    gc, gw = grids["small"]

    nao = S.shape[0]
    rng = np.random.default_rng(0)             # the C of water_ref.npz
    C, _ = np.linalg.qr(rng.standard_normal((nao, 5)))
    P = 2.0 * C @ C.T
    ao, dao = _ao(R, orb, gc)
    print(f"AO values {time.time() - t0:.1f}s", flush=True)
    xc = R.xc.PBE0()

    def exc(Pm):
        rho = np.einsum("gm,mn,gn->g", ao, Pm, ao)
        grad = 2.0 * np.einsum("gm,mn,gnx->gx", ao, Pm, dao)
        return float(R.egrid.xc_energy(xc, rho, gw, grad_rho=grad))

    e_xc = exc(P)
    qrng = np.random.default_rng(42)
    Qs, dE = [], []
    for _ in range(3):
        A = qrng.standard_normal((nao, nao)) * 0.05
        Q = A + A.T
        Qs.append(Q)
        dE.append(_richardson(lambda t: exc(P + t * Q), 1e-4))
    print(f"E_xc {e_xc:.12f} {time.time() - t0:.1f}s", flush=True)

    # PBE0 at seeded inputs: eps and the derivatives of rho * eps
    prng = np.random.default_rng(7)
    n = 60
    rho_s = 10.0 ** prng.uniform(-6, 2, n)
    grad_s = prng.standard_normal((n, 3)) * rho_s[:, None] ** (4 / 3) * 10.0 ** prng.uniform(-1, 1, (n, 1))
    eps_s = np.array([float(xc(r, g)) for r, g in zip(rho_s, grad_s)])
    d_rho = np.zeros(n)
    d_grad = np.zeros((n, 3))
    for i in range(n):
        r, g = rho_s[i], grad_s[i]
        d_rho[i] = _richardson(lambda t: (r + t) * float(xc(r + t, g)), 1e-4 * r)
        for x in range(3):
            e = np.zeros(3)
            e[x] = 1.0
            hg = 1e-4 * np.linalg.norm(g)
            d_grad[i, x] = _richardson(lambda t: r * float(xc(r, g + t * e)), hg)

    sample = np.random.default_rng(3).choice(gc.shape[0], size=400, replace=False)
    np.savez(out, symbols=np.array(sym), coords=xyz, charges=charges, C=C, S=S, T=T, V=V,
             e_nn=e_nn, grid_small_coords=gc, grid_small_weights=gw,
             grid_default_coords=grids["default"][0], grid_default_weights=grids["default"][1],
             ao_sample_idx=sample, ao_sample=ao[sample], dao_sample=dao[sample],
             e_xc=e_xc, dexc_Q=np.stack(Qs), dexc=np.array(dE),
             pbe0_rho=rho_s, pbe0_grad=grad_s, pbe0_eps=eps_s, pbe0_drho=d_rho,
             pbe0_dgrad=d_grad)
    print(f"water_scf: E_xc={e_xc:.12f} e_nn={e_nn:.12f} {time.time() - t0:.1f}s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of a dftax checkout")
    a = ap.parse_args()
    R = load(a.ref)
    make(R, os.path.join(HERE, "water_scf_ref.npz"))


if __name__ == "__main__":
    main()
