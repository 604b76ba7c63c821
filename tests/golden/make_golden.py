"""Generate the golden fixtures by running dftax's own DF code (the reference).

Run from the repository root, in a checkout that has the reference sources:

    python tests/golden/make_golden.py --ref PATH_TO_DFTAX_CHECKOUT

dftax needs JAX, which is not installed here; ``jax_numpy_shim`` stands in for
the handful of JAX features the DF path uses, so every number in the fixtures
is computed by the reference's unmodified functions:

* ``dftax/energy/boys.py``: ``_build_table``, ``boys``, ``_boys_ref``;
* ``dftax/basis/loader.py``: ``build_basis_data`` (fed by a stand-in for the
  Basis Set Exchange package that serves the even-tempered sets of
  ``dftax_b200.systems``), with ``dftax/energy/gto.py`` normalization;
* ``dftax/integrals/eri3c_bucketed.py``: ``plan_eri3c``,
  ``eri3c_matrix_bucketed``, ``eri2c_matrix_bucketed``, ``_shell_pair_keep``
  (through ``dftax/integrals/eri4c.py:schwarz_diagonal``);
* ``dftax/ks/terms.py``: ``_metric_pinv``, ``_rik_cholesky``,
  ``_rik_occ_orbitals``, ``_exchange_quadratic``, ``DFCoulomb.energy``;
* ``dftax/energy/hybrid.py``: ``df_k_matrix``.

J is the analytic P-gradient of the RI-J energy, ``J = int3c . (V+ gamma)``,
formed here from the reference's ``int3c`` and ``V+``; K is the reference's
``df_k_matrix``. Outputs: ``boys_ref.npz``, ``water_ref.npz``, ``water_rsh_ref.npz``
(the range-separated erf(omega r)/r form), ``ch2_ref.npz``.
The fixtures are read by the tests only; nothing at run time needs the
reference.
"""

from __future__ import annotations

import __future__
import argparse
import ast
import importlib
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

import jax_numpy_shim as shim  # noqa: E402

from dftax_b200 import systems  # noqa: E402


def _fake_package(name, path):
    mod = types.ModuleType(name)
    mod.__path__ = [path]
    spec = importlib.machinery.ModuleSpec(name, None, is_package=True)
    spec.submodule_search_locations = [path]
    mod.__spec__ = spec
    sys.modules[name] = mod
    return mod


def _install(ref):
    shim.install()
    pkg = os.path.join(ref, "dftax")
    _fake_package("dftax", pkg)
    _fake_package("dftax.integrals", os.path.join(pkg, "integrals"))
    _fake_package("dftax.utils", os.path.join(pkg, "utils"))
    _fake_package("dftax.ks", os.path.join(pkg, "ks"))
    vm = types.ModuleType("dftax.utils.vmap")
    vm.vmap = lambda fun, in_axes=0, out_axes=0, chunk_size=None, checkpoint=False, **k: \
        shim.vmap(fun, in_axes)
    sys.modules["dftax.utils.vmap"] = vm

    # periodictable stand-in (only symbol -> Z is used)
    pt = types.ModuleType("periodictable")
    zs = {"H": 1, "C": 6, "N": 7, "O": 8}
    pt.elements = types.SimpleNamespace(
        symbol=lambda s: types.SimpleNamespace(number=zs[s]))
    sys.modules["periodictable"] = pt

    # Basis Set Exchange stand-in serving this project's even-tempered sets
    bse = types.ModuleType("basis_set_exchange")
    zsym = {v: k for k, v in zs.items()}

    def get_basis(name, elements, header=False):
        sets = systems.ORBITAL_SETS if name == "even-tempered-orbital" else systems.AUX_SETS
        out = {}
        for z in elements:
            shells = []
            for l, exps, cs in sets[zsym[int(z)]]:
                shells.append({"angular_momentum": [l], "exponents": list(exps),
                               "coefficients": [list(cs)]})
            out[str(z)] = {"electron_shells": shells}
        return {"elements": out}

    bse.get_basis = get_basis
    sys.modules["basis_set_exchange"] = bse


def _extract(path, names, namespace):
    """Exec the named top-level defs/classes of a reference module into namespace."""
    src = open(path).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body
            if isinstance(n, (ast.FunctionDef, ast.ClassDef)) and n.name in names]
    missing = set(names) - {n.name for n in keep}
    if missing:
        raise RuntimeError(f"{path}: missing {sorted(missing)}")
    mod = ast.Module(body=keep, type_ignores=[])
    code = compile(mod, path, "exec", flags=__future__.annotations.compiler_flag,
                   dont_inherit=True)
    exec(code, namespace)
    return namespace


def load_reference(ref):
    _install(ref)
    boys = importlib.import_module("dftax.energy.boys")
    gto = importlib.import_module("dftax.energy.gto")
    loader = importlib.import_module("dftax.basis.loader")
    eb = importlib.import_module("dftax.integrals.eri3c_bucketed")
    hybrid = importlib.import_module("dftax.energy.hybrid")
    ns = {"jax": shim.jax, "jnp": shim.jnp, "eqx": shim.eqx, "abc": importlib.import_module("abc"),
          "Array": shim.jaxtyping.Array, "Float": shim.jaxtyping.Float,
          "Scalar": shim.jaxtyping.Scalar}
    terms = _extract(os.path.join(ref, "dftax", "ks", "terms.py"),
                     ["_metric_pinv", "_metric_pinv_jvp", "_rik_cholesky",
                      "_rik_occ_orbitals", "_exchange_quadratic", "CoulombTerm",
                      "DFCoulomb"], ns)
    return types.SimpleNamespace(boys=boys, gto=gto, loader=loader, eb=eb,
                                 hybrid=hybrid, terms=types.SimpleNamespace(**terms))


def _basis_arrays(prefix, b):
    return {f"{prefix}_centers": np.asarray(b.centers),
            f"{prefix}_exponents": np.asarray(b.exponents),
            f"{prefix}_coefficients": np.asarray(b.coefficients),
            f"{prefix}_angular": np.asarray(b.angular),
            f"{prefix}_cart2sph": np.asarray(b.cart2sph)}


def make_boys(R, out):
    tbl = np.asarray(R.boys._TBL_NP)
    rng = np.random.default_rng(7)
    t = np.concatenate([np.array([0.0, 1e-12, 1e-6, 0.05, 0.1, 0.15, 39.95, 40.0, 40.0 + 1e-9,
                                  45.0, 60.0, 200.0, 1e4]),
                        rng.uniform(0.0, 45.0, 400), rng.uniform(0.0, 2.0, 100)])
    vals = np.stack([np.asarray(R.boys.boys(n, t)) for n in range(19)])
    exact = np.stack([np.asarray(R.boys._boys_ref(n, t)) for n in range(19)])
    np.savez(out, table=tbl, t=t, boys=vals, boys_exact=exact)


def make_system(R, name, sym, xyz, nocc, out, seed, sample=None, screen=None):
    t0 = time.time()
    orb = R.loader.build_basis_data(sym, xyz, "even-tempered-orbital", spherical=True)
    aux = R.loader.build_basis_data(sym, xyz, "even-tempered-aux", spherical=True)
    plan = R.eb.plan_eri3c(orb, aux)
    int3c = np.asarray(R.eb.eri3c_matrix_bucketed(orb, aux, plan=plan))
    t1 = time.time()
    int2c = np.asarray(R.eb.eri2c_matrix_bucketed(aux))
    vinv = np.asarray(R.terms["_metric_pinv"](int2c) if isinstance(R.terms, dict)
                      else R.terms._metric_pinv(int2c))
    nao, naux = int3c.shape[0], int3c.shape[2]
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.standard_normal((nao, nocc)))
    D = C @ C.T
    P = 2.0 * D
    dfc = R.terms.DFCoulomb(int3c=int3c, int2c_inv=vinv, hf_coeff=0.25)
    e_total = float(dfc.energy(P[None], None, (nocc,)))
    e_j = float(R.terms.DFCoulomb(int3c=int3c, int2c_inv=vinv, hf_coeff=0.0)
                .energy(P[None], None, (nocc,)))
    gamma = np.einsum("mnP,mn->P", int3c, D)
    J = np.einsum("mnP,P->mn", int3c, vinv @ gamma)
    K = np.asarray(R.hybrid.df_k_matrix(D, int3c, vinv))
    w = np.linalg.eigvalsh(int2c)
    data = dict(symbols=np.array(sym), coords=xyz, nocc=nocc, C=C, int2c=int2c,
                vinv=vinv, e_total=e_total, e_j=e_j, J=J, K=K, metric_w=w,
                n_kept=int(np.sum(w > 1e-7 * w[-1])),
                **_basis_arrays("orb", orb), **_basis_arrays("aux", aux))
    pa, pb = np.tril_indices(nao)
    if sample is None:
        data["int3c_tril"] = int3c[pa, pb, :]
    else:
        idx = rng.choice(len(pa) * naux, size=sample, replace=False)
        pi, xi = np.divmod(idx, naux)
        data["sample_m"] = pa[pi].astype(np.int32)
        data["sample_n"] = pb[pi].astype(np.int32)
        data["sample_P"] = xi.astype(np.int32)
        data["sample_val"] = int3c[pa[pi], pb[pi], xi]
    if screen is not None:
        keep = R.eb._shell_pair_keep(orb, screen)
        data["screen_thresh"] = screen
        data["screen_keep"] = np.array(sorted(keep), dtype=np.int32)
    np.savez(out, **data)
    print(f"{name}: nao={nao} naux={naux} eri3c {t1 - t0:.1f}s total {time.time() - t0:.1f}s "
          f"E={e_total:.12f}", flush=True)


def make_rsh(R, out, omega=0.3, hf=0.2, hf_lr=0.8, seed=0, nocc=5):
    """Range-separated form of the water monomer: the erf(omega r)/r 3-center
    tensor and metric (``eri3c_matrix_bucketed(..., omega=)``,
    ``eri2c_matrix_bucketed(..., omega=)``), their pseudo-inverse, the
    long-range K and the DFCoulomb energy with both exchange terms."""
    t0 = time.time()
    sym, xyz = systems.water_monomer()
    orb = R.loader.build_basis_data(sym, xyz, "even-tempered-orbital", spherical=True)
    aux = R.loader.build_basis_data(sym, xyz, "even-tempered-aux", spherical=True)
    plan = R.eb.plan_eri3c(orb, aux)
    int3c = np.asarray(R.eb.eri3c_matrix_bucketed(orb, aux, plan=plan))
    int3c_lr = np.asarray(R.eb.eri3c_matrix_bucketed(orb, aux, omega=omega, plan=plan))
    int2c = np.asarray(R.eb.eri2c_matrix_bucketed(aux))
    int2c_lr = np.asarray(R.eb.eri2c_matrix_bucketed(aux, omega=omega))
    vinv = np.asarray(R.terms._metric_pinv(int2c))
    vinv_lr = np.asarray(R.terms._metric_pinv(int2c_lr))
    nao = int3c.shape[0]
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.standard_normal((nao, nocc)))
    D = C @ C.T
    P = 2.0 * D
    dfc = R.terms.DFCoulomb(int3c=int3c, int2c_inv=vinv, hf_coeff=hf, int3c_lr=int3c_lr,
                            int2c_inv_lr=vinv_lr, hf_coeff_lr=hf_lr)
    e_total = float(dfc.energy(P[None], None, (nocc,)))
    K_lr = np.asarray(R.hybrid.df_k_matrix(D, int3c_lr, vinv_lr))
    w = np.linalg.eigvalsh(int2c_lr)
    pa, pb = np.tril_indices(nao)
    np.savez(out, omega=omega, hf_coeff=hf, hf_coeff_lr=hf_lr, C=C, e_total=e_total,
             int3c_lr_tril=int3c_lr[pa, pb, :], int2c_lr=int2c_lr, vinv_lr=vinv_lr,
             K_lr=K_lr, metric_w_lr=w, n_kept_lr=int(np.sum(w > 1e-7 * w[-1])))
    print(f"water_rsh: omega={omega} E={e_total:.12f} kept={int(np.sum(w > 1e-7 * w[-1]))} "
          f"{time.time() - t0:.1f}s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of a dftax checkout")
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    R = load_reference(a.ref)
    if a.only in (None, "boys"):
        make_boys(R, os.path.join(HERE, "boys_ref.npz"))
    if a.only in (None, "water"):
        sym, xyz = systems.water_monomer()
        make_system(R, "water", sym, xyz, 5, os.path.join(HERE, "water_ref.npz"), seed=0,
                    screen=1e-3)
    if a.only in (None, "water_rsh"):
        make_rsh(R, os.path.join(HERE, "water_rsh_ref.npz"))
    if a.only in (None, "ch2"):
        ang = systems.ANGSTROM_TO_BOHR
        s = 1.09 / np.sqrt(3.0)
        sym = ["C", "H", "H"]
        xyz = np.array([[0.0, 0.0, 0.0], [s, s, s], [s, -s, -s]]) * ang
        make_system(R, "ch2", sym, xyz, 4, os.path.join(HERE, "ch2_ref.npz"), seed=1,
                    sample=20000)


if __name__ == "__main__":
    main()
