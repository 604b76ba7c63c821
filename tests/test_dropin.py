"""The dftax-facing layer: ``df()``, ``make_coulomb`` and ``B200DFCoulomb``
(the mirror of ``DFCoulomb``, ``dftax/ks/terms.py:576-613``, and of
``_make_coulomb``, ``terms.py:951-988``).

The argument checks run on any machine; the energy and Fock checks need the
GPU and compare with the reference's golden water values (closed shell) and
with the oracle's formula (open shell), at NOISE_REL in float64 and at the
mixed tolerances in mixed precision.
"""

import numpy as np
import pytest

from conftest import golden_basis, unpack_tril

NOISE_REL = 5e-10


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_df_spec_defaults_and_fields():
    from dftax_b200 import df

    s = df("aux", screen=1e-10, precision="mixed")
    assert (s.auxbasis, s.screen, s.backend, s.precision, s.chunk) == ("aux", 1e-10, "b200",
                                                                          "mixed", None)
    assert df().precision == "fp64"
    assert df(chunk="auto").chunk is None   # "auto" resolves to materialized B
    assert df(chunk=4096).chunk == 4096     # an integer chunk selects the streamed form


@pytest.mark.parametrize("kw,msg", [
    ({"backend": "jax"}, "backend"),
    ({"chunk": -1}, "chunk"),
    ({"chunk": "big"}, "chunk"),
    ({"spherical": False}, "spherical"),
    ({"precision": "bf16"}, "precision"),
])
def test_df_rejects_unsupported_arguments(kw, msg):
    from dftax_b200 import df

    with pytest.raises(ValueError, match=msg):
        df("aux", **kw)


def test_make_coulomb_type_checks(water_golden):
    from dftax_b200 import df, make_coulomb

    orb = golden_basis(water_golden, "orb")
    with pytest.raises(TypeError):
        make_coulomb({"auxbasis": None}, orb, 0.25)
    with pytest.raises(TypeError):
        make_coulomb(df("not a basis"), orb, 0.25)


def test_range_separated_needs_omega(water_golden):
    from dftax_b200 import B200DFCoulomb

    g = water_golden
    with pytest.raises(ValueError, match="omega"):
        B200DFCoulomb(golden_basis(g, "orb"), golden_basis(g, "aux"), 0.2, hf_coeff_lr=0.8)


def test_ks_rejects_an_unknown_density_route(water_golden):
    """Checked before any device work."""
    from dftax_b200 import df
    from dftax_b200.ks import KS

    orb, aux = golden_basis(water_golden, "orb"), golden_basis(water_golden, "aux")
    with pytest.raises(ValueError, match="density must be one of"):
        KS(["O", "H", "H"], np.zeros((3, 3)), orb, coulomb=df(aux), density="diagonalize")


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", NOISE_REL), ("mixed", 1e-7)])
def test_make_coulomb_energy_and_fock_vs_reference(water_golden, precision, tol):
    from dftax_b200 import B200DFCoulomb, df, make_coulomb

    g = water_golden
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    term = make_coulomb(df(aux, precision=precision), orb, 0.25)
    assert isinstance(term, B200DFCoulomb)
    C = g["C"]
    P = 2.0 * C @ C.T
    e = term.energy(P[None], None, (5,))
    assert abs(e - g["e_total"]) < tol * abs(g["e_total"])
    e2, F = term.fock(P[None])
    assert e2 == e
    assert tuple(F.shape) == (1,) + P.shape
    assert rel(F[0].cpu().numpy(), 2.0 * g["J"] - 0.25 * g["K"]) < tol
    J, K = term.jk(C)
    assert rel(J.cpu().numpy(), g["J"]) < tol
    assert rel(K.cpu().numpy(), g["K"]) < max(tol, 1e-7)


@pytest.mark.gpu
def test_make_coulomb_open_shell_vs_oracle(water_golden):
    from dftax_b200 import df, make_coulomb
    from oracle import df as odf

    g = water_golden
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    term = make_coulomb(df(aux), orb, 0.25)
    rng = np.random.default_rng(31)
    n = g["C"].shape[0]
    Ca = np.linalg.qr(rng.standard_normal((n, 5)))[0]
    Cb = np.linalg.qr(rng.standard_normal((n, 4)))[0]
    P = np.stack([Ca @ Ca.T, Cb @ Cb.T])
    e, F = term.fock(P)
    I3 = unpack_tril(g["int3c_tril"], n)
    er = odf.df_energy(I3, g["vinv"], P, 0.25)
    assert abs(e - er) < NOISE_REL * abs(er)
    Jt, _ = odf.df_jk(I3, g["vinv"], P.sum(0))
    for s in range(2):
        assert rel(F[s].cpu().numpy(), Jt - 0.25 * odf.df_k(I3, g["vinv"], P[s])) < NOISE_REL


@pytest.mark.gpu
def test_make_coulomb_screened_matches_reference_screen(water_golden):
    """df(screen=...) reaches the plan: its kept pairs are the reference's."""
    from dftax_b200 import df, make_coulomb

    g = water_golden
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    term = make_coulomb(df(aux, screen=float(g["screen_thresh"])), orb, 0.25)
    assert term.plan.kept_pairs() == {(int(a), int(b)) for a, b in g["screen_keep"]}
