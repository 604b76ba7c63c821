"""The compiled CPU restatement (oracle/cpu_df.cpp + oracle/cpu.py), the timed
CPU baseline of bench.py, pinned like the numpy oracle: against the
reference's golden fixtures and against the numpy oracle on multi-molecule
inputs. Tolerances: integrals 1e-13 absolute, (P|Q) 1e-12, J/K/E 1e-12
relative (same integrals and metric, different contraction order)."""

import numpy as np
import pytest

from conftest import golden_basis, load_golden, unpack_tril


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def cpu():
    from oracle import cpu as ocpu

    ocpu.build_lib()
    return ocpu


def test_water_matches_reference_golden(cpu):
    g = load_golden("water")
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    I3 = cpu.eri3c_dense(orb, aux, nthreads=2)
    assert np.abs(I3 - unpack_tril(g["int3c_tril"], I3.shape[0])).max() < 1e-13
    assert np.abs(cpu.eri2c(aux, nthreads=2) - g["int2c"]).max() < 1e-12


def test_ch2_high_l_matches_reference_golden(cpu):
    g = load_golden("ch2")
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    I3 = cpu.eri3c_dense(orb, aux, nthreads=3)
    v = I3[g["sample_m"], g["sample_n"], g["sample_P"]]
    assert np.abs(v - g["sample_val"]).max() < 1e-13
    assert np.abs(cpu.eri2c(aux) - g["int2c"]).max() < 1e-12


@pytest.mark.parametrize("name", ["water3", "alkane2"])
def test_matches_numpy_oracle(cpu, name):
    from dftax_b200 import systems
    from oracle import md as omd

    _, _, orb, aux, _ = systems.workload(name, seed=2)
    assert np.abs(cpu.eri3c_dense(orb, aux) - omd.eri3c(orb, aux)).max() < 1e-13
    assert np.abs(cpu.eri2c(aux) - omd.eri2c(aux)).max() < 1e-12


def test_screened_pairs_stay_zero(cpu):
    g = load_golden("water")
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    keep = {(int(a), int(b)) for a, b in g["screen_keep"]}
    I3s = cpu.eri3c_dense(orb, aux, keep_pairs=keep)
    I3 = unpack_tril(g["int3c_tril"], I3s.shape[0])
    nz = np.abs(I3s).max(axis=2) > 0
    assert np.abs(I3s[nz] - I3[nz]).max() < 1e-13
    assert np.all(I3s[~nz] == 0.0) and (~nz).any()


def test_build_jk_matches_reference_energy(cpu):
    """The full build (metric, V+, 3-center, J, K by dftax's einsum path)
    against the reference's golden J, K and DFCoulomb energy."""
    g = load_golden("water")
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    r = cpu.df_build_jk(orb, aux, g["C"], hf_coeff=0.25)
    assert rel(r["J"], g["J"]) < 5e-10
    assert rel(r["K"], g["K"]) < 5e-10
    assert abs(r["E"] - g["e_total"]) < 5e-10 * abs(g["e_total"])
    assert set(r["seconds"]) == {"eri2c", "metric", "eri3c", "j", "k"}


def test_k_path_equals_einsum(cpu):
    from oracle import df as odf

    rng = np.random.default_rng(4)
    I3 = rng.standard_normal((7, 7, 11))
    I3 = I3 + I3.transpose(1, 0, 2)
    A = rng.standard_normal((11, 11))
    vinv = A @ A.T
    D = rng.standard_normal((7, 7))
    D = D + D.T
    assert rel(cpu.k_reference_path(I3, vinv, D), odf.df_k(I3, vinv, D)) < 1e-13


@pytest.mark.parametrize("nspin", [1, 2])
def test_gradient_oracle_equals_finite_differences(cpu, nspin):
    """The oracle's DF gradient (weights G, W contracted with integral
    derivatives) against central differences of the whole oracle energy, on
    the water molecule with its own orbital basis as the fitting basis: that
    metric is well conditioned and drops no direction, so the pseudo-inverse
    rule d(V+) = -V+ dV V+ is the exact derivative and both must agree."""
    from dftax_b200 import systems

    _, xyz, orb, _, nocc = systems.workload("water", seed=0)
    aux = orb
    C = systems.random_occupied(orb.nao, nocc, seed=1)
    P = 2.0 * C @ C.T if nspin == 1 else np.stack([C @ C.T, C[:, :-1] @ C[:, :-1].T])
    E, g = cpu.df_energy_grad(orb, aux, P, 0.25, xyz)
    assert abs(E - cpu.df_energy(orb, aux, P, 0.25)) < 1e-12 * abs(E)
    h = 1e-3
    fd = np.zeros_like(g)
    for A in range(len(xyz)):
        for x in range(3):
            def e(d):
                return cpu.df_energy(cpu._moved(orb, xyz, A, x, d), cpu._moved(aux, xyz, A, x, d),
                                     P, 0.25)
            d1 = (e(h) - e(-h)) / (2 * h)
            d2 = (e(h / 2) - e(-h / 2)) / h
            fd[A, x] = (4 * d2 - d1) / 3
    assert np.abs(fd - g).max() < 1e-7 * np.abs(g).max()
    assert np.abs(g.sum(axis=0)).max() < 1e-9 * np.abs(g).max()
