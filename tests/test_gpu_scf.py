"""The device Kohn-Sham pieces and SCF (include/dfscf.h) against dftax's own
outputs (tests/golden/water_scf_ref.npz) and against the oracle
(oracle/ks.py, pinned to the same fixtures in test_oracle_ks.py).

Tolerances: one-electron integrals 1e-13 absolute (V 1e-12); the grid's
points 1e-12 and weights 1e-13 relative; E_xc 1e-12 relative and Tr(Vxc Q)
1e-7 relative against the reference's difference quotient; E(P) and F(P)
5e-10 relative (the DF Coulomb floor); converged SCF energies 1e-8 Ha apart
with e_tol 1e-10 on both sides; mixed against float64 SCF 1 uHa.
"""

import numpy as np
import pytest

from conftest import golden_basis, load_golden, unpack_tril

pytestmark = pytest.mark.gpu

NOISE_REL = 5e-10


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def g():
    return load_golden("water_scf")


@pytest.fixture(scope="module")
def ks_small(g, water_golden):
    from dftax_b200 import df
    from dftax_b200.ks import KS

    orb, aux = golden_basis(water_golden, "orb"), golden_basis(water_golden, "aux")
    return KS(list(g["symbols"]), g["coords"], orb, coulomb=df(aux),
              grid=(g["grid_small_coords"], g["grid_small_weights"]))


@pytest.fixture(scope="module")
def oracle_small(g, water_golden):
    from oracle import ks as oks

    orb, aux = golden_basis(water_golden, "orb"), golden_basis(water_golden, "aux")
    I3 = unpack_tril(water_golden["int3c_tril"], orb.nao)
    return oks.KSEnergy(orb, aux, g["coords"], g["charges"], g["grid_small_coords"],
                        g["grid_small_weights"], I3=I3, vinv=water_golden["vinv"])


def test_one_electron_vs_reference(ks_small, g):
    S, T, V = (x.cpu().numpy() for x in ks_small.one_electron())
    assert np.abs(S - g["S"]).max() < 1e-13
    assert np.abs(T - g["T"]).max() < 1e-13
    assert np.abs(V - g["V"]).max() < 1e-12


def test_becke_grid_vs_reference(g):
    from scipy.spatial import cKDTree

    from dftax_b200.grid import becke_grid

    pts, w = becke_grid(list(g["symbols"]), g["coords"])
    ref_p, ref_w = g["grid_default_coords"], g["grid_default_weights"]
    assert pts.shape == ref_p.shape
    d, i = cKDTree(pts).query(ref_p)
    assert d.max() < 1e-12 and len(np.unique(i)) == len(i)
    assert np.abs(w[i] - ref_w).max() < 1e-13 * np.abs(ref_w).max()


def test_xc_energy_and_fock_vs_reference(ks_small, g):
    P = 2.0 * g["C"] @ g["C"].T
    e, V = ks_small.xc_energy(P)
    V = V.cpu().numpy()
    assert abs(e - g["e_xc"]) < 1e-12 * abs(g["e_xc"])
    assert np.abs(V - V.T).max() < 1e-14
    for Q, dE in zip(g["dexc_Q"], g["dexc"]):
        assert abs(np.sum(V * Q) - dE) < 1e-7 * abs(dE)


def test_energy_and_fock_vs_oracle(ks_small, oracle_small, g):
    rng = np.random.default_rng(12)
    C = np.linalg.qr(rng.standard_normal((ks_small.nao, 5)))[0]
    P = 2.0 * C @ C.T
    e, F = ks_small.total(P)
    er, Fr = oracle_small.energy_fock(P)
    assert abs(e - er) < NOISE_REL * abs(er)
    assert rel(F.cpu().numpy(), Fr) < NOISE_REL


def test_scf_vs_oracle_on_reference_grid(ks_small, oracle_small):
    from dftax_b200.ks import scf
    from oracle import ks as oks

    r = scf(ks_small, e_tol=1e-10, d_tol=1e-8)
    er, Pr, epsr, _, nr, convr = oks.scf(oracle_small, 5, e_tol=1e-10, d_tol=1e-8)
    assert r.converged and convr
    assert abs(r.e_tot - er) < 1e-8
    assert np.abs(r.P[0] - Pr).max() < 1e-6
    assert np.abs(r.mo_energy[0][:8] - epsr[:8]).max() < 1e-6
    assert abs(r.n_iter - nr) <= 2
    # the energy reported is the energy of the returned density
    e2, _ = ks_small.total(r.P[0])
    assert abs(e2 - r.e_tot) < 1e-10


def test_scf_default_grid_and_warm_restart(g, water_golden):
    """The product's own Becke grid (75 radial, 302 Lebedev, NWChem pruning),
    then a restart from the converged density converges at once."""
    from dftax_b200 import df
    from dftax_b200.ks import KS, scf

    orb, aux = golden_basis(water_golden, "orb"), golden_basis(water_golden, "aux")
    ks = KS(list(g["symbols"]), g["coords"], orb, coulomb=df(aux))
    r = scf(ks)
    assert r.converged
    r2 = scf(ks, guess=r.P)
    assert r2.converged and r2.n_iter <= 3
    assert abs(r2.e_tot - r.e_tot) < 1e-8


@pytest.mark.parametrize("xc,hf,xs,cs", [("PBE", 0.0, 1.0, 1.0), ("HF", 1.0, 0.0, 0.0)])
def test_other_functionals_vs_oracle(g, water_golden, xc, hf, xs, cs):
    """PBE (no exact exchange) and HF (no XC) through the same energy and Fock."""
    from dftax_b200 import df
    from dftax_b200.ks import KS
    from oracle import ks as oks

    orb, aux = golden_basis(water_golden, "orb"), golden_basis(water_golden, "aux")
    ks = KS(list(g["symbols"]), g["coords"], orb, coulomb=df(aux), xc=xc,
            grid=(g["grid_small_coords"], g["grid_small_weights"]))
    I3 = unpack_tril(water_golden["int3c_tril"], orb.nao)
    model = oks.KSEnergy(orb, aux, g["coords"], g["charges"], g["grid_small_coords"],
                         g["grid_small_weights"], hf_coeff=hf, I3=I3, vinv=water_golden["vinv"],
                         xs=xs, cs=cs)
    rng = np.random.default_rng(3)
    C = np.linalg.qr(rng.standard_normal((ks.nao, 5)))[0]
    P = 2.0 * C @ C.T
    e, F = ks.total(P)
    er, Fr = model.energy_fock(P)
    assert abs(e - er) < NOISE_REL * abs(er)
    assert rel(F.cpu().numpy(), Fr) < NOISE_REL


def test_mixed_precision_scf_within_one_microhartree():
    """(H2O)_4: the same SCF with the int8 tensor-core J/K plan against float64."""
    from dftax_b200 import df, systems
    from dftax_b200.grid import becke
    from dftax_b200.ks import KS, scf

    sym, xyz, orb, aux, nocc = systems.workload("water4", seed=1)
    grid = becke(50, 194)
    r64 = scf(KS(sym, xyz, orb, coulomb=df(aux), grid=grid))
    rmx = scf(KS(sym, xyz, orb, coulomb=df(aux, precision="mixed"), grid=grid))
    assert r64.converged and rmx.converged
    assert abs(rmx.e_tot - r64.e_tot) < 1e-6


def test_screened_xc_equals_dense_quadrature():
    """(H2O)_8 on the default grid: the spatially sorted, shell-screened XC
    (ao_thresh 1e-14, 8192-point chunks) against the dense quadrature
    (ao_thresh 0, one shell list for all points) at 1e-12 relative."""
    from dftax_b200 import df, systems
    from dftax_b200.ks import KS

    sym, xyz, orb, aux, nocc = systems.workload("water8", seed=2)
    sparse = KS(sym, xyz, orb, coulomb=df(aux))
    dense = KS(sym, xyz, orb, coulomb=df(aux), plan=sparse.plan, ao_thresh=0.0,
               grid=(sparse.grid_coords, sparse.grid_weights))
    C = systems.random_occupied(orb.nao, nocc, seed=5)
    P = 2.0 * C @ C.T
    e1, V1 = sparse.xc_energy(P)
    e2, V2 = dense.xc_energy(P)
    assert abs(e1 - e2) < 1e-12 * abs(e2)
    assert rel(V1.cpu().numpy(), V2.cpu().numpy()) < 1e-12


def test_xc_graph_replay_is_bitwise_equal(ks_small, g):
    """The same P and V buffers three times: the first evaluation launches
    directly, the second captures its launches in a CUDA graph, the third
    replays it; all three give the same bits."""
    import ctypes

    import torch

    from dftax_b200 import _lib

    P = torch.as_tensor(2.0 * g["C"] @ g["C"].T, device=ks_small.dev)
    V = torch.empty_like(P)
    out = []
    for _ in range(3):
        e = ctypes.c_double()
        _lib.check(ks_small.lib.dfscf_xc(ks_small.h, P.data_ptr(), ctypes.byref(e), V.data_ptr(),
                                         None), ks_small.ctx.h)
        torch.cuda.synchronize()
        out.append((e.value, V.cpu().numpy().copy()))
    assert out[0][0] == out[1][0] == out[2][0]
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][1], out[2][1])


def test_autotuned_chunk_scf_matches_fixed_chunk():
    """(H2O)_3: the SCF with the autotuned XC chunk (and its CUDA graph)
    against 8192-point chunks: the same energy to 1e-10 Ha."""
    from dftax_b200 import df, systems
    from dftax_b200.grid import becke
    from dftax_b200.ks import KS, scf

    sym, xyz, orb, aux, nocc = systems.workload("water3", seed=4)
    grid = becke(50, 194)
    a = KS(sym, xyz, orb, coulomb=df(aux), grid=grid)
    ra = scf(a)
    b = KS(sym, xyz, orb, coulomb=df(aux), grid=(a.grid_coords, a.grid_weights),
           plan=a.plan, grid_chunk=8192)
    rb = scf(b)
    assert ra.converged and rb.converged
    assert ra.xc_chunk in (4096, 8192, 16384) and rb.xc_chunk == 8192
    assert ra.xc_graph and rb.xc_graph
    assert abs(ra.e_tot - rb.e_tot) < 1e-10
