"""The oracle's Kohn-Sham pieces (oracle/ks.py) against dftax's own outputs
(tests/golden/water_scf_ref.npz, made by tests/golden/make_golden_scf.py).

Tolerances: one-electron integrals 1e-13 absolute; grid points 1e-13 and
weights 1e-13 relative (the Lebedev rules come from SciPy, matched point by
point to dftax's vendored tables); AO values 1e-14 and gradients 1e-12
(complex-step on dftax's side); PBE0 eps 1e-14 relative and its derivatives
1e-7 (rho) and 1e-6 (grad rho) relative: the reference side is a
Richardson-extrapolated central difference whose round-off, eps |rho e_xc| / h,
reaches 2e-7 of the derivative at the low-density samples; E_xc 1e-12
relative; Tr(V_xc Q) against the reference's difference quotient of E_xc along
Q, 1e-7 relative.
"""

import numpy as np
import pytest

from conftest import golden_basis, load_golden


@pytest.fixture(scope="module")
def scf_golden():
    return load_golden("water_scf")


@pytest.fixture(scope="module")
def orb(water_golden):
    return golden_basis(water_golden, "orb")


def test_one_electron_matches_reference(scf_golden, orb):
    from oracle import ks

    g = scf_golden
    S, T, V = ks.one_electron(orb, g["coords"], g["charges"])
    assert np.abs(S - g["S"]).max() < 1e-13
    assert np.abs(T - g["T"]).max() < 1e-13
    assert np.abs(V - g["V"]).max() < 1e-12
    assert abs(ks.nuclear_repulsion(g["coords"], g["charges"]) - g["e_nn"]) < 1e-13


def _match(a, b):
    """index of the point of b nearest each point of a"""
    from scipy.spatial import cKDTree

    d, i = cKDTree(b).query(a)
    return d, i


@pytest.mark.parametrize("tag,spec", [("small", (40, 110)), ("default", (75, 302))])
def test_becke_grid_matches_reference(scf_golden, tag, spec):
    from oracle import ks

    g = scf_golden
    pts, w = ks.becke_grid(list(g["symbols"]), g["coords"], spec[0], spec[1])
    ref_p, ref_w = g[f"grid_{tag}_coords"], g[f"grid_{tag}_weights"]
    assert pts.shape == ref_p.shape
    d, i = _match(ref_p, pts)
    assert d.max() < 1e-12
    assert len(np.unique(i)) == len(i)
    assert np.abs(w[i] - ref_w).max() < 1e-13 * np.abs(ref_w).max()


def test_ao_values_and_gradients_match_reference(scf_golden, orb):
    from oracle import ks

    g = scf_golden
    pts = g["grid_small_coords"][g["ao_sample_idx"]]
    val, grad = ks.eval_ao(orb, pts)
    assert np.abs(val - g["ao_sample"]).max() < 1e-14
    assert np.abs(grad - g["dao_sample"]).max() < 1e-12


def test_pbe0_matches_reference_pointwise(scf_golden):
    import torch

    from oracle import ks

    g = scf_golden
    rho = torch.tensor(g["pbe0_rho"], requires_grad=True)
    grad = torch.tensor(g["pbe0_grad"], requires_grad=True)
    eps = ks.pbe0_eps(torch, rho, grad)
    assert np.allclose(eps.detach().numpy(), g["pbe0_eps"], rtol=1e-14, atol=0)
    (rho * eps).sum().backward()
    np.testing.assert_allclose(rho.grad.numpy(), g["pbe0_drho"], rtol=1e-7)
    dg = grad.grad.numpy()
    scale = np.abs(g["pbe0_dgrad"]).max(axis=1, keepdims=True)
    assert np.all(np.abs(dg - g["pbe0_dgrad"]) <= 1e-6 * scale)


def test_exc_and_vxc_match_reference(scf_golden, orb):
    from oracle import ks

    g = scf_golden
    P = 2.0 * g["C"] @ g["C"].T
    e, vxc = ks.exc_and_vxc(orb, g["grid_small_coords"], g["grid_small_weights"], P)
    assert abs(e - g["e_xc"]) < 1e-12 * abs(g["e_xc"])
    for Q, dE in zip(g["dexc_Q"], g["dexc"]):
        assert abs(np.sum(vxc * Q) - dE) < 1e-7 * abs(dE)


def test_scf_converges_to_a_stationary_density(scf_golden, orb, water_golden):
    """The oracle SCF on the water monomer (golden grid): converged, the
    commutator at the solution below d_tol, and E(P*) equal to the sum of the
    reference's own terms at P* (one-electron, DFCoulomb, E_xc, nuclear)."""
    from oracle import df as odf
    from oracle import ks

    g = scf_golden
    aux = golden_basis(water_golden, "aux")
    from conftest import unpack_tril

    I3 = unpack_tril(water_golden["int3c_tril"], orb.nao)
    model = ks.KSEnergy(orb, aux, g["coords"], g["charges"], g["grid_small_coords"],
                        g["grid_small_weights"], I3=I3, vinv=water_golden["vinv"])
    e, P, eps, C, n_iter, conv = ks.scf(model, 5)
    assert conv and n_iter < 40
    # the reference's terms at P*
    e_ref = (np.sum(P * (g["T"] + g["V"])) + g["e_nn"]
             + odf.df_energy(I3, water_golden["vinv"], P[None], 0.25)
             + ks.exc_and_vxc(orb, g["grid_small_coords"], g["grid_small_weights"], P)[0])
    assert abs(e - e_ref) < 1e-10
    _, F = model.energy_fock(P)
    S = g["S"]
    X = ks.canonical_orthonormalizer(S)
    assert np.linalg.norm(X.T @ (F @ P @ S - S @ P @ F) @ X) < 1e-6
    # aufbau: the occupied orbitals lie below the virtual ones (the synthetic
    # even-tempered basis has no tight O 1s exponents, so E is about -60 Ha)
    assert eps[4] < 0.0 < eps[5] or eps[4] < eps[5]


def test_ground_state_configurations():
    """Madelung filling with the s -> d promotions of Cr, Cu and the 4d row."""
    from dftax_b200.guess import ground_state

    assert ground_state(1) == [(1, 0, 1)]
    assert ground_state(8) == [(1, 0, 2), (2, 0, 2), (2, 1, 4)]
    assert dict(((n, l), c) for n, l, c in ground_state(24))[(3, 2)] == 5
    assert dict(((n, l), c) for n, l, c in ground_state(29))[(4, 0)] == 1
    assert (5, 0) not in dict(((n, l), c) for n, l, c in ground_state(46))
    for Z in range(1, 55):
        assert sum(c for _, _, c in ground_state(Z)) == Z


def test_config_occupations_fill_channels_by_energy():
    """A synthetic spherical atom: orbitals of pure l, the lowest s pair and
    the p triplet of oxygen's 1s2 2s2 2p4."""
    import numpy as np

    from dftax_b200.guess import config_occupations

    ao_l = [0, 0, 0, 1, 1, 1]
    S = np.eye(6)
    C = np.eye(6)[:, [0, 3, 4, 5, 1, 2]]   # energy order: s, p, p, p, s, s
    occ = config_occupations(C, S, ao_l, 8)
    assert np.allclose(occ, [2, 4 / 3, 4 / 3, 4 / 3, 2, 0])


def _atom_blocks_loop(b, xyz, tol=1e-10):
    """The per-shell restatement: nearest atom of each shell center, then each
    atom's contiguous run of shells."""
    from dftax_b200.guess import _shells

    cen = np.asarray(b.centers)
    sph = b.cart2sph is not None
    owner, c0, f0 = [], [0], [0]
    for start, l in _shells(b):
        d = np.linalg.norm(xyz - cen[start], axis=1)
        a = int(np.argmin(d))
        assert d[a] <= tol
        owner.append(a)
        c0.append(c0[-1] + (l + 1) * (l + 2) // 2)
        f0.append(f0[-1] + (2 * l + 1 if sph else (l + 1) * (l + 2) // 2))
    out = []
    for a in range(len(xyz)):
        ks = [k for k, o in enumerate(owner) if o == a]
        out.append((slice(c0[ks[0]], c0[ks[-1] + 1]), slice(f0[ks[0]], f0[ks[-1] + 1])))
    return out


@pytest.mark.parametrize("name", ["water3", "alkane2"])
def test_atom_blocks_match_the_per_shell_form(name):
    """The SAD guess's atomic blocks (orbital and auxiliary, spherical and
    cartesian) against the per-shell restatement, and its two errors."""
    from dftax_b200 import systems
    from dftax_b200.guess import atom_blocks

    sym, xyz, orb, aux, _ = systems.workload(name, seed=0)
    for b in (orb, aux, systems.basis_for(sym, xyz, spherical=False)[0]):
        assert atom_blocks(b, xyz) == _atom_blocks_loop(b, np.asarray(xyz))
    with pytest.raises(ValueError, match="on no atom"):
        atom_blocks(orb, np.asarray(xyz) + 0.1)
    with pytest.raises(ValueError, match="no shells"):
        atom_blocks(orb, np.vstack([xyz, [[50.0, 50.0, 50.0]]]))
