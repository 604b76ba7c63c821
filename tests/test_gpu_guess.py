"""The superposition-of-atomic-densities guess (dftax_b200.guess.sad, dftax's
``guess.sad``, dftax/ks/guess.py:115-123, :382-452, :529-546).

* each atomic block holds Z electrons in its own functions (Tr(P_A S_AA) = Z)
  and is symmetric;
* an SCF started from it converges to the energy reached from the core guess
  (1e-8 Ha: the converged state does not depend on the start) in fewer
  iterations, for water clusters (O d shells) and ethane (C f shells), in
  float64 and mixed precision;
* batched solves given the same guess equal the solo solve (1e-10 Ha).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_atomic_blocks_hold_the_atoms_electrons():
    import torch

    from dftax_b200 import df, systems
    from dftax_b200.guess import atom_blocks, sad_density
    from dftax_b200.ks import KS

    sym, xyz, orb, aux, _ = systems.workload("alkane2", seed=0)
    P = sad_density(sym, xyz, orb, aux)
    ks = KS(sym, xyz, orb, coulomb=df(aux), xc="HF")
    S = ks.one_electron()[0].cpu().numpy()
    assert np.abs(P - P.T).max() < 1e-12
    for s, (_, fs) in zip(sym, atom_blocks(orb, xyz)):
        Z = {"H": 1, "C": 6}[s]
        assert abs(np.sum(P[fs, fs] * S[fs, fs]) - Z) < 1e-8
    ks.close()
    torch.cuda.synchronize()


@pytest.mark.parametrize("name,precision", [("water3", "fp64"), ("water5", "mixed"),
                                            ("alkane2", "fp64")])
def test_sad_converges_to_the_core_guess_energy_in_fewer_iterations(name, precision):
    from dftax_b200 import df, systems
    from dftax_b200.grid import becke
    from dftax_b200.ks import KS, scf

    sym, xyz, orb, aux, _ = systems.workload(name, seed=3)
    ks = KS(sym, xyz, orb, coulomb=df(aux, precision=precision), grid=becke(50, 194))
    r0 = scf(ks)
    r1 = scf(ks, guess="sad")
    assert r0.converged and r1.converged
    assert abs(r1.e_tot - r0.e_tot) < 1e-8
    assert r1.n_iter < r0.n_iter, (r1.n_iter, r0.n_iter)
    ks.close()


def test_batch_with_sad_equals_solo():
    from dftax_b200 import df, systems
    from dftax_b200.batch import scf_batch
    from dftax_b200.grid import becke
    from dftax_b200.ks import KS, scf

    g = becke(50, 194)
    mols = [systems.workload(nm, seed=4)[:4] for nm in ("water3", "alkane3", "water2")]
    solo = []
    for sym, xyz, orb, aux in mols:
        ks = KS(sym, xyz, orb, coulomb=df(aux), grid=g, xc_streams=1)   # as the engine runs it
        solo.append(scf(ks, guess="sad").e_tot)
        ks.close()
    res = scf_batch(mols, grid=g, workers=3, guess="sad")
    for r, e in zip(res, solo):
        assert r.status == 0, r.message
        assert abs(r.e_tot - e) < 1e-10
