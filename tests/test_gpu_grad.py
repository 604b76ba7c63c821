"""Nuclear gradient of the DF energy at a fixed density (dfjk_energy_grad).

dftax's forces() differentiate the DF energy through its integral build
(dftax/ks/forces.py:245-270) with d(V+) = -V+ dV V+ for the metric
pseudo-inverse (dftax/ks/terms.py:196-204). The oracle restates that
derivative: the weights G and W of the energy (numpy, float64) contracted with
the integral derivatives, taken by central differences of the compiled CPU
integrals with one Richardson step (oracle/cpu.py ``df_energy_grad``; it
agrees with finite differences of the whole oracle energy to 1e-8 where the
metric drops no direction, tests/test_oracle_cpu.py). The device gradient
is checked against it per atom, for closed and open shells, pure Coulomb and
hybrid exchange, on the even-tempered water (d shells, aux up to f) and on
ethane (carbon f shells, aux up to g), and for translational invariance on
(H2O)_8.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _density(nao, nocc, seed, nspin=1):
    from dftax_b200 import systems

    if nspin == 1:
        C = systems.random_occupied(nao, nocc, seed=seed)
        return 2.0 * C @ C.T
    Ca = systems.random_occupied(nao, nocc, seed=seed)
    Cb = systems.random_occupied(nao, nocc - 1, seed=seed + 1)
    return np.stack([Ca @ Ca.T, Cb @ Cb.T])


@pytest.mark.parametrize("name,nspin,hf", [("water", 1, 0.25), ("water", 1, 0.0),
                                           ("water", 2, 0.25), ("alkane2", 1, 0.0),
                                           ("alkane2", 1, 0.25)])
def test_gradient_matches_oracle(name, nspin, hf):
    """Two comparisons. With the oracle given the device's metric
    pseudo-inverse, the contractions agree to 1e-9 of the largest component
    for pure Coulomb; with exchange the metric term W = V+ M V+ carries V+
    twice (condition number 1.5e8), and two algebraically equal forms of V+
    (U diag(1/w) U^T and L L^T) already move the oracle's own gradient by
    6e-9 of its largest component, so 5e-8 is allowed. With the oracle's own
    (LAPACK) pseudo-inverse the two V+ differ at the metric's conditioning and
    so do the gradients (2e-7 allowed), while the energies agree to 1e-10."""
    from dftax_b200 import Plan, systems
    from oracle import cpu

    _, xyz, orb, aux, nocc = systems.workload(name, seed=0)
    P = _density(orb.nao, nocc, seed=4, nspin=nspin)
    plan = Plan(orb, aux).build()
    E, g = plan.energy_grad(P, hf, xyz)
    scale = max(np.abs(g).max(), 1.0)
    _, gv = cpu.df_energy_grad(orb, aux, P, hf, xyz, vinv=plan.metric_pinv().cpu().numpy())
    # ethane's fit drops 36 of 456 directions (condition 8e6 over the kept
    # ones): there the two forms of V+ already move the oracle by 4e-8
    tol = 1e-9 if hf == 0.0 else (5e-8 if name == "water" else 4e-7)
    assert np.abs(g - gv).max() <= tol * scale, (np.abs(g - gv).max(), scale)
    E0, g0 = cpu.df_energy_grad(orb, aux, P, hf, xyz)
    assert abs(E - E0) <= 1e-10 * abs(E0)
    assert np.abs(g - g0).max() <= 2e-7 * scale, (np.abs(g - g0).max(), scale)
    assert np.abs(g.sum(axis=0)).max() <= 1e-9 * scale
    plan.close()


@pytest.mark.parametrize("name,nspin", [("water", 1), ("water", 2), ("alkane2", 1)])
def test_exchange_gradient_with_well_conditioned_fit(name, nspin):
    """With the orbital basis itself as the fitting basis (d and f shells on
    both sides, metric condition ~1e4, no direction dropped) the exchange
    part has no conditioning floor: the device gradient equals the oracle's
    to 1e-9 of the largest component."""
    from dftax_b200 import Plan, systems
    from oracle import cpu

    _, xyz, orb, _, nocc = systems.workload(name, seed=0)
    P = _density(orb.nao, nocc, seed=7, nspin=nspin)
    plan = Plan(orb, orb).build()
    E, g = plan.energy_grad(P, 0.25, xyz)
    E0, g0 = cpu.df_energy_grad(orb, orb, P, 0.25, xyz)
    scale = max(np.abs(g0).max(), 1.0)
    assert abs(E - E0) <= 1e-11 * abs(E0)
    assert np.abs(g - g0).max() <= 1e-9 * scale, (np.abs(g - g0).max(), scale)
    plan.close()


def test_gradient_energy_equals_dfjk_energy_and_is_translation_free():
    from dftax_b200 import Plan, systems

    _, xyz, orb, aux, nocc = systems.workload("water8", seed=2)
    P = _density(orb.nao, nocc, seed=9)
    plan = Plan(orb, aux).build()
    E, g = plan.energy_grad(P, 0.25, xyz)
    E1, _ = plan.energy(P, 0.25, want_grad=False)
    assert abs(E - E1) <= 1e-11 * abs(E1)
    assert np.abs(g.sum(axis=0)).max() <= 1e-9 * np.abs(g).max()
    # the shell-resolved form sums to the same atom gradient
    _, go, ga = plan.energy_grad(P, 0.25)
    from dftax_b200.coulomb import shells_to_atoms

    g2 = shells_to_atoms(go, plan.orb_centers, xyz) + shells_to_atoms(ga, plan.aux_centers, xyz)
    assert np.abs(g2 - g).max() <= 1e-12 * np.abs(g).max()
    plan.close()


def test_mixed_plan_gradient_close_to_fp64():
    """A mixed-precision plan's B carries 5 int8 digits per value; its
    gradient stays within 1e-7 of the float64 plan's."""
    from dftax_b200 import Plan, systems

    _, xyz, orb, aux, nocc = systems.workload("water3", seed=1)
    P = _density(orb.nao, nocc, seed=3)
    g64 = Plan(orb, aux).build().energy_grad(P, 0.25, xyz)[1]
    gmx = Plan(orb, aux, precision="mixed").build().energy_grad(P, 0.25, xyz)[1]
    assert np.abs(gmx - g64).max() <= 1e-7 * max(np.abs(g64).max(), 1.0)


def test_gradient_requires_a_build():
    from dftax_b200 import Plan, _lib, systems

    _, xyz, orb, aux, nocc = systems.workload("water", seed=0)
    plan = Plan(orb, aux)
    with pytest.raises(_lib.DfjkError) as e:
        plan.energy_grad(_density(orb.nao, nocc, 1), 0.25, xyz)
    assert e.value.status == _lib.DFJK_ERR_STATE
