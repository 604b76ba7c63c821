"""Float64 parity on the benchmark workloads, not only on the small fixtures.

  * (H2O)_8 (240 AOs, 1128 auxiliary functions) in full: every (ij|P) against
    the oracle (1e-13 absolute), (P|Q) (1e-12), the kept metric directions,
    and J, K, E, dE/dP of P = 2 C C^T with a_x = 0.25 against the oracle's
    formula (NOISE_REL, the float64 floor of the reference's own formula);
  * (H2O)_16, (H2O)_32, C10H22, C20H42: whole blocks of a seeded sample of
    shell pairs (every auxiliary shell) against the oracle at 1e-13, and a
    sample of the metric's auxiliary shells at 1e-12;
  * (H2O)_16: J and K of the built plan against a float64 torch contraction
    of the device's own dense integrals and a pseudo-inverse of its own
    metric (the contraction path at a size the oracle cannot finish quickly).

The workloads and seeds are those of bench.py (geometry seed 0).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOISE_REL = 5e-10
INT_ABS = 1e-13
METRIC_ABS = 1e-12


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def water8():
    from dftax_b200 import Plan, systems
    from oracle import md as omd

    sym, xyz, orb, aux, nocc = systems.workload("water8", seed=0)
    plan = Plan(orb, aux).build()
    return {"orb": orb, "aux": aux, "nocc": nocc, "plan": plan,
            "I3": omd.eri3c(orb, aux), "V": omd.eri2c(aux)}


def test_water8_eri3c_full_vs_oracle(water8):
    I3 = water8["plan"].eri3c_dense().cpu().numpy()
    assert I3.shape == water8["I3"].shape
    assert np.abs(I3 - water8["I3"]).max() < INT_ABS


def test_water8_metric_vs_oracle(water8):
    from oracle import df as odf

    plan = water8["plan"]
    V = plan.eri2c_dense().cpu().numpy()
    assert np.abs(V - water8["V"]).max() < METRIC_ABS
    w = np.linalg.eigvalsh(water8["V"])
    kept = int(np.sum(w > 1e-7 * w.max()))
    assert plan.info()["nfit"] == kept
    vinv = plan.metric_pinv().cpu().numpy()
    assert rel(vinv, odf.metric_pinv(water8["V"])) < 2e-8


def test_water8_jk_energy_vs_oracle(water8):
    from dftax_b200 import systems
    from oracle import df as odf

    plan = water8["plan"]
    vinv = odf.metric_pinv(water8["V"])
    C = systems.random_occupied(plan.nao, water8["nocc"], seed=100)
    D = C @ C.T
    Jr, Kr = odf.df_jk(water8["I3"], vinv, D)
    J, K = (x.cpu().numpy() for x in plan.jk(C))
    assert rel(J, Jr) < NOISE_REL
    assert rel(K, Kr) < NOISE_REL
    P = 2.0 * D
    e, F = plan.energy(P, 0.25)
    er = odf.df_energy(water8["I3"], vinv, P[None], 0.25)
    assert abs(e - er) < NOISE_REL * abs(er)
    assert rel(F[0].cpu().numpy(), 2.0 * Jr - 0.25 * Kr) < NOISE_REL


def _sample_pairs(orb, n, seed):
    from oracle import md as omd

    ns = len(omd.shells(orb))
    ia, ib = np.triu_indices(ns)
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(ia), size=min(n, len(ia)), replace=False)
    return {(int(ia[i]), int(ib[i])) for i in pick}


def _sub_aux(aux, shells_picked):
    """The auxiliary basis restricted to whole shells, with its cart2sph block
    columns; returns the sub-basis and the spherical columns it covers."""
    from dftax_b200.basis import BasisData
    from oracle import md as omd

    sa = omd.shells(aux)
    sas, _ = omd.sph_starts(sa, aux.cart2sph)
    rows = np.concatenate([np.arange(sa[s][1], sa[s][1] + sa[s][2]) for s in shells_picked])
    cols = np.concatenate([np.arange(sas[s], sas[s] + 2 * sa[s][0] + 1) for s in shells_picked])
    sub = BasisData(aux.centers[rows], aux.exponents[rows], aux.coefficients[rows],
                    aux.angular[rows], aux.cart2sph[np.ix_(rows, cols)], aux.max_l)
    return sub, cols


@pytest.mark.parametrize("name", ["water16", "water32", "alkane10", "alkane20"])
def test_sampled_blocks_vs_oracle(name):
    """Seeded sample of whole shell-pair blocks (all auxiliary shells) and of
    the metric, compared on the device-resident dense tensor."""
    import torch

    from dftax_b200 import Plan, systems
    from oracle import md as omd

    sym, xyz, orb, aux, nocc = systems.workload(name, seed=0)
    plan = Plan(orb, aux)
    I3 = plan.eri3c_dense()
    keep = _sample_pairs(orb, 200, seed=17)
    worst = 0.0
    nblk = 0
    for ra, rb, rc, v in omd.eri3c_blocks(orb, aux, keep):
        ia = torch.as_tensor(ra, device=I3.device)[:, :, None, None]
        ib = torch.as_tensor(rb, device=I3.device)[:, None, :, None]
        ic = torch.as_tensor(rc, device=I3.device)[:, None, None, :]
        d = I3[ia, ib, ic].cpu().numpy()
        worst = max(worst, float(np.abs(d - v).max()))
        # the mirrored block (ba|P) of the dense output
        dm = I3[ib.transpose(1, 2), ia.transpose(1, 2), ic].cpu().numpy()
        worst = max(worst, float(np.abs(dm - v.transpose(0, 2, 1, 3)).max()))
        nblk += v.shape[0]
    assert nblk > 0
    assert worst < INT_ABS, worst
    del I3
    torch.cuda.empty_cache()
    # metric: a seeded sample of 120 auxiliary shells
    nsa = len(omd.shells(aux))
    pick = sorted(np.random.default_rng(23).choice(nsa, size=min(120, nsa), replace=False).tolist())
    sub, cols = _sub_aux(aux, pick)
    Vr = omd.eri2c(sub)
    V = plan.eri2c_dense()
    ci = torch.as_tensor(cols, device=V.device)
    Vd = V[ci[:, None], ci[None, :]].cpu().numpy()
    assert np.abs(Vd - Vr).max() < METRIC_ABS
    plan.close()


def test_water16_jk_vs_torch_contraction():
    """J and K through B = (ij|P) L (DMMA half transform, split-k X X^T) against
    J = I3 . V+ (I3 . D) and K_mn = sum_PQ (ml|P) V+_PQ (ns|Q) D_ls evaluated
    in float64 with torch from the plan's own dense integrals and metric."""
    import torch

    from dftax_b200 import Plan, systems

    sym, xyz, orb, aux, nocc = systems.workload("water16", seed=0)
    plan = Plan(orb, aux).build()
    C = systems.random_occupied(plan.nao, nocc, seed=100)
    J, K = (x.cpu().numpy() for x in plan.jk(C))
    I3 = plan.eri3c_dense()
    V = plan.eri2c_dense()
    w, U = torch.linalg.eigh(V)
    keepw = w > 1e-7 * w.max()
    assert int(keepw.sum()) == plan.info()["nfit"]
    Uk = U[:, keepw] / torch.sqrt(w[keepw])[None, :]
    nao, naux = I3.shape[0], I3.shape[2]
    Cd = torch.as_tensor(C, device=I3.device)
    D = Cd @ Cd.T
    Bt = (I3.reshape(nao * nao, naux) @ Uk)           # (mn, x)
    del I3
    gamma = Bt.T @ D.reshape(-1)
    Jr = (Bt @ gamma).reshape(nao, nao)
    X = Bt.reshape(nao, nao, -1).permute(2, 0, 1) @ Cd     # (x, m, i)
    Kr = torch.einsum("xmi,xni->mn", X, X)
    assert rel(J, Jr.cpu().numpy()) < NOISE_REL
    assert rel(K, Kr.cpu().numpy()) < NOISE_REL
    plan.close()
