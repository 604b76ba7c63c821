"""Plans built together (dfjk_build_batch, Plan.build_many): the 3-center
integrals of every plan whose rows fit in one staging chunk are computed in
shared launches, one per integral class, over a work queue of (plan, run of
shell pairs) segments. Each queue entry runs the plain launch's block, so
every plan must end exactly as its own dfjk_build leaves it: J and K from
the two builds are compared bit for bit, for molecules of different sizes and
compositions (d and f shells), both precisions, with a plan whose rows span
several chunks and a streamed plan in the same batch (both built alone).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["water", "water3", "alkane2", "water5", "alkane3", "water2"]


def _plans(precision, **kw):
    from dftax_b200 import Plan, systems

    out = []
    for i, nm in enumerate(NAMES):
        _, _, orb, aux, nocc = systems.workload(nm, seed=i)
        out.append((Plan(orb, aux, precision=precision, **kw), orb.nao, nocc))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_build_equals_single_builds(precision):
    import torch

    from dftax_b200 import Plan, systems

    solo = _plans(precision)
    for p, _, _ in solo:
        p.build()
    together = _plans(precision)
    # one plan staged in several chunks and one streamed plan ride along
    _, _, orb, aux, nocc = systems.workload("water3", seed=9)
    chunked = Plan(orb, aux, precision=precision, chunk_bytes=2 << 20)
    streamed = Plan(orb, aux, precision=precision, streamed=True)
    Plan.build_many([p for p, _, _ in together] + [chunked, streamed])
    ref = Plan(orb, aux, precision=precision).build()
    for (a, nao, nocc_i), (b, _, _) in zip(solo, together):
        C = systems.random_occupied(nao, nocc_i, seed=3)
        Ja, Ka = a.jk(C)
        Jb, Kb = b.jk(C)
        torch.cuda.synchronize()
        assert torch.equal(Ja, Jb) and torch.equal(Ka, Kb)
        assert b.info()["built"] == 1
    C = systems.random_occupied(orb.nao, nocc, seed=4)
    J0, K0 = (x.cpu().numpy() for x in ref.jk(C))
    for p in (chunked, streamed):
        J1, K1 = (x.cpu().numpy() for x in p.jk(C))
        assert np.abs(J1 - J0).max() <= 1e-12 * np.abs(J0).max()
        tol = 1e-12 if precision == "fp64" else 3e-8   # streamed K runs in float64
        assert np.abs(K1 - K0).max() <= tol * np.abs(K0).max()


def test_batched_build_rejects_a_repeated_plan():
    from dftax_b200 import _lib

    (p, _, _), = _plans("fp64")[:1]
    with pytest.raises(_lib.DfjkError) as e:
        from dftax_b200 import Plan

        Plan.build_many([p, p])
    assert e.value.status == _lib.DFJK_ERR_INVALID
