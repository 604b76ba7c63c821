"""Batched and served SCF solves (include/dfbatch.h, dftax_b200/batch.py).

  * every result of a batch of molecules of uneven size (monomer to (H2O)_5,
    ethane) equals the same molecule solved alone: |dE| <= 1e-10 Ha and the
    density to 1e-8 (the same kernels with fixed-order reductions run either
    way; the engine runs each solve's XC on one stream, so the solo solves
    here do too);
  * with room for several, solves overlap in time, and the estimated bytes of
    the solves running at once never exceed the budget;
  * with room for one, they run one after another;
  * a request the library refuses (an orbital g shell) fails alone;
  * a seeded Poisson stream of requests, each submitted while others run,
    gives the results of solo solves, with latencies reported.
The grid is Becke 50 x 194 (NWChem pruning) to keep the solves short.
"""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_TOL = 1e-10


def molecules():
    from dftax_b200 import systems

    out = []
    for name, seed in (("water3", 1), ("alkane2", 0), ("water", 0), ("water5", 2), ("water2", 3)):
        sym, xyz, orb, aux, _ = systems.workload(name, seed=seed)
        out.append((sym, xyz, orb, aux))
    return out


@pytest.fixture(scope="module")
def grid():
    from dftax_b200.grid import becke

    return becke(50, 194)


@pytest.fixture(scope="module")
def solo(grid):
    from dftax_b200 import df
    from dftax_b200.ks import KS, scf

    res = []
    for sym, xyz, orb, aux in molecules():
        ks = KS(sym, xyz, orb, coulomb=df(aux), grid=grid, xc_streams=1)
        r = scf(ks)
        res.append((r.e_tot, r.P[0]))
        ks.close()
        ks.plan.close()
    return res


def _overlaps(results):
    iv = sorted((r.t_start, r.t_end) for r in results)
    return any(iv[i + 1][0] < iv[i][1] for i in range(len(iv) - 1))


def _max_concurrent_bytes(results):
    worst = 0
    for r in results:
        t = r.t_start
        worst = max(worst, sum(q.bytes for q in results if q.t_start <= t < q.t_end))
    return worst


def test_batch_equals_solo_runs(solo, grid):
    from dftax_b200.batch import scf_batch

    res = scf_batch(molecules(), workers=3, grid=grid, want_density=True)
    for r, (e, P) in zip(res, solo):
        assert r.status == 0, r.message
        assert r.converged
        assert abs(r.e_tot - e) < E_TOL
        assert np.abs(r.P - P).max() < 1e-8
    assert _overlaps(res)


def test_budget_bounds_the_running_solves(grid):
    from dftax_b200.batch import BatchEngine

    mols = molecules()
    with BatchEngine(workers=4) as probe:
        est = sorted(probe.estimate(*m, grid=grid) for m in mols)
    budget = est[-1] + est[-2]           # room for the two largest at once
    with BatchEngine(workers=4, hbm_budget=budget) as eng:
        ids = [eng.submit(*m, grid=grid) for m in mols]
        res = [eng.wait(i) for i in ids]
    assert all(r.status == 0 for r in res)
    assert _max_concurrent_bytes(res) <= budget
    assert _overlaps(res)


def test_budget_for_one_serializes(grid):
    from dftax_b200.batch import BatchEngine

    mols = molecules()[3:]               # (H2O)_5 and (H2O)_2
    with BatchEngine(workers=4) as probe:
        est = [probe.estimate(*m, grid=grid) for m in mols]
    with BatchEngine(workers=4, hbm_budget=max(est) + min(est) - 1) as eng:
        ids = [eng.submit(*m, grid=grid) for m in mols]
        res = [eng.wait(i) for i in ids]
    assert all(r.status == 0 for r in res)
    assert not _overlaps(res)


def test_refused_request_fails_alone(grid):
    from dftax_b200.basis import build_basis_data
    from dftax_b200.batch import BatchEngine

    mols = molecules()[:2]
    sym, xyz, orb, aux = mols[0]
    bad = build_basis_data(["O"], np.zeros((1, 3)), {"O": [(4, [1.0], [1.0])]})
    with BatchEngine(workers=2) as eng:
        ids = [eng.submit(*mols[0], grid=grid),
               eng.submit(["O"], np.zeros((1, 3)), bad, mols[0][3], xc="HF"),
               eng.submit(*mols[1], grid=grid)]
        res = [eng.wait(i) for i in ids]
    assert res[0].status == 0 and res[2].status == 0
    assert res[1].status == 2 and "angular momentum" in res[1].message   # UNSUPPORTED


def test_poisson_stream_matches_solo(solo, grid):
    """Requests arrive with seeded exponential gaps (mean 0.15 s) while
    earlier ones are on the GPU; each is admitted as memory frees up."""
    from dftax_b200.batch import BatchEngine

    rng = np.random.default_rng(8)
    mols = molecules()
    order = [0, 3, 1, 4, 2, 3, 0]
    with BatchEngine(workers=3) as eng:
        ids = []
        for k in order:
            ids.append((k, eng.submit(*mols[k], grid=grid)))
            time.sleep(float(rng.exponential(0.15)))
        res = [(k, eng.wait(i)) for k, i in ids]
    lat = []
    for k, r in res:
        assert r.status == 0, r.message
        assert abs(r.e_tot - solo[k][0]) < E_TOL
        lat.append(r.latency)
    assert np.percentile(lat, 50) <= np.percentile(lat, 99)
    assert _overlaps([r for _, r in res])


def test_stream_with_buffer_reuse_across_workers(grid):
    """Alkanes (carbon f shells) and water clusters, each twice, four workers:
    the device buffers of finished solves are reused by solves on other
    streams while work is still queued. Every result is the solo result."""
    from dftax_b200 import df, systems
    from dftax_b200.batch import BatchEngine
    from dftax_b200.ks import KS, scf

    names = ["alkane4", "water5", "alkane6", "water3", "alkane5", "water4"]
    mols = [systems.workload(nm, seed=7)[:4] for nm in names]
    solo = []
    for sym, xyz, orb, aux in mols:
        ks = KS(sym, xyz, orb, coulomb=df(aux, precision="mixed"), grid=grid, xc_streams=1)
        solo.append(scf(ks).e_tot)
        ks.close()
        ks.plan.close()
    order = [0, 1, 2, 3, 4, 5, 2, 0, 5, 1, 4, 3]
    with BatchEngine(workers=4) as eng:
        ids = [(k, eng.submit(*mols[k], grid=grid, precision="mixed")) for k in order]
        res = [(k, eng.wait(i)) for k, i in ids]
    for k, r in res:
        assert r.status == 0, (names[k], r.message)
        assert abs(r.e_tot - solo[k]) < E_TOL, names[k]
