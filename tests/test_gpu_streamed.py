"""Streamed plans (dfjk_options.streamed = 1, dftax's StreamedDFCoulomb,
dftax/ks/terms.py:716-761): B is not stored; every J/K evaluation rebuilds it
chunk by chunk of bra pairs with the build's own kernels, sums gamma and the
K half transform over the chunks and forms J in a second pass.

Checks: J, K and the DF energy (with its Fock) of a streamed plan equal those
of the materialized plan of the same bases, in float64 and mixed precision,
with several chunks (a small chunk budget), open shell, range-separated
exchange and a Schwarz-screened plan; the streamed plan holds no B; an SCF
solve through ``df(aux, chunk=...)`` converges to the materialized energy;
the entry points that need a resident B refuse a streamed plan.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _plans(name, precision="fp64", seed=0, **kw):
    from dftax_b200 import Plan, systems

    _, xyz, orb, aux, nocc = systems.workload(name, seed=seed)
    full = Plan(orb, aux, precision=precision, **kw).build()
    # a 4 MB row budget splits B into many chunks
    st = Plan(orb, aux, precision=precision, streamed=True, chunk_bytes=4 << 20, **kw).build()
    return full, st, orb, nocc, xyz


@pytest.mark.parametrize("name,precision", [("water3", "fp64"), ("alkane2", "fp64"),
                                            ("water8", "fp64"), ("water3", "mixed")])
def test_streamed_jk_equals_materialized(name, precision):
    from dftax_b200 import systems

    full, st, orb, nocc, _ = _plans(name, precision)
    assert st.info()["b_bytes"] == 0 and full.info()["b_bytes"] > 0
    C = systems.random_occupied(orb.nao, nocc, seed=2)
    J0, K0 = (x.cpu().numpy() for x in full.jk(C))
    J1, K1 = (x.cpu().numpy() for x in st.jk(C))
    assert _rel(J1, J0) < 1e-12
    # a mixed materialized plan runs K on int8 digits (5e-9 relative here); the
    # streamed one runs it in float64
    assert _rel(K1, K0) < (1e-12 if precision == "fp64" else 3e-8)


@pytest.mark.parametrize("nspin", [1, 2])
def test_streamed_energy_and_fock(nspin):
    from dftax_b200 import systems

    full, st, orb, nocc, _ = _plans("water3")
    C = systems.random_occupied(orb.nao, nocc, seed=5)
    P = 2 * C @ C.T if nspin == 1 else np.stack([C @ C.T, C[:, :-1] @ C[:, :-1].T])
    e0, F0 = full.energy(P, 0.25)
    e1, F1 = st.energy(P, 0.25)
    assert abs(e1 - e0) < 1e-12 * abs(e0)
    assert _rel(F1.cpu().numpy(), F0.cpu().numpy()) < 1e-12


def test_streamed_screened_and_range_separated():
    from dftax_b200 import systems

    full, st, orb, nocc, _ = _plans("water3", screen=1e-10, omega=0.3)
    C = systems.random_occupied(orb.nao, nocc, seed=6)
    P = 2 * C @ C.T
    e0, F0 = full.energy(P, 0.2, hf_coeff_lr=0.5)
    e1, F1 = st.energy(P, 0.2, hf_coeff_lr=0.5)
    assert abs(e1 - e0) < 1e-12 * abs(e0)
    assert _rel(F1.cpu().numpy(), F0.cpu().numpy()) < 1e-12


def test_streamed_scf_through_df_chunk():
    from dftax_b200 import df, systems
    from dftax_b200.grid import becke
    from dftax_b200.ks import KS, scf

    sym, xyz, orb, aux, _ = systems.workload("water2", seed=1)
    g = becke(50, 194)
    r0 = scf(KS(sym, xyz, orb, coulomb=df(aux), grid=g))
    ks = KS(sym, xyz, orb, coulomb=df(aux, chunk=512), grid=g)
    assert ks.plan.streamed
    r1 = scf(ks)
    assert r1.converged and abs(r1.e_tot - r0.e_tot) < 1e-9


def test_streamed_plan_refuses_resident_b_entry_points():
    import ctypes

    import torch

    from dftax_b200 import _lib, systems

    _, st, orb, nocc, xyz = _plans("water")
    C = systems.random_occupied(orb.nao, nocc, seed=1)
    with pytest.raises(_lib.DfjkError) as e:
        st.energy_grad(2 * C @ C.T, 0.25, xyz)
    assert e.value.status == _lib.DFJK_ERR_UNSUPPORTED
    Cd = torch.as_tensor(C, device=st.dev)
    J = torch.empty((orb.nao, orb.nao), dtype=torch.float64, device=st.dev)
    s = st.lib.dfjk_j_noalloc(st.h, Cd.data_ptr(), None, C.shape[1], J.data_ptr(),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert s == _lib.DFJK_ERR_UNSUPPORTED
