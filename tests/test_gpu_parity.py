"""Parity of the CUDA library (through the C ABI) with the reference's golden
fixtures and with the oracle.

Tolerances:
  * integrals (P|Q), (ij|P): 1e-13 absolute (float64, different operation order);
  * Boys: 5e-14 relative (table + Taylor in a different operation order);
  * J, K, energy with the metric recomputed on the device: NOISE_REL = 5e-10
    relative — the float64 floor of the reference's own formula (a 3e-16
    relative change of (P|Q) moves J by ~1.2e-10 through the condition-1.9e8
    metric, measured oracle-vs-reference in test_oracle_golden.py);
  * J, K against the oracle fed the device's own integrals and V+: NOISE_REL too.
"""

import numpy as np
import pytest

from conftest import golden_basis, load_golden, unpack_tril

pytestmark = pytest.mark.gpu

NOISE_REL = 5e-10


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def water_plan(water_golden):
    from dftax_b200 import Plan

    g = water_golden
    return Plan(golden_basis(g, "orb"), golden_basis(g, "aux")).build()


@pytest.fixture(scope="module")
def ch2_plan(ch2_golden):
    from dftax_b200 import Plan

    g = ch2_golden
    return Plan(golden_basis(g, "orb"), golden_basis(g, "aux")).build()


def test_boys_device_vs_reference():
    from dftax_b200 import Context

    g = load_golden("boys")
    out = Context.get(0).boys(g["t"], 18)
    np.testing.assert_allclose(out.T, g["boys"], rtol=5e-14, atol=1e-300)


def test_water_eri3c_vs_reference(water_plan, water_golden):
    g = water_golden
    I3 = water_plan.eri3c_dense().cpu().numpy()
    ref = unpack_tril(g["int3c_tril"], I3.shape[0])
    assert np.abs(I3 - ref).max() < 1e-13


def test_ch2_eri3c_high_l_vs_reference(ch2_plan, ch2_golden):
    g = ch2_golden
    I3 = ch2_plan.eri3c_dense().cpu().numpy()
    v = I3[g["sample_m"], g["sample_n"], g["sample_P"]]
    assert np.abs(v - g["sample_val"]).max() < 1e-13
    assert np.abs(I3 - I3.transpose(1, 0, 2)).max() < 1e-14


@pytest.mark.parametrize("name", ["water", "ch2"])
def test_eri2c_vs_reference(name, request):
    plan = request.getfixturevalue(f"{name}_plan")
    g = load_golden(name)
    V = plan.eri2c_dense().cpu().numpy()
    assert np.abs(V - g["int2c"]).max() < 1e-12


@pytest.mark.parametrize("name", ["water", "ch2"])
def test_metric_pinv_vs_reference(name, request):
    plan = request.getfixturevalue(f"{name}_plan")
    g = load_golden(name)
    vinv = plan.metric_pinv().cpu().numpy()
    assert plan.info()["nfit"] == int(g["n_kept"])
    assert rel(vinv, g["vinv"]) < 2e-8   # condition ~1e8 times float64 rounding


@pytest.mark.parametrize("name", ["water", "ch2"])
def test_jk_vs_reference(name, request):
    plan = request.getfixturevalue(f"{name}_plan")
    g = load_golden(name)
    J, K = plan.jk(g["C"])
    J, K = J.cpu().numpy(), K.cpu().numpy()
    assert rel(J, g["J"]) < NOISE_REL
    assert rel(K, g["K"]) < NOISE_REL
    assert np.abs(J - J.T).max() < 1e-13 and np.abs(K - K.T).max() < 1e-13


@pytest.mark.parametrize("name", ["water", "ch2"])
def test_jk_vs_oracle_with_device_metric(name, request):
    """The device's own integrals and V+ = L L^T fed to the oracle's formula.

    Contracting through B = (ij|P) L instead of through V+ reorders a product
    with the same ill-conditioned factor, so the two agree only to the float64
    floor (3.4e-10 measured on CH2), not to machine precision."""
    from oracle import df as odf

    plan = request.getfixturevalue(f"{name}_plan")
    g = load_golden(name)
    I3 = plan.eri3c_dense().cpu().numpy()
    vinv = plan.metric_pinv().cpu().numpy()
    Jr, Kr = odf.df_jk(I3, vinv, g["C"] @ g["C"].T)
    J, K = plan.jk(g["C"])
    assert rel(J.cpu().numpy(), Jr) < NOISE_REL
    assert rel(K.cpu().numpy(), Kr) < NOISE_REL


@pytest.mark.parametrize("name", ["water", "ch2"])
def test_energy_and_fock_vs_reference(name, request):
    plan = request.getfixturevalue(f"{name}_plan")
    g = load_golden(name)
    C = g["C"]
    P = 2.0 * C @ C.T
    e, F = plan.energy(P, 0.25)
    assert abs(e - g["e_total"]) < NOISE_REL * abs(g["e_total"])
    e0, _ = plan.energy(P, 0.0, want_grad=False)
    assert abs(e0 - g["e_j"]) < NOISE_REL * abs(g["e_j"])
    # dE/dP = J(P) - a_x/2 K(P) = 2 J(D) - 0.25 K(D) for P = 2D, a_x = 0.25
    assert rel(F[0].cpu().numpy(), 2.0 * g["J"] - 0.25 * g["K"]) < NOISE_REL


def test_open_shell_energy_vs_oracle(water_plan, water_golden):
    from oracle import df as odf

    g = water_golden
    rng = np.random.default_rng(5)
    n = g["C"].shape[0]
    Ca = np.linalg.qr(rng.standard_normal((n, 5)))[0]
    Cb = np.linalg.qr(rng.standard_normal((n, 4)))[0]
    P = np.stack([Ca @ Ca.T, Cb @ Cb.T])
    e, F = water_plan.energy(P, 0.25)
    I3 = unpack_tril(g["int3c_tril"], n)
    er = odf.df_energy(I3, g["vinv"], P, 0.25)
    assert abs(e - er) < NOISE_REL * abs(er)
    Jt, _ = odf.df_jk(I3, g["vinv"], P.sum(0))
    for s in range(2):
        Fr = Jt - 0.25 * odf.df_k(I3, g["vinv"], P[s])
        assert rel(F[s].cpu().numpy(), Fr) < NOISE_REL


def test_nonidempotent_density_exact(water_plan, water_golden):
    """Any symmetric P (e.g. a DIIS extrapolation) is handled exactly."""
    from oracle import df as odf

    g = water_golden
    n = g["C"].shape[0]
    rng = np.random.default_rng(9)
    A = rng.standard_normal((n, n)) * 0.1
    P = A + A.T
    e, F = water_plan.energy(P, 0.25)
    I3 = unpack_tril(g["int3c_tril"], n)
    er = odf.df_energy(I3, g["vinv"], P[None], 0.25)
    assert abs(e - er) < NOISE_REL * abs(er)


def test_signed_weights_linearity(water_plan, water_golden):
    g = water_golden
    C = g["C"]
    w = np.array([1.0, -0.5, 2.0, 0.0, -1.5])
    J, K = water_plan.jk(C, w)
    Js, Ks = 0.0, 0.0
    for i in range(5):
        Ji, Ki = water_plan.jk(C[:, i:i + 1])
        Js = Js + w[i] * Ji.cpu().numpy()
        Ks = Ks + w[i] * Ki.cpu().numpy()
    assert rel(J.cpu().numpy(), Js) < 1e-12
    assert rel(K.cpu().numpy(), Ks) < 1e-12


def test_host_entry_matches_device(water_plan, water_golden):
    C = water_golden["C"]
    Jh, Kh = water_plan.jk_host(C)
    Jd, Kd = water_plan.jk(C)
    assert np.array_equal(Jh, Jd.cpu().numpy()) and np.array_equal(Kh, Kd.cpu().numpy())


def test_screening_kept_pairs_vs_reference(water_golden):
    from dftax_b200 import Plan

    g = water_golden
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    plan = Plan(orb, aux, screen=float(g["screen_thresh"]))
    ref = {(int(a), int(b)) for a, b in g["screen_keep"]}
    assert plan.kept_pairs() == ref
    # kept blocks equal the dense build, dropped blocks exactly zero (test_screening.py:67-88)
    I3s = plan.eri3c_dense().cpu().numpy()
    I3 = unpack_tril(g["int3c_tril"], I3s.shape[0])
    nz = np.abs(I3s).max(axis=2) > 0
    assert np.abs(I3s[nz] - I3[nz]).max() < 1e-13
    assert np.all(I3s[~nz] == 0.0)


def test_chunked_build_matches(water_golden):
    from dftax_b200 import Plan

    g = water_golden
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    a = Plan(orb, aux).build()
    b = Plan(orb, aux, chunk_bytes=40_000).build()
    Ja, Ka = a.jk(g["C"])
    Jb, Kb = b.jk(g["C"])
    assert rel(Jb.cpu().numpy(), Ja.cpu().numpy()) < 1e-14
    assert rel(Kb.cpu().numpy(), Ka.cpu().numpy()) < 1e-14


@pytest.mark.parametrize("name", ["water3", "alkane2"])
def test_small_systems_vs_oracle(name):
    """Multi-molecule inputs: device integrals vs the oracle, J/K at the noise floor."""
    from dftax_b200 import Plan, systems
    from oracle import df as odf
    from oracle import md as omd

    sym, xyz, orb, aux, nocc = systems.workload(name, seed=2)
    plan = Plan(orb, aux).build()
    I3 = plan.eri3c_dense().cpu().numpy()
    I3r = omd.eri3c(orb, aux)
    assert np.abs(I3 - I3r).max() < 1e-13
    V = plan.eri2c_dense().cpu().numpy()
    Vr = omd.eri2c(aux)
    assert np.abs(V - Vr).max() < 1e-12
    C = systems.random_occupied(orb.nao, nocc, seed=4)
    J, K = plan.jk(C)
    Jr, Kr = odf.df_jk(I3r, odf.metric_pinv(Vr), C @ C.T)
    assert rel(J.cpu().numpy(), Jr) < NOISE_REL
    assert rel(K.cpu().numpy(), Kr) < NOISE_REL


def test_errors_are_reported_not_trapped(water_golden):
    from dftax_b200 import Plan
    from dftax_b200._lib import DfjkError
    from dftax_b200.basis import build_basis_data

    g = water_golden
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    # unsupported angular momentum: an orbital g shell
    sym = ["O"]
    gsets = {"O": [(4, [1.0], [1.0])]}
    gorb = build_basis_data(sym, np.zeros((1, 3)), gsets)
    with pytest.raises(DfjkError) as ei:
        Plan(gorb, aux)
    assert ei.value.status_name == "UNSUPPORTED"
    # non-finite coordinate
    bad = golden_basis(g, "orb")
    bad.centers = bad.centers.copy()
    bad.centers[0, 0] = np.nan
    with pytest.raises(DfjkError) as ei:
        Plan(bad, aux)
    assert ei.value.status_name == "NUMERIC"
    # broken row order
    bad = golden_basis(g, "orb")
    bad.angular = bad.angular[::-1].copy()
    with pytest.raises(DfjkError) as ei:
        Plan(bad, aux)
    assert ei.value.status_name == "INVALID"
    # J/K before build
    p = Plan(orb, aux)
    with pytest.raises(DfjkError) as ei:
        p.jk(g["C"])
    assert ei.value.status_name == "STATE"


def test_fp64_k_is_bitwise_reproducible():
    """The float64 X X^T sums its k slices in a fixed order."""
    from dftax_b200 import Plan, systems

    sym, xyz, orb, aux, nocc = systems.workload("water8", seed=4)
    plan = Plan(orb, aux).build()
    C = systems.random_occupied(plan.nao, nocc, seed=8)
    _, K1 = plan.jk(C)
    _, K2 = plan.jk(C)
    K1 = K1.cpu().numpy()
    assert np.array_equal(K1, K2.cpu().numpy())
    assert np.array_equal(K1, K1.T)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_first_build_uses_creation_metric_bitwise(precision):
    """Plan creation computes the metric factor on a stream of its own and the
    first build uses it; a second build recomputes it on the caller's stream.
    Both builds give the same J and K, bit for bit, and the same kept count."""
    from dftax_b200 import Plan, systems

    sym, xyz, orb, aux, nocc = systems.workload("water8", seed=6)
    plan = Plan(orb, aux, precision=precision)
    C = systems.random_occupied(orb.nao, nocc, seed=9)
    plan.build()
    nfit1 = plan.info()["nfit"]
    J1, K1 = (x.cpu().numpy() for x in plan.jk(C))
    assert plan.phase_times()["metric"] > 0.0
    plan.build()
    J2, K2 = (x.cpu().numpy() for x in plan.jk(C))
    assert plan.info()["nfit"] == nfit1
    assert np.array_equal(J1, J2) and np.array_equal(K1, K2)
    plan.close()


def test_trim_and_rebuild(water_golden):
    """Cached device memory goes back to the driver; later plans still work."""
    from dftax_b200 import Context, Plan

    g = water_golden
    orb, aux = golden_basis(g, "orb"), golden_basis(g, "aux")
    a = Plan(orb, aux).build()
    Ja, Ka = a.jk(g["C"])
    a.close()
    Context.get(0).trim()
    b = Plan(orb, aux).build()
    Jb, Kb = b.jk(g["C"])
    assert np.array_equal(Ja.cpu().numpy(), Jb.cpu().numpy())
    assert np.array_equal(Ka.cpu().numpy(), Kb.cpu().numpy())


def test_oversized_plan_reports_memory(water_golden):
    """C40H82 unscreened in mixed precision needs ~136 GB for B plus ~136 GB of
    digit planes, more than one B200 holds: the build reports MEMORY (after
    emptying the device-memory cache and retrying), and the context stays
    usable."""
    from dftax_b200 import Context, Plan, systems
    from dftax_b200._lib import DfjkError

    sym, xyz, orb, aux, nocc = systems.workload("alkane40")
    plan = Plan(orb, aux, precision="mixed")
    with pytest.raises(DfjkError) as ei:
        plan.build()
    assert ei.value.status_name == "MEMORY"
    plan.close()
    Context.get(0).trim()
    g = water_golden
    small = Plan(golden_basis(g, "orb"), golden_basis(g, "aux")).build()
    J, K = small.jk(g["C"])
    assert rel(K.cpu().numpy(), g["K"]) < NOISE_REL
