"""C ABI and host logic, no GPU needed: the library loads and exports every
entry point include/dfjk.h, include/dfscf.h and include/dfbatch.h declare; the synthetic workloads are what the
configs describe."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from dftax_b200 import _lib, systems


def header_functions():
    names = set()
    for h in ("dfjk.h", "dfscf.h", "dfbatch.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b((?:dfjk|dfscf|dfbatch)_[a-z0-9_]+)\s*\(", src))
    return names


def test_exports_match_header():
    assert header_functions() == set(_lib.EXPORTS)


def test_library_loads_and_exports_every_symbol():
    lib = _lib.load()
    for name in header_functions():
        assert getattr(lib, name) is not None
    raw = ctypes.CDLL(_lib.LIB_PATH)
    for name in header_functions():
        ctypes.cast(getattr(raw, name), ctypes.c_void_p)


def test_default_options():
    lib = _lib.load()
    o = _lib.Options()
    lib.dfjk_default_options(ctypes.byref(o))
    assert o.screen == 0.0 and o.metric_cutoff == 1e-7 and o.precision == _lib.DFJK_FP64


def test_null_arguments_are_rejected_without_a_device():
    lib = _lib.load()
    assert lib.dfjk_create(0, None) == 1                     # INVALID
    assert lib.dfjk_plan_get_info(None, None) == 1
    assert lib.dfjk_build(None, None) == 1
    assert lib.dfjk_jk(None, None, None, 0, None, None, None) == 1
    assert lib.dfjk_last_error(None) == b"null context"


def test_create_reports_missing_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.dfjk_create(0, ctypes.byref(h)) != 0
    assert not h.value


def test_water_cluster_geometry():
    sym, xyz = systems.water_cluster(32, seed=0)
    o = xyz[0::3] / systems.ANGSTROM_TO_BOHR
    d = np.linalg.norm(o[:, None] - o[None], axis=-1)
    np.fill_diagonal(d, 99.0)
    assert d.min() >= 2.6
    side = (32 * systems.WATER_MASS / (systems.AVOGADRO * 1.0)) ** (1 / 3) * 1e8
    assert abs(side - 9.86) < 0.01
    # rigid monomers: O-H 0.9579 A
    for k in range(32):
        for h in (1, 2):
            r = np.linalg.norm(xyz[3 * k + h] - xyz[3 * k]) / systems.ANGSTROM_TO_BOHR
            assert abs(r - 0.957924) < 1e-5


def test_alkane_geometry():
    sym, xyz = systems.alkane(10, seed=0)
    assert sym.count("C") == 10 and sym.count("H") == 22
    a = xyz / systems.ANGSTROM_TO_BOHR
    c = a[:10]
    for i in range(9):
        assert abs(np.linalg.norm(c[i + 1] - c[i]) - 1.54) < 1e-9
    for h in a[10:]:
        assert abs(np.min(np.linalg.norm(c - h, axis=1)) - 1.09) < 1e-9


@pytest.mark.parametrize("name,nao,naux,nocc", [("water", 30, 141, 5), ("water8", 240, 1128, 40),
                                                ("water32", 960, 4512, 160),
                                                ("alkane10", 522, 2056, 41)])
def test_workload_sizes(name, nao, naux, nocc):
    _, _, orb, aux, no = systems.workload(name)
    assert (orb.nao, aux.nao, no) == (nao, naux, nocc)


def test_scf_default_options():
    lib = _lib.load()
    o = _lib.ScfOptions()
    lib.dfscf_default_options(ctypes.byref(o))
    assert (o.hf_coeff, o.x_scale, o.c_scale) == (0.25, 0.75, 1.0)       # PBE0
    assert (o.e_tol, o.d_tol, o.max_iter, o.diis_space) == (1e-8, 1e-6, 128, 8)
    assert o.lindep == 1e-7 and o.rho_thresh == 1e-10 and o.ao_thresh == 1e-14


def test_scf_null_arguments_are_rejected():
    lib = _lib.load()
    assert lib.dfscf_create(None, 0, None, None, 0, None, None, 0, None, None, None) == 1
    assert lib.dfscf_run(None, None, None, None) == 1
    assert lib.dfscf_destroy(None) == 0


def test_batch_estimate_grows_with_the_molecule():
    """The admission estimate of a solve needs no device and grows with the
    system: at least B (rows x fitted columns x 8 bytes) and the mixed form's
    extra K digit planes."""
    from dftax_b200.batch import make_request

    lib = _lib.load()
    est = {}
    for name in ("water3", "water8"):
        sym, xyz, orb, aux, nocc = systems.workload(name, seed=0)
        for prec in ("fp64", "mixed"):
            r, keep, nao = make_request(sym, xyz, orb, aux, precision=prec,
                                        grid=(np.zeros((0, 3)), np.zeros(0)))
            b = ctypes.c_int64()
            assert lib.dfbatch_estimate(ctypes.byref(r), ctypes.byref(b)) == 0
            est[name, prec] = b.value
            assert b.value > (nao * (nao + 1) // 2) * aux.nao * 8
    assert est["water8", "fp64"] > 2 * est["water3", "fp64"]
    assert est["water8", "mixed"] > est["water8", "fp64"]


def test_batch_null_arguments_are_rejected():
    lib = _lib.load()
    assert lib.dfbatch_create(0, None, None) == 1
    assert lib.dfbatch_submit(None, None, None) == 1
    assert lib.dfbatch_wait(None, 0, None) == 1
    assert lib.dfbatch_destroy(None) == 0
