"""The SCF density by SP2 purification (``KS(density="purify")``, the default)
against the eigensolver route (``density="eigh"``, cuSOLVER syevd and aufbau
occupations as dftax's scf.py:319-327).

With a HOMO-LUMO gap the projection of X^T F X onto its nocc lowest
eigenvalues is the aufbau density itself, so the two routes follow the same
iterations. In float64: the same iteration count, energies within 1e-10 Ha,
densities within 1e-9 and the same orbital energies (both routes
diagonalize the last DIIS Fock matrix for the orbitals). In mixed precision
the int8 digits of K are taken of C_occ, and the two routes give C_occ in
different rotations of the occupied space, so K differs at the mixed form's
own error: energies within 1e-7 Ha (its bound against float64), densities
within 1e-6, iteration counts within one.

Without a gap the projection stalls at fractional occupations and the
iteration falls back to the eigensolver, bit for bit the eigensolver route:
a closed-shell carbon atom from its spherically averaged atomic density
(the SAD guess), whose Fock matrix has the three 2p levels degenerate to
rounding with one of them to be occupied. (In float64 a split below about
1e-10 of the spectral range stays unresolved within the 96 projection
steps; the first iteration's density breaks the symmetry, so only one
iteration is run.)
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(sym, xyz, orb, aux, density, precision="fp64", xc="PBE0", guess=None, **kw):
    import torch

    from dftax_b200 import df
    from dftax_b200.ks import KS, scf

    ks = KS(sym, xyz, orb, coulomb=df(aux, precision=precision), xc=xc, density=density)
    r = scf(ks, guess=guess, **kw)
    ks.close()
    ks.plan.close()
    torch.cuda.synchronize()
    return r


@pytest.mark.parametrize("name,precision,guess", [("water3", "fp64", None),
                                                  ("water8", "mixed", "sad"),
                                                  ("alkane2", "fp64", "sad")])
def test_purification_follows_the_eigensolver(name, precision, guess):
    from dftax_b200 import systems

    sym, xyz, orb, aux, _ = systems.workload(name, seed=0)
    a = _solve(sym, xyz, orb, aux, "eigh", precision, guess=guess)
    b = _solve(sym, xyz, orb, aux, "purify", precision, guess=guess)
    assert a.converged and b.converged
    exact = precision == "fp64"
    assert abs(a.n_iter - b.n_iter) <= (0 if exact else 1)
    assert abs(a.e_tot - b.e_tot) < (1e-10 if exact else 1e-7)
    assert np.abs(a.P - b.P).max() < (1e-9 if exact else 1e-6)
    assert np.abs(a.mo_energy - b.mo_energy).max() < (1e-8 if exact else 1e-6)
    # every iteration and the core guess (when used) on the eigensolver route;
    # only the core guess on the projection route
    assert a.n_eig == a.n_iter + (1 if guess is None else 0)
    assert b.n_iter > 0
    assert b.n_eig == (1 if guess is None else 0)
    # the projected density is idempotent in the metric: P S P = 2 P
    S = _overlap(sym, xyz, orb, aux)
    P = b.P[0]
    assert np.abs(P @ S @ P - 2.0 * P).max() < 1e-9


def _overlap(sym, xyz, orb, aux):
    from dftax_b200 import df
    from dftax_b200.ks import KS

    ks = KS(sym, xyz, orb, coulomb=df(aux), xc="HF")
    S = ks.one_electron()[0].cpu().numpy()
    ks.close()
    ks.plan.close()
    return S


def test_no_gap_falls_back_to_the_eigensolver():
    from dftax_b200 import systems

    sym, xyz = ["C"], np.zeros((1, 3))
    orb, aux = systems.basis_for(sym, xyz)
    a = _solve(sym, xyz, orb, aux, "eigh", xc="HF", guess="sad", max_iter=1)
    b = _solve(sym, xyz, orb, aux, "purify", xc="HF", guess="sad", max_iter=1)
    assert a.n_iter == b.n_iter == 1
    assert b.n_eig == a.n_eig == 1
    assert a.e_tot == b.e_tot
    assert np.array_equal(a.P, b.P)
    assert np.array_equal(a.mo_energy, b.mo_energy)


def test_density_option_is_checked_and_xc_work_reported():
    """dfscf_create refuses a density route other than 0 or 1 (INVALID), and
    the result reports the XC DGEMM work of one evaluation (none for HF)."""
    import ctypes
    from ctypes import byref

    import torch

    from dftax_b200 import _lib, df, systems
    from dftax_b200.coulomb import _stream_ptr
    from dftax_b200.ks import KS, scf

    sym, xyz, orb, aux, _ = systems.workload("water", seed=0)
    ks = KS(sym, xyz, orb, coulomb=df(aux))
    o = _lib.ScfOptions()
    ctypes.memmove(byref(o), byref(ks._opts), ctypes.sizeof(o))
    o.density = 5
    h = ctypes.c_void_p()
    st = ks.lib.dfscf_create(ks.plan.h, len(ks.charges), ks.coords.ctypes.data,
                             ks.charges.ctypes.data, len(ks.grid_weights),
                             ks.grid_coords.ctypes.data, ks.grid_weights.ctypes.data,
                             ks.nocc[0], byref(o), byref(h), _stream_ptr(torch))
    assert st == _lib.DFJK_ERR_INVALID
    assert "density must be 0 or 1" in ks.ctx.last_error()
    r = scf(ks)
    assert r.converged and r.xc_gemm_flop > 0
    ks.close()
    hf = KS(sym, xyz, orb, coulomb=df(aux), xc="HF")
    assert scf(hf).xc_gemm_flop == 0
    hf.close()
