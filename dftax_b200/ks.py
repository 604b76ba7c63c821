"""Closed-shell Kohn-Sham model and SCF on the device, with dftax's names.

``KS(symbols, coords, basis, coulomb=df(aux), xc="PBE0", grid=becke())``
mirrors dftax's ``KS`` (``dftax/ks/energy.py:549-723``) for a closed shell:
one-electron integrals, the DF Coulomb/exchange plan (``dfjk``), the XC
quadrature grid and the canonical orthonormalizer, all on the device
(``include/dfscf.h``). ``scf(ks, ...)`` mirrors ``dftax.ks.scf.scf``
(``scf.py:394-495``) with Pulay DIIS and returns a ``KSResult``.

Functionals: ``"PBE0"`` (0.75 PBE exchange + PBE correlation + 0.25 exact
exchange, ``xc.py:584-601``), ``"PBE"`` and ``"HF"`` (exact exchange only, no
grid). The guess is the core Hamiltonian (``guess.core()``, the default),
a superposition of atomic densities (``guess.sad()`` or ``"sad"``) or an
explicit density; dftax's minao guess is not provided.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from ctypes import byref

import numpy as np

from . import _lib
from .basis import BasisData
from .coulomb import DFSpec, Plan, _stream_ptr, _torch
from .grid import ATOMIC_NUMBER, Becke, becke_grid
from .guess import CoreSpec, SADSpec, initial_density

XC_FUNCTIONALS = {
    # name: (hf_coeff, x_scale, c_scale)
    "PBE0": (0.25, 0.75, 1.0),
    "PBE": (0.0, 1.0, 1.0),
    "HF": (1.0, 0.0, 0.0),
}


@dataclass
class KSResult:
    """Outcome of a closed-shell solve, spin-stacked like dftax's (nspin = 1)."""

    e_tot: float
    e_elec: float
    converged: bool
    n_iter: int
    nocc: tuple
    mo_energy: np.ndarray     # (1, nmo)
    mo_coeff: np.ndarray      # (1, nao, nmo)
    P: np.ndarray             # (1, nao, nao)
    e_xc: float = 0.0
    e_coul: float = 0.0
    timings_ms: dict | None = None   # J/K, XC, diagonalization, DIIS of the run
    xc_chunk: int = 0                # grid points per XC chunk (set or autotuned)
    xc_graph: bool = False           # XC evaluations replayed a captured CUDA graph
    n_eig: int = 0                   # densities built by the eigensolver (guess, fallbacks)
    xc_gemm_flop: float = 0.0        # float64 FLOP of one XC evaluation's two DGEMMs


DENSITY_ROUTES = {"eigh": 0, "purify": 1}


class KS:
    """Closed-shell DF Kohn-Sham energy functional on one GPU."""

    def __init__(self, symbols, coords_bohr, basis: BasisData, *, coulomb: DFSpec, xc="PBE0",
                 grid=None, charges=None, device: int = 0, diis_space: int = 8,
                 lindep_thresh: float = 1e-7, plan: Plan | None = None,
                 ao_thresh: float = 1e-14, grid_chunk: int = 0, xc_streams: int = 0,
                 density: str = "purify"):
        if xc not in XC_FUNCTIONALS:
            raise ValueError(f"xc must be one of {sorted(XC_FUNCTIONALS)}")
        # each iteration's aufbau density: "purify" (SP2 projection, the
        # eigensolver when it does not converge) or "eigh" (the eigensolver)
        if density not in DENSITY_ROUTES:
            raise ValueError(f"density must be one of {sorted(DENSITY_ROUTES)}")
        if not isinstance(coulomb, DFSpec) or not isinstance(coulomb.auxbasis, BasisData):
            raise TypeError("coulomb must be df(aux) with a built auxiliary BasisData")
        self.torch = _torch()
        self.symbols = list(symbols)
        self.coords = np.ascontiguousarray(np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3))
        self.charges = np.ascontiguousarray(
            np.asarray(charges if charges is not None else
                       [float(ATOMIC_NUMBER[s]) for s in self.symbols], dtype=np.float64))
        nelec = int(round(self.charges.sum()))
        if nelec % 2:
            raise NotImplementedError("this SCF is closed-shell: an even electron count is needed")
        self.nocc = (nelec // 2,)
        self.xc = xc
        self.basis, self.aux = basis, coulomb.auxbasis
        self.plan = plan or Plan(basis, coulomb.auxbasis, screen=coulomb.screen,
                                 precision=coulomb.precision,
                                 streamed=coulomb.chunk is not None, device=device)
        if not self.plan.info()["built"]:
            self.plan.build()
        self.ctx, self.lib, self.dev = self.plan.ctx, self.plan.lib, self.plan.dev
        hf, xs, cs = XC_FUNCTIONALS[xc]
        if xs == 0.0 and cs == 0.0:
            self.grid_coords = np.zeros((0, 3))
            self.grid_weights = np.zeros(0)
        elif isinstance(grid, tuple):
            self.grid_coords = np.ascontiguousarray(grid[0], dtype=np.float64)
            self.grid_weights = np.ascontiguousarray(grid[1], dtype=np.float64)
        else:
            self.grid_coords, self.grid_weights = becke_grid(self.symbols, self.coords,
                                                             grid if isinstance(grid, Becke) else None,
                                                             device=self.ctx.device)
        self._diis, self._lindep = diis_space, lindep_thresh
        self._ao_thresh, self._grid_chunk = float(ao_thresh), int(grid_chunk)
        self._xc_streams = int(xc_streams)   # 0: 8 concurrent XC streams; the batch engine uses 1
        self._density = DENSITY_ROUTES[density]
        self.h = ctypes.c_void_p()
        self._create()

    def _create(self):
        if self.h.value:
            self.lib.dfscf_destroy(self.h)
            self.h = ctypes.c_void_p()
        o = _lib.ScfOptions()
        self.lib.dfscf_default_options(byref(o))
        o.hf_coeff, o.x_scale, o.c_scale = XC_FUNCTIONALS[self.xc]
        o.diis_space = int(self._diis)
        o.lindep = float(self._lindep)
        o.ao_thresh = self._ao_thresh
        o.grid_chunk = self._grid_chunk
        o.xc_streams = self._xc_streams
        o.density = self._density
        self._opts = o
        _lib.check(self.lib.dfscf_create(self.plan.h, len(self.charges), self.coords.ctypes.data,
                                         self.charges.ctypes.data, len(self.grid_weights),
                                         self.grid_coords.ctypes.data,
                                         self.grid_weights.ctypes.data, self.nocc[0], byref(o),
                                         byref(self.h), _stream_ptr(self.torch)), self.ctx.h)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.dfscf_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    @property
    def nao(self) -> int:
        return self.plan.nao

    def _dev(self, x):
        t = self.torch
        if isinstance(x, t.Tensor):
            return x.to(device=self.dev, dtype=t.float64).contiguous()
        return t.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=self.dev)

    # -- parity entry points ----------------------------------------------
    def one_electron(self):
        t = self.torch
        S, T, V = (t.empty((self.nao, self.nao), dtype=t.float64, device=self.dev) for _ in range(3))
        _lib.check(self.lib.dfscf_one_electron(self.h, S.data_ptr(), T.data_ptr(), V.data_ptr(),
                                               _stream_ptr(t)), self.ctx.h)
        return S, T, V

    def xc_energy(self, P, want_fock: bool = True):
        t = self.torch
        P = self._dev(P)
        if P.ndim == 3:
            P = P[0]
        V = t.empty_like(P) if want_fock else None
        e = ctypes.c_double()
        _lib.check(self.lib.dfscf_xc(self.h, P.data_ptr(), byref(e),
                                     None if V is None else V.data_ptr(), _stream_ptr(t)),
                   self.ctx.h)
        return e.value, V

    def total(self, P):
        """(E(P), F(P)) of the closed-shell density P (KS.total and its Fock)."""
        t = self.torch
        P = self._dev(P)
        if P.ndim == 3:
            P = P[0]
        F = t.empty_like(P)
        e = ctypes.c_double()
        _lib.check(self.lib.dfscf_energy_fock(self.h, P.data_ptr(), byref(e), F.data_ptr(),
                                              _stream_ptr(t)), self.ctx.h)
        return e.value, F


def scf(ks: KS, *, max_iter: int = 128, e_tol: float = 1e-8, d_tol: float = 1e-6,
        diis_space: int = 8, lindep_thresh: float = 1e-7, level_shift: float = 0.0,
        guess=None, stream=None) -> KSResult:
    """Run the SCF to self-consistency (dftax ``scf``, closed shell)."""
    t = ks.torch
    if diis_space != ks._diis or lindep_thresh != ks._lindep:
        ks._diis, ks._lindep = diis_space, lindep_thresh
        ks._create()
    # per-run options (the other fields were fixed when the handle was made)
    o = _lib.ScfOptions()
    ctypes.memmove(byref(o), byref(ks._opts), ctypes.sizeof(o))
    o.max_iter, o.e_tol, o.d_tol, o.level_shift = int(max_iter), float(e_tol), float(d_tol), \
        float(level_shift)
    P0 = None
    if isinstance(guess, (str, SADSpec, CoreSpec)):
        guess = initial_density(guess, ks.symbols, ks.coords, ks.basis, ks.aux,
                                2 * ks.nocc[0], ks.ctx.device)
    if guess is not None:
        P0 = ks._dev(guess)
        if P0.ndim == 3:
            P0 = P0[0]
    _lib.check(ks.lib.dfscf_run(ks.h, None if P0 is None else P0.data_ptr(), byref(o),
                                _stream_ptr(t, stream)), ks.ctx.h)
    r = _lib.ScfResult()
    _lib.check(ks.lib.dfscf_get_result(ks.h, byref(r)), ks.ctx.h)
    n, m = ks.nao, r.nmo
    P = t.empty((n, n), dtype=t.float64, device=ks.dev)
    eps = t.empty(m, dtype=t.float64, device=ks.dev)
    C = t.empty((m, n), dtype=t.float64, device=ks.dev)   # column-major nao x nmo
    _lib.check(ks.lib.dfscf_get_density(ks.h, P.data_ptr(), _stream_ptr(t, stream)), ks.ctx.h)
    _lib.check(ks.lib.dfscf_get_orbitals(ks.h, eps.data_ptr(), C.data_ptr(),
                                         _stream_ptr(t, stream)), ks.ctx.h)
    return KSResult(e_tot=r.e_tot, e_elec=r.e_tot - r.e_nn, converged=bool(r.converged),
                    n_iter=r.n_iter, nocc=ks.nocc, mo_energy=eps.cpu().numpy()[None],
                    mo_coeff=C.T.cpu().numpy()[None], P=P.cpu().numpy()[None], e_xc=r.e_xc,
                    e_coul=r.e_coul,
                    timings_ms={"jk": r.ms_jk, "xc": r.ms_xc, "diag": r.ms_diag,
                                "diis": r.ms_diis},
                    xc_chunk=int(r.xc_chunk), xc_graph=bool(r.xc_graph), n_eig=int(r.n_eig),
                    xc_gemm_flop=float(r.xc_gemm_flop))


__all__ = ["KS", "KSResult", "scf", "XC_FUNCTIONALS", "DENSITY_ROUTES"]


def _main(argv=None):
    """``python -m dftax_b200.ks water8 --precision mixed``: one SCF solve of a
    named workload (``systems.workload``) from geometry, printed as JSON."""
    import argparse
    import json
    import time

    from . import df, systems
    from .grid import becke

    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("workload")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--xc", default="PBE0", choices=sorted(XC_FUNCTIONALS))
    ap.add_argument("--radial", type=int, default=75)
    ap.add_argument("--lebedev", type=int, default=302)
    ap.add_argument("--repeat", type=int, default=1, help="solves (the last one is reported)")
    ap.add_argument("--guess", default="core", choices=["core", "sad"])
    ap.add_argument("--density", default="purify", choices=sorted(DENSITY_ROUTES))
    ap.add_argument("--xc-streams", type=int, default=0,
                    help="concurrent streams of the XC chunks (0: 8; the batch engine uses 1)")
    ap.add_argument("--streamed", action="store_true",
                    help="streamed DF (B rebuilt per J/K call, not held): df(aux, chunk=...)")
    a = ap.parse_args(argv)
    sym, xyz, orb, aux, nocc = systems.workload(a.workload, seed=0)
    for _ in range(a.repeat):
        t0 = time.perf_counter()
        ks = KS(sym, xyz, orb, coulomb=df(aux, precision=a.precision,
                                           chunk=1 if a.streamed else None), xc=a.xc,
                grid=becke(a.radial, a.lebedev), density=a.density, xc_streams=a.xc_streams)
        r = scf(ks, guess=a.guess)
        sec = time.perf_counter() - t0
        ks.close()
        ks.plan.close()
    print(json.dumps({"workload": a.workload, "precision": a.precision, "xc": a.xc,
                      "guess": a.guess, "density": a.density, "streamed": a.streamed,
                      "e_tot": r.e_tot, "converged": r.converged, "n_iter": r.n_iter,
                      "seconds": round(sec, 3), "parts_ms": r.timings_ms,
                      "xc_chunk": r.xc_chunk, "xc_graph": r.xc_graph, "n_eig": r.n_eig,
                      "xc_gemm_tflop": round(r.xc_gemm_flop / 1e12, 4)}))


if __name__ == "__main__":
    _main()
