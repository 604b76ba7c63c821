"""Batched and served SCF solves of molecules of uneven size on one GPU.

``BatchEngine`` wraps ``include/dfbatch.h``: W workers, each with its own
library context and CUDA stream, take submitted solves first-in, first-out as
their estimated device memory fits in a budget beside the running ones, and
the running solves' device work overlaps. ``submit`` returns at once;
``wait`` blocks for one result. ``scf_batch`` solves a list of molecules this
way (dftax's ``scf_batched``, ``dftax/ks/batched.py:82-304``, solves
conformers of one molecule; here sizes and compositions may differ).
"""

from __future__ import annotations

import ctypes
from ctypes import byref
from dataclasses import dataclass

import numpy as np

from . import _lib
from .basis import BasisData
from .coulomb import PRECISIONS, _basis_struct
from .grid import ATOMIC_NUMBER, Becke, becke_grid
from .guess import initial_density
from .ks import XC_FUNCTIONALS


@dataclass
class BatchResult:
    id: int
    status: int
    message: str
    e_tot: float
    converged: bool
    n_iter: int
    worker: int
    t_submit: float       # seconds since the engine started
    t_start: float
    t_end: float
    bytes: int            # device bytes reserved for the solve
    P: np.ndarray | None = None

    @property
    def latency(self) -> float:
        """Submission to completion, seconds."""
        return self.t_end - self.t_submit


class BatchEngine:
    def __init__(self, device: int = 0, workers: int = 4, hbm_budget: int = 0):
        self.lib = _lib.load()
        self.device = device
        o = _lib.BatchOptions()
        self.lib.dfbatch_default_options(byref(o))
        o.workers = int(workers)
        o.hbm_budget = int(hbm_budget)
        self.h = ctypes.c_void_p()
        _lib.check(self.lib.dfbatch_create(device, byref(o), byref(self.h)))
        self._P = {}

    def request(self, symbols, coords_bohr, orb: BasisData, aux: BasisData, *, grid=None, **kw):
        """A filled dfbatch_request and the arrays it points into (the Becke
        grid, unless given, built here)."""
        if not isinstance(grid, tuple) and XC_FUNCTIONALS[kw.get("xc", "PBE0")][1:] != (0.0, 0.0):
            coords = np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3)
            grid = becke_grid(symbols, coords, grid if isinstance(grid, Becke) else None,
                              device=self.device)
        return make_request(symbols, coords_bohr, orb, aux, grid=grid, **kw)

    def estimate(self, *args, **kw) -> int:
        r, keep, _ = self.request(*args, **kw)
        b = ctypes.c_int64()
        _lib.check(self.lib.dfbatch_estimate(byref(r), byref(b)))
        return b.value

    def submit(self, symbols, coords_bohr, orb, aux, *, want_density=False, **kw) -> int:
        req = self.request(symbols, coords_bohr, orb, aux, **kw)
        return self.submit_request(req, want_density=want_density)

    def submit_request(self, req, *, want_density=False) -> int:
        """Submit a request made by ``request``/``make_request`` (its arrays
        are copied by the engine)."""
        r, keep, nao = req
        P = np.empty((nao, nao)) if want_density else None
        r.P_out = P.ctypes.data if P is not None else None
        jid = ctypes.c_int64()
        _lib.check(self.lib.dfbatch_submit(self.h, byref(r), byref(jid)))
        self._P[jid.value] = P
        return jid.value

    def wait(self, jid: int) -> BatchResult:
        res = _lib.BatchResult()
        _lib.check(self.lib.dfbatch_wait(self.h, int(jid), byref(res)))
        return BatchResult(id=jid, status=res.status, message=res.message.decode(),
                           e_tot=res.scf.e_tot, converged=bool(res.scf.converged),
                           n_iter=res.scf.n_iter, worker=res.worker, t_submit=res.t_submit,
                           t_start=res.t_start, t_end=res.t_end, bytes=res.bytes,
                           P=self._P.pop(jid, None))

    def done(self, jid: int) -> bool:
        d = ctypes.c_int32()
        _lib.check(self.lib.dfbatch_poll(self.h, int(jid), byref(d)))
        return bool(d.value)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.dfbatch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass


def make_request(symbols, coords_bohr, orb: BasisData, aux: BasisData, *, xc="PBE0",
                 precision="fp64", grid=None, screen=None, scf_opts=None, guess=None):
    """A dfbatch_request for an explicit grid (points, weights) and the arrays
    it points into (kept alive by the caller until it is submitted).
    ``guess``: None/``"core"`` (core Hamiltonian), ``"sad"`` (superposition of
    atomic densities, built here) or an explicit (nao, nao) density."""
    lib = _lib.load()
    coords = np.ascontiguousarray(np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3))
    charges = np.ascontiguousarray([float(ATOMIC_NUMBER[s]) for s in symbols])
    nelec = int(round(charges.sum()))
    if nelec % 2:
        raise NotImplementedError("closed-shell solves only")
    hf, xs, cs = XC_FUNCTIONALS[xc]
    if (xs == 0.0 and cs == 0.0) or grid is None:
        pts, w = np.zeros((0, 3)), np.zeros(0)
    else:
        pts, w = (np.ascontiguousarray(a, dtype=np.float64) for a in grid)
    keep: list = [coords, charges, pts, w]
    ob, ab = _basis_struct(orb, keep), _basis_struct(aux, keep)
    keep += [ob, ab]
    r = _lib.BatchRequest()
    r.orb = ctypes.pointer(ob)
    r.aux = ctypes.pointer(ab)
    lib.dfjk_default_options(byref(r.plan_opts))
    r.plan_opts.precision = PRECISIONS[precision]
    r.plan_opts.screen = float(screen) if screen else 0.0
    r.natom, r.nocc = len(symbols), nelec // 2
    r.atom_xyz, r.atom_charge = coords.ctypes.data, charges.ctypes.data
    r.npoint = len(w)
    r.grid_xyz = pts.ctypes.data if len(w) else None
    r.grid_w = w.ctypes.data if len(w) else None
    lib.dfscf_default_options(byref(r.scf_opts))
    r.scf_opts.hf_coeff, r.scf_opts.x_scale, r.scf_opts.c_scale = hf, xs, cs
    for k, v in (scf_opts or {}).items():
        setattr(r.scf_opts, k, v)
    P0 = initial_density(guess, list(symbols), coords, orb, aux, nelec)
    if P0 is not None:
        P0 = np.ascontiguousarray(P0, dtype=np.float64).reshape(orb.nao, orb.nao)
        keep.append(P0)
        r.P_guess = P0.ctypes.data
    return r, keep, orb.nao


def scf_batch(molecules, *, precision="fp64", xc="PBE0", grid=None, workers: int = 4,
              hbm_budget: int = 0, device: int = 0, want_density=False, guess=None):
    """Solve every (symbols, coords, orb, aux) of ``molecules``; results in order."""
    with BatchEngine(device, workers, hbm_budget) as eng:
        ids = [eng.submit(s, x, o, a, precision=precision, xc=xc, grid=grid, guess=guess,
                          want_density=want_density) for (s, x, o, a) in molecules]
        return [eng.wait(i) for i in ids]


__all__ = ["BatchEngine", "BatchResult", "scf_batch", "make_request"]
