"""Host-side mirror of dftax's density-fitting Coulomb backend, on the C ABI.

dftax selects its Coulomb strategy with a spec value (``df(...)``,
``dftax/ks/terms.py:63-148``), assembles the matching ``CoulombTerm``
(``_make_coulomb``, ``terms.py:951-988``) and evaluates
``CoulombTerm.energy(P, S, nocc)`` (``terms.py:512-527``) under ``jax.grad``
to get the two-electron Fock matrix (``dftax/ks/scf.py:345``). This module
mirrors that surface for the B200 library:

* :func:`df` / :class:`DFSpec` — the spec, with ``backend="b200"`` and
  ``precision`` ("fp64" or "mixed");
* :class:`B200DFCoulomb` — the drop-in for ``DFCoulomb`` (``terms.py:576-613``):
  ``energy(P, S, nocc)`` returns ``E_J + a_x E_K`` and ``fock(P, S, nocc)``
  returns ``(E, dE/dP)``, i.e. ``J - a_x/2 K`` for a closed shell and
  ``J - a_x K_sigma`` per spin channel (the VJP dftax obtains by autodiff);
* :class:`Plan` — the library handle: build, J/K from occupied orbitals, and
  the parity entry points (dense 3-center, metric, its pseudo-inverse, Boys).

Device memory is held in torch CUDA tensors (plumbing only); all arithmetic
runs in ``libdfjk.so``. Without the library or a GPU, construction raises.
"""

from __future__ import annotations

import abc
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import Basis, Options, PlanInfo, byref, check
from .basis import BasisData


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("dftax_b200 needs a CUDA device; none is available")
    return torch


def _stream_ptr(torch, stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


class Context:
    """A device, its cuBLAS/cuSOLVER handles and the Boys table."""

    _by_device: dict[int, "Context"] = {}

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        self.device = device
        self.h = ctypes.c_void_p()
        _torch().cuda.set_device(device)
        check(self.lib.dfjk_create(device, byref(self.h)))

    @classmethod
    def get(cls, device: int = 0) -> "Context":
        if device not in cls._by_device:
            cls._by_device[device] = cls(device)
        return cls._by_device[device]

    def last_error(self) -> str:
        return self.lib.dfjk_last_error(self.h).decode()

    def trim(self):
        """Return the device memory cached from destroyed plans to the driver."""
        check(self.lib.dfjk_trim(self.h), self.h)

    def boys(self, t, nmax: int):
        """F_0..F_nmax at the points t (host array in, host array out)."""
        torch = _torch()
        tt = torch.as_tensor(np.ascontiguousarray(t, dtype=np.float64), device=f"cuda:{self.device}")
        out = torch.empty((tt.numel(), nmax + 1), dtype=torch.float64, device=tt.device)
        check(self.lib.dfjk_boys(self.h, tt.data_ptr(), tt.numel(), nmax, out.data_ptr(),
                                 _stream_ptr(torch)), self.h)
        return out.cpu().numpy()


def _basis_struct(b: BasisData, keep: list):
    cen = np.ascontiguousarray(b.centers, dtype=np.float64)
    ex = np.ascontiguousarray(b.exponents, dtype=np.float64)
    co = np.ascontiguousarray(b.coefficients, dtype=np.float64)
    an = np.ascontiguousarray(b.angular, dtype=np.int32)
    c2s = None if b.cart2sph is None else np.ascontiguousarray(b.cart2sph, dtype=np.float64)
    keep.extend([cen, ex, co, an, c2s])
    s = Basis()
    s.ncart = an.shape[0]
    s.max_prim = ex.shape[1]
    s.nsph = 0 if c2s is None else c2s.shape[1]
    s.centers = cen.ctypes.data
    s.exponents = ex.ctypes.data
    s.coefficients = co.ctypes.data
    s.angular = an.ctypes.data
    s.cart2sph = None if c2s is None else c2s.ctypes.data
    return s


PRECISIONS = {"fp64": _lib.DFJK_FP64, "mixed": _lib.DFJK_MIXED}


def shell_centers(b: BasisData) -> np.ndarray:
    """(nshell, 3) centers of a basis's shells in the order the library reads
    them: a shell starts at each cartesian row whose angular part is (l, 0, 0)."""
    an = np.asarray(b.angular)
    starts = np.nonzero((an[:, 1] == 0) & (an[:, 2] == 0))[0]
    return np.asarray(b.centers, dtype=np.float64)[starts]


def shells_to_atoms(shell_grad, centers, atom_xyz, tol: float = 1e-8) -> np.ndarray:
    """Sum per-shell gradients (nshell, 3) onto the atoms whose positions
    (natom, 3) the shell centers sit on."""
    atom_xyz = np.asarray(atom_xyz, dtype=np.float64).reshape(-1, 3)
    d = np.linalg.norm(np.asarray(centers)[:, None, :] - atom_xyz[None, :, :], axis=2)
    idx = np.argmin(d, axis=1)
    if len(idx) and d[np.arange(len(idx)), idx].max() > tol:
        raise ValueError("a shell center is on no atom")
    out = np.zeros_like(atom_xyz)
    np.add.at(out, idx, np.asarray(shell_grad, dtype=np.float64))
    return out


class Plan:
    """One molecule's density-fitting plan on the device (``dfjk_plan``)."""

    def __init__(self, orb: BasisData, aux: BasisData, *, screen: float | None = None,
                 precision: str = "fp64", metric_cutoff: float = 1e-7, chunk_bytes: int = 0,
                 omega: float = 0.0, streamed: bool = False, device: int = 0,
                 ctx: Context | None = None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.ctx = ctx or Context.get(device)
        self.lib = self.ctx.lib
        self.torch = _torch()
        self.dev = f"cuda:{self.ctx.device}"
        keep: list = []
        ob, ab = _basis_struct(orb, keep), _basis_struct(aux, keep)
        opts = Options()
        self.lib.dfjk_default_options(byref(opts))
        opts.screen = float(screen) if screen else 0.0
        opts.metric_cutoff = float(metric_cutoff)
        opts.precision = PRECISIONS[precision]
        opts.chunk_bytes = int(chunk_bytes)
        opts.omega = float(omega)
        opts.streamed = 1 if streamed else 0
        self.omega = float(omega)
        self.streamed = bool(streamed)
        self._parent = None
        self.h = ctypes.c_void_p()
        check(self.lib.dfjk_plan_create(self.ctx.h, byref(ob), byref(ab), byref(opts),
                                        byref(self.h)), self.ctx.h)
        self.precision = precision
        self.orb_centers, self.aux_centers = shell_centers(orb), shell_centers(aux)

    # -- lifecycle -------------------------------------------------------
    def close(self):
        if getattr(self, "_parent", None) is not None:   # owned by the parent plan
            self.h = ctypes.c_void_p()
            return
        if getattr(self, "h", None) and self.h.value:
            self.lib.dfjk_plan_destroy(self.h)
            self.h = ctypes.c_void_p()

    @property
    def long_range(self) -> "Plan":
        """The erf(omega r)/r plan of a plan made with omega > 0 (built by this
        plan's ``build``): its ``jk`` gives K_lr, its diagnostics the
        attenuated tensors. Valid while this plan lives."""
        h = ctypes.c_void_p()
        check(self.lib.dfjk_plan_long_range(self.h, byref(h)), self.ctx.h)
        lr = Plan.__new__(Plan)
        lr.ctx, lr.lib, lr.torch, lr.dev = self.ctx, self.lib, self.torch, self.dev
        lr.precision, lr.omega, lr._parent, lr.h = self.precision, self.omega, self, h
        return lr

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        i = PlanInfo()
        check(self.lib.dfjk_plan_get_info(self.h, byref(i)), self.ctx.h)
        return {f: getattr(i, f) for f, _ in PlanInfo._fields_}

    @property
    def nao(self) -> int:
        return self.info()["nao"]

    @property
    def naux(self) -> int:
        return self.info()["naux"]

    def phase_times(self) -> dict:
        """Milliseconds per phase of the last build and the last J/K call."""
        arr = (ctypes.c_double * len(_lib.PHASES))()
        check(self.lib.dfjk_phase_times(self.h, arr, len(_lib.PHASES)), self.ctx.h)
        return dict(zip(_lib.PHASES, list(arr)))

    @staticmethod
    def build_many(plans, stream=None):
        """Build several plans of one context together (``dfjk_build_batch``):
        the 3-center integrals of the small ones share their launches."""
        plans = list(plans)
        if not plans:
            return plans
        arr = (ctypes.c_void_p * len(plans))(*[p.h.value for p in plans])
        t = plans[0].torch
        check(plans[0].lib.dfjk_build_batch(arr, len(plans), _stream_ptr(t, stream)),
              plans[0].ctx.h)
        return plans

    def build(self, stream=None):
        check(self.lib.dfjk_build(self.h, _stream_ptr(self.torch, stream)), self.ctx.h)
        return self

    # -- contractions ----------------------------------------------------
    def _dev(self, x):
        t = self.torch
        if isinstance(x, t.Tensor):
            return x.to(device=self.dev, dtype=t.float64).contiguous()
        return t.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=self.dev)

    def jk(self, C, w=None, *, want_j=True, want_k=True, out=None, stream=None):
        """J and K of D = C diag(w) C^T (device tensors in and out)."""
        t = self.torch
        C = self._dev(C)
        nao, ncol = C.shape
        wv = None if w is None else self._dev(w)
        if out is None:
            J = t.empty((nao, nao), dtype=t.float64, device=self.dev) if want_j else None
            K = t.empty((nao, nao), dtype=t.float64, device=self.dev) if want_k else None
        else:
            J, K = out
        check(self.lib.dfjk_jk(self.h, C.data_ptr(), None if wv is None else wv.data_ptr(), ncol,
                               None if J is None else J.data_ptr(),
                               None if K is None else K.data_ptr(),
                               _stream_ptr(t, stream)), self.ctx.h)
        return J, K

    def jk_host(self, C, w=None, *, J=None, K=None, stream=None):
        """J and K through the host-buffer entry point (copies inside the call)."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        nao, ncol = C.shape
        wv = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        J = np.empty((nao, nao)) if J is None else J
        K = np.empty((nao, nao)) if K is None else K
        check(self.lib.dfjk_jk_host(self.h, C.ctypes.data, None if wv is None else wv.ctypes.data,
                                    ncol, J.ctypes.data, K.ctypes.data,
                                    _stream_ptr(self.torch, stream)), self.ctx.h)
        return J, K

    def energy(self, P, hf_coeff: float, *, hf_coeff_lr: float = 0.0, want_grad: bool = True,
               stream=None):
        """(E, dE/dP) of DFCoulomb.energy for the spin-stacked density P;
        ``hf_coeff_lr`` adds the long-range exchange (plans made with omega)."""
        t = self.torch
        P = self._dev(P)
        if P.ndim == 2:
            P = P[None]
        nspin = P.shape[0]
        F = t.empty_like(P) if want_grad else None
        e = ctypes.c_double()
        check(self.lib.dfjk_energy_rsh(self.h, P.data_ptr(), nspin, float(hf_coeff),
                                       float(hf_coeff_lr), byref(e),
                                       None if F is None else F.data_ptr(),
                                       _stream_ptr(t, stream)), self.ctx.h)
        return e.value, F

    def energy_grad(self, P, hf_coeff: float, atom_xyz=None, *, stream=None):
        """Energy and nuclear gradient of the DF energy at the fixed symmetric
        density P (``dfjk_energy_grad``). With ``atom_xyz`` (natom, 3) the
        gradient is summed per atom, (E, (natom, 3)); otherwise per shell,
        (E, (norb_shell, 3), (naux_shell, 3))."""
        t = self.torch
        P = self._dev(P)
        if P.ndim == 2:
            P = P[None]
        go = t.empty((len(self.orb_centers), 3), dtype=t.float64, device=self.dev)
        ga = t.empty((len(self.aux_centers), 3), dtype=t.float64, device=self.dev)
        e = ctypes.c_double()
        check(self.lib.dfjk_energy_grad(self.h, P.data_ptr(), P.shape[0], float(hf_coeff),
                                        byref(e), go.data_ptr(), ga.data_ptr(),
                                        _stream_ptr(t, stream)), self.ctx.h)
        go, ga = go.cpu().numpy(), ga.cpu().numpy()
        if atom_xyz is None:
            return e.value, go, ga
        return e.value, (shells_to_atoms(go, self.orb_centers, atom_xyz)
                         + shells_to_atoms(ga, self.aux_centers, atom_xyz))

    # -- parity entry points --------------------------------------------
    def eri3c_dense(self):
        t = self.torch
        i = self.info()
        out = t.empty((i["nao"], i["nao"], i["naux"]), dtype=t.float64, device=self.dev)
        check(self.lib.dfjk_eri3c_dense(self.h, out.data_ptr(), _stream_ptr(t)), self.ctx.h)
        return out

    def eri2c_dense(self):
        t = self.torch
        n = self.naux
        out = t.empty((n, n), dtype=t.float64, device=self.dev)
        check(self.lib.dfjk_eri2c_dense(self.h, out.data_ptr(), _stream_ptr(t)), self.ctx.h)
        return out

    def metric_pinv(self):
        t = self.torch
        n = self.naux
        out = t.empty((n, n), dtype=t.float64, device=self.dev)
        check(self.lib.dfjk_metric_pinv(self.h, out.data_ptr(), _stream_ptr(t)), self.ctx.h)
        return out

    def kept_pairs(self) -> set[tuple[int, int]]:
        n = self.info()["npair_shell"]
        out = np.empty((max(n, 1), 2), dtype=np.int32)
        check(self.lib.dfjk_kept_pairs(self.h, out.ctypes.data), self.ctx.h)
        return {(int(a), int(b)) for a, b in out[:n]}


# ---------------------------------------------------------------------------
# dftax-style spec and Coulomb term
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class DFSpec:
    """Density-fitting spec (``dftax/ks/terms.py:63-76``) with the B200 backend.

    ``chunk=None`` or ``"auto"``: B is built once and held in device memory
    (dftax's materialized ``DFCoulomb``). An integer ``chunk`` selects the
    streamed form (``StreamedDFCoulomb``, ``terms.py:716-761``): B is not
    stored and every J/K evaluation rebuilds it chunk by chunk of bra pairs
    (the chunk size is the library's own: the value only selects the form).
    """

    auxbasis: object = None
    chunk: int | str | None = None
    screen: float | None = None
    spherical: bool | None = None
    backend: str = "b200"
    precision: str = "fp64"


def df(auxbasis=None, *, chunk=None, screen=None, spherical=None, backend="b200",
       precision="fp64") -> DFSpec:
    """``dftax.df`` (``terms.py:96-148``) plus ``backend``/``precision``."""
    if backend != "b200":
        raise ValueError("this package provides only backend='b200'")
    if chunk not in (None, "auto") and not (isinstance(chunk, int) and chunk > 0):
        raise ValueError("chunk must be None, 'auto' or a positive int (streamed)")
    if spherical is False:
        raise ValueError("the b200 backend fits in the spherical auxiliary span")
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    return DFSpec(auxbasis=auxbasis, chunk=chunk if isinstance(chunk, int) else None,
                  screen=screen, spherical=spherical, backend=backend, precision=precision)


class CoulombTerm(abc.ABC):
    """``E_J + a_x E_x`` of a spin-stacked density (``terms.py:512-527``)."""

    @abc.abstractmethod
    def energy(self, P, S, nocc) -> float:
        raise NotImplementedError


class B200DFCoulomb(CoulombTerm):
    """Materialized RI-J (+ RI-K for hybrids) on the B200 library.

    Same energy as ``DFCoulomb.energy`` (``terms.py:592-613``):
    ``E = 1/2 gamma^T V+ gamma - 1/4 a_x Tr(P K(P))`` for one channel,
    ``- 1/2 a_x sum_s Tr(P_s K(P_s))`` for two; ``fock`` adds its P-gradient.
    Range-separated hybrids (``hf_coeff_lr`` with ``omega``) add the same
    exchange quadratic of the erf(omega r)/r fit (``terms.py:604-612``).
    """

    def __init__(self, basis: BasisData, aux_basis: BasisData, hf_coeff: float, *,
                 hf_coeff_lr: float = 0.0, omega: float = 0.0, screen: float | None = None,
                 precision: str = "fp64", streamed: bool = False, device: int = 0):
        if hf_coeff_lr != 0.0 and omega <= 0.0:
            raise ValueError("hf_coeff_lr needs omega > 0 (terms.py:953-978)")
        self.hf_coeff = float(hf_coeff)
        self.hf_coeff_lr = float(hf_coeff_lr)
        self.plan = Plan(basis, aux_basis, screen=screen, precision=precision,
                         omega=omega if hf_coeff_lr != 0.0 else 0.0, streamed=streamed,
                         device=device)
        self.plan.build()

    def energy(self, P, S=None, nocc=None) -> float:
        e, _ = self.plan.energy(P, self.hf_coeff, hf_coeff_lr=self.hf_coeff_lr, want_grad=False)
        return e

    def fock(self, P, S=None, nocc=None):
        """(E, dE/dP) with dE/dP on the device, shaped like P."""
        return self.plan.energy(P, self.hf_coeff, hf_coeff_lr=self.hf_coeff_lr, want_grad=True)

    def jk(self, C, w=None):
        return self.plan.jk(C, w)

    def geometry_gradient(self, P, atom_xyz):
        """dE/dR (natom, 3) of this term at the fixed density P: the part of
        dftax's forces() that flows through the DF integral build
        (``forces.py:245-270``). Long-range exchange is not included."""
        if self.hf_coeff_lr != 0.0:
            raise NotImplementedError("geometry gradient of the long-range exchange")
        return self.plan.energy_grad(P, self.hf_coeff, atom_xyz)[1]


def make_coulomb(spec: DFSpec, basis: BasisData, hf_coeff: float, *, hf_coeff_lr: float = 0.0,
                 omega: float = 0.0, device: int = 0):
    """``_make_coulomb`` (``terms.py:951-988``) for a resolved b200 spec."""
    if not isinstance(spec, DFSpec):
        raise TypeError("make_coulomb expects a DFSpec from dftax_b200.df()")
    if not isinstance(spec.auxbasis, BasisData):
        raise TypeError("spec.auxbasis must be a built BasisData")
    return B200DFCoulomb(basis, spec.auxbasis, hf_coeff, hf_coeff_lr=hf_coeff_lr, omega=omega,
                         screen=spec.screen, precision=spec.precision,
                         streamed=spec.chunk is not None, device=device)


__all__ = ["Context", "Plan", "DFSpec", "df", "CoulombTerm", "B200DFCoulomb", "make_coulomb"]
