"""ctypes bindings of the C ABI declared in ``include/dfjk.h``, ``include/dfscf.h`` and
``include/dfbatch.h``.

The library ``libdfjk.so`` is built in-tree by ``dftax_b200.build``. There is
no fallback: if the library is missing or fails to load, every entry point
raises :class:`LibraryNotLoaded`.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, byref, c_char_p, c_double, c_int, c_int32, c_int64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdfjk.so")

DFJK_OK = 0
(DFJK_ERR_INVALID, DFJK_ERR_UNSUPPORTED, DFJK_ERR_CUDA, DFJK_ERR_MEMORY, DFJK_ERR_NUMERIC,
 DFJK_ERR_STATE) = range(1, 7)
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "UNSUPPORTED", 3: "CUDA", 4: "MEMORY", 5: "NUMERIC",
                6: "STATE"}
DFJK_FP64 = 0
DFJK_MIXED = 1

# every symbol include/dfjk.h declares
EXPORTS = (
    "dfjk_default_options", "dfjk_create", "dfjk_destroy", "dfjk_last_error",
    "dfjk_plan_create", "dfjk_plan_destroy", "dfjk_plan_get_info", "dfjk_build", "dfjk_jk",
    "dfjk_jk_host", "dfjk_energy", "dfjk_eri3c_dense", "dfjk_eri2c_dense", "dfjk_metric_pinv",
    "dfjk_kept_pairs", "dfjk_boys", "dfjk_phase_times", "dfjk_kernel_launches",
    "dfjk_wait_selftest", "dfjk_energy_grad", "dfjk_build_batch",
    "dfjk_j_noalloc", "dfjk_trim", "dfjk_plan_long_range", "dfjk_energy_rsh",
    # include/dfscf.h
    "dfscf_default_options", "dfscf_create", "dfscf_destroy", "dfscf_run", "dfscf_get_result",
    "dfscf_get_density", "dfscf_get_orbitals", "dfscf_one_electron", "dfscf_xc",
    "dfscf_energy_fock", "dfjk_becke_partition",
    # include/dfbatch.h
    "dfbatch_default_options", "dfbatch_create", "dfbatch_destroy", "dfbatch_submit",
    "dfbatch_wait", "dfbatch_poll", "dfbatch_estimate",
)
PHASES = ("metric", "pairs", "eri3c", "bgemm", "j", "khalf", "ksyrk", "kplanes")


class LibraryNotLoaded(RuntimeError):
    pass


class DfjkError(RuntimeError):
    """A non-OK dfjk_status, with the library's last error message."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"dfjk {self.status_name}: {message}")


class Basis(ctypes.Structure):
    _fields_ = [("ncart", c_int64), ("max_prim", c_int32), ("nsph", c_int32),
                ("centers", c_void_p), ("exponents", c_void_p), ("coefficients", c_void_p),
                ("angular", c_void_p), ("cart2sph", c_void_p)]


class Options(ctypes.Structure):
    _fields_ = [("screen", c_double), ("metric_cutoff", c_double), ("precision", c_int32),
                ("streamed", c_int32), ("chunk_bytes", c_int64), ("omega", c_double)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("nao", c_int64), ("naux", c_int64), ("nao_cart", c_int64),
                ("naux_cart", c_int64), ("nshell", c_int64), ("naux_shell", c_int64),
                ("npair_shell", c_int64), ("nrows", c_int64), ("nfit", c_int64),
                ("b_bytes", c_int64), ("built", c_int32), ("precision", c_int32)]


class ScfOptions(ctypes.Structure):
    _fields_ = [("hf_coeff", c_double), ("x_scale", c_double), ("c_scale", c_double),
                ("e_tol", c_double), ("d_tol", c_double), ("lindep", c_double),
                ("level_shift", c_double), ("rho_thresh", c_double), ("ao_thresh", c_double),
                ("max_iter", c_int32),
                ("diis_space", c_int32), ("grid_chunk", c_int64), ("xc_streams", c_int32),
                ("density", c_int32)]


class ScfResult(ctypes.Structure):
    _fields_ = [("e_tot", c_double), ("e_one", c_double), ("e_coul", c_double),
                ("e_xc", c_double), ("e_nn", c_double), ("derr", c_double),
                ("n_iter", c_int32), ("converged", c_int32), ("nmo", c_int32),
                ("nocc", c_int32), ("ms_jk", c_double), ("ms_xc", c_double),
                ("ms_diag", c_double), ("ms_diis", c_double), ("xc_chunk", c_int64),
                ("xc_graph", c_int32), ("n_eig", c_int32),
                ("xc_gemm_flop", c_double)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("workers", c_int32), ("reserved", c_int32), ("hbm_budget", c_int64)]


class BatchRequest(ctypes.Structure):
    _fields_ = [("orb", POINTER(Basis)), ("aux", POINTER(Basis)), ("plan_opts", Options),
                ("natom", c_int32), ("nocc", c_int32), ("atom_xyz", c_void_p),
                ("atom_charge", c_void_p), ("npoint", c_int64), ("grid_xyz", c_void_p),
                ("grid_w", c_void_p), ("scf_opts", ScfOptions), ("P_out", c_void_p),
                ("P_guess", c_void_p)]


class BatchResult(ctypes.Structure):
    _fields_ = [("status", c_int32), ("worker", c_int32), ("scf", ScfResult),
                ("t_submit", c_double), ("t_start", c_double), ("t_end", c_double),
                ("bytes", c_int64), ("message", ctypes.c_char * 256)]


_lib = None


def load(path: str | None = None):
    """Load (once) and return the ctypes library with argtypes set."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or os.environ.get("DFJK_LIB", LIB_PATH)
    if not os.path.exists(p):
        raise LibraryNotLoaded(f"{p} not found; build it with `python -m dftax_b200.build`")
    try:
        lib = ctypes.CDLL(p)
    except OSError as e:  # pragma: no cover - depends on the environment
        raise LibraryNotLoaded(f"cannot load {p}: {e}") from e
    V, P = c_void_p, POINTER
    sig = {
        "dfjk_default_options": (None, [P(Options)]),
        "dfjk_create": (c_int, [c_int, P(c_void_p)]),
        "dfjk_destroy": (c_int, [V]),
        "dfjk_last_error": (c_char_p, [V]),
        "dfjk_plan_create": (c_int, [V, P(Basis), P(Basis), P(Options), P(c_void_p)]),
        "dfjk_plan_destroy": (c_int, [V]),
        "dfjk_plan_get_info": (c_int, [V, P(PlanInfo)]),
        "dfjk_build": (c_int, [V, V]),
        "dfjk_jk": (c_int, [V, V, V, c_int64, V, V, V]),
        "dfjk_jk_host": (c_int, [V, V, V, c_int64, V, V, V]),
        "dfjk_energy": (c_int, [V, V, c_int32, c_double, P(c_double), V, V]),
        "dfjk_eri3c_dense": (c_int, [V, V, V]),
        "dfjk_eri2c_dense": (c_int, [V, V, V]),
        "dfjk_metric_pinv": (c_int, [V, V, V]),
        "dfjk_kept_pairs": (c_int, [V, V]),
        "dfjk_boys": (c_int, [V, V, c_int64, c_int32, V, V]),
        "dfjk_wait_selftest": (c_int, [V, c_int64, V, V]),
        "dfjk_energy_grad": (c_int, [V, V, c_int32, c_double, V, V, V, V]),
        "dfjk_build_batch": (c_int, [V, c_int32, V]),
        "dfjk_phase_times": (c_int, [V, P(c_double), c_int32]),
        "dfjk_kernel_launches": (c_int64, []),
        "dfjk_j_noalloc": (c_int, [V, V, V, c_int64, V, V]),
        "dfjk_trim": (c_int, [V]),
        "dfjk_plan_long_range": (c_int, [V, P(c_void_p)]),
        "dfjk_energy_rsh": (c_int, [V, V, c_int32, c_double, c_double, P(c_double), V, V]),
        "dfscf_default_options": (None, [P(ScfOptions)]),
        "dfscf_create": (c_int, [V, c_int32, V, V, c_int64, V, V, c_int32, P(ScfOptions),
                                 P(c_void_p), V]),
        "dfscf_destroy": (c_int, [V]),
        "dfscf_run": (c_int, [V, V, P(ScfOptions), V]),
        "dfscf_get_result": (c_int, [V, P(ScfResult)]),
        "dfscf_get_density": (c_int, [V, V, V]),
        "dfscf_get_orbitals": (c_int, [V, V, V, V]),
        "dfscf_one_electron": (c_int, [V, V, V, V, V]),
        "dfscf_xc": (c_int, [V, V, P(c_double), V, V]),
        "dfscf_energy_fock": (c_int, [V, V, P(c_double), V, V]),
        "dfjk_becke_partition": (c_int, [V, V, V, V, c_int64, c_int32, V, V, V, V]),
        "dfbatch_default_options": (None, [P(BatchOptions)]),
        "dfbatch_create": (c_int, [c_int, P(BatchOptions), P(c_void_p)]),
        "dfbatch_destroy": (c_int, [V]),
        "dfbatch_submit": (c_int, [V, P(BatchRequest), P(c_int64)]),
        "dfbatch_wait": (c_int, [V, c_int64, P(BatchResult)]),
        "dfbatch_poll": (c_int, [V, c_int64, P(c_int32)]),
        "dfbatch_estimate": (c_int, [P(BatchRequest), P(c_int64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status: int, ctx=None):
    if status != DFJK_OK:
        lib = load()
        msg = lib.dfjk_last_error(ctx).decode() if ctx else ""
        raise DfjkError(status, msg)


__all__ = ["load", "check", "Basis", "Options", "PlanInfo", "ScfOptions", "ScfResult",
           "BatchOptions", "BatchRequest", "BatchResult", "DfjkError",
           "LibraryNotLoaded",
           "EXPORTS", "DFJK_FP64", "DFJK_MIXED", "byref", "DFJK_OK", "DFJK_ERR_INVALID",
           "DFJK_ERR_UNSUPPORTED", "DFJK_ERR_CUDA", "DFJK_ERR_MEMORY", "DFJK_ERR_NUMERIC",
           "DFJK_ERR_STATE"]
