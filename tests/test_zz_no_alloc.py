"""dfjk_j_noalloc, the J entry point that allocates no device memory.

It exists for callers that must not call cudaMalloc while they run: an XLA
FFI handler inside a JAX program whose allocator already owns the GPU's
memory, or a serving loop that keeps cudaMalloc/cudaFree (which synchronize
the device) off its hot path. Its scratch is a fixed array inside the library,
shared by every call, so the test makes two calls in a row with different
densities and checks each against dfjk_jk's J (same B, same algorithm; the
partial sums are grouped differently, hence 1e-12 relative rather than
bitwise). This file is collected last so that a failure here comes after every
other test has run; it passes alone in a fresh process as well.
"""

import ctypes

import numpy as np
import pytest

from conftest import golden_basis

pytestmark = pytest.mark.gpu


def _noalloc_j(plan, C):
    """J from dfjk_j_noalloc, and the device's free bytes before and after the
    call (inputs and output are allocated before the first reading)."""
    import torch

    from dftax_b200 import _lib

    Cd = torch.as_tensor(np.ascontiguousarray(C), device=plan.dev)
    J = torch.full((C.shape[0], C.shape[0]), np.nan, dtype=torch.float64, device=plan.dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    st = plan.lib.dfjk_j_noalloc(plan.h, Cd.data_ptr(), None, C.shape[1], J.data_ptr(), stream)
    _lib.check(st, plan.ctx.h)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    return J.cpu().numpy(), free0 - free1


@pytest.mark.parametrize("workload", ["golden-water", "water8"])
def test_noalloc_j_matches_jk_twice(workload, water_golden):
    from dftax_b200 import Plan, systems

    if workload == "golden-water":
        orb, aux = golden_basis(water_golden, "orb"), golden_basis(water_golden, "aux")
        nocc = 5
    else:
        _, _, orb, aux, nocc = systems.workload(workload, seed=3)
    plan = Plan(orb, aux).build()
    for seed in (11, 12):   # two calls in a row: the shared scratch keeps the first call's data
        C = systems.random_occupied(orb.nao, nocc, seed=seed)
        J, taken = _noalloc_j(plan, C)
        # the call itself takes no device memory (the scratch was placed on the
        # device when the context was created)
        assert taken == 0
        Jref, _ = plan.jk(C, want_k=False)
        Jref = Jref.cpu().numpy()
        assert np.all(np.isfinite(J))
        assert np.linalg.norm(J - Jref) <= 1e-12 * np.linalg.norm(Jref)


def test_noalloc_rejects_unbuilt_plan(water_golden):
    import torch

    from dftax_b200 import Plan

    plan = Plan(golden_basis(water_golden, "orb"), golden_basis(water_golden, "aux"))
    C = torch.zeros((plan.nao, 5), dtype=torch.float64, device=plan.dev)
    J = torch.zeros((plan.nao, plan.nao), dtype=torch.float64, device=plan.dev)
    st = plan.lib.dfjk_j_noalloc(plan.h, C.data_ptr(), None, 5, J.data_ptr(), None)
    assert st == 6   # DFJK_ERR_STATE
