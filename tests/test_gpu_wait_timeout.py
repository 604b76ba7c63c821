"""The bounded device wait of the tensor-core pipelines, made to run out.

The int8 tcgen05 GEMMs wait on mbarriers with a %globaltimer limit (4 s): a
wait that runs out flags an error word, the other warps see the flag and stop
waiting, and the host call returns DFJK_ERR_CUDA. ``dfjk_wait_selftest`` runs
that same wait on a barrier that nothing completes, with no copy or MMA in
flight, so the limit is reached without any fault. The test checks the status
and message, that the warp holding the 4 s limit returned as soon as the short
wait was flagged, and that the same context and plan then give the same mixed
(tensor-core) J and K bit for bit as before.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _selftest(ctx, limit_ns):
    import torch

    waited = (ctypes.c_double * 2)()
    st = ctx.lib.dfjk_wait_selftest(ctx.h, int(limit_ns), waited,
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, list(waited)


def test_wait_runs_out_and_the_context_survives():
    import torch

    from dftax_b200 import Plan, _lib, systems

    _, _, orb, aux, nocc = systems.workload("water8", seed=5)
    plan = Plan(orb, aux, precision="mixed").build()
    C = systems.random_occupied(orb.nao, nocc, seed=5)
    J0, K0 = (x.clone() for x in plan.jk(C))

    st, waited = _selftest(plan.ctx, 2_000_000)            # 2 ms
    assert st == _lib.DFJK_ERR_CUDA
    assert "gave up waiting (code 90)" in plan.ctx.last_error()
    assert 2.0 <= waited[0] < 1000.0
    # the warp with the pipelines' 4 s limit stopped on the flag, not its own limit
    assert waited[1] < 1000.0

    J1, K1 = plan.jk(C)
    torch.cuda.synchronize()
    assert torch.equal(J0, J1) and torch.equal(K0, K1)
    assert np.isfinite(J1.cpu().numpy()).all()


def test_wait_limit_is_checked():
    from dftax_b200 import _lib
    from dftax_b200.coulomb import Context

    ctx = Context.get(0)
    for bad in (0, 999, 4_000_000_001):
        st, _ = _selftest(ctx, bad)
        assert st == _lib.DFJK_ERR_INVALID
