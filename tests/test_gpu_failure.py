"""Failure detection on the device without faulting the GPU: the bounded
mbarrier wait the tensor-core kernels use (2^24 polls or 2 s) is run alone
with a short limit on a barrier nothing arrives on.  The kernel must give
up, record its error word and return; the call must report FMG_ERR_CUDA with
the timed-out message, and the context must stay usable.  With an arrival the
same wait completes.  No MMA or bulk copy is in flight in the kernel."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_reports():
    import gnu_femlisp_b200 as G
    ctx = G.Context(0)
    lib = G._capi.load()
    assert lib.fmg_wait_selftest(ctx.h, 1, 4096, 1000000) == 0          # an arrival: the wait completes
    t0 = time.perf_counter()
    rc = lib.fmg_wait_selftest(ctx.h, 0, 1 << 20, 1000000)               # nothing arrives: 1 ms limit
    dt = time.perf_counter() - t0
    assert rc == -2 and dt < 5.0, (rc, dt)
    with pytest.raises(G.FmgError, match="FMG_ERR_CUDA.*timed out"):
        ctx.check(rc, "fmg_wait_selftest")
    # the poll limit alone also ends the wait
    assert lib.fmg_wait_selftest(ctx.h, 0, 256, 2000000000) == -2
    # the context is still usable: a small solve after the give-up
    g = G.Grid(ctx, 2, 1, 4, base_level=0).assemble()
    x = g.vector()
    C = G._capi
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 50, C.FMG_MULTIPLICATIVE)
    hist, steps, st = g.solve(cfg, x)
    assert st == 0 and np.isfinite(hist).all()
    assert lib.fmg_wait_selftest(ctx.h, 1, 4096, 1000000) == 0


def test_bounded_wait_rejects_out_of_range_limits():
    import gnu_femlisp_b200 as G
    ctx = G.Context(0)
    lib = G._capi.load()
    assert lib.fmg_wait_selftest(ctx.h, 0, 0, 1000) == -1
    assert lib.fmg_wait_selftest(ctx.h, 0, 100, 3000000000) == -1
