"""fmg_dot_noalloc: the dot product for callers that cannot allocate device
memory (their device memory belongs to their own pool allocator, or they run
a latency-critical loop that must not take the device synchronisation of
cudaMalloc/cudaFree).  It must give the result of fmg_dot, call after call,
with the caller's own device buffers and the library's fixed scratch, take no
device memory while it runs, and leave the caller's current device as it was.

Kept in a file of its own that pytest collects last, so that a run stopping at
its first failure has run every other test before this one.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12


def _noalloc(lib, ctx, xd, yd, n, outd):
    return lib.fmg_dot_noalloc(ctx.h, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()), n,
                               ctypes.c_void_p(outd.data_ptr()))


def test_dot_noalloc_matches_dot_on_consecutive_calls():
    import torch

    import gnu_femlisp_b200 as G
    ctx = G.Context(0)
    lib = G._capi.load()
    g = G.Grid(ctx, 2, 1, 9, 0).assemble()          # 513^2 = 263,169 nodes
    n = g.nnodes()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    dev0 = torch.cuda.current_device()
    for call in range(2):
        rng = np.random.default_rng(100 + call)
        x, y = rng.standard_normal(n), rng.standard_normal(n)
        ref = g.vector(values=x).dot(g.vector(values=y))            # fmg_dot
        xd = torch.from_numpy(x).to("cuda")
        yd = torch.from_numpy(y).to("cuda")
        torch.cuda.synchronize()
        ctx.check(_noalloc(lib, ctx, xd, yd, n, out), "fmg_dot_noalloc")
        ctx.synchronize()
        got = float(out.item())
        assert abs(got - ref) <= REL * abs(ref), (call, got, ref)
        assert got == ref, (call, got, ref)        # same reduction order: bitwise
        assert torch.cuda.current_device() == dev0


def test_dot_noalloc_takes_no_device_memory_and_runs_on_any_context_stream():
    import torch

    import gnu_femlisp_b200 as G
    lib = G._capi.load()
    ctx_a, ctx_b = G.Context(0), G.Context(0)      # each context has its own (non-default) stream
    g = G.Grid(ctx_a, 3, 1, 6, 0).assemble()        # 65^3 = 274,625 nodes
    n = g.nnodes()
    rng = np.random.default_rng(7)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    ref = g.vector(values=x).dot(g.vector(values=y))
    xd = torch.from_numpy(x).to("cuda")
    yd = torch.from_numpy(y).to("cuda")
    outs = torch.zeros(8, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    # the first call on the device (in a fresh process this is the first call
    # at all) looks up the fixed array; the CUDA runtime may load the module
    # holding it at that point, which is the array's own storage
    ctx_a.check(_noalloc(lib, ctx_a, xd, yd, n, outs[0:1]), "fmg_dot_noalloc")
    ctx_a.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(1, 8):
        c = ctx_a if k % 2 else ctx_b
        c.check(_noalloc(lib, c, xd, yd, n, outs[k:k + 1]), "fmg_dot_noalloc")
        c.synchronize()                            # calls on the two streams must not overlap
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    got = outs.cpu().numpy()
    assert np.all(got == ref), (got, ref)


def test_dot_noalloc_rejects_oversized_input():
    import torch

    import gnu_femlisp_b200 as G
    ctx = G.Context(0)
    lib = G._capi.load()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = lib.fmg_dot_noalloc(ctx.h, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()),
                             134217728 + 1, ctypes.c_void_p(buf.data_ptr()))
    assert rc == -1
    with pytest.raises(G.FmgError, match="FMG_NOALLOC_MAX_N"):
        ctx.check(rc, "fmg_dot_noalloc")
