"""Batches (fmg_batch_create / _load / _solve): B independent 2D Q1 problems
solved in the same launches give, problem by problem, exactly what fmg_solve
gives on the problem's own grid -- the defnorm history, the step count, the
status and the iterate, bit for bit -- for CG + MG, the MG iteration and
plain CG (solve.lisp:139-164, krylow.lisp:72-132, multigrid.lisp:254-288),
with scalar and per-node damping, and with problems that stop at different
steps (a problem that has stopped keeps its iterate while the others go on)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gnu_femlisp_b200 as G
    return G


@pytest.fixture(scope="module")
def ctx(G):
    return G.Context(0)


def _cfg(G, method, maxsteps=200):
    C = G._capi
    return G.SolveCfg(method, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, maxsteps, C.FMG_MULTIPLICATIVE)


def _fields(level, nprob, seed0, lo=-3.0, hi=3.0):
    from gnu_femlisp_b200 import learn
    n = 2 ** level
    return [learn.block_field(seed0 + k, n=n, blocks=8 if n >= 8 else n, lo=lo, hi=hi) for k in range(nprob)]


def _damping(rng, g, level):
    return rng.uniform(0.45, 0.75, g.nnodes(level))


@pytest.mark.parametrize("method", ["cg_mg", "mg", "cg"])
@pytest.mark.parametrize("damped", [False, True])
def test_batch_equals_single_solves(G, ctx, method, damped):
    C = G._capi
    meth = {"cg_mg": C.FMG_METHOD_CG_MG, "mg": C.FMG_METHOD_MG, "cg": C.FMG_METHOD_CG}[method]
    level, base, nprob = 6, 2, 5
    cfg = _cfg(G, meth, maxsteps=400 if method != "cg_mg" else 200)
    fields = _fields(level, nprob, 4242, lo=-1.0, hi=1.0)  # contrast the MG iteration converges on
    rng = np.random.default_rng(7)
    g = G.Grid(ctx, 2, 1, level, base_level=base)
    x = g.vector()
    batch = G.Grid.batch(g, nprob)
    single = []
    for k, kc in enumerate(fields):
        g.set_coefficient(C.FMG_K_CELL, kc)
        g.assemble()
        for lev in range(base + 1, level + 1):
            g.set_node_damping(lev, _damping(rng, g, lev) if damped else None)
        x.fill(0.0)
        hist, steps, st = g.solve(cfg, x)
        single.append((hist, steps, st, x.get()))
        batch.batch_load(k, g)
    xb = batch.vector()
    hb, sb, stb = batch.batch_solve(cfg, xb)
    xs = xb.get().reshape(nprob, -1)
    assert len(set(int(s) for s in sb)) > 1 or method == "cg", "problems should stop at different steps"
    for k, (hist, steps, st, xk) in enumerate(single):
        assert sb[k] == steps and stb[k] == st, (k, sb[k], steps, stb[k], st)
        assert np.array_equal(hb[k, : steps + 1], hist), k
        assert np.array_equal(xs[k], xk), (k, np.max(np.abs(xs[k] - xk)))
    xb.close()
    batch.close()
    x.close()
    g.close()


def test_batch_of_c4_size_fields_with_the_network(G, ctx):
    """The learned smoother's configuration (128^2 cells, 8 x 8 blocks): the
    damping network on every level of each problem's own grid, then the batch
    against each problem's fmg_solve."""
    import os
    from gnu_femlisp_b200 import learn
    C = G._capi
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    net = learn.DampingNet.load(ctx, os.path.join(root, "gnu_femlisp_b200", "weights", "damping2d.fmgnet"))
    level, base, nprob = 7, 2, 4
    cfg = _cfg(G, C.FMG_METHOD_CG_MG)
    g = G.Grid(ctx, 2, 1, level, base_level=base)
    x = g.vector()
    batch = G.Grid.batch(g, nprob)
    single = []
    for k, kc in enumerate(_fields(level, nprob, 1000000)):
        g.set_coefficient(C.FMG_K_CELL, kc)
        g.assemble()
        net.apply(g)
        x.fill(0.0)
        single.append(g.solve(cfg, x) + (x.get(),))
        batch.batch_load(k, g)
    xb = batch.vector()
    hb, sb, stb = batch.batch_solve(cfg, xb)
    xs = xb.get().reshape(nprob, -1)
    for k, (hist, steps, st, xk) in enumerate(single):
        assert sb[k] == steps and stb[k] == st == 0
        assert np.array_equal(hb[k, : steps + 1], hist)
        assert np.array_equal(xs[k], xk)
    net.close()


def test_batch_refusals(G, ctx):
    C = G._capi
    g = G.Grid(ctx, 2, 1, 4, base_level=1)
    g.assemble()
    batch = G.Grid.batch(g, 3)
    x = batch.vector()
    with pytest.raises(G._capi.FmgError):  # not every problem loaded
        batch.batch_solve(_cfg(G, C.FMG_METHOD_CG_MG), x)
    for k in range(3):
        batch.batch_load(k, g)
    with pytest.raises(G._capi.FmgError):  # single-problem entry points refuse a batch
        batch.solve(_cfg(G, C.FMG_METHOD_CG_MG), x)
    other = G.Grid(ctx, 2, 1, 5, base_level=1)
    other.assemble()
    with pytest.raises(G._capi.FmgError):  # another geometry
        batch.batch_load(0, other)
    g3 = G.Grid(ctx, 3, 1, 3, base_level=1)
    with pytest.raises(G._capi.FmgError):  # 3D grids are not batched
        G.Grid.batch(g3, 2)
