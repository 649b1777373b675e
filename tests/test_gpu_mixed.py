"""Mixed-precision solve (FP64 flexible CG preconditioned by the FP32/BF16
V-cycle): it must reach the FP64 residual tolerance in the true residual of
the assembled FP64 matrix, and its solution must agree with the FP64 path's."""
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


def _cfg(G, rtol, maxsteps=400, damp=0.6, pre=1, post=1):
    C = G._capi
    return G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, damp, pre, post, 1, 0, 1.0, rtol, 0.0, maxsteps,
                      C.FMG_MULTIPLICATIVE)


def _grid(G, ctx, dim, level, base, seed=0, field="fourier"):
    from gnu_femlisp_b200 import problems
    g = G.Grid(ctx, dim, 1, level, base_level=base)
    n = 1 << level
    if field == "fourier":
        k = np.exp(problems.fourier_log_field(n, dim, seed))
    else:
        k = np.ones(n ** dim)
    g.set_coefficient(G._capi.FMG_K_CELL, k)
    return g.assemble()


@pytest.mark.parametrize("matrix_free", [True, False])
def test_mixed_reaches_tolerance_and_matches_fp64(G, ctx, matrix_free):
    g = _grid(G, ctx, 3, 5, 2, seed=3)
    x64 = g.vector()
    h64, s64, st64 = g.solve(_cfg(G, 1e-13), x64)
    assert st64 == 0
    xm = g.vector()
    hist, nouter, ninner, st = g.solve_mixed(_cfg(G, 1e-10), xm, inner_rtol=1e-5, matrix_free=matrix_free)
    assert st == 0, (hist, nouter, ninner)
    assert hist[-1] / hist[0] < 1e-10          # true FP64 residual reduction
    a, b = xm.get(), x64.get()
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel <= 1e-10, rel                     # the north star's bound on the mixed result
    assert 1 <= nouter <= 3
    assert ninner <= 30


@pytest.mark.parametrize("dmask", [21, 42, 7, 56, 45])
def test_mixed_matrix_free_boundary_masks(G, ctx, dmask):
    # Dirichlet on some faces only: the padded layout's front, the face CTAs
    # and the transfers at Neumann faces; the matrix-free solve takes the
    # stored solve's steps and reaches the FP64 solution
    from gnu_femlisp_b200 import problems
    g = G.Grid(ctx, 3, 1, 5, base_level=2, dirichlet_mask=dmask)
    g.set_coefficient(G._capi.FMG_K_CELL, np.exp(problems.fourier_log_field(32, 3, 5)))
    g.assemble()
    x64 = g.vector()
    _, _, st64 = g.solve(_cfg(G, 1e-13), x64)
    assert st64 == 0
    steps = {}
    for mf in (True, False):
        xm = g.vector()
        hist, nouter, ninner, st = g.solve_mixed(_cfg(G, 1e-10), xm, matrix_free=mf)
        assert st == 0 and hist[-1] / hist[0] < 1e-10, (mf, hist)
        rel = np.linalg.norm(xm.get() - x64.get()) / np.linalg.norm(x64.get())
        assert rel <= 1e-10, (mf, rel)
        steps[mf] = ninner
    assert abs(steps[True] - steps[False]) <= 1, steps


def test_mixed_tight_tolerance_error_vs_fp64(G, ctx):
    # both driven to 1e-13: the mixed result agrees with FP64 to 1e-10
    g = _grid(G, ctx, 3, 6, 2, seed=1)
    x64, xm = g.vector(), g.vector()
    g.solve(_cfg(G, 1e-13), x64)
    hist, nouter, ninner, st = g.solve_mixed(_cfg(G, 1e-13), xm)
    assert st == 0
    rel = np.linalg.norm(xm.get() - x64.get()) / np.linalg.norm(x64.get())
    assert rel <= 1e-10, rel


def test_mixed_2d_stored_levels(G, ctx):
    g = _grid(G, ctx, 2, 7, 1, seed=2)
    x64, xm = g.vector(), g.vector()
    g.solve(_cfg(G, 1e-12), x64)
    hist, nouter, ninner, st = g.solve_mixed(_cfg(G, 1e-10), xm)
    assert st == 0 and hist[-1] / hist[0] < 1e-10
    rel = np.linalg.norm(xm.get() - x64.get()) / np.linalg.norm(x64.get())
    assert rel < 1e-8


def test_mixed_rejects_unsupported_cycle(G, ctx):
    g = _grid(G, ctx, 2, 4, 1, field="const")
    C = G._capi
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_SOR, 1.0, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 50, C.FMG_MULTIPLICATIVE)
    with pytest.raises(G.FmgError, match="UNSUPPORTED"):
        g.solve_mixed(cfg, g.vector())


def test_handles_released_in_any_order(G):
    # a context closed before its grid and vectors stays valid for them
    ctx2 = G.Context(0)
    g = G.Grid(ctx2, 2, 1, 4, 1).assemble()
    v = g.vector(values=np.ones(g.nnodes()))
    ctx2.close()
    assert abs(v.dot(v) - g.nnodes()) < 1e-9
    g.close()
    assert v.l2_norm() > 0
    v.close()
