"""Galerkin coarse operators on the GPU (multilevel-decomposition with
:galerkin-p t, geomg.lisp:122-123; the product I^T A I of galerkin-product,
amg.lisp:247-285) for the forms beyond scalar Q1: scalar Q2 in its
colour-major sliced storage and 3 x 3 node blocks (Q1 and Q2 elasticity),
with variable coefficients and partial Dirichlet boundaries.  Every level
matrix and a CG solve preconditioned by the Galerkin hierarchy must equal the
oracle's bit for bit."""
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


def assert_same(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.max(np.abs(a)), 1e-300)
    diff = np.max(np.abs(a - b)) if a.size else 0.0
    assert diff <= 1e-12 * scale, f"{what}: max diff {diff:.3e} (scale {scale:.3e})"
    assert np.array_equal(a, b), f"{what}: within 1e-12 but not bitwise (max diff {diff:.3e})"


def _pair(O, G, ctx, dim, order, level, base, nc, n0, dmask, seed):
    kw = dict(ncomp=nc, n0=n0, dirichlet_mask=dmask)
    o = O.Oracle(dim, order, level, base_level=base, **kw)
    g = G.Grid(ctx, dim, order, level, base_level=base, **kw)
    ncell = (n0 << level) ** dim
    k = np.exp(0.5 * np.random.default_rng(seed).standard_normal(ncell))
    if nc == 3:
        o.set_coefficient(O.LAMBDA_MU_CELL, k)
        g.set_coefficient(G._capi.FMG_LAMBDA_MU_CELL, k)
        o.set_coefficient(O.F_VEC, [0.0, 0.0, -1.0])
        g.set_coefficient(G._capi.FMG_F_VEC, [0.0, 0.0, -1.0])
    else:
        o.set_coefficient(O.K_CELL, k)
        g.set_coefficient(1, k)
    o.assemble(galerkin=True)
    g.assemble(galerkin=True)
    return o, g


# dim, order, level, base, components, cells of level 0 per direction, Dirichlet faces
CASES = [
    (1, 2, 5, 0, 1, 1, None),
    (2, 2, 4, 1, 1, 1, None),
    (2, 2, 4, 0, 1, 1, 0b0110),
    (3, 2, 3, 1, 1, 1, None),
    (3, 2, 3, 0, 1, 1, 0b000001),
    (3, 1, 2, 0, 3, 2, 0b000001),
    (3, 2, 1, 0, 3, 2, 0b000001),
    (3, 2, 2, 1, 3, 1, 0b000011),
]


@pytest.mark.parametrize("dim,order,level,base,nc,n0,dmask", CASES)
def test_galerkin_levels_and_solve(oracle_mod, G, ctx, dim, order, level, base, nc, n0, dmask):
    O = oracle_mod
    o, g = _pair(O, G, ctx, dim, order, level, base, nc, n0, dmask, seed=dim * 10 + order + nc)
    for l in range(base, level + 1):
        assert_same(g.matrix(l), o.matrix(l), f"A level {l}")
    damp, pre = (0.6, 2)
    oc = O.solve_cfg(method=O.METHOD_CG_MG, damp=damp, pre=pre, post=pre, compat=False, rtol=1e-10,
                     maxsteps=200)
    gc = G.SolveCfg(O.METHOD_CG_MG, 0, damp, pre, pre, 1, 0, 1.0, 1e-10, 0.0, 200, 0)
    ro = o.solve(oc)
    X = g.vector()
    hist, steps, status = g.solve(gc, X)
    assert status == 0 and ro.status == 0 and steps == ro.steps
    assert_same(hist, ro.history, "defnorm history")
    assert_same(X.get(), ro.x, "solution")


def test_galerkin_q2_sor_cycle(oracle_mod, G, ctx):
    # the colour-major Q2 storage read by the multicolour SOR of the Galerkin levels
    O = oracle_mod
    o, g = _pair(O, G, ctx, 3, 2, 3, 1, 1, 1, None, seed=7)
    oc = O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.SOR, damp=1.2, pre=2, post=2, compat=False,
                     rtol=1e-10, maxsteps=100)
    gc = G.SolveCfg(O.METHOD_CG_MG, 1, 1.2, 2, 2, 1, 0, 1.0, 1e-10, 0.0, 100, 0)
    ro = o.solve(oc)
    X = g.vector()
    hist, steps, status = g.solve(gc, X)
    assert status == 0 and steps == ro.steps
    assert_same(hist, ro.history, "defnorm history")
    assert_same(X.get(), ro.x, "solution")
