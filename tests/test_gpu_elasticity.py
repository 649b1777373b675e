"""The vector (linear elasticity, 3 x 3 nodal blocks) form of the FP64 GPU
path against the oracle, through the C-ABI, bitwise: assembly of every level
with the Lame field lambda = mu = E per cell and a constant body force, the
level operators (block matvec, block Jacobi, componentwise transfers, the
dense coarse solve of more than 1024 unknowns), and CG preconditioned by the
block-Jacobi V(2,2) cycle on the clamped cube of 3 x 2^l cells per
direction."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORCE = [0.0, 0.0, -1.0]


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


def make_pair(O, G, ctx, order, level, base, n0, seed=0, dmask=0b000001, const=False):
    o = O.Oracle(3, order, level, base_level=base, ncomp=3, n0=n0, dirichlet_mask=dmask)
    g = G.Grid(ctx, 3, order, level, base_level=base, n0=n0, ncomp=3, dirichlet_mask=dmask)
    ncell = (n0 << level) ** 3
    if not const:
        e = np.exp(0.5 * np.random.default_rng(seed).standard_normal(ncell))
        o.set_coefficient(O.LAMBDA_MU_CELL, e)
        g.set_coefficient(G._capi.FMG_LAMBDA_MU_CELL, e)
    o.set_coefficient(O.F_VEC, FORCE)
    g.set_coefficient(G._capi.FMG_F_VEC, FORCE)
    o.assemble()
    g.assemble()
    return o, g


CASES = [(2, 1, 0, 3, False), (1, 2, 0, 2, False), (2, 1, 0, 3, True), (2, 2, 1, 1, False)]


@pytest.mark.parametrize("order,level,base,n0,const", CASES)
def test_assembly(oracle_mod, G, ctx, order, level, base, n0, const):
    o, g = make_pair(oracle_mod, G, ctx, order, level, base, n0, const=const)
    for l in range(base, level + 1):
        assert_same(g.matrix(l), o.matrix(l), f"A level {l}")
    assert_same(g.rhs(), o.rhs(), "rhs")
    assert np.abs(g.rhs()).max() > 0


def test_level_operators(oracle_mod, G, ctx):
    o, g = make_pair(oracle_mod, G, ctx, 2, 1, 0, 3, seed=3)
    rng = np.random.default_rng(5)
    for l in (0, 1):
        n = 3 * g.nnodes(l)
        x, b = rng.standard_normal(n), rng.standard_normal(n)
        X, B, Y = g.vector(l, x), g.vector(l, b), g.vector(l)
        g.matvec(X, Y)
        assert_same(Y.get(), o.matvec(x, l), f"matvec l={l}")
        g.residual(X, B, Y)
        assert_same(Y.get(), o.residual(x, b, l), f"residual l={l}")
        if l > 0:
            R = g.vector(l, b)
            g.jacobi(X, R, 0.5)
            xo, ro = o.jacobi(x, b, 0.5, l)
            assert_same(X.get(), xo, "block jacobi x")
            assert_same(R.get(), ro, "block jacobi r")
            rc = g.vector(l - 1)
            g.restrict(g.vector(l, x), rc)
            assert_same(rc.get(), o.restrict(x, l), "restrict")
            xc = rng.standard_normal(3 * g.nnodes(l - 1))
            XF = g.vector(l, b)
            g.prolongate(g.vector(l - 1, xc), XF)
            assert_same(XF.get(), o.prolongate(xc, b, l - 1), "prolongate")
    nb = 3 * g.nnodes(0)
    assert nb > 1024  # the dense coarse solve beyond one thread per unknown
    x, r = rng.standard_normal(nb), rng.standard_normal(nb)
    X, R = g.vector(0, x), g.vector(0, r)
    g.coarse_solve(X, R, 1.0)
    xo, ro = o.coarse_solve(x, r, 1.0)
    assert_same(R.get(), ro, "coarse r")
    assert_same(X.get(), xo, "coarse x")


@pytest.mark.parametrize("method,pre,post", [(1, 2, 2), (0, 2, 2), (1, 1, 1)])
def test_solve_history(oracle_mod, G, ctx, method, pre, post):
    O = oracle_mod
    o, g = make_pair(O, G, ctx, 2, 1, 0, 3, seed=4)
    oc = O.solve_cfg(method=method, smoother=O.JACOBI, damp=0.5, pre=pre, post=post, compat=False,
                     rtol=1e-10, maxsteps=300)
    gc = G.SolveCfg(method, G._capi.FMG_JACOBI, 0.5, pre, post, 1, 0, 1.0, 1e-10, 0.0, 300,
                    G._capi.FMG_MULTIPLICATIVE)
    ro = o.solve(oc)
    X = g.vector()
    hist, steps, status = g.solve(gc, X)
    assert status == 0 and steps == ro.steps and status == ro.status
    assert_same(hist, ro.history, "defnorm history")
    assert_same(X.get(), ro.x, "solution")


def test_unsupported_forms_fail_loudly(G, ctx):
    g = G.Grid(ctx, 3, 2, 1, base_level=0, n0=3, ncomp=3, dirichlet_mask=1)
    g.set_coefficient(G._capi.FMG_F_VEC, FORCE)
    g.assemble()
    sor = G.SolveCfg(0, G._capi.FMG_SOR, 1.2, 2, 2, 1, 0, 1.0, 1e-10, 0.0, 10, 0)
    with pytest.raises(G.FmgError):
        g.solve(sor, g.vector())
    mg = G.SolveCfg(0, G._capi.FMG_JACOBI, 0.5, 2, 2, 1, 0, 1.0, 1e-10, 0.0, 10, 0)
    with pytest.raises(G.FmgError):
        g.solve_mixed(mg, g.vector())  # the mixed form is CG + cycle
    with pytest.raises(G.FmgError):
        G.Grid(ctx, 2, 2, 1, ncomp=3)


@pytest.mark.parametrize("order,level,n0", [(2, 1, 3), (2, 2, 3), (1, 2, 3)])
def test_mixed_solve_matches_fp64(oracle_mod, G, ctx, order, level, n0):
    # FP32 block-Jacobi V(2,2) cycle inside FP64 flexible CG: the same discrete
    # solution as the FP64 path, in about as many CG steps
    _, g = make_pair(oracle_mod, G, ctx, order, level, 0, n0, seed=6)
    cfg = G.SolveCfg(1, G._capi.FMG_JACOBI, 0.6, 2, 2, 1, 0, 1.0, 1e-10, 0.0, 300, G._capi.FMG_MULTIPLICATIVE)
    X = g.vector()
    hist, steps, status = g.solve(cfg, X)
    assert status == 0
    XM = g.vector()
    mh, nouter, ninner, mst = g.solve_mixed(cfg, XM)
    assert mst == 0 and mh[-1] / mh[0] < 1e-10, (mh[-3:], nouter, ninner)
    assert ninner <= steps + 3, (steps, ninner)
    a, b = XM.get(), X.get()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8
    # the true residual of the mixed solution
    B, R = g.vector(values=g.rhs()), g.vector()
    g.residual(XM, B, R)
    assert np.linalg.norm(R.get()) / np.linalg.norm(g.rhs()) < 1e-9
