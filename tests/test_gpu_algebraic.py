"""Algebraic grids on the GPU (fmg_grid_create_algebraic: matrices and
interpolations handed over as compressed rows, the path for unstructured and
adaptively refined meshes): a structured hierarchy given this way iterates
bit for bit like the structured oracle, an irregular problem bit for bit like
the oracle's algebraic hierarchy, the level operators match, the
multicolour SOR and one-unknown SSC sweeps over the greedy colouring of the
matrix graph match the oracle's, and geometry-bound calls are refused."""
import numpy as np
import pytest

from _hier import from_structured, irregular, oracle_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gnu_femlisp_b200 as G
    return G


@pytest.fixture(scope="module")
def ctx(G):
    return G.Context(0)


def gpu_of(G, ctx, sizes, mats, interp, rhs, layout="csr"):
    g = G.Grid.algebraic(ctx, sizes)
    for l, (s_, i_, v_) in mats.items():
        if layout == "ccs":
            import scipy.sparse as sp
            m = sp.csr_matrix((v_, i_, s_), shape=(sizes[l], sizes[l])).tocsc()
            g.set_matrix(l, m.indptr, m.indices, m.data, layout="ccs")
        else:
            g.set_matrix(l, s_, i_, v_)
    for l, (s_, i_, v_) in interp.items():
        g.set_interpolation(l, s_, i_, v_, sizes[l - 1])
    g.set_rhs(rhs)
    return g


def _cfg(G, method, compat, damp=0.6, pre=1, post=1, maxsteps=60):
    C = G._capi
    m = C.FMG_METHOD_CG_MG if method == "cg" else C.FMG_METHOD_MG
    return G.SolveCfg(m, C.FMG_JACOBI, damp, pre, post, 1, 1 if compat else 0, 1.0, 1e-10, 0.0, maxsteps,
                      C.FMG_MULTIPLICATIVE, 0)


@pytest.mark.parametrize("dim,order,level,base,layout", [(2, 1, 5, 1, "csr"), (3, 1, 3, 1, "ccs"),
                                                         (2, 2, 4, 1, "csr"), (3, 2, 2, 0, "csr")])
@pytest.mark.parametrize("method,compat", [("cg", False), ("cg", True), ("mg", False)])
def test_structured_hierarchy_as_algebraic(oracle_mod, G, ctx, dim, order, level, base, layout, method, compat):
    O = oracle_mod
    o = O.Oracle(dim, order, level, base_level=base)
    o.set_coefficient(O.K_CELL, np.exp(np.random.default_rng(dim + order).standard_normal((1 << level) ** dim)))
    o.assemble()
    g = gpu_of(G, ctx, *from_structured(o, dim, order), layout=layout)
    m = O.METHOD_CG_MG if method == "cg" else O.METHOD_MG
    r = o.solve(O.solve_cfg(method=m, smoother=O.JACOBI, damp=0.6, pre=1, post=1, compat=compat, rtol=1e-10,
                            maxsteps=60))
    x = g.vector()
    hist, steps, st = g.solve(_cfg(G, method, compat), x)
    assert steps == r.steps and st == r.status
    assert np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)


def test_irregular_problem(oracle_mod, G, ctx):
    O = oracle_mod
    h = irregular(n=2000, levels=4, seed=3)
    a = oracle_of(O, *h)
    g = gpu_of(G, ctx, *h)
    for pre, damp in ((1, 0.6), (2, 0.5)):
        r = a.solve(O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.JACOBI, damp=damp, pre=pre, post=pre,
                                compat=False, rtol=1e-10, maxsteps=200))
        x = g.vector()
        hist, steps, st = g.solve(_cfg(G, "cg", False, damp=damp, pre=pre, post=pre, maxsteps=200), x)
        assert st == 0 and r.status == 0
        assert np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)


def test_level_operators(oracle_mod, G, ctx):
    O = oracle_mod
    sizes, mats, interp, rhs = irregular(n=700, levels=3, seed=5)
    a = oracle_of(O, sizes, mats, interp, rhs)
    g = gpu_of(G, ctx, sizes, mats, interp, rhs)
    rng = np.random.default_rng(1)
    top = len(sizes) - 1
    n = sizes[top]
    xv, bv = rng.standard_normal(n), rng.standard_normal(n)
    X, B, Y = g.vector(values=xv), g.vector(values=bv), g.vector()
    g.matvec(X, Y)
    assert np.array_equal(Y.get(), a.matvec(xv))
    g.residual(X, B, Y)
    assert np.array_equal(Y.get(), a.residual(xv, bv))
    R = g.vector(values=bv)
    g.jacobi(X, R, 0.7)
    xo, ro = a.jacobi(xv, bv, 0.7)
    assert np.array_equal(X.get(), xo) and np.array_equal(R.get(), ro)
    rc = g.vector(top - 1)
    g.restrict(B, rc)
    assert np.array_equal(rc.get(), a.restrict(bv, top))
    xc = rng.standard_normal(sizes[top - 1])
    XF = g.vector(values=xv)
    g.prolongate(g.vector(top - 1, values=xc), XF)
    assert np.array_equal(XF.get(), a.prolongate(xc, xv, top - 1))


def test_refusals_and_incomplete_hierarchy(G, ctx):
    C = G._capi
    sizes, mats, interp, rhs = irregular(n=200, levels=2, seed=7)
    g = G.Grid.algebraic(ctx, sizes)
    for l, (s_, i_, v_) in mats.items():
        g.set_matrix(l, s_, i_, v_)
    x = g.vector()
    with pytest.raises(G.FmgError) as e:  # the interpolation is missing
        g.solve(_cfg(G, "cg", False), x)
    assert e.value.code == -3
    s_, i_, v_ = interp[1]
    with pytest.raises(G.FmgError) as e:  # wrong shape
        g.set_interpolation(1, s_, i_, v_, sizes[0] + 1)
    assert e.value.code == -1
    g.set_interpolation(1, s_, i_, v_, sizes[0])
    g.set_rhs(rhs)
    psc = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_PSC, 0.5, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 60, C.FMG_MULTIPLICATIVE, 0)
    for call in (lambda: g.solve(psc, x), lambda: g.assemble(), lambda: g.set_coefficient(C.FMG_K_CONST, 1.0),
                 lambda: g.matrix(1)):
        with pytest.raises(G.FmgError) as e:
            call()
        assert e.value.code == -6
    hist, steps, st = g.solve(_cfg(G, "cg", False), x)
    assert st == 0


@pytest.mark.parametrize("gamma,fmg,comb", [(2, False, 0), (1, True, 0), (1, False, 1)])
def test_algebraic_cycles(oracle_mod, G, ctx, gamma, fmg, comb):
    O = oracle_mod
    C = G._capi
    o = O.Oracle(3, 1, 3, base_level=1)
    o.set_coefficient(O.K_CELL, np.exp(np.random.default_rng(12).standard_normal(8 ** 3)))
    o.assemble()
    g = gpu_of(G, ctx, *from_structured(o, 3, 1))
    post = 1 if comb == 0 else 0
    r = o.solve(O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.JACOBI, damp=0.6, pre=1, post=post, gamma=gamma,
                            fmg=fmg, combination=comb, compat=False, rtol=1e-10, maxsteps=60))
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, post, gamma, 0, 1.0, 1e-10, 0.0, 60, comb,
                     1 if fmg else 0)
    x = g.vector()
    hist, steps, st = g.solve(cfg, x)
    assert st == r.status == 0
    assert np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)


@pytest.mark.parametrize("smoother", ["sor", "ssc"])
@pytest.mark.parametrize("case", ["structured", "irregular"])
def test_algebraic_sor_and_ssc(oracle_mod, G, ctx, smoother, case):
    """<sor> with the rows ordered by colour (linit.lisp:288-323) and the
    one-unknown-block SSC sweep (blockit.lisp:118-204) on algebraic levels:
    one sweep, then the MG iteration with V(1,1), against the oracle's
    algebraic hierarchy (the same greedy colouring), bit for bit."""
    O = oracle_mod
    C = G._capi
    if case == "structured":
        o = O.Oracle(2, 1, 5, base_level=1)
        o.set_coefficient(O.K_CELL, np.exp(np.random.default_rng(21).standard_normal(32 ** 2)))
        o.assemble()
        h = from_structured(o, 2, 1)
    else:
        h = irregular(n=2000, levels=4, seed=3)
    a = oracle_of(O, *h)
    g = gpu_of(G, ctx, *h)
    sizes = h[0]
    top = len(sizes) - 1
    rng = np.random.default_rng(2)
    xv, bv = rng.standard_normal(sizes[top]), rng.standard_normal(sizes[top])
    X, B, R = g.vector(values=xv), g.vector(values=bv), g.vector()
    if smoother == "sor":
        g.sor(X, B, R, 1.1)
        xo, ro = a.sor(xv, bv, np.zeros(sizes[top]), 1.1)
    else:
        g.ssc(X, B, R, 1.0)
        xo, ro = a.ssc(xv, bv, np.zeros(sizes[top]), 1.0)
    assert np.array_equal(X.get(), xo) and np.array_equal(R.get(), ro)
    sm_o, sm_g = (O.SOR, C.FMG_SOR) if smoother == "sor" else (O.SSC, C.FMG_SSC)
    r = a.solve(O.solve_cfg(method=O.METHOD_MG, smoother=sm_o, damp=1.0, pre=1, post=1, compat=False, rtol=1e-10,
                            maxsteps=150))
    x = g.vector()
    cfg = G.SolveCfg(C.FMG_METHOD_MG, sm_g, 1.0, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 150, C.FMG_MULTIPLICATIVE, 0)
    hist, steps, st = g.solve(cfg, x)
    assert st == r.status and steps == r.steps, (st, r.status, steps, r.steps)
    assert np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)
