"""The vertex-centred successive and parallel subspace corrections
(geometric-ssc / geometric-psc, geoblock.lisp:37-158, blockit.lisp:118-204)
on the GPU against the oracle,
bitwise: single sweeps (separate b and r, and b aliased to r as inside
<cg>), Q1 (one-node blocks) and Q2 (3^d boxes) in 1, 2 and 3 dimensions, a
partially clamped boundary (blocks cut by Neumann faces), and whole
multigrid / CG solves with it as the smoother."""
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


def make_pair(O, G, ctx, dim, order, level, base, seed=0, dmask=None):
    o = O.Oracle(dim, order, level, base_level=base, dirichlet_mask=dmask)
    g = G.Grid(ctx, dim, order, level, base_level=base, dirichlet_mask=dmask)
    k = np.exp(np.random.default_rng(seed).standard_normal((1 << level) ** dim))
    o.set_coefficient(O.K_CELL, k)
    g.set_coefficient(G._capi.FMG_K_CELL, k)
    o.assemble()
    g.assemble()
    return o, g


SWEEPS = [(1, 2, 4), (2, 2, 3), (3, 2, 2), (3, 2, 3), (2, 1, 4), (3, 1, 3)]


@pytest.mark.parametrize("dim,order,level", SWEEPS)
@pytest.mark.parametrize("dmask", [None, 0b000001])
@pytest.mark.parametrize("alias", [False, True])
def test_ssc_sweep(oracle_mod, G, ctx, dim, order, level, dmask, alias):
    o, g = make_pair(oracle_mod, G, ctx, dim, order, level, 0, seed=dim + level, dmask=dmask)
    n = g.nnodes()
    rng = np.random.default_rng(17)
    x0, b0, r0 = rng.standard_normal(n), rng.standard_normal(n), rng.standard_normal(n)
    x, b, r = g.vector(values=x0), g.vector(values=b0), g.vector(values=r0)
    if alias:
        xo, ro = _oracle_alias(o, x0, r0, 1.1)
        g.ssc(x, r, r, omega=1.1)
    else:
        xo, ro = o.ssc(x0, b0, r0, omega=1.1)
        g.ssc(x, b, r, omega=1.1)
        assert np.array_equal(b.get(), b0)
    assert np.array_equal(x.get(), xo), np.max(np.abs(x.get() - xo))
    assert np.array_equal(r.get(), ro), np.max(np.abs(r.get() - ro))
    assert not np.array_equal(xo, x0)


def _oracle_alias(o, x0, r0, omega):
    r = np.array(r0, copy=True)
    return o.ssc(x0, r, r, omega=omega)


@pytest.mark.parametrize("dim,level,base", [(2, 4, 1), (3, 3, 1)])
@pytest.mark.parametrize("method,compat", [("mg", True), ("cg", True), ("cg", False)])
def test_ssc_solve_histories(oracle_mod, G, ctx, dim, level, base, method, compat):
    O = oracle_mod
    o, g = make_pair(O, G, ctx, dim, 2, level, base, seed=3)
    C = G._capi
    m_o = O.METHOD_MG if method == "mg" else O.METHOD_CG_MG
    m_g = C.FMG_METHOD_MG if method == "mg" else C.FMG_METHOD_CG_MG
    pre, post = (1, 0) if method == "mg" else (1, 1)
    r = o.solve(O.solve_cfg(method=m_o, smoother=O.SSC, damp=1.0, pre=pre, post=post, compat=compat,
                            rtol=1e-10, maxsteps=60))
    cfg = G.SolveCfg(m_g, C.FMG_SSC, 1.0, pre, post, 1, 1 if compat else 0, 1.0, 1e-10, 0.0, 60,
                     C.FMG_MULTIPLICATIVE, 0)
    x = g.vector()
    hist, steps, st = g.solve(cfg, x)
    assert np.array_equal(hist, r.history), (hist[-3:], r.history[-3:])
    assert np.array_equal(x.get(), r.x)
    if not (method == "cg" and compat):   # the alias spoils the preconditioner inside <cg>
        assert st == 0 and r.status == 0


def test_ssc_two_steps_and_vcycle_literal(oracle_mod, G, ctx):
    # V(2,2) applied once on user vectors: every residual write is kept
    O = oracle_mod
    o, g = make_pair(O, G, ctx, 3, 2, 3, 1, seed=4)
    C = G._capi
    n = g.nnodes()
    rng = np.random.default_rng(5)
    x0, b0 = rng.standard_normal(n), rng.standard_normal(n)
    cfgo = O.solve_cfg(method=O.METHOD_MG, smoother=O.SSC, damp=0.9, pre=2, post=2, compat=False)
    xo, bo, ro = o.vcycle(cfgo, x0, b0, np.zeros(n))
    cfg = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_SSC, 0.9, 2, 2, 1, 0, 1.0, 0.0, 0.0, 1, C.FMG_MULTIPLICATIVE, 0)
    x, b, rr = g.vector(values=x0), g.vector(values=b0), g.vector(values=np.zeros(n))
    g.vcycle(cfg, x, b, rr)
    assert np.array_equal(x.get(), xo)
    assert np.array_equal(rr.get(), ro)


def test_default_smoother_of_q2_is_ssc(G, ctx):
    # select-smoother (geomg.lisp:48-60): order 1 -> Gauss-Seidel, higher -> SSC
    from gnu_femlisp_b200 import iteration as I
    cs = I.geometric_cs(base_level=1)
    cfg1, _, _ = I.make_cfg(I.CG(preconditioner=cs), "(< :reduction 1e-10)", "(> :step 50)", order=1)
    cfg2, _, _ = I.make_cfg(I.CG(preconditioner=cs), "(< :reduction 1e-10)", "(> :step 50)", order=2)
    assert cfg1.smoother == G._capi.FMG_SOR and cfg2.smoother == G._capi.FMG_SSC
    problem = I.cdr_model_problem(2)
    mesh = I.uniformly_refined_hierarchical_mesh(2, 4)
    A, _ = I.discretize_globally(problem, mesh, I.lagrange_fe(2), ctx=ctx)
    solver = I.LinearSolver(iteration=I.CG(preconditioner=cs), success_if="(< :reduction 1e-10)",
                            failure_if="(> :step 50)")
    bb = I.solve({"matrix": A, "solver": solver})
    assert bb["report"].status == "success"
    assert bb["report"].steps < 20


# ---------------------------------------------------------------- geometric PSC

@pytest.mark.parametrize("dim,order,level", SWEEPS)
@pytest.mark.parametrize("dmask", [None, 0b000001])
def test_psc_sweep(oracle_mod, G, ctx, dim, order, level, dmask):
    o, g = make_pair(oracle_mod, G, ctx, dim, order, level, 0, seed=dim + 2 * level, dmask=dmask)
    n = g.nnodes()
    rng = np.random.default_rng(23)
    x0, r0 = rng.standard_normal(n), rng.standard_normal(n)
    x, r = g.vector(values=x0), g.vector(values=r0)
    xo = o.psc(x0, r0, damp=0.7)
    g.psc(x, r, damp=0.7)
    assert np.array_equal(x.get(), xo), np.max(np.abs(x.get() - xo))
    assert np.array_equal(r.get(), r0)   # the residual is read, not written
    assert not np.array_equal(xo, x0)


@pytest.mark.parametrize("dim,level,base", [(2, 4, 1), (3, 3, 1)])
def test_psc_cg_histories(oracle_mod, G, ctx, dim, level, base):
    # additive Schwarz over the vertex blocks is symmetric: CG + V(1,1) PSC
    O = oracle_mod
    o, g = make_pair(O, G, ctx, dim, 2, level, base, seed=6)
    C = G._capi
    damp = 0.4 if dim == 2 else 0.2  # a node lies in up to 2^d blocks
    r = o.solve(O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.PSC, damp=damp, pre=1, post=1, compat=False,
                            rtol=1e-10, maxsteps=80))
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_PSC, damp, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 80, C.FMG_MULTIPLICATIVE, 0)
    x = g.vector()
    hist, steps, st = g.solve(cfg, x)
    assert st == 0 and r.status == 0
    assert np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)
