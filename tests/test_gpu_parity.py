"""GPU FP64 path against the oracle, through the C-ABI.

Both sides follow the same operation order (explicit fma, fixed stencil
slot order, DR4096 reductions), so the results are compared bitwise; the
acceptance bound of the plain path is 1e-12 relative, checked as well.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12


@pytest.fixture(scope="module")
def G():
    import gnu_femlisp_b200 as G
    return G


@pytest.fixture(scope="module")
def ctx(G):
    return G.Context(0)


def _nq(dim, order):
    return (order + 1) ** dim


def make_pair(O, G, ctx, dim, order, level, base, kcell=False, fip=False, seed=0, dmask=None):
    o = O.Oracle(dim, order, level, base_level=base, dirichlet_mask=dmask)
    g = G.Grid(ctx, dim, order, level, base_level=base, dirichlet_mask=dmask)
    rng = np.random.default_rng(seed)
    ncell = (1 << level) ** dim
    if kcell:
        k = np.exp(rng.standard_normal(ncell))
        o.set_coefficient(O.K_CELL, k)
        g.set_coefficient(1, k)
    if fip:
        f = rng.standard_normal(ncell * _nq(dim, order))
        o.set_coefficient(O.F_IP, f)
        g.set_coefficient(3, f)
    o.assemble()
    g.assemble()
    return o, g


def assert_same(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.max(np.abs(a)), 1e-300)
    diff = np.max(np.abs(a - b)) if a.size else 0.0
    assert diff <= REL * scale, f"{what}: max diff {diff:.3e} (scale {scale:.3e})"
    assert np.array_equal(a, b), f"{what}: within {REL} but not bitwise (max diff {diff:.3e})"


CASES = [(1, 1, 5, 0), (2, 1, 4, 1), (3, 1, 3, 1), (1, 2, 3, 0), (2, 2, 3, 1), (3, 2, 2, 0)]


@pytest.mark.parametrize("dim,order,level,base", CASES)
@pytest.mark.parametrize("kcell", [False, True])
def test_assembly(oracle_mod, G, ctx, dim, order, level, base, kcell):
    o, g = make_pair(oracle_mod, G, ctx, dim, order, level, base, kcell=kcell, fip=kcell, seed=dim)
    for l in range(base, level + 1):
        assert_same(g.matrix(l), o.matrix(l), f"A level {l}")
    assert_same(g.rhs(), o.rhs(), "rhs")


def test_assembly_partial_dirichlet(oracle_mod, G, ctx):
    # only the x=0 face is essential (the clamped face of the elasticity case)
    o, g = make_pair(oracle_mod, G, ctx, 3, 1, 3, 1, kcell=True, seed=5, dmask=0b000001)
    for l in range(1, 4):
        assert_same(g.matrix(l), o.matrix(l), f"A level {l}")


@pytest.mark.parametrize("dim,order,level,base", CASES)
def test_level_operators(oracle_mod, G, ctx, dim, order, level, base):
    o, g = make_pair(oracle_mod, G, ctx, dim, order, level, base, kcell=True, seed=11)
    rng = np.random.default_rng(3)
    for l in range(base, level + 1):
        n = g.nnodes(l)
        x, b = rng.standard_normal(n), rng.standard_normal(n)
        X, B, Y = g.vector(l, x), g.vector(l, b), g.vector(l)
        g.matvec(X, Y)
        assert_same(Y.get(), o.matvec(x, l), f"matvec l={l}")
        g.residual(X, B, Y)
        assert_same(Y.get(), o.residual(x, b, l), f"residual l={l}")
        g.residual(X, B, B)  # aliased b == r: r := r - A x
        assert_same(B.get(), o.residual(x, b, l), f"aliased residual l={l}")
        if l > base:
            X.set(x)
            R = g.vector(l, b)
            g.jacobi(X, R, 0.6)
            xo, ro = o.jacobi(x, b, 0.6, l)
            assert_same(X.get(), xo, "jacobi x")
            assert_same(R.get(), ro, "jacobi r")
            X.set(x)
            B.set(b)
            R = g.vector(l)
            g.sor(X, B, R, 1.2)
            xo, ro = o.sor(x, b, np.zeros(n), 1.2, l)
            assert_same(X.get(), xo, "sor x")
            assert_same(R.get(), ro, "sor r")
            rc = g.vector(l - 1)
            g.restrict(g.vector(l, x), rc)
            assert_same(rc.get(), o.restrict(x, l), f"restrict {l}")
            xc = rng.standard_normal(g.nnodes(l - 1))
            XF = g.vector(l, b)
            g.prolongate(g.vector(l - 1, xc), XF)
            assert_same(XF.get(), o.prolongate(xc, b, l - 1), f"prolongate {l - 1}")
    nb = g.nnodes(base)
    x, r = rng.standard_normal(nb), rng.standard_normal(nb)
    X, R = g.vector(base, x), g.vector(base, r)
    g.coarse_solve(X, R, 1.0)
    xo, ro = o.coarse_solve(x, r, 1.0)
    assert_same(R.get(), ro, "coarse r")
    assert_same(X.get(), xo, "coarse x")


@pytest.mark.parametrize("n", [1, 5, 4095, 4096, 4097, 65537, 1_000_003])
def test_dot_is_bitwise(oracle_mod, G, ctx, n):
    # vectors are sized by a level: take a 2D Q1 level with >= n nodes and
    # zero the tail (zeros add nothing in the fixed reduction order either)
    rng = np.random.default_rng(n)
    level = max(1, int(np.ceil(np.log2(max(np.sqrt(n) - 1.0, 1.0)))))
    g = G.Grid(ctx, 2, 1, level, 0).assemble()
    m = g.nnodes()
    x, y = np.zeros(m), np.zeros(m)
    x[:n], y[:n] = rng.standard_normal(n), rng.standard_normal(n)
    X, Y = g.vector(values=x), g.vector(values=y)
    assert X.dot(Y) == oracle_mod.dot(x, y)


def _cfg(O, G, method, smoother, damp, pre, post, compat, comb=0, gamma=1, rtol=1e-10, atol=0.0,
         maxsteps=60):
    oc = O.solve_cfg(method=method, smoother=smoother, damp=damp, pre=pre, post=post, gamma=gamma,
                     compat=compat, rtol=rtol, atol=atol, maxsteps=maxsteps, combination=comb)
    gc = G.SolveCfg(method, smoother, damp, pre, post, gamma, 1 if compat else 0, 1.0, rtol, atol,
                    maxsteps, comb)
    return oc, gc


VCYCLES = [
    # smoother, damp, pre, post, combination, gamma
    (0, 0.6, 1, 1, 0, 1),
    (0, 0.6, 2, 2, 0, 1),
    (1, 1.2, 2, 2, 0, 1),
    (0, 1.0, 1, 0, 1, 1),
    (0, 0.6, 1, 1, 0, 2),
]


@pytest.mark.parametrize("sm,damp,pre,post,comb,gamma", VCYCLES)
@pytest.mark.parametrize("alias", [False, True])
def test_vcycle(oracle_mod, G, ctx, sm, damp, pre, post, comb, gamma, alias):
    O = oracle_mod
    o, g = make_pair(O, G, ctx, 3, 1, 4, 1, kcell=True, seed=2)
    oc, gc = _cfg(O, G, 0, sm, damp, pre, post, alias, comb, gamma)
    rng = np.random.default_rng(7)
    n = g.nnodes()
    b = rng.standard_normal(n)
    X, B = g.vector(), g.vector(values=b)
    if alias:
        g.vcycle(gc, X, B, B)
        xo, bo, _ = o.vcycle(oc, np.zeros(n), b, None)
        assert_same(B.get(), bo, "aliased rhs/res after the cycle")
    else:
        R = g.vector(values=b)
        g.vcycle(gc, X, B, R)
        xo, bo, ro = o.vcycle(oc, np.zeros(n), b, b)
        assert_same(R.get(), ro, "res after the cycle")
    assert_same(X.get(), xo, "x after the cycle")


SOLVES = [
    # dim, order, level, base, method, smoother, damp, pre, post, compat, comb
    (2, 1, 6, 0, 1, 0, 0.6, 1, 1, False, 0),   # C1: CG + V(1,1) Jacobi 0.6, 64x64 Q1
    (2, 1, 6, 0, 1, 0, 0.6, 1, 1, True, 0),    # C1 with the reference's alias
    (2, 1, 5, 1, 1, 0, 1.0, 1, 0, True, 1),    # BPX-style additive cycle under <cg>
    (3, 1, 4, 1, 1, 0, 0.6, 2, 2, False, 0),
    (3, 2, 3, 1, 1, 1, 1.2, 2, 2, False, 0),   # Q2, multicolour SOR
    (3, 1, 4, 1, 0, 1, 1.0, 1, 1, False, 0),   # bare V-cycle iteration
    (2, 1, 5, 0, 2, 0, 0.6, 1, 1, False, 0),   # unpreconditioned CG
]


@pytest.mark.parametrize("dim,order,level,base,method,sm,damp,pre,post,compat,comb", SOLVES)
def test_solve_history(oracle_mod, G, ctx, dim, order, level, base, method, sm, damp, pre, post, compat,
                       comb):
    O = oracle_mod
    o, g = make_pair(O, G, ctx, dim, order, level, base, kcell=(dim == 3), seed=4)
    oc, gc = _cfg(O, G, method, sm, damp, pre, post, compat, comb, maxsteps=80)
    ro = o.solve(oc)
    X = g.vector()
    hist, steps, status = g.solve(gc, X)
    assert steps == ro.steps and status == ro.status
    assert_same(hist, ro.history, "defnorm history")
    assert_same(X.get(), ro.x, "solution")


def test_v_cycle_convergence_rate_on_gpu(G, ctx):
    # mg-cdr.lisp:85-87 through the Femlisp-style API
    A, b = G.discretize_globally(G.cdr_model_problem(1), G.uniformly_refined_hierarchical_mesh(1, 3),
                                 G.lagrange_fe(1), ctx)
    cs = G.geometric_cs(gamma=1, smoother=G.Jacobi(damp=0.5), pre_steps=1, post_steps=0, base_level=2)
    solver = G.LinearSolver(cs, success_if="(or (< :defnorm 1.0e-12) (> :step 10))")
    res = G.solve({"matrix": A, "rhs": b, "solver": solver})
    cr = res["report"].convergence_rate
    assert cr < 0.3941 and abs(cr - 0.39407) < 1e-5


def test_exact_nodal_value_on_gpu(G, ctx):
    # ellsys-fe.lisp:249-256: u_h(1/2) = 0.125 for 1D Q1 level 2
    A, b = G.discretize_globally(G.cdr_model_problem(1), G.uniformly_refined_hierarchical_mesh(1, 2),
                                 G.lagrange_fe(1), ctx)
    cs = G.geometric_cs(smoother=G.Jacobi(damp=0.6), base_level=2)
    res = G.solve({"matrix": A, "rhs": b, "solver": G.LinearSolver(cs, "(< :reduction 1.0e-14)",
                                                                   "(> :step 3)")})
    assert res["solution"][2] == 0.125


@pytest.mark.parametrize("dim,level,base,dmask", [(1, 5, 0, None), (2, 4, 1, None), (3, 3, 1, None),
                                                  (3, 3, 0, 0b000001)])
def test_galerkin_levels(oracle_mod, G, ctx, dim, level, base, dmask):
    # multilevel-decomposition with :galerkin-p t: I^T A I from the top level down
    O = oracle_mod
    o = O.Oracle(dim, 1, level, base_level=base, dirichlet_mask=dmask)
    g = G.Grid(ctx, dim, 1, level, base_level=base, dirichlet_mask=dmask)
    k = np.exp(np.random.default_rng(dim).standard_normal((1 << level) ** dim))
    o.set_coefficient(O.K_CELL, k)
    g.set_coefficient(1, k)
    o.assemble(galerkin=True)
    g.assemble(galerkin=True)
    for l in range(base, level + 1):
        assert_same(g.matrix(l), o.matrix(l), f"A level {l}")
    oc, gc = _cfg(O, G, 1, 0, 0.6, 1, 1, False, maxsteps=80)
    ro = o.solve(oc)
    X = g.vector()
    hist, steps, status = g.solve(gc, X)
    assert status == 0 and steps == ro.steps
    assert_same(hist, ro.history, "defnorm history")
    assert_same(X.get(), ro.x, "solution")


@pytest.mark.parametrize("dim,order,level,base,method,sm,damp", [(2, 1, 6, 1, 0, 0, 0.6), (3, 1, 4, 1, 1, 0, 0.6),
                                                                  (3, 2, 3, 1, 0, 1, 1.2), (2, 1, 5, 0, 1, 0, 0.6)])
def test_f_cycle_solve_history(oracle_mod, G, ctx, dim, order, level, base, method, sm, damp):
    # the f-cycle (:fmg t, multigrid.lisp:290-297) as the iteration and as the preconditioner
    O = oracle_mod
    o, g = make_pair(O, G, ctx, dim, order, level, base, kcell=(dim == 3), seed=12)
    oc, gc = _cfg(O, G, method, sm, damp, 1, 1, False, maxsteps=80)
    oc.fmg = 1
    gc.fmg = 1
    ro = o.solve(oc)
    X = g.vector()
    hist, steps, status = g.solve(gc, X)
    assert status == 0 and steps == ro.steps
    assert_same(hist, ro.history, "defnorm history")
    assert_same(X.get(), ro.x, "solution")
    with pytest.raises(G.FmgError):
        g.solve_mixed(gc, g.vector())  # the mixed cycle is a V/W cycle


def test_deferred_top_level_matrix(oracle_mod, G, ctx):
    # 3D scalar Q1: the top level's matrix is formed on its first use; a
    # mixed solve (matrix-free top level) before it, then the FP64 solve and
    # the matrices, all as the oracle has them
    O = oracle_mod
    o, g = make_pair(O, G, ctx, 3, 1, 4, 1, kcell=True, seed=21)
    C = G._capi
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 100,
                     C.FMG_MULTIPLICATIVE, 0)
    xm = g.vector()
    hist_m, _, _, st_m = g.solve_mixed(cfg, xm, matrix_free=True)
    assert st_m == 0
    x = g.vector()
    hist, steps, st = g.solve(cfg, x)
    r = o.solve(O.solve_cfg(damp=0.6, compat=False, rtol=1e-10, maxsteps=100))
    assert st == 0 and np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)
    assert_same(g.matrix(4), o.matrix(4), "top level")
    assert np.linalg.norm(xm.get() - r.x) <= 1e-8 * np.linalg.norm(r.x)

