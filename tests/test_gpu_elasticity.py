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


def _vcfg11(G):
    return G.SolveCfg(1, G._capi.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 200, G._capi.FMG_MULTIPLICATIVE)


def test_block_cycle_gradient_matches_finite_differences(oracle_mod, G, ctx):
    # dL/domega of the per-node damping of the 3 x 3 block Jacobi, through the
    # whole V(1,1) cycle (the recorded cycle's adjoint with block solves), on
    # the top level and the level below, against central differences
    from gnu_femlisp_b200.learn import learn_loss_levels
    _, g = make_pair(oracle_mod, G, ctx, 2, 2, 0, 3, seed=8)
    cfg = _vcfg11(G)
    rng = np.random.default_rng(4)
    ws = {}
    for lev in range(g.base + 1, g.top + 1):
        ws[lev] = rng.uniform(0.4, 0.8, g.nnodes(lev))
        g.set_node_damping(lev, ws[lev])
    n = g.nnodes()
    m = round(n ** (1 / 3))
    e0 = rng.uniform(-1, 1, (n, 3))
    e0[np.arange(n) % m == 0] = 0.0  # the clamped face x = 0
    ev = g.vector(values=e0.reshape(-1))
    for lev in (g.top - 1, g.top):
        L0, grad = learn_loss_levels(g, cfg, ev, lev)
        assert 0 < L0 < 1 and grad.shape == (g.nnodes(lev),)
        d = rng.standard_normal(ws[lev].size)
        eps = 1e-5
        g.set_node_damping(lev, ws[lev] + eps * d)
        Lp, _ = learn_loss_levels(g, cfg, ev, lev, want_grad=False)
        g.set_node_damping(lev, ws[lev] - eps * d)
        Lm, _ = learn_loss_levels(g, cfg, ev, lev, want_grad=False)
        g.set_node_damping(lev, ws[lev])
        fd = (Lp - Lm) / (2 * eps)
        assert abs(fd - grad @ d) <= 1e-6 * max(1e-3, abs(fd)), (lev, fd, grad @ d)


def test_network_damping_on_elasticity_levels(oracle_mod, G, ctx):
    # the damping network on Q2 node grids (features from E on each node's 8
    # half-cells), the judge with both probes, and solves with the damping
    from gnu_femlisp_b200.learn import DampingNet
    _, g = make_pair(oracle_mod, G, ctx, 2, 2, 0, 3, seed=9)
    net = DampingNet(ctx, 3, seed=5)
    om = net.damping(g, g.top)
    assert om.shape == (g.nnodes(),) and om.min() >= 0.1 and om.max() <= 1.3
    net.apply(g)
    cfg = G.SolveCfg(1, G._capi.FMG_JACOBI, 0.6, 2, 2, 1, 0, 1.0, 1e-10, 0.0, 300, G._capi.FMG_MULTIPLICATIVE)
    ok, rp, rl = g.learned_judge(cfg)
    assert 0 < rp < 1 and np.isfinite(rl)
    net.apply(g)
    ok2, rp2, rl2 = g.learned_judge_mixed(cfg)
    assert 0 < rp2 < 1 and np.isfinite(rl2)
    if not ok2:
        net.apply(g)  # install it anyway: the solves must still reach the tolerance
    X = g.vector()
    hist, _, _, st = g.solve_mixed(cfg, X)
    assert st == 0 and hist[-1] / hist[0] < 1e-10


def test_trained_elasticity_net_beats_the_plain_cycle(G, ctx):
    # the shipped network (trained on fields of seeds 1000-1007) on the
    # benchmark's field recipe with its seed 0, at 24^3 cells: the judge keeps
    # it, and CG + V(2,2) block Jacobi needs fewer steps, FP64 and mixed
    import os
    from gnu_femlisp_b200 import problems
    from gnu_femlisp_b200.learn import DampingNet
    C = G._capi
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    net = DampingNet.load(ctx, os.path.join(root, "gnu_femlisp_b200", "weights", "damping3d_elastic.fmgnet"))
    wl = problems.c5(level=3)
    g = G.Grid(ctx, 3, 2, wl.level, base_level=0, n0=3, ncomp=3, dirichlet_mask=wl.dirichlet_mask)
    g.set_coefficient(C.FMG_LAMBDA_MU_CELL, wl.ecell)
    g.set_coefficient(C.FMG_F_VEC, list(wl.force))
    g.assemble()
    cfg = G.SolveCfg(1, C.FMG_JACOBI, 0.6, 2, 2, 1, 0, 1.0, 1e-10, 0.0, 300, C.FMG_MULTIPLICATIVE)
    x = g.vector()
    _, ns_p, st = g.solve(cfg, x)
    xp = x.get()
    _, _, ni_p, _ = g.solve_mixed(cfg, g.vector())
    net.apply(g)
    ok, rp, rl = g.learned_judge_mixed(cfg)
    assert ok and rl < rp, (rp, rl)
    x.fill(0.0)
    _, ns_l, st = g.solve(cfg, x)
    assert st == 0 and ns_l < ns_p, (ns_p, ns_l)
    assert np.linalg.norm(x.get() - xp) / np.linalg.norm(xp) < 1e-8
    _, _, ni_l, st = g.solve_mixed(cfg, g.vector())
    assert st == 0 and ni_l < ni_p and g.learned_status()["reverts"] == 0, (ni_p, ni_l)
