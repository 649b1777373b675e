"""Locally refined meshes with hanging nodes on the GPU: the hierarchy of a
2D Q1 problem refined towards a corner (gnu_femlisp_b200.adaptive; the
hanging-node and Dirichlet constraints eliminated on the host as
constraints.lisp:78-151,323-411 does) through fmg_grid_create_algebraic
solves bit for bit like the oracle's algebraic hierarchy -- CG + MG and the
MG iteration with Jacobi, multicolour SOR and one-unknown SSC
(multigrid.lisp:254-288, krylow.lisp:72-132) -- and the blackboard solve
with local_mg (<local-mg>, geomg.lisp:161-168) reaches the same iterate."""
import numpy as np
import pytest

from _hier import oracle_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gnu_femlisp_b200 as G
    return G


@pytest.fixture(scope="module")
def ctx(G):
    return G.Context(0)


def _k(x, y):
    return 1.0 + 9.0 * (x > 0.5) * (y > 0.5)


@pytest.fixture(scope="module")
def hier():
    from gnu_femlisp_b200 import adaptive as AD
    return AD.hierarchy(n0=4, levels=6, kcoef=_k)[:4]


def _grid(G, ctx, sizes, mats, interp, rhs):
    g = G.Grid.algebraic(ctx, sizes)
    for l, (s_, i_, v_) in mats.items():
        g.set_matrix(l, s_, i_, v_)
    for l, (s_, i_, v_) in interp.items():
        g.set_interpolation(l, s_, i_, v_, sizes[l - 1])
    g.set_rhs(rhs)
    return g


@pytest.mark.parametrize("smoother,damp", [("jacobi", 0.6), ("sor", 1.0), ("ssc", 1.0)])
@pytest.mark.parametrize("method", ["cg", "mg"])
def test_adaptive_hierarchy_bitwise(oracle_mod, G, ctx, hier, smoother, damp, method):
    O = oracle_mod
    C = G._capi
    a = oracle_of(O, *hier)
    g = _grid(G, ctx, *hier)
    sm_o = {"jacobi": O.JACOBI, "sor": O.SOR, "ssc": O.SSC}[smoother]
    sm_g = {"jacobi": C.FMG_JACOBI, "sor": C.FMG_SOR, "ssc": C.FMG_SSC}[smoother]
    m_o, m_g = (O.METHOD_CG_MG, C.FMG_METHOD_CG_MG) if method == "cg" else (O.METHOD_MG, C.FMG_METHOD_MG)
    r = a.solve(O.solve_cfg(method=m_o, smoother=sm_o, damp=damp, pre=1, post=1, compat=False, rtol=1e-10,
                            maxsteps=100))
    x = g.vector()
    hist, steps, st = g.solve(G.SolveCfg(m_g, sm_g, damp, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 100,
                                         C.FMG_MULTIPLICATIVE, 0), x)
    assert st == r.status == 0 and steps == r.steps
    assert np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)


def test_blackboard_solve_with_local_mg(oracle_mod, G, ctx):
    """(solve (blackboard :matrix A :solver (make-instance '<linear-solver>
    :iteration (make-instance '<cg> :preconditioner (local-mg ...))))) on the
    AlgebraicSystem of the refined mesh: the default smoother of order 1 is
    Gauss-Seidel (geomg.lisp:48-60), here the multicolour SOR(1)."""
    from gnu_femlisp_b200 import adaptive as AD
    O = oracle_mod
    A = AD.system(n0=4, levels=5, kcoef=_k, ctx=ctx)
    solver = G.LinearSolver(G.CG(preconditioner=G.local_mg(base_level=1)),
                            success_if="(< :reduction 1.0e-10)", failure_if="(> :step 100)")
    out = G.solve({"matrix": A, "solver": solver})
    assert out["report"].status == "success"
    mats = {l: m for l, m in enumerate(A.matrices[1:])}
    interp = {l: p for l, p in enumerate(A.interpolations[1:], start=1)}
    o = oracle_of(O, A.sizes[1:], mats, interp, A.rhs)
    r = o.solve(O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.SOR, damp=1.0, pre=1, post=1, compat=False,
                            rtol=1e-10, maxsteps=100))
    assert out["report"].steps == r.steps
    assert np.array_equal(out["history"], r.history) and np.array_equal(out["solution"], r.x)
