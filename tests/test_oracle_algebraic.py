"""The oracle's algebraic hierarchies (no GPU): a structured hierarchy given as
compressed rows (its level matrices and its constrained interpolations)
iterates bit for bit like the structured one, and an irregular problem with
no grid behind it (a graph Laplacian on random points, aggregation
interpolations, Galerkin coarse matrices) is solved by CG + V(1,1) Jacobi."""
import numpy as np
import pytest

from _hier import from_structured, irregular, oracle_of


@pytest.mark.parametrize("dim,order,level,base", [(2, 1, 4, 1), (3, 1, 3, 1), (2, 2, 3, 1)])
@pytest.mark.parametrize("method,compat", [("cg", False), ("cg", True), ("mg", False)])
def test_structured_as_algebraic(oracle_mod, dim, order, level, base, method, compat):
    O = oracle_mod
    o = O.Oracle(dim, order, level, base_level=base)
    o.set_coefficient(O.K_CELL, np.exp(np.random.default_rng(dim).standard_normal((1 << level) ** dim)))
    o.assemble()
    a = oracle_of(O, *from_structured(o, dim, order))
    m = O.METHOD_CG_MG if method == "cg" else O.METHOD_MG
    cfg = O.solve_cfg(method=m, smoother=O.JACOBI, damp=0.6, pre=1, post=1, compat=compat, rtol=1e-10,
                      maxsteps=60)
    rs, ra = o.solve(cfg), a.solve(cfg)
    assert np.array_equal(rs.history, ra.history) and np.array_equal(rs.x, ra.x)


def test_irregular_problem_converges(oracle_mod):
    O = oracle_mod
    sizes, mats, interp, rhs = irregular()
    a = oracle_of(O, sizes, mats, interp, rhs)
    r = a.solve(O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.JACOBI, damp=0.6, pre=2, post=2, compat=False,
                            rtol=1e-10, maxsteps=200))
    assert r.status == 0, r.steps
    import scipy.sparse as sp
    s_, i_, v_ = mats[len(sizes) - 1]
    A = sp.csr_matrix((v_, i_, s_), shape=(sizes[-1], sizes[-1]))
    assert np.linalg.norm(A @ r.x - rhs) <= 1e-9 * np.linalg.norm(rhs)


@pytest.mark.parametrize("gamma,fmg,comb", [(2, False, 0), (1, True, 0), (1, False, 1)])
def test_structured_as_algebraic_cycles(oracle_mod, gamma, fmg, comb):
    # W-cycle, F-cycle and the additive combination through the same
    # algebraic levels
    O = oracle_mod
    o = O.Oracle(2, 1, 5, base_level=1)
    o.set_coefficient(O.K_CELL, np.exp(np.random.default_rng(11).standard_normal(32 * 32)))
    o.assemble()
    a = oracle_of(O, *from_structured(o, 2, 1))
    cfg = O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.JACOBI, damp=0.6, pre=1, post=1 if comb == 0 else 0,
                      gamma=gamma, fmg=fmg, combination=comb, compat=False, rtol=1e-10, maxsteps=60)
    rs, ra = o.solve(cfg), a.solve(cfg)
    assert rs.status == 0
    assert np.array_equal(rs.history, ra.history) and np.array_equal(rs.x, ra.x)


def test_algebraic_level_operators_against_scipy(oracle_mod):
    # the oracle's compressed-row operators against plain sparse arithmetic
    import scipy.sparse as sp
    O = oracle_mod
    sizes, mats, interp, rhs = irregular(n=500, levels=3, seed=2)
    a = oracle_of(O, sizes, mats, interp, rhs)
    top = len(sizes) - 1
    A = sp.csr_matrix((mats[top][2], mats[top][1], mats[top][0]), shape=(sizes[top], sizes[top]))
    P = sp.csr_matrix((interp[top][2], interp[top][1], interp[top][0]), shape=(sizes[top], sizes[top - 1]))
    rng = np.random.default_rng(4)
    x, b = rng.standard_normal(sizes[top]), rng.standard_normal(sizes[top])
    tol = 1e-13 * np.abs(A).sum(axis=1).max() * np.abs(x).max()
    assert np.max(np.abs(a.matvec(x) - A @ x)) <= tol
    assert np.max(np.abs(a.residual(x, b) - (b - A @ x))) <= tol
    assert np.max(np.abs(a.restrict(b, top) - P.T @ b)) <= 1e-13 * np.abs(P).sum(axis=0).max() * np.abs(b).max()
    xc = rng.standard_normal(sizes[top - 1])
    assert np.max(np.abs(a.prolongate(xc, x, top - 1) - (x + P @ xc))) <= 1e-13 * (1 + np.abs(x).max())
    xj, rj = a.jacobi(x, b, 0.7)
    d = A.diagonal()
    assert np.allclose(rj, b / d, rtol=0, atol=0) and np.max(np.abs(xj - (x + 0.7 * b / d))) <= 1e-15 * np.abs(xj).max()
