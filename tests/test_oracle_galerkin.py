"""Galerkin coarse operators of the oracle (multilevel-decomposition with
:galerkin-p t, geomg.lisp:122-123; galerkin-product, amg.lisp:247-285) for
every Lagrange form the path has: scalar Q1/Q2 and 3 x 3 node blocks.  With
constant coefficients nested conforming spaces give the variational
property I^T A_fine I = A_coarse, so the products must equal the
re-discretised coarse matrices to rounding; with a variable coefficient the
Galerkin hierarchy must still make a working preconditioner."""
import numpy as np
import pytest

CASES = [(2, 1, 4, 1, 1, 1), (2, 2, 3, 0, 1, 1), (3, 2, 2, 0, 1, 1), (3, 1, 2, 0, 3, 2), (3, 2, 1, 0, 3, 2)]


def _pair(O, dim, order, level, base, nc, n0, galerkin, k=None):
    kw = dict(ncomp=nc, n0=n0) if nc == 3 else {}
    o = O.Oracle(dim, order, level, base_level=base, dirichlet_mask=1 if nc == 3 else None, **kw)
    if nc == 3:
        o.set_coefficient(O.LAMBDA_MU_CELL, np.ones((n0 << level) ** 3) if k is None else k)
        o.set_coefficient(O.F_VEC, [0.0, 0.0, -1.0])
    elif k is not None:
        o.set_coefficient(O.K_CELL, k)
    return o.assemble(galerkin=galerkin)


@pytest.mark.parametrize("dim,order,level,base,nc,n0", CASES)
def test_variational_property(oracle_mod, dim, order, level, base, nc, n0):
    O = oracle_mod
    a = _pair(O, dim, order, level, base, nc, n0, False)
    b = _pair(O, dim, order, level, base, nc, n0, True)
    assert np.array_equal(a.matrix(level), b.matrix(level))     # the top level is assembled in both
    for lev in range(base, level):
        A, B = a.matrix(lev), b.matrix(lev)
        assert np.max(np.abs(A - B)) <= 1e-13 * np.max(np.abs(A)), lev


def test_galerkin_q2_hierarchy_preconditions_cg(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(2)
    k = np.exp(rng.standard_normal(8 ** 3))
    o = _pair(O, 3, 2, 3, 1, 1, 1, True, k=k)
    r = o.solve(O.solve_cfg(method=O.METHOD_CG_MG, damp=0.6, pre=2, post=2, compat=False, rtol=1e-10,
                            maxsteps=100))
    assert r.status == 0 and r.steps <= 40, r.steps
