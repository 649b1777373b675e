"""The drop-in path of the Python mirror, driven the way Femlisp's own
<linear-solver> loop drives an iterator (linsolve.lisp:58-73,
solve.lisp:139-155): make_iterator of a GeometricCS (one fmg_vcycle per
iterate) and of a CG (fmg_cg_start / fmg_cg_step), each step's :defnorm taken
on the host from the returned residual.  The iterates are those of the
library's own loop (fmg_solve) bit for bit; the host-side norms agree with
the device's to rounding.  The vector (elasticity) form reaches the GPU
through discretize_globally and solve like the scalar one, and matches the
oracle bitwise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def I():
    from gnu_femlisp_b200 import iteration as I
    return I


@pytest.fixture(scope="module")
def ctx():
    import gnu_femlisp_b200 as G
    return G.Context(0)


def _system(I, ctx, dim=2, level=6):
    prob = I.cdr_model_problem(dim)
    return I.discretize_globally(prob, I.uniformly_refined_hierarchical_mesh(dim, level), I.lagrange_fe(1), ctx)


def test_cg_iterator_steps_like_the_device_loop(I, ctx):
    A, b = _system(I, ctx)
    cs = I.geometric_cs(smoother=I.Jacobi(0.6), pre_steps=1, post_steps=1, base_level=0)
    solver = I.LinearSolver(I.CG(preconditioner=cs), "(< :reduction 1.0e-10)", "(> :step 100)")
    it = I.solve_iterating({"matrix": A, "rhs": b, "solver": solver})
    ref = I.solve({"matrix": A, "rhs": b, "solver": solver})
    assert it["report"].status == ref["report"].status == "success"
    assert it["report"].steps == ref["report"].steps
    assert np.array_equal(it["solution"], ref["solution"])          # the same device arithmetic
    rel = np.max(np.abs(it["history"] - ref["history"]) / ref["history"])
    assert rel <= 1e-13, rel                                        # host norm vs the device reduction


def test_cg_iterator_with_the_alias(I, ctx):
    # (iterate q w w): rhs and residual of the preconditioner aliased
    A, b = _system(I, ctx, level=4)
    cs = I.geometric_cs(smoother=I.Jacobi(0.5), pre_steps=1, post_steps=0, base_level=0,
                        combination="additive")
    solver = I.LinearSolver(I.CG(preconditioner=cs, compat_alias=True), "(< :reduction 1.0e-10)",
                            "(> :step 60)")
    it = I.solve_iterating({"matrix": A, "rhs": b, "solver": solver})
    ref = I.solve({"matrix": A, "rhs": b, "solver": solver})
    assert it["report"].steps == ref["report"].steps
    assert np.array_equal(it["solution"], ref["solution"])


def test_mg_iterator_steps_like_the_device_loop(I, ctx):
    A, b = _system(I, ctx, dim=3, level=4)
    cs = I.geometric_cs(smoother=I.Jacobi(0.6), pre_steps=2, post_steps=2, base_level=1)
    solver = I.LinearSolver(cs, "(< :reduction 1.0e-8)", "(> :step 100)")
    it = I.solve_iterating({"matrix": A, "rhs": b, "solver": solver})
    ref = I.solve({"matrix": A, "rhs": b, "solver": solver})
    assert it["report"].steps == ref["report"].steps and it["report"].status == "success"
    assert np.array_equal(it["solution"], ref["solution"])


def test_mg_iterator_alias_matches_the_oracle(I, ctx, oracle_mod):
    # one application with b and r the same array, as <cg> calls its preconditioner
    O = oracle_mod
    A, b = _system(I, ctx, dim=2, level=5)
    cs = I.geometric_cs(smoother=I.Jacobi(0.6), pre_steps=1, post_steps=1, base_level=0)
    it = I.make_iterator(cs, A)
    rng = np.random.default_rng(4)
    w = rng.standard_normal(b.size)
    w[np.abs(b) == 0] = 0.0                      # Dirichlet rows carry no residual
    q = np.zeros_like(w)
    w0 = w.copy()
    it.iterate(q, w, w)
    o = O.Oracle(2, 1, 5, base_level=0).assemble()
    xo, bo, _ = o.vcycle(O.solve_cfg(method=O.METHOD_MG, damp=0.6, compat=True), np.zeros_like(w0), w0)
    assert np.array_equal(q, xo) and np.array_equal(w, bo)


def test_elasticity_through_the_mirror_matches_the_oracle(I, ctx, oracle_mod):
    O = oracle_mod
    n0, level = 3, 1
    ncell = (n0 << level) ** 3
    e = np.exp(0.5 * np.random.default_rng(9).standard_normal(ncell))
    prob = I.elasticity_model_problem(3, lame=e)
    A, b = I.discretize_globally(prob, I.uniformly_refined_hierarchical_mesh(3, level, n0=n0),
                                 I.lagrange_fe(2, nr_comps=3), ctx)
    cs = I.geometric_cs(smoother=I.Jacobi(0.6), pre_steps=2, post_steps=2, base_level=0)
    solver = I.LinearSolver(I.CG(preconditioner=cs), "(< :reduction 1.0e-10)", "(> :step 200)")
    out = I.solve({"matrix": A, "rhs": b, "solver": solver})
    o = O.Oracle(3, 2, level, base_level=0, ncomp=3, n0=n0, dirichlet_mask=0b000001)
    o.set_coefficient(O.LAMBDA_MU_CELL, e)
    o.set_coefficient(O.F_VEC, [0.0, 0.0, -1.0])
    o.assemble()
    ref = o.solve(O.solve_cfg(method=O.METHOD_CG_MG, damp=0.6, pre=2, post=2, compat=False, rtol=1e-10,
                              maxsteps=200))
    assert out["report"].status == "success" and out["report"].steps == ref.steps
    assert np.array_equal(out["history"], ref.history) and np.array_equal(out["solution"], ref.x)
    # and the iterator path of the same system
    it = I.solve_iterating({"matrix": A, "rhs": b, "solver": solver})
    assert it["report"].steps == ref.steps and np.array_equal(it["solution"], ref.x)
