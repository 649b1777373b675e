"""Locally refined 2D Q1 hierarchies with hanging nodes
(gnu_femlisp_b200.adaptive), checked against the mathematics they restate
and solved by the oracle's algebraic hierarchy:

* the meshes are 2:1 balanced and do carry hanging vertices;
* with the hanging-node constraints eliminated (constraints.lisp:78-151) the
  space holds the bilinear functions exactly: constants are in the kernel of
  the stiffness matrix, and u^T A u is the energy of x, x + 2y and xy (1, 5
  and 2/3); the load vector of f = 1 sums to the area;
* the constrained nodal interpolation (constraints.lisp:58-72) reproduces
  bilinear functions, and, as the coarse space is a subspace of the fine
  one, P^T A_fine P equals the re-discretised coarse matrix (the Galerkin
  identity) on the unknowns off the Dirichlet boundary;
* CG preconditioned by the V-cycle over these levels (Jacobi, multicolour
  SOR, one-unknown SSC) converges in few steps, independently of the depth
  of the refinement, to the sparse direct solution, and the discrete
  solution of -Laplace u = 2 pi^2 sin(pi x) sin(pi y) approaches the exact
  one as the mesh is refined."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from _hier import oracle_of
from gnu_femlisp_b200 import adaptive as AD


def _mat(triple, n, m=None):
    s, i, v = triple
    return sp.csr_matrix((v, i, s), shape=(n, n if m is None else m))


@pytest.fixture(scope="module")
def hier():
    return AD.hierarchy(n0=4, levels=5)


def test_meshes_balanced_with_hanging_vertices(hier):
    sizes, mats, interp, rhs, meshes = hier
    assert sizes == sorted(sizes) and len(set(sizes)) == len(sizes)
    top = meshes[-1]
    assert {c[0] for c in top.leaves} == set(range(1, 6))
    order_, free = AD._space(top)[1], AD._space(top)[3]
    assert len(order_) - len(free) > 10  # hanging vertices
    n = top.n0 << top.depth
    for c in top.leaves:
        x, y, s = top.span(c)
        for X, Y in ((x - 1, y), (x + s, y), (x, y - 1), (x, y + s)):
            if 0 <= X < n and 0 <= Y < n:
                assert abs(top.leaf_at(X, Y)[0] - c[0]) <= 1


@pytest.mark.parametrize("level", [1, 3, 5])
def test_energy_of_bilinear_functions(hier, level):
    mesh = hier[4][level]
    A, b, free, _ = AD.level_system(mesh, lambda x, y: 1.0, boundary=False)
    n = mesh.n0 << mesh.depth
    X = np.array([v[0] for v in free]) / n
    Y = np.array([v[1] for v in free]) / n
    assert np.abs(A @ np.ones(len(free))).max() < 1e-13
    for u, e in ((X, 1.0), (X + 2 * Y, 5.0), (X * Y, 2.0 / 3.0)):
        assert abs(u @ (A @ u) - e) < 1e-12
    assert abs(b.sum() - 1.0) < 1e-14


@pytest.mark.parametrize("level", [1, 3, 5])
def test_interpolation_reproduces_bilinear_functions(hier, level):
    meshes = hier[4]
    _, _, cfree, cdir = AD.level_system(meshes[level - 1], lambda x, y: 1.0)
    _, _, ffree, fdir = AD.level_system(meshes[level], lambda x, y: 1.0)
    P = AD.interpolation(meshes[level - 1], cfree, np.zeros(len(cfree), bool), ffree, np.zeros(len(ffree), bool))
    n = meshes[0].n0 << meshes[0].depth
    for fn in (lambda x, y: 1.0 + 0 * x, lambda x, y: x - 3 * y, lambda x, y: x * y):
        uc = fn(np.array([v[0] for v in cfree]) / n, np.array([v[1] for v in cfree]) / n)
        uf = fn(np.array([v[0] for v in ffree]) / n, np.array([v[1] for v in ffree]) / n)
        assert np.abs(P @ uc - uf).max() < 1e-14


def test_galerkin_identity(hier):
    sizes, mats, interp, rhs, meshes = hier
    for l in range(1, len(sizes)):
        P = _mat(interp[l], sizes[l], sizes[l - 1])
        G = (P.T @ _mat(mats[l], sizes[l]) @ P).toarray()
        Ac = _mat(mats[l - 1], sizes[l - 1]).toarray()
        inner = ~AD.level_system(meshes[l - 1], lambda x, y: 1.0)[3]
        assert np.abs(G[np.ix_(inner, inner)] - Ac[np.ix_(inner, inner)]).max() < 1e-14


@pytest.mark.parametrize("smoother,damp", [("jacobi", 0.6), ("sor", 1.0), ("ssc", 1.0)])
def test_oracle_cg_mg_on_the_hierarchy(oracle_mod, smoother, damp):
    O = oracle_mod
    steps = []
    for levels in (4, 6):
        sizes, mats, interp, rhs, _ = AD.hierarchy(n0=4, levels=levels,
                                                   kcoef=lambda x, y: 1.0 + 9.0 * (x > 0.5) * (y > 0.5))
        o = oracle_of(O, sizes, mats, interp, rhs)
        sm = {"jacobi": O.JACOBI, "sor": O.SOR, "ssc": O.SSC}[smoother]
        r = o.solve(O.solve_cfg(method=O.METHOD_CG_MG, smoother=sm, damp=damp, pre=1, post=1, compat=False,
                                rtol=1e-10, maxsteps=100))
        assert r.status == 0
        A = _mat(mats[levels], sizes[-1]).tocsc()
        exact = spla.spsolve(A, rhs)
        assert np.abs(r.x - exact).max() <= 1e-8 * np.abs(exact).max()
        steps.append(r.steps)
    assert max(steps) <= 16 and steps[1] <= steps[0] + 3, steps


def test_discretisation_converges_to_the_continuum():
    """-Laplace u = 2 pi^2 sin(pi x) sin(pi y), u = sin(pi x) sin(pi y):
    refined everywhere once more, the nodal error falls by about 4."""
    def f(x, y):
        return 2 * np.pi ** 2 * np.sin(np.pi * x) * np.sin(np.pi * y)
    errs = []
    for uniform in (2, 3):
        def refine(l, xc, yc, side, uniform=uniform):
            return l <= uniform or (xc * xc + yc * yc) ** 0.5 < 0.25 + side
        mesh_levels = uniform + 2
        sizes, mats, interp, rhs, meshes = AD.hierarchy(n0=2, levels=mesh_levels, refine=refine, f=f)
        A = _mat(mats[mesh_levels], sizes[-1]).tocsc()
        u = spla.spsolve(A, rhs)
        free = AD._space(meshes[-1])[3]
        n = meshes[-1].n0 << meshes[-1].depth
        ex = np.array([np.sin(np.pi * v[0] / n) * np.sin(np.pi * v[1] / n) for v in free])
        errs.append(np.abs(u - ex).max())
    assert errs[0] < 0.05 and 3.0 < errs[0] / errs[1] < 5.0, errs
