"""Level matrices uploaded through fmg_set_matrix (the parity path for
matrices Femlisp assembles itself, handed over in the compressed-column form
of sparse-matrix->ccs, sparselu.lisp:226-263).

- Round trip: the CSR / CCS of every level of an assembled grid, uploaded
  into a fresh grid, gives back the same slot storage bitwise and the same
  CG + V-cycle history bitwise (scalar Q1 and Q2, the elasticity blocks).
- The oracle's own matrices, uploaded, solve with the oracle's history.
- A Q2 Galerkin hierarchy (I^T A I with the constrained interpolation,
  geomg.lisp:122-123), formed on the host, solves on the GPU with the same
  history as the oracle given the same matrices.
- Malformed input fails with FMG_ERR_ARG, an incomplete hierarchy with
  FMG_ERR_STATE.
"""
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


def _cfg(G, smoother=0, damp=0.6, pre=1, post=1, rtol=1e-10, maxsteps=200):
    C = G._capi
    # a separate residual for the preconditioner (with the alias of krylow.lisp:120
    # CG stagnates under the multiplicative cycle)
    return G.SolveCfg(C.FMG_METHOD_CG_MG, smoother, damp, pre, post, 1, 0, 1.0, rtol, 0.0, maxsteps,
                      C.FMG_MULTIPLICATIVE, 0)


def _upload_all(G, ctx, src, layout="csr", **kw):
    g = G.Grid(ctx, src.dim, src.order, src.top, base_level=src.base, **kw)
    for l in range(src.base, src.top + 1):
        start, index, values = src.matrix_csr(l)
        if layout == "ccs":  # the transpose's rows are the columns
            import scipy.sparse as sp
            n = start.size - 1
            m = sp.csr_matrix((values, index, start), shape=(n, n)).tocsc()
            start, index, values = m.indptr, m.indices, m.data
        g.set_matrix(l, start, index, values, layout=layout)
    g.set_rhs(src.rhs())
    return g


def _solve(G, g, cfg):
    x = g.vector()
    hist, steps, st = g.solve(cfg, x)
    return hist, x.get(), st


def _kgrid(G, ctx, dim, order, level, base, seed, **kw):
    g = G.Grid(ctx, dim, order, level, base_level=base, **kw)
    k = np.exp(np.random.default_rng(seed).standard_normal((1 << level) ** dim))
    g.set_coefficient(G._capi.FMG_K_CELL, k)
    return g.assemble()


@pytest.mark.parametrize("dim,order,level,base,layout,smoother", [
    (3, 1, 4, 1, "csr", 0), (2, 1, 5, 1, "ccs", 0), (2, 2, 4, 1, "csr", 1), (3, 2, 3, 1, "ccs", 1)])
def test_round_trip_scalar(G, ctx, dim, order, level, base, layout, smoother):
    a = _kgrid(G, ctx, dim, order, level, base, seed=dim + order)
    b = _upload_all(G, ctx, a, layout=layout)
    for l in range(base, level + 1):
        assert np.array_equal(a.matrix(l), b.matrix(l)), l
    cfg = _cfg(G) if smoother == 0 else _cfg(G, smoother=1, damp=1.0, pre=2, post=2)
    ha, xa, sa = _solve(G, a, cfg)
    hb, xb, sb = _solve(G, b, cfg)
    assert sa == 0 and sb == 0
    assert np.array_equal(ha, hb) and np.array_equal(xa, xb)


def test_round_trip_elasticity(G, ctx):
    C = G._capi
    a = G.Grid(ctx, 3, 2, 1, base_level=0, n0=2, ncomp=3, dirichlet_mask=0b000001)
    e = np.exp(0.5 * np.random.default_rng(4).standard_normal((2 << 1) ** 3))
    a.set_coefficient(C.FMG_LAMBDA_MU_CELL, e)
    a.set_coefficient(C.FMG_F_VEC, [0.0, 0.0, -1.0])
    a.assemble()
    b = _upload_all(G, ctx, a, n0=2, ncomp=3, dirichlet_mask=0b000001)
    for l in range(0, 2):
        assert np.array_equal(a.matrix(l), b.matrix(l)), l
    cfg = _cfg(G, damp=0.5, pre=2, post=2)
    ha, xa, sa = _solve(G, a, cfg)
    hb, xb, sb = _solve(G, b, cfg)
    assert sa == 0 and np.array_equal(ha, hb) and np.array_equal(xa, xb)


def test_oracle_matrices_solve_like_the_oracle(oracle_mod, G, ctx):
    O = oracle_mod
    o = O.Oracle(3, 1, 4, base_level=1)
    k = np.exp(np.random.default_rng(9).standard_normal(16 ** 3))
    o.set_coefficient(O.K_CELL, k)
    o.assemble()
    g = G.Grid(ctx, 3, 1, 4, base_level=1)
    for l in range(1, 5):
        g.set_matrix(l, *G.slots_to_csr(o.matrix(l), 3, 1))
    g.set_rhs(o.rhs())
    r = o.solve(O.solve_cfg(damp=0.6, compat=False))
    hist, x, st = _solve(G, g, _cfg(G))
    assert st == 0 and np.array_equal(hist, r.history) and np.array_equal(x, r.x)


def _prolongation(O, o, coarse_level):
    nc_, nf = o.nnodes(coarse_level), o.nnodes(coarse_level + 1)
    P = np.zeros((nf, nc_))
    for j in range(nc_):
        e = np.zeros(nc_)
        e[j] = 1.0
        P[:, j] = o.prolongate(e, np.zeros(nf), coarse_level, constrained=True)
    return P


def _dense_to_slots(A, dim, order):
    w = 2 * order + 1
    N = A.shape[0]
    M = int(round(N ** (1.0 / dim)))
    idx = np.arange(N)
    c = np.stack([(idx // M ** d) % M for d in range(dim)], 1)
    S = np.zeros((w ** dim, N))
    for s in range(w ** dim):
        off = np.array([(s // w ** d) % w - order for d in range(dim)])
        cj = c + off
        ok = np.all((cj >= 0) & (cj < M), 1)
        j = sum(cj[:, d] * M ** d for d in range(dim))
        S[s, ok] = A[idx[ok], j[ok]]
    return S


def _slots_to_dense(S, dim, order):
    start, index, values = __import__("gnu_femlisp_b200").slots_to_csr(S, dim, order)
    n = start.size - 1
    D = np.zeros((n, n))
    for i in range(n):
        D[i, index[start[i]:start[i + 1]]] = values[start[i]:start[i + 1]]
    return D


@pytest.mark.parametrize("dim,level", [(2, 4), (3, 2)])
def test_q2_galerkin_hierarchy(oracle_mod, G, ctx, dim, level):
    O = oracle_mod
    base = 1 if dim == 2 else 0
    o = O.Oracle(dim, 2, level, base_level=base)
    k = np.exp(np.random.default_rng(5).standard_normal((1 << level) ** dim))
    o.set_coefficient(O.K_CELL, k)
    o.assemble()
    mats = {level: o.matrix(level)}
    A = _slots_to_dense(mats[level], dim, 2)
    for l in range(level - 1, base - 1, -1):
        P = _prolongation(O, o, l)
        Ac = P.T @ A @ P
        dirichlet = ~np.any(P != 0.0, axis=0)
        Ac[dirichlet, dirichlet] = 1.0
        mats[l] = _dense_to_slots(Ac, dim, 2)
        assert np.array_equal(_slots_to_dense(mats[l], dim, 2), Ac), "Galerkin product outside the Q2 stencil"
        A = Ac
    rhs = o.rhs()
    o.set_levels(mats, rhs)
    g = G.Grid(ctx, dim, 2, level, base_level=base)
    for l, S in mats.items():
        g.set_matrix(l, *G.slots_to_csr(S, dim, 2))
    g.set_rhs(rhs)
    for l in mats:
        assert np.array_equal(g.matrix(l), o.matrix(l)), l
    r = o.solve(O.solve_cfg(smoother=O.SOR, damp=1.2, pre=2, post=2, compat=False))
    hist, x, st = _solve(G, g, _cfg(G, smoother=1, damp=1.2, pre=2, post=2))
    assert st == 0 and r.status == 0
    assert np.array_equal(hist, r.history) and np.array_equal(x, r.x)


def test_upload_errors(G, ctx):
    g = G.Grid(ctx, 2, 1, 3, base_level=1)
    n = g.nnodes(3)
    eye = (np.arange(n + 1), np.arange(n), np.ones(n))
    with pytest.raises(G.FmgError) as e:  # wrong row count
        g.set_matrix(3, np.arange(n), np.arange(n - 1), np.ones(n - 1))
    assert e.value.code == -1
    with pytest.raises(G.FmgError) as e:  # coupling of distance 2 in a Q1 level
        g.set_matrix(3, np.r_[0, np.arange(2, n + 2)], np.r_[0, 2, np.arange(1, n)], np.ones(n + 1))
    assert e.value.code == -1
    with pytest.raises(G.FmgError) as e:  # column index out of range
        g.set_matrix(3, eye[0], np.r_[np.arange(n - 1), n], eye[2])
    assert e.value.code == -1
    g.set_matrix(3, *eye)  # an explicit zero outside the stencil is dropped
    g.set_matrix(3, np.r_[0, np.arange(2, n + 2)], np.r_[0, 2, np.arange(1, n)], np.r_[1.0, 0.0, np.ones(n - 1)])
    x = g.vector()
    with pytest.raises(G.FmgError) as e:  # levels 1, 2 missing
        g.solve(_cfg(G), x)
    assert e.value.code == -3
    for l in (1, 2):
        m = g.nnodes(l)
        g.set_matrix(l, np.arange(m + 1), np.arange(m), np.ones(m))
    g.set_rhs(np.ones(n))
    hist, steps, st = g.solve(_cfg(G), x)  # identity at every level
    assert st == 0 and np.allclose(x.get(), 1.0)
