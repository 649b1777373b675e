"""Algebraic hierarchies for the tests: compressed rows of the level matrices
and interpolations, either read off a structured oracle hierarchy (so the
algebraic solve can be held against the structured one) or built for an
irregular problem with no grid behind it."""
import numpy as np
import scipy.sparse as sp

from gnu_femlisp_b200.core import slots_to_csr


def csr_of(m):
    m = sp.csr_matrix(m)
    m.sum_duplicates()
    m.eliminate_zeros()
    m.sort_indices()
    return m.indptr.astype(np.int64), m.indices.astype(np.int32), m.data.astype(np.float64)


def prolongation(o, coarse_level):
    """The oracle's constrained interpolation from coarse_level as a matrix
    (columns = prolongated unit vectors)."""
    nc_, nf = o.nnodes(coarse_level), o.nnodes(coarse_level + 1)
    P = np.zeros((nf, nc_))
    for j in range(nc_):
        e = np.zeros(nc_)
        e[j] = 1.0
        P[:, j] = o.prolongate(e, np.zeros(nf), coarse_level, constrained=True)
    return P


def from_structured(o, dim, order):
    """(sizes, {level: A csr}, {fine level: P csr}, rhs) of an assembled
    structured oracle hierarchy, levels renumbered from 0 at its base."""
    base, top = o.base, o.top
    sizes = [o.nnodes(l) for l in range(base, top + 1)]
    mats = {l - base: slots_to_csr(o.matrix(l), dim, order) for l in range(base, top + 1)}
    interp = {l - base: csr_of(prolongation(o, l - 1)) for l in range(base + 1, top + 1)}
    return sizes, mats, interp, o.rhs()


def irregular(n=600, levels=3, seed=0):
    """A weighted graph Laplacian plus a small shift on n random points
    (k nearest neighbours, no grid), smoothed-aggregation interpolations
    (pairs of unknowns after a random permutation, then consecutive pairs,
    the tentative prolongator smoothed by one damped Jacobi step) and
    Galerkin coarse matrices P^T A P."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    d2 = ((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
    nb = np.argsort(d2, axis=1)[:, 1:6]
    rows = np.repeat(np.arange(n), 5)
    cols = nb.ravel()
    w = np.exp(rng.standard_normal(rows.size))
    W = sp.coo_matrix((w, (rows, cols)), shape=(n, n)).tocsr()
    W = W + W.T
    A = sp.diags(np.asarray(W.sum(axis=1)).ravel() + 1e-2) - W
    mats_dense = [A.tocsr()]
    interps = []
    size = n
    perm = rng.permutation(n)
    for _ in range(levels - 1):
        nc_ = (size + 1) // 2
        agg = np.empty(size, dtype=np.int64)
        agg[perm[:size] if size == n else np.arange(size)] = np.arange(size) // 2
        P0 = sp.coo_matrix((np.ones(size), (np.arange(size), agg)), shape=(size, nc_)).tocsr()
        Af = mats_dense[-1]
        P = (P0 - (2.0 / 3.0) * sp.diags(1.0 / Af.diagonal()) @ Af @ P0).tocsr()  # smoothed aggregation
        interps.append(P)
        mats_dense.append((P.T @ mats_dense[-1] @ P).tocsr())
        size = nc_
    mats_dense = mats_dense[::-1]
    interps = interps[::-1]
    sizes = [m.shape[0] for m in mats_dense]
    mats = {l: csr_of(m) for l, m in enumerate(mats_dense)}
    interp = {l + 1: csr_of(P) for l, P in enumerate(interps)}
    rhs = rng.standard_normal(n)
    return sizes, mats, interp, rhs


def oracle_of(O, sizes, mats, interp, rhs):
    o = O.Oracle.algebraic(sizes)
    for l, (s_, i_, v_) in mats.items():
        o.set_csr_matrix(l, s_, i_, v_)
    for l, (s_, i_, v_) in interp.items():
        o.set_interpolation(l, s_, i_, v_)
    return o.finish(rhs)
