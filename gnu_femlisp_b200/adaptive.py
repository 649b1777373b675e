"""Multilevel systems of adaptively refined meshes with hanging nodes, formed
on the host as Femlisp forms them, for the algebraic-grid path
(fmg_grid_create_algebraic): 2D Q1 on the unit square, a quadtree of cells
refined level by level where a predicate asks for it (kept 2:1 balanced),
the level matrices re-discretised on every level's mesh with the hanging-node
constraints eliminated, the Dirichlet boundary as identity rows, and the
constrained nodal interpolation between consecutive levels.

Restated from the reference: hanging-node constraints (constraints.lisp:78-151:
a hanging vertex, the midpoint of an edge of a coarser neighbour cell, takes
the mean of that edge's end values; eliminate-hanging-node-constraints-from-matrix
forms C^T A C), the Dirichlet identity rows (constraints.lisp:323-411), the
constrained interpolation matrix (constraints.lisp:58-72, fetransfer.lisp:73-195:
nodal values of the coarse function, rows of constrained fine unknowns and
columns of constrained coarse ones empty) and the multilevel decomposition
(geomg.lisp:109-142: one system per level of the refinement hierarchy)."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

# the Q1 stiffness of a square cell (independent of its size in 2D) and the
# local vertex order (0,0), (1,0), (0,1), (1,1)
_KQ1 = np.array([[4.0, -1.0, -1.0, -2.0],
                 [-1.0, 4.0, -2.0, -1.0],
                 [-1.0, -2.0, 4.0, -1.0],
                 [-2.0, -1.0, -1.0, 4.0]]) / 6.0


class Mesh:
    """The leaves of a quadtree over the unit square, n0 x n0 root cells;
    a cell is (level, i, j) with side 1/(n0 2^level).  Vertices are points
    of the lattice of the finest possible level `depth` (integer coordinates,
    spacing 1/(n0 2^depth))."""

    def __init__(self, n0: int, depth: int):
        self.n0, self.depth = n0, depth
        self.leaves = {(0, i, j) for i in range(n0) for j in range(n0)}

    def span(self, c):
        lev, i, j = c
        s = 1 << (self.depth - lev)
        return i * s, j * s, s  # lower-left corner on the finest lattice, side

    def refine(self, cells):
        for c in cells:
            if c in self.leaves:
                lev, i, j = c
                self.leaves.remove(c)
                for di in (0, 1):
                    for dj in (0, 1):
                        self.leaves.add((lev + 1, 2 * i + di, 2 * j + dj))

    def leaf_at(self, X, Y):
        """The leaf containing the finest-lattice point (X, Y) (lower-left
        convention: the leaf whose half-open box [x, x+s) x [y, y+s) holds
        it, boxes at the upper domain edges closed)."""
        top = self.n0 << self.depth
        for lev in range(self.depth + 1):
            s = 1 << (self.depth - lev)
            i, j = min(X // s, (top - 1) // s), min(Y // s, (top - 1) // s)
            if (lev, i, j) in self.leaves:
                return (lev, i, j)
        raise KeyError((X, Y))

    def balance(self):
        """Refine until neighbouring leaves differ by at most one level."""
        while True:
            todo = set()
            for c in self.leaves:
                x, y, s = self.span(c)
                for (X, Y) in ((x - 1, y), (x + s, y), (x, y - 1), (x, y + s)):
                    if 0 <= X < (self.n0 << self.depth) and 0 <= Y < (self.n0 << self.depth):
                        nb = self.leaf_at(X, Y)
                        if nb[0] < c[0] - 1:
                            todo.add(nb)
            if not todo:
                return
            self.refine(todo)


def _space(mesh: Mesh):
    """Vertices, free (unconstrained) vertices and the constraint matrix of
    the Q1 space on the mesh's leaves: C maps the free vertex values to all
    vertex values (hanging vertices: the mean of the coarse edge's ends)."""
    top = mesh.n0 << mesh.depth
    verts = set()
    cells = sorted(mesh.leaves, key=lambda c: (c[0], c[2], c[1]))
    for c in cells:
        x, y, s = mesh.span(c)
        verts.update({(x, y), (x + s, y), (x, y + s), (x + s, y + s)})
    # hanging: a vertex interior to an edge of a leaf
    hang = {}
    for c in cells:
        x, y, s = mesh.span(c)
        h = s // 2
        if h == 0:
            continue
        for (a, b, m) in (((x, y), (x + s, y), (x + h, y)), ((x, y + s), (x + s, y + s), (x + h, y + s)),
                          ((x, y), (x, y + s), (x, y + h)), ((x + s, y), (x + s, y + s), (x + s, y + h))):
            if m in verts:
                hang[m] = (a, b)
    order = sorted(verts, key=lambda v: (v[1], v[0]))
    free = [v for v in order if v not in hang]
    fidx = {v: k for k, v in enumerate(free)}
    vidx = {v: k for k, v in enumerate(order)}
    rows, cols, vals = [], [], []
    for v in order:
        if v in hang:
            for w in hang[v]:
                rows.append(vidx[v]); cols.append(fidx[w]); vals.append(0.5)
        else:
            rows.append(vidx[v]); cols.append(fidx[v]); vals.append(1.0)
    C = sp.csr_matrix((vals, (rows, cols)), shape=(len(order), len(free)))
    return cells, order, vidx, free, fidx, C, top


def level_system(mesh: Mesh, kcoef, f=1.0, boundary: bool = True):
    """The Q1 system of -div(k grad u) = f, u = 0 on the boundary, on the
    mesh's leaves: assembled over all vertices, the hanging-node constraints
    eliminated (C^T A C, C^T b), Dirichlet rows made identity rows with their
    columns removed (``boundary=False``: left as assembled).  kcoef(xc, yc) is
    the coefficient of the cell with centre (xc, yc); f a number or f(x, y),
    integrated by the vertex rule (a quarter of the cell's area at each
    vertex).  Returns (A csr over the free vertices, b, free vertices,
    Dirichlet flags)."""
    cells, order, vidx, free, fidx, C, top = _space(mesh)
    n = len(order)
    rows, cols, vals = [], [], []
    b = np.zeros(n)
    hgrid = 1.0 / top
    fv = f if callable(f) else (lambda x, y: f)
    for c in cells:
        x, y, s = mesh.span(c)
        corners = ((x, y), (x + s, y), (x, y + s), (x + s, y + s))
        loc = [vidx[v] for v in corners]
        k = kcoef((x + s / 2) * hgrid, (y + s / 2) * hgrid)
        area = (s * hgrid) ** 2
        for a in range(4):
            b[loc[a]] += fv(corners[a][0] * hgrid, corners[a][1] * hgrid) * area / 4.0
            for q in range(4):
                rows.append(loc[a]); cols.append(loc[q]); vals.append(k * _KQ1[a, q])
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    Af = (C.T @ A @ C).tocsr()
    bf = C.T @ b
    dirichlet = np.array([v[0] in (0, top) or v[1] in (0, top) for v in free])
    if not boundary:
        Af.sum_duplicates()
        Af.sort_indices()
        return Af, bf, free, dirichlet
    D = sp.diags((~dirichlet).astype(float))
    Af = (D @ Af @ D + sp.diags(dirichlet.astype(float))).tocsr()
    bf = np.where(dirichlet, 0.0, bf)
    Af.sum_duplicates()
    Af.eliminate_zeros()
    Af.sort_indices()
    return Af, bf, free, dirichlet


def interpolation(coarse: Mesh, coarse_free, coarse_dir, fine_free, fine_dir):
    """The constrained nodal interpolation from the coarse mesh's free
    vertices to the fine mesh's: the coarse Q1 function (hanging vertices
    through their constraints) evaluated at each fine free vertex; rows of
    fine Dirichlet vertices and columns of coarse Dirichlet vertices empty."""
    cells, order, vidx, free, fidx, C, top = _space(coarse)
    assert free == list(coarse_free)
    rows, cols, vals = [], [], []
    for r, (X, Y) in enumerate(fine_free):
        if fine_dir[r]:
            continue
        lev, i, j = coarse.leaf_at(X, Y)
        x, y, s = coarse.span((lev, i, j))
        tx, ty = (X - x) / s, (Y - y) / s
        wts = ((1 - tx) * (1 - ty), tx * (1 - ty), (1 - tx) * ty, tx * ty)
        for wv, v in zip(wts, ((x, y), (x + s, y), (x, y + s), (x + s, y + s))):
            if wv == 0.0:
                continue
            crow = C.getrow(vidx[v])
            for cj, cw in zip(crow.indices, crow.data):
                if not coarse_dir[cj]:
                    rows.append(r); cols.append(cj); vals.append(wv * cw)
    P = sp.csr_matrix((vals, (rows, cols)), shape=(len(fine_free), len(coarse_free)))
    P.sum_duplicates()
    P.eliminate_zeros()
    P.sort_indices()
    return P


def hierarchy(n0: int = 4, levels: int = 4, refine=None, kcoef=None, f=1.0):
    """The multilevel system of a mesh refined `levels` times: level 0 the
    n0 x n0 root mesh, level l the mesh after the l-th refinement of the
    leaves refine(l, xc, yc, side) selects (default: uniform first, then the
    cells within 0.3 of the corner (0, 0)), 2:1 balanced.  Returns (sizes,
    {level: (start, index, values)}, {fine level: (start, index, values)},
    rhs of the top level, meshes) in the form AlgebraicSystem and the
    oracle's algebraic hierarchy take."""
    if refine is None:
        def refine(l, xc, yc, side):
            return l == 1 or (xc * xc + yc * yc) ** 0.5 < 0.3 + side
    if kcoef is None:
        def kcoef(xc, yc):
            return 1.0
    mesh = Mesh(n0, levels)
    meshes, systems = [], []
    for l in range(levels + 1):
        if l > 0:
            top = n0 << levels
            pick = []
            for c in mesh.leaves:
                x, y, s = mesh.span(c)
                if c[0] == l - 1 and refine(l, (x + s / 2) / top, (y + s / 2) / top, s / top):
                    pick.append(c)
            mesh.refine(pick)
            mesh.balance()
        snap = Mesh(n0, levels)
        snap.leaves = set(mesh.leaves)
        meshes.append(snap)
        systems.append(level_system(snap, kcoef, f))
    sizes = [len(s[2]) for s in systems]

    def csr(m):
        return m.indptr.astype(np.int64), m.indices.astype(np.int32), m.data.astype(np.float64)
    mats = {l: csr(systems[l][0]) for l in range(levels + 1)}
    interp = {l: csr(interpolation(meshes[l - 1], systems[l - 1][2], systems[l - 1][3], systems[l][2],
                                   systems[l][3]))
              for l in range(1, levels + 1)}
    return sizes, mats, interp, systems[-1][1], meshes


def system(n0: int = 4, levels: int = 4, refine=None, kcoef=None, f=1.0, ctx=None):
    """The hierarchy as the blackboard solve's matrix: an AlgebraicSystem of
    order 1 (select-smoother's Gauss-Seidel by default), to be solved with
    local_mg / a CG preconditioned by it."""
    from .iteration import AlgebraicSystem
    sizes, mats, interp, rhs, _ = hierarchy(n0, levels, refine, kcoef, f)
    return AlgebraicSystem([mats[l] for l in range(len(sizes))], [interp[l] for l in range(1, len(sizes))], rhs,
                           ctx=ctx, order=1)
