"""Host-side mirror of Femlisp's problem, discretization and iteration API
for the multigrid solve path, running on the B200 through libfmgpu.

The names and meanings follow the reference so that code written against
Femlisp reads the same here:

  cdr_model_problem                 src/problem/cdr.lisp:153-204
  uniformly_refined_hierarchical_mesh  src/mesh/meshgen.lisp:180-183
  lagrange_fe                       src/discretization/lagrange.lisp:176-202
  discretize_globally               src/discretization/fedisc.lisp:307-316
  Jacobi, SOR, GaussSeidel, LU      src/iteration/linit.lisp:132-385
  geometric_cs / GeometricCS        src/iteration/geomg.lisp:148-155,
                                    multigrid.lisp:55-70
  local_mg / LocalMG                src/iteration/geomg.lisp:161-168 (on an
                                    AlgebraicSystem of a locally refined mesh)
  CG                                src/iteration/krylow.lisp:67-132
  LinearSolver, solve               src/iteration/linsolve.lisp:40-73,
                                    solve.lisp:113-164, iterate.lisp:105-250
  elasticity_model_problem          src/problem/elasticity.lisp:71-123
  Iterator, make_iterator           src/iteration/linit.lisp:48-67 (<iterator>,
                                    make-iterator), multigrid.lisp:303-393,
                                    krylow.lisp:72-132
  solve_iterating                   the <linear-solver> loop driving an
                                    iterator: linsolve.lisp:58-73,
                                    solve.lisp:139-155, iterate.lisp:239-250

Success/failure conditions are given as Femlisp forms, e.g.
``"(or (< :defnorm 1.0e-12) (> :step 10))"``.  Coefficients are sampled on
the host (a Lisp coefficient closure cannot run on the device): diffusion
as a constant or one value per top-level cell, source as a constant or its
values at the Gauss points of every top-level cell.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np

from . import _capi as C
from .core import Context, Grid, Vector

# ------------------------------------------------------------------ problem


@dataclass
class CdrProblem:
    """-div(k grad u) = f on the unit dim-cube with Dirichlet data 0 on the
    faces in ``dirichlet_mask`` (cdr-model-problem defaults: k = 1, f = 1,
    u = 0 on the whole boundary)."""
    dim: int
    diffusion: Any = 1.0           # float, or array of per-cell values, or callable(x) -> k
    source: Any = 1.0              # float, or callable(x) -> f evaluated at Gauss points
    dirichlet_mask: int | None = None


def cdr_model_problem(dim: int, diffusion=None, source=None, dirichlet_mask=None) -> CdrProblem:
    return CdrProblem(dim, 1.0 if diffusion is None else diffusion, 1.0 if source is None else source,
                      dirichlet_mask)


@dataclass
class ElasticityProblem:
    """Linear elasticity -div(C : eps(u)) = f on the unit 3-cube with the
    isotropic elasticity tensor of Lame parameters lambda = mu = E
    (isotropic-elasticity-tensor, elasticity.lisp:71-88): E a constant, one
    value per top-level cell, or callable(x) at the cell centres; a constant
    body force; every component clamped (u = 0) on the faces in
    ``dirichlet_mask`` (bit 0: x = 0)."""
    dim: int
    lame: Any = 1.0
    force: tuple = (0.0, 0.0, -1.0)
    dirichlet_mask: int = 0b000001


def elasticity_model_problem(dim: int = 3, lame=None, force=None, dirichlet_mask=0b000001) -> ElasticityProblem:
    """elasticity-model-problem (elasticity.lisp:112-123) with lambda = mu = E."""
    if dim != 3:
        raise ValueError("the vector form is built for 3D")
    return ElasticityProblem(dim, 1.0 if lame is None else lame,
                             (0.0, 0.0, -1.0) if force is None else tuple(force), dirichlet_mask)


@dataclass
class Mesh:
    """Uniformly refined hierarchical mesh of the unit n-cube: level l has
    n0 * 2^l cells per direction."""
    dim: int
    level: int
    n0: int = 1


def uniformly_refined_hierarchical_mesh(dim: int, level: int, n0: int = 1) -> Mesh:
    return Mesh(dim, level, n0)


@dataclass
class LagrangeFE:
    order: int
    nr_comps: int = 1


def lagrange_fe(order: int, nr_comps: int = 1) -> LagrangeFE:
    return LagrangeFE(order, nr_comps)


def gauss_points_1d(order: int) -> np.ndarray:
    """Gauss points on [0,1] in the order of the quadrature rule
    (quadrature.lisp:202-215): (1 - t)/2 for ascending Legendre roots t."""
    if order == 1:
        t = math.sqrt(1.0 / 3.0)
        ts = [-t, t]
    else:
        t = math.sqrt(0.6)
        ts = [-t, 0.0, t]
    return np.array([0.5 * (1.0 - v) for v in ts])


def sample_at_gauss_points(f: Callable[[np.ndarray], np.ndarray], dim: int, order: int,
                           n_cells: int) -> np.ndarray:
    """Values of f at the Gauss points of every cell, layout [cell][q] with
    cells and points numbered x fastest; f maps points [..., dim] to values."""
    xi = gauss_points_1d(order)
    npt = len(xi)
    h = 1.0 / n_cells
    c = np.arange(n_cells ** dim)[:, None]
    q = np.arange(npt ** dim)[None, :]
    pts = [((c // n_cells ** k) % n_cells + xi[(q // npt ** k) % npt]) * h for k in range(dim)]
    return np.ascontiguousarray(f(np.stack(pts, axis=-1))).reshape(-1)


def cell_centres(dim: int, n_cells: int) -> np.ndarray:
    """Cell midpoints [cell, dim], cells numbered x fastest."""
    c = np.arange(n_cells ** dim)
    return np.stack([((c // n_cells ** k) % n_cells + 0.5) / n_cells for k in range(dim)], axis=-1)


class DiscreteSystem:
    """The assembled system A x = b of discretize_globally.  The level
    hierarchy is assembled on the device lazily, once per coarse level a
    solver asks for (the reference assembles coarse levels when the
    multigrid iterator is made, geomg.lisp:109-142)."""

    def __init__(self, problem, mesh: Mesh, fe: LagrangeFE, ctx: Context | None = None):
        vector = isinstance(problem, ElasticityProblem)
        if vector != (fe.nr_comps == 3):
            raise ValueError("an elasticity problem takes lagrange_fe(order, nr_comps=3), a cdr problem nr_comps=1")
        self.problem, self.mesh, self.fe = problem, mesh, fe
        self.ctx = ctx or Context()
        self._grids: dict[int, Grid] = {}

    def grid(self, base_level: int = 0) -> Grid:
        if base_level not in self._grids:
            p, m = self.problem, self.mesh
            if isinstance(p, ElasticityProblem):
                self._grids[base_level] = self._elasticity_grid(base_level)
                return self._grids[base_level]
            g = Grid(self.ctx, p.dim, self.fe.order, m.level, base_level=base_level, n0=m.n0,
                     dirichlet_mask=p.dirichlet_mask)
            ncell = g.n_cells
            k = p.diffusion
            if callable(k):
                g.set_coefficient(C.FMG_K_CELL, np.ascontiguousarray(k(cell_centres(p.dim, ncell))).ravel())
            elif np.ndim(k) == 0:
                g.set_coefficient(C.FMG_K_CONST, [float(k)])
            else:
                g.set_coefficient(C.FMG_K_CELL, np.asarray(k, dtype=np.float64).ravel())
            f = p.source
            if callable(f):
                g.set_coefficient(C.FMG_F_IP, sample_at_gauss_points(f, p.dim, self.fe.order, ncell))
            else:
                g.set_coefficient(C.FMG_F_CONST, [float(f)])
            self._grids[base_level] = g.assemble()
        return self._grids[base_level]

    def _elasticity_grid(self, base_level: int) -> Grid:
        """Vector Q1/Q2 with 3 x 3 node blocks: E per top-level cell, the body
        force, the clamped faces (ellsys-fe.lisp:68-218 with the tensor of
        elasticity.lisp:71-88)."""
        p, m = self.problem, self.mesh
        g = Grid(self.ctx, 3, self.fe.order, m.level, base_level=base_level, n0=m.n0, ncomp=3,
                 dirichlet_mask=p.dirichlet_mask)
        ncell = g.n_cells
        e = p.lame
        if callable(e):
            e = np.ascontiguousarray(e(cell_centres(3, ncell))).ravel()
        elif np.ndim(e) == 0:
            e = np.full(ncell ** 3, float(e))
        g.set_coefficient(C.FMG_LAMBDA_MU_CELL, np.asarray(e, dtype=np.float64).ravel())
        g.set_coefficient(C.FMG_F_VEC, list(p.force))
        return g.assemble()


def _csr_triple(m):
    """(start, index, values) of a scipy sparse matrix or of such a triple."""
    if hasattr(m, "tocsr"):
        m = m.tocsr()
        return m.indptr, m.indices, m.data
    return tuple(m)


class AlgebraicSystem:
    """A multilevel decomposition formed elsewhere -- the level matrices,
    coarsest first, the interpolation into each level above the coarsest, and
    the top-level rhs -- as Femlisp forms it on an unstructured or adaptively
    refined mesh (multilevel-decomposition, geomg.lisp:109-142).  Matrices are
    scipy sparse matrices or (start, index, values) compressed rows.  The
    blackboard solve runs it on an algebraic grid (fmg_grid_create_algebraic);
    with no ansatz space to choose from, the default smoother is <jacobi>."""

    fe = None

    def __init__(self, matrices, interpolations, rhs, ctx: Context | None = None, order: int | None = None):
        """order: the discretisation order of a scalar Lagrange space behind
        the matrices (select-smoother then picks Gauss-Seidel for order 1 and
        SSC above, geomg.lisp:48-60); None: <jacobi>."""
        if order is not None:
            self.fe = lagrange_fe(order)
        if len(interpolations) != len(matrices) - 1:
            raise ValueError("one interpolation per level above the coarsest")
        self.matrices = [_csr_triple(m) for m in matrices]
        self.interpolations = [_csr_triple(p) for p in interpolations]
        self.sizes = [len(s) - 1 for s, _, _ in self.matrices]
        for l, (s, _, _) in enumerate(self.interpolations, start=1):
            if len(s) - 1 != self.sizes[l]:
                raise ValueError(f"interpolation into level {l} has {len(s) - 1} rows, the level {self.sizes[l]}")
        self.rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        if self.rhs.size != self.sizes[-1]:
            raise ValueError("rhs size differs from the top level's")
        self.ctx = ctx
        self._grids: dict[int, Grid] = {}

    def grid(self, base_level: int = 0) -> Grid:
        """The algebraic grid of levels base_level .. top (renumbered from 0)."""
        if base_level not in self._grids:
            if self.ctx is None:
                self.ctx = Context()
            g = Grid.algebraic(self.ctx, self.sizes[base_level:])
            for l, (s, i, v) in enumerate(self.matrices[base_level:]):
                g.set_matrix(l, s, i, v)
            for l, (s, i, v) in enumerate(self.interpolations[base_level:], start=1):
                g.set_interpolation(l, s, i, v, self.sizes[base_level + l - 1])
            g.set_rhs(self.rhs)
            self._grids[base_level] = g
        return self._grids[base_level]


def discretize_globally(problem, mesh: Mesh, fe: LagrangeFE, ctx: Context | None = None):
    """Returns (A, b) like Femlisp; here A is the DiscreteSystem and b its
    assembled right-hand side on the host."""
    sysm = DiscreteSystem(problem, mesh, fe, ctx)
    return sysm, sysm.grid(0).rhs()


# ---------------------------------------------------------------- iterations


@dataclass
class Jacobi:
    damp: float = 1.0


@dataclass
class SOR:
    omega: float = 1.0


class GaussSeidel(SOR):
    def __init__(self):
        super().__init__(1.0)


@dataclass
class GeometricSSC:
    """(geometric-ssc) -- successive subspace correction over the
    vertex-centred blocks (geoblock.lisp:37-158, blockit.lisp:118-204): the
    default smoother of higher-order discretisations (geomg.lisp:48-60)."""
    omega: float = 1.0


def geometric_ssc(**kw) -> GeometricSSC:
    return GeometricSSC(**kw)


@dataclass
class GeometricPSC:
    """(geometric-psc) -- parallel subspace correction over the vertex-centred
    blocks (geoblock.lisp:37-158, blockit.lisp:118-204), damped by :damp."""
    damp: float = 1.0


def geometric_psc(**kw) -> GeometricPSC:
    return GeometricPSC(**kw)


@dataclass
class LU:
    damp: float = 1.0


@dataclass
class GeometricCS:
    smoother: Any = None
    pre_steps: int = 1
    post_steps: int = 1
    gamma: int = 1
    base_level: int = 0
    coarse_grid_iteration: Any = None
    combination: str = "multiplicative"
    fmg: bool = False            # the f-cycle of :fmg t (multigrid.lisp:290-297)


def geometric_cs(**kw) -> GeometricCS:
    return GeometricCS(**kw)


@dataclass
class LocalMG(GeometricCS):
    """<local-mg> (geomg.lisp:161-168): the correction scheme on the levels of
    a locally refined mesh.  Its systems come as an AlgebraicSystem (the
    level matrices and constrained interpolations with the hanging-node and
    essential constraints eliminated); smoothers <jacobi>, <sor> /
    Gauss-Seidel (multicolour order) and geometric SSC (one-unknown
    blocks)."""


def local_mg(**kw) -> LocalMG:
    return LocalMG(**kw)


@dataclass
class CG:
    preconditioner: Any = None
    # True: call the preconditioner as (iterate q w w), rhs and residual
    # aliased exactly as krylow.lisp:120 does; False: a separate residual.
    compat_alias: bool = False


# ------------------------------------------------------------ solver forms

def _parse_form(text: str):
    toks = text.replace("(", " ( ").replace(")", " ) ").split()

    def rd(i):
        if toks[i] == "(":
            out, i = [], i + 1
            while toks[i] != ")":
                e, i = rd(i)
                out.append(e)
            return out, i + 1
        t = toks[i]
        try:
            return float(t), i + 1
        except ValueError:
            return t.lower(), i + 1

    form, _ = rd(0)
    return form


def _conditions(form) -> dict:
    """Flatten (or (< :defnorm a) (< :reduction b) (> :step n)) into bounds."""
    out: dict = {}
    if isinstance(form, str):
        form = _parse_form(form)
    if not form:
        return out
    if form[0] == "or":
        for f in form[1:]:
            out.update(_conditions(f))
        return out
    op, key, val = form
    if op == "<" and key == ":defnorm":
        out["atol"] = val
    elif op == "<" and key == ":reduction":
        out["rtol"] = val
    elif op in (">", ">=") and key == ":step":
        out["maxsteps"] = int(val) if op == ">" else int(val) - 1
    else:
        raise ValueError(f"unsupported condition {form}")
    return out


@dataclass
class LinearSolver:
    iteration: Any
    success_if: str = "(< :reduction 1.0e-10)"
    failure_if: str = "(> :step 100)"
    output: bool = False


@dataclass
class SolveReport:
    status: str
    steps: int
    history: np.ndarray
    convergence_rate: float
    extra: dict = field(default_factory=dict)


def make_cfg(iteration, success_if: str, failure_if: str, order: int | None = 1,
             vector: bool = False) -> tuple[C.SolveCfg, int, bool]:
    """The fmg_solve_cfg of an iteration and the solver's forms.  The default
    smoother is select-smoother's (geomg.lisp:48-60): Gauss-Seidel for order
    1, geometric SSC above; for an algebraic system, and for node blocks (the
    GPU's block smoother is <jacobi> on the 3 x 3 diagonal blocks, linit.lisp:234),
    <jacobi>."""
    cs = iteration.preconditioner if isinstance(iteration, CG) else iteration
    cfg = C.SolveCfg()
    if isinstance(iteration, CG):
        cfg.method = C.FMG_METHOD_CG_MG if cs is not None else C.FMG_METHOD_CG
        cfg.compat_alias = 1 if iteration.compat_alias else 0
    else:
        cfg.method = C.FMG_METHOD_MG
    base = 0
    if cs is not None:
        # select-smoother (geomg.lisp:48-60): Gauss-Seidel for order 1, SSC
        # above; <jacobi> for an algebraic system (order None)
        sm = cs.smoother or (Jacobi() if (order is None or vector) else GaussSeidel() if order == 1
                             else GeometricSSC())
        if isinstance(sm, Jacobi):
            cfg.smoother, cfg.damp = C.FMG_JACOBI, sm.damp
        elif isinstance(sm, GeometricSSC):
            cfg.smoother, cfg.damp = C.FMG_SSC, sm.omega
        elif isinstance(sm, GeometricPSC):
            cfg.smoother, cfg.damp = C.FMG_PSC, sm.damp
        elif isinstance(sm, SOR):
            cfg.smoother, cfg.damp = C.FMG_SOR, sm.omega
        else:
            raise NotImplementedError(f"smoother {sm!r}")
        cfg.pre_steps, cfg.post_steps, cfg.gamma = cs.pre_steps, cs.post_steps, cs.gamma
        cfg.combination = C.FMG_ADDITIVE if cs.combination == "additive" else C.FMG_MULTIPLICATIVE
        cfg.fmg = 1 if cs.fmg else 0
        cgi = cs.coarse_grid_iteration or LU()
        if not isinstance(cgi, LU):
            raise NotImplementedError("only the <lu> coarse-grid iteration is built")
        cfg.coarse_damp = cgi.damp
        base = cs.base_level
    succ, fail = _conditions(success_if), _conditions(failure_if)
    cfg.rtol = succ.get("rtol", 0.0)
    cfg.atol = succ.get("atol", 0.0)
    step_success = "maxsteps" in succ
    cfg.maxsteps = succ.get("maxsteps", fail.get("maxsteps", 100))
    return cfg, base, step_success


def solve(blackboard: dict) -> dict:
    """(solve (blackboard :matrix A :rhs b :solver solver)) -- returns the
    blackboard with :solution, :report and :history filled in."""
    A: DiscreteSystem | AlgebraicSystem = blackboard["matrix"]
    solver: LinearSolver = blackboard["solver"]
    order = A.fe.order if A.fe is not None else None
    vector = A.fe is not None and A.fe.nr_comps > 1
    cfg, base, step_success = make_cfg(solver.iteration, solver.success_if, solver.failure_if, order, vector)
    g = A.grid(base)
    x = g.vector()
    if "solution" in blackboard and blackboard["solution"] is not None:
        x.set(blackboard["solution"])
    hist, steps, status = g.solve(cfg, x)
    st = "success" if (status == 0 or step_success) else "failure"
    red = hist[-1] / hist[0] if hist[0] != 0 else 0.0
    rate = red ** (1.0 / steps) if steps > 0 else float("nan")
    out = dict(blackboard)
    out["solution"] = x.get()
    out["history"] = hist
    out["report"] = SolveReport(st, steps, hist, rate)
    return out


# ------------------------------------------------------------- iterators


@dataclass
class Iterator:
    """<iterator> (linit.lisp:48-67): what make_iterator returns -- the
    matrix, an initialize function (or None) and an iterate function of
    (x, b, r), and whether the residual must be up to date before a step and
    is up to date after it.  Vectors are host arrays in the grid's node
    order (node-major for node blocks), updated in place."""
    matrix: Any
    initialize: Callable | None
    iterate: Callable
    residual_before: bool
    residual_after: bool
    initializedp: bool = False


def _system_of(A):
    order = A.fe.order if A.fe is not None else None
    vector = A.fe is not None and A.fe.nr_comps > 1
    return order, vector


def make_iterator(linit, A) -> Iterator:
    """make-iterator (linit.lisp:48-67) of a GeometricCS or a CG on the
    system A (a DiscreteSystem or an AlgebraicSystem).

    GeometricCS: one cycle of the <mg-iteration> iterator per iterate
    (multigrid.lisp:366-386, fmg_vcycle): the top-level solution, rhs and
    residual are the given arrays; passing the same array as b and r is the
    alias of <cg>'s preconditioner call (krylow.lisp:120).  :residual-after
    nil.

    CG (preconditioned by a GeometricCS): initialize restarts from the
    residual (fmg_cg_start), iterate is one CG step (fmg_cg_step) with x and
    r brought back up to date; :residual-before and :residual-after t
    (krylow.lisp:72-132)."""
    order, vector = _system_of(A)
    if isinstance(linit, CG):
        cfg, base, _ = make_cfg(linit, "(< :reduction 0.0)", "(> :step 0)", order, vector)
        g = A.grid(base)
        X, R = g.vector(), g.vector()

        def initialize(x, b, r):
            X.set(x)
            R.set(r)
            g.cg_start(cfg, R)

        def iterate(x, b, r):
            g.cg_step(X, R)
            X.get(out=x)
            R.get(out=r)
            return {"residual_after": True}

        it = Iterator(A, initialize, iterate, True, True)
        it.grid, it.vectors = g, (X, R)
        return it
    if isinstance(linit, GeometricCS):
        cfg, base, _ = make_cfg(linit, "(< :reduction 0.0)", "(> :step 0)", order, vector)
        g = A.grid(base)
        X, B, R = g.vector(), g.vector(), g.vector()

        def iterate(x, b, r):
            alias = b is r
            X.set(x)
            B.set(b)
            if not alias:
                R.set(r)
            g.vcycle(cfg, X, B, B if alias else R)
            X.get(out=x)
            B.get(out=b)
            if not alias:
                R.get(out=r)
            return {}

        it = Iterator(A, None, iterate, True, False)
        it.grid, it.vectors = g, (X, B, R)
        return it
    raise NotImplementedError(f"no GPU iterator for {linit!r}")


def solve_iterating(blackboard: dict) -> dict:
    """The <linear-solver> loop with the solver's iterator, step by step as
    Femlisp runs it: (solve (blackboard :matrix A :rhs b :solver solver)).
    Each step: ensure the residual (r = b - A x when it is not up to date;
    ensure-residual, solve.lisp:139-155), :defnorm = l2 norm of r on the host,
    the success/failure forms, then next-step (linsolve.lisp:58-73):
    initialize once, iterate, and the iterator's :residual-after flag.
    Returns the blackboard with :solution, :history and :report."""
    A = blackboard["matrix"]
    solver: LinearSolver = blackboard["solver"]
    order, vector = _system_of(A)
    cfg, base, step_success = make_cfg(solver.iteration, solver.success_if, solver.failure_if, order, vector)
    it = make_iterator(solver.iteration, A)
    g = it.grid
    b = np.array(blackboard["rhs"] if blackboard.get("rhs") is not None else g.rhs(), dtype=np.float64)
    x = np.array(blackboard.get("solution") if blackboard.get("solution") is not None else np.zeros(b.size))
    Xv, Bv, Rv = g.vector(), g.vector(values=b), g.vector()
    r = np.zeros_like(b)
    residual_p = False
    hist = []
    status = "failure"
    step = 0
    while True:
        if not residual_p:  # compute-residual (linit.lisp:73-80) on the device
            Xv.set(x)
            g.residual(Xv, Bv, Rv)
            Rv.get(out=r)
            residual_p = True
        defnorm = float(np.sqrt(np.dot(r, r)))
        hist.append(defnorm)
        red = defnorm / hist[0] if hist[0] != 0 else 0.0
        if (cfg.rtol > 0 and red < cfg.rtol) or (cfg.atol > 0 and defnorm < cfg.atol):
            status = "success"
            break
        if step > cfg.maxsteps:
            status = "success" if step_success else "failure"
            break
        if not it.initializedp:
            if it.initialize is not None:
                it.initialize(x, b, r)
            it.initializedp = True
        flags = it.iterate(x, b, r)
        residual_p = it.residual_after and bool(flags.get("residual_after"))
        step += 1
    hist = np.array(hist)
    rate = (hist[-1] / hist[0]) ** (1.0 / step) if step > 0 and hist[0] != 0 else float("nan")
    out = dict(blackboard)
    out["solution"] = x
    out["history"] = hist
    out["report"] = SolveReport(status, step, hist, rate)
    return out
