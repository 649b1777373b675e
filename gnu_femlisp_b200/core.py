"""Device handles: context, level hierarchy (grid) and level vectors.

Thin, checked wrappers of the C-ABI: every non-zero status becomes an
:class:`FmgError` carrying the library's message.
"""
from __future__ import annotations

import ctypes

import numpy as np

import atexit

from . import _capi as C
from ._capi import FmgError

# At interpreter exit handles may be collected in any order; the process is
# ending and the driver reclaims device memory, so destructors do nothing.
_EXITING = False


def _mark_exit():
    global _EXITING
    _EXITING = True


atexit.register(_mark_exit)


class Context:
    """One CUDA device and the stream all work is queued on
    (``fmg_init``)."""

    def __init__(self, device: int = 0):
        self._lib = C.load()
        h = ctypes.c_void_p()
        rc = self._lib.fmg_init(device, ctypes.byref(h))
        if rc != C.FMG_OK:
            raise FmgError(rc, f"fmg_init(device={device}) failed (no CUDA device?)")
        self.h = h
        self.device = device

    def check(self, rc: int, what: str = ""):
        if rc != C.FMG_OK:
            buf = ctypes.create_string_buffer(512)
            self._lib.fmg_last_error(self.h, buf, 512)
            raise FmgError(rc, f"{what}: {buf.value.decode(errors='replace')}")

    def synchronize(self):
        self.check(self._lib.fmg_synchronize(self.h), "synchronize")

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self.check(self._lib.fmg_get_stream(self.h, ctypes.byref(s)), "get_stream")
        return s.value or 0

    def close(self):
        if getattr(self, "h", None):
            self._lib.fmg_finalize(self.h)
            self.h = None

    def __del__(self):
        if _EXITING:
            return
        try:
            self.close()
        except Exception:
            pass


def slots_to_csr(A: np.ndarray, dim: int, order: int, nc: int = 1):
    """Stencil-slot storage ``[slot][k][l][node]`` (slot = sum over directions
    of (offset + order) * (2 order + 1)^d, the layout ``fmg_get_matrix``
    returns) to compressed rows ``(start, index, values)``, node-major dofs,
    exact zeros left out."""
    w = 2 * order + 1
    nslots = w ** dim
    A = np.asarray(A).reshape(nslots, nc, nc, -1)
    N = A.shape[-1]
    M = int(round(N ** (1.0 / dim)))
    assert M ** dim == N, "level is not a full n-cube"
    idx = np.arange(N, dtype=np.int64)
    c = np.stack([(idx // M ** d) % M for d in range(dim)], 1)
    rows, cols, vals = [], [], []
    for s in range(nslots):
        off = np.array([(s // w ** d) % w - order for d in range(dim)])
        cj = c + off
        ok = np.all((cj >= 0) & (cj < M), 1)
        j = sum(cj[:, d] * M ** d for d in range(dim))
        for k in range(nc):
            for l in range(nc):
                v = A[s, k, l]
                m = ok & (v != 0.0)
                rows.append(idx[m] * nc + k)
                cols.append(j[m] * nc + l)
                vals.append(v[m])
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    order_ = np.lexsort((cols, rows))
    rows, cols, vals = rows[order_], cols[order_], vals[order_]
    start = np.zeros(N * nc + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=N * nc), out=start[1:])
    return start, cols, vals


def _compressed(start, index, values):
    """Compressed rows (or columns) as the C-ABI reads them: 32-bit starts and
    indices, FP64 values.  The starts must begin at 0 and never decrease, and
    the index and value arrays must hold the start[-1] entries they promise
    (the library reads that many)."""
    st = np.ascontiguousarray(start, dtype=np.int32)
    ix = np.ascontiguousarray(index, dtype=np.int32)
    va = np.ascontiguousarray(values, dtype=np.float64)
    if st.ndim != 1 or st.size < 1:
        raise ValueError("start must be a 1-D array of at least one entry")
    if st[0] != 0 or np.any(np.diff(st) < 0):
        raise ValueError("start must begin at 0 and be nondecreasing")
    nnz = int(st[-1])
    if ix.size < nnz or va.size < nnz:
        raise ValueError(f"start promises {nnz} entries; index holds {ix.size}, values hold {va.size}")
    return st, ix, va


class Grid:
    """A level hierarchy of the uniformly refined unit n-cube with a Lagrange
    Q1/Q2 space (``fmg_grid_create``); levels base_level..level."""

    def __init__(self, ctx: Context, dim: int, order: int, level: int, base_level: int = 0,
                 n0: int = 1, ncomp: int = 1, dirichlet_mask: int | None = None):
        self.ctx, self.dim, self.order, self.top, self.base = ctx, dim, order, level, base_level
        self.nc = ncomp
        if dirichlet_mask is None:
            dirichlet_mask = (1 << (2 * dim)) - 1
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.fmg_grid_create(ctx.h, dim, order, ncomp, n0, level, base_level,
                                           dirichlet_mask, ctypes.byref(h)), "grid_create")
        self.h = h
        self.n_cells = n0 << level
        self.assembled = False

    nb = 1  # problems held (a batch: ``Grid.batch``)

    @classmethod
    def batch(cls, like: "Grid", nbatch: int) -> "Grid":
        """``fmg_batch_create``: nbatch independent problems with the geometry
        of ``like`` (1D/2D scalar Q1), loaded one by one from assembled grids
        (``batch_load``) and solved together (``batch_solve``)."""
        g = cls.__new__(cls)
        g.ctx, g.dim, g.order, g.top, g.base, g.nc = like.ctx, like.dim, like.order, like.top, like.base, 1
        h = ctypes.c_void_p()
        like.ctx.check(like._lib.fmg_batch_create(like.h, int(nbatch), ctypes.byref(h)), "batch_create")
        g.h = h
        g.n_cells = like.n_cells
        g.assembled = False
        g.nb = int(nbatch)
        return g

    def batch_load(self, index: int, src: "Grid") -> "Grid":
        """``fmg_batch_load``: problem ``index`` from the assembled grid ``src``
        (its matrices, rhs, coarse inverse and node damping)."""
        self.ctx.check(self._lib.fmg_batch_load(self.h, int(index), src.h), "batch_load")
        return self

    def batch_solve(self, cfg: C.SolveCfg, x: "Vector"):
        """``fmg_batch_solve``: every problem from x to cfg's tolerance at once;
        returns (defnorm histories, one row per problem, padded with zeros;
        steps; status), each row as ``solve`` on the problem's own grid."""
        hl = cfg.maxsteps + 2
        hist = np.zeros(self.nb * hl)
        steps = np.zeros(self.nb, dtype=np.int32)
        status = np.zeros(self.nb, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        self.ctx.check(self._lib.fmg_batch_solve(self.h, ctypes.byref(cfg), x.h, C.dptr(hist), hl,
                                                 steps.ctypes.data_as(ip), status.ctypes.data_as(ip)), "batch_solve")
        return hist.reshape(self.nb, hl), steps, status

    @classmethod
    def algebraic(cls, ctx: Context, sizes) -> "Grid":
        """``fmg_grid_create_algebraic``: levels 0 .. len(sizes)-1 without
        geometry; matrices by ``set_matrix``, interpolations by
        ``set_interpolation``, the rhs by ``set_rhs``."""
        g = cls.__new__(cls)
        sz = np.ascontiguousarray(sizes, dtype=np.int64)
        g.ctx, g.dim, g.order, g.top, g.base, g.nc = ctx, 0, 1, sz.size - 1, 0, 1
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.fmg_grid_create_algebraic(ctx.h, int(sz.size), sz.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                                     ctypes.byref(h)), "grid_create_algebraic")
        g.h = h
        g.n_cells = 0
        g.assembled = False
        return g

    def set_interpolation(self, fine_level: int, start, index, values, ncoarse: int, layout: str = "csr") -> "Grid":
        """``fmg_set_interpolation``: I from level fine_level-1 to fine_level
        (rows fine, columns coarse; ``"ccs"``: the arrays of the transpose's
        rows)."""
        lay = {"csr": C.FMG_CSR, "ccs": C.FMG_CCS}[layout]
        st, ix, va = _compressed(start, index, values)
        ip = ctypes.POINTER(ctypes.c_int)
        nfine = self.nnodes(fine_level)
        self.ctx.check(self._lib.fmg_set_interpolation(self.h, fine_level, lay, st.ctypes.data_as(ip),
                                                       ix.ctypes.data_as(ip), C.dptr(va), nfine, ncoarse),
                       "set_interpolation")
        return self

    @property
    def _lib(self):
        return self.ctx._lib

    def nnodes(self, level: int | None = None) -> int:
        return int(self._lib.fmg_grid_nnodes(self.h, self.top if level is None else level))

    @property
    def nslots(self) -> int:
        return int(self._lib.fmg_grid_nslots(self.h))

    def set_coefficient(self, kind: int, values):
        v = np.ascontiguousarray(np.atleast_1d(np.asarray(values, dtype=np.float64)).ravel())
        self.ctx.check(self._lib.fmg_set_coefficient(self.h, kind, C.dptr(v), v.size), "set_coefficient")
        self.assembled = False

    def assemble(self, galerkin: bool = False) -> "Grid":
        """``fmg_assemble_levels``: coarse levels re-discretised, or Galerkin
        products I^T A I of the level above (``galerkin=True``; every
        structured form: Q1, Q2, 3 x 3 node blocks)."""
        mode = C.FMG_ASSEMBLE_GALERKIN if galerkin else C.FMG_ASSEMBLE_REDISCRETIZE
        self.ctx.check(self._lib.fmg_assemble_levels(self.h, mode), "assemble")
        self.assembled = True
        return self

    def matrix(self, level: int | None = None) -> np.ndarray:
        level = self.top if level is None else level
        out = np.zeros(self.nslots * self.nc * self.nc * self.nnodes(level))
        self.ctx.check(self._lib.fmg_get_matrix(self.h, level, C.dptr(out)), "get_matrix")
        return out.reshape(self.nslots * self.nc * self.nc, -1)

    def matrix_csr(self, level: int | None = None):
        """The level matrix as compressed rows ``(start, index, values)`` in the
        grid's node-major lexicographic numbering (the inverse of
        ``set_matrix``); exact zeros are left out."""
        level = self.top if level is None else level
        return slots_to_csr(self.matrix(level), self.dim, self.order, self.nc)

    def set_matrix(self, level: int, start, index, values, layout: str = "csr") -> "Grid":
        """``fmg_set_matrix``: a level matrix from compressed rows (``"csr"``)
        or columns (``"ccs"``, the form of Femlisp's ``sparse-matrix->ccs``)
        in the grid's node-major lexicographic numbering.  The grid counts as
        assembled once every level has a matrix."""
        lay = {"csr": C.FMG_CSR, "ccs": C.FMG_CCS}[layout]
        st, ix, va = _compressed(start, index, values)
        ip = ctypes.POINTER(ctypes.c_int)
        self.ctx.check(self._lib.fmg_set_matrix(self.h, level, lay, st.ctypes.data_as(ip), ix.ctypes.data_as(ip),
                                                C.dptr(va), st.size - 1), "set_matrix")
        return self

    def set_rhs(self, values) -> "Grid":
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        self.ctx.check(self._lib.fmg_set_rhs(self.h, C.dptr(v), v.size), "set_rhs")
        return self

    def rhs(self) -> np.ndarray:
        out = np.zeros(self.nnodes() * self.nc)
        self.ctx.check(self._lib.fmg_get_rhs(self.h, C.dptr(out)), "get_rhs")
        return out

    def set_node_damping(self, level: int, w):
        if w is None:
            self.ctx.check(self._lib.fmg_set_node_damping(self.h, level, None, 0), "set_node_damping")
            return
        w = np.ascontiguousarray(w, dtype=np.float64)
        self.ctx.check(self._lib.fmg_set_node_damping(self.h, level, C.dptr(w), w.size),
                       "set_node_damping")

    def vector(self, level: int | None = None, values=None) -> "Vector":
        v = Vector(self, self.top if level is None else level)
        if values is not None:
            v.set(values)
        return v

    # operators of one level ---------------------------------------------
    def matvec(self, x: "Vector", y: "Vector"):
        self.ctx.check(self._lib.fmg_matvec(self.h, x.level, x.h, y.h), "matvec")

    def residual(self, x: "Vector", b: "Vector", r: "Vector"):
        self.ctx.check(self._lib.fmg_residual(self.h, x.level, x.h, b.h, r.h), "residual")

    def matvec_mf(self, x: "Vector", y: "Vector", b: "Vector" = None, fp32=False):
        """y = A x (b None) or y = b - A x on the top level, matrix-free from
        the cell coefficients as the mixed solve applies it: FP64 difference
        form (fp32 False), FP32 with the result widened (True), or FP64 on x
        rounded to FP32 (2: the mixed solve's CG operator; b must be None)."""
        mode = 2 if fp32 == 2 else (1 if fp32 else 0)
        self.ctx.check(self._lib.fmg_matvec_mf(self.h, mode, x.h, b.h if b is not None else None, y.h),
                       "matvec_mf")

    def restrict(self, rf: "Vector", rc: "Vector"):
        self.ctx.check(self._lib.fmg_restrict(self.h, rf.level, rf.h, rc.h), "restrict")

    def prolongate(self, xc: "Vector", xf: "Vector"):
        self.ctx.check(self._lib.fmg_prolongate(self.h, xc.level, xc.h, xf.h), "prolongate")

    def jacobi(self, x: "Vector", r: "Vector", damp: float):
        self.ctx.check(self._lib.fmg_jacobi(self.h, x.level, damp, x.h, r.h), "jacobi")

    def sor(self, x: "Vector", b: "Vector", r: "Vector", omega: float):
        self.ctx.check(self._lib.fmg_sor(self.h, x.level, omega, x.h, b.h, r.h), "sor")

    def ssc(self, x: "Vector", b: "Vector", r: "Vector", omega: float = 1.0):
        """One <geometric-ssc> sweep (vertex-centred blocks); b may be r."""
        self.ctx.check(self._lib.fmg_ssc(self.h, x.level, omega, x.h, b.h, r.h), "ssc")

    def psc(self, x: "Vector", r: "Vector", damp: float = 1.0):
        """One <geometric-psc> sweep (vertex-centred blocks) with the residual r."""
        self.ctx.check(self._lib.fmg_psc(self.h, x.level, damp, x.h, r.h), "psc")

    def coarse_solve(self, x: "Vector", r: "Vector", damp: float = 1.0):
        self.ctx.check(self._lib.fmg_coarse_solve(self.h, damp, x.h, r.h), "coarse_solve")

    def vcycle(self, cfg: C.SolveCfg, x: "Vector", b: "Vector", r: "Vector"):
        self.ctx.check(self._lib.fmg_vcycle(self.h, ctypes.byref(cfg), x.h, b.h, r.h), "vcycle")

    def solve(self, cfg: C.SolveCfg, x: "Vector"):
        hist = np.zeros(cfg.maxsteps + 2)
        ns, st = ctypes.c_int(0), ctypes.c_int(0)
        self.ctx.check(self._lib.fmg_solve(self.h, ctypes.byref(cfg), x.h, C.dptr(hist), hist.size,
                                           ctypes.byref(ns), ctypes.byref(st)), "solve")
        return hist[: ns.value + 1].copy(), ns.value, st.value

    def cg_start(self, cfg: C.SolveCfg, r: "Vector"):
        """``fmg_cg_start``: the <cg> iterator's initialize (restart from r)."""
        self.ctx.check(self._lib.fmg_cg_start(self.h, ctypes.byref(cfg), r.h), "cg_start")

    def cg_step(self, x: "Vector", r: "Vector") -> float:
        """``fmg_cg_step``: one <cg> iterate on x and its residual r; returns ||r||."""
        dn = ctypes.c_double()
        self.ctx.check(self._lib.fmg_cg_step(self.h, x.h, r.h, ctypes.byref(dn)), "cg_step")
        return dn.value

    def solve_mixed(self, cfg: C.SolveCfg, x: "Vector", inner_rtol: float = 1e-5, max_inner: int = 200,
                    max_outer: int = 20, matrix_free: bool = True, judge: int = 0):
        """FP64 flexible CG preconditioned by the FP32/BF16 V-cycle; returns
        (defnorm history: true FP64 residuals at the start and at every
        restart, recursive residuals in between; restarts; CG iterations;
        status).  judge > 0: installed node damping is judged against the
        plain cycle on that many CG steps after each (re)start, inside the
        solve (reverted when the plain cycle does better)."""
        mc = C.MixedCfg(inner_rtol, max_inner, max_outer, 1 if matrix_free else 0, int(judge))
        hist = np.zeros(cfg.maxsteps + max_outer + 4)
        no, ni, st = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        self.ctx.check(self._lib.fmg_solve_mixed(self.h, ctypes.byref(cfg), ctypes.byref(mc), x.h, C.dptr(hist),
                                                 hist.size, ctypes.byref(no), ctypes.byref(ni), ctypes.byref(st)),
                       "solve_mixed")
        return hist[: no.value + ni.value + 1].copy(), no.value, ni.value, st.value

    def mixed_top_kernel(self, kind: int, reps: int = 1):
        """``fmg_mixed_top_kernel``: `reps` launches of one top-level kernel of
        the mixed solve (FMG_MXK_RESIDUAL, FMG_MXK_SMOOTH, FMG_MXK_MATVEC64) on
        the buffers the last matrix-free mixed solve left; nothing waits."""
        self.ctx.check(self._lib.fmg_mixed_top_kernel(self.h, kind, reps), "mixed_top_kernel")

    def learned_judge(self, cfg: C.SolveCfg):
        """Plain cycle vs the installed node damping (``fmg_learned_judge``);
        returns (accepted, rho_plain, rho_learned)."""
        rp, rl, ok = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self.ctx.check(self._lib.fmg_learned_judge(self.h, ctypes.byref(cfg), ctypes.byref(rp), ctypes.byref(rl),
                                                   ctypes.byref(ok)), "learned_judge")
        return bool(ok.value), rp.value, rl.value

    def learned_judge_mixed(self, cfg: C.SolveCfg, matrix_free: bool = True):
        """``fmg_learned_judge_mixed``: the judge's CG probe run with the
        mixed-precision cycle of ``solve_mixed``; returns (accepted,
        rho_plain, rho_learned)."""
        mc = C.MixedCfg(0.0, 0, 1, 1 if matrix_free else 0, 0)
        rp, rl, ok = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self.ctx.check(self._lib.fmg_learned_judge_mixed(self.h, ctypes.byref(cfg), ctypes.byref(mc), ctypes.byref(rp),
                                                         ctypes.byref(rl), ctypes.byref(ok)), "learned_judge_mixed")
        return bool(ok.value), rp.value, rl.value

    def learned_status(self) -> dict:
        a, rp, rl, rv = ctypes.c_int(), ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self.ctx.check(self._lib.fmg_learned_status(self.h, ctypes.byref(a), ctypes.byref(rp), ctypes.byref(rl),
                                                    ctypes.byref(rv)), "learned_status")
        return {"active": bool(a.value), "rho_plain": rp.value, "rho_learned": rl.value, "reverts": rv.value}

    def close(self):
        if getattr(self, "h", None):
            self._lib.fmg_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        if _EXITING:
            return
        try:
            self.close()
        except Exception:
            pass


class Vector:
    """A device vector of one level (``fmg_vec_create``)."""

    def __init__(self, grid: Grid, level: int):
        self.grid, self.level = grid, level
        self.n = grid.nnodes(level) * grid.nc * grid.nb
        h = ctypes.c_void_p()
        grid.ctx.check(grid._lib.fmg_vec_create(grid.h, level, ctypes.byref(h)), "vec_create")
        self.h = h

    @property
    def _lib(self):
        return self.grid._lib

    def set(self, values):
        v = np.ascontiguousarray(np.asarray(values, dtype=np.float64).ravel())
        self.grid.ctx.check(self._lib.fmg_vec_set(self.h, C.dptr(v), v.size), "vec_set")
        return self

    def get(self, out: np.ndarray | None = None) -> np.ndarray:
        """Copy to the host (into `out`, e.g. a pinned buffer, when given)."""
        if out is None:
            out = np.zeros(self.n)
        self.grid.ctx.check(self._lib.fmg_vec_get(self.h, C.dptr(out), self.n), "vec_get")
        return out

    def fill(self, value: float = 0.0):
        self.grid.ctx.check(self._lib.fmg_vec_fill(self.h, value), "fill")
        return self

    def copy_to(self, y: "Vector"):
        self.grid.ctx.check(self._lib.fmg_copy(self.h, y.h), "copy")

    def axpy(self, alpha: float, x: "Vector"):
        """self := self + alpha x"""
        self.grid.ctx.check(self._lib.fmg_axpy(alpha, x.h, self.h), "axpy")

    def dot(self, y: "Vector") -> float:
        out = ctypes.c_double()
        self.grid.ctx.check(self._lib.fmg_dot(self.h, y.h, ctypes.byref(out)), "dot")
        return out.value

    def l2_norm(self) -> float:
        out = ctypes.c_double()
        self.grid.ctx.check(self._lib.fmg_l2_norm(self.h, ctypes.byref(out)), "l2_norm")
        return out.value

    def close(self):
        if getattr(self, "h", None):
            self._lib.fmg_vec_destroy(self.h)
            self.h = None

    def __del__(self):
        if _EXITING:
            return
        try:
            self.close()
        except Exception:
            pass
