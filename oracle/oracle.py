"""ctypes wrapper of the CPU oracle (oracle/libfmg_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker of the GPU path.  Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this module; the product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libfmg_oracle.so")

K_CONST, K_CELL, F_CONST, F_IP, LAMBDA_MU_CELL, F_VEC = 0, 1, 2, 3, 4, 5
JACOBI, SOR, SSC, PSC = 0, 1, 2, 3
METHOD_MG, METHOD_CG_MG, METHOD_CG = 0, 1, 2

_dp = ctypes.POINTER(ctypes.c_double)


class SolveCfg(ctypes.Structure):
    _fields_ = [
        ("method", ctypes.c_int),
        ("smoother", ctypes.c_int),
        ("damp", ctypes.c_double),
        ("pre_steps", ctypes.c_int),
        ("post_steps", ctypes.c_int),
        ("gamma", ctypes.c_int),
        ("compat_alias", ctypes.c_int),
        ("coarse_damp", ctypes.c_double),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("maxsteps", ctypes.c_int),
        ("combination", ctypes.c_int),
        ("fmg", ctypes.c_int),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.ora_create.restype = ctypes.c_void_p
        L.ora_create.argtypes = [ctypes.c_int] * 7
        L.ora_destroy.argtypes = [ctypes.c_void_p]
        L.ora_set_coefficient.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_long]
        L.ora_assemble.argtypes = [ctypes.c_void_p]
        L.ora_assemble_levels.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_set_node_damping.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_long]
        L.ora_nnodes.restype = ctypes.c_long
        L.ora_nnodes.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_nslots.argtypes = [ctypes.c_void_p]
        for name in ("ora_get_matrix", "ora_set_matrix"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.ora_set_rhs.argtypes = [ctypes.c_void_p, _dp]
        L.ora_create_algebraic.restype = ctypes.c_void_p
        L.ora_create_algebraic.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_long)]
        _lp, _ip = ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int)
        L.ora_set_csr_matrix.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _ip, _dp]
        L.ora_set_interpolation.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _ip, _dp]
        L.ora_finish_levels.argtypes = [ctypes.c_void_p]
        L.ora_get_rhs.argtypes = [ctypes.c_void_p, _dp]
        L.ora_get_coarse_inverse.argtypes = [ctypes.c_void_p, _dp]
        L.ora_matvec.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.ora_residual.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]
        L.ora_restrict.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.ora_prolongate.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.ora_inject.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.ora_jacobi.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.ora_sor.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.ora_ssc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.ora_psc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.ora_coarse_solve.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, _dp]
        L.ora_dot.restype = ctypes.c_double
        L.ora_dot.argtypes = [_dp, _dp, ctypes.c_long]
        L.ora_dot_par.restype = ctypes.c_double
        L.ora_dot_par.argtypes = [_dp, _dp, ctypes.c_long]
        L.ora_mf_apply.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp]
        L.ora_mf_apply.restype = None
        L.ora_vcycle.argtypes = [ctypes.c_void_p, ctypes.POINTER(SolveCfg), _dp, _dp, _dp]
        L.ora_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(SolveCfg), _dp, _dp, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_int)]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


@dataclass
class SolveResult:
    x: np.ndarray
    history: np.ndarray
    steps: int
    status: int

    @property
    def reduction(self) -> float:
        return float(self.history[-1] / self.history[0]) if self.history[0] != 0 else 0.0

    @property
    def convergence_rate(self) -> float:
        """reduction^(1/steps) as in solve.lisp:157-164."""
        return self.reduction ** (1.0 / self.steps) if self.steps > 0 else float("nan")


MULTIPLICATIVE, ADDITIVE = 0, 1


def solve_cfg(method=METHOD_CG_MG, smoother=JACOBI, damp=0.6, pre=1, post=1, gamma=1,
              compat=True, coarse_damp=1.0, rtol=1e-10, atol=0.0, maxsteps=200,
              combination=MULTIPLICATIVE, fmg=False) -> SolveCfg:
    return SolveCfg(method, smoother, damp, pre, post, gamma, 1 if compat else 0, coarse_damp,
                    rtol, atol, maxsteps, combination, 1 if fmg else 0)


class Oracle:
    """A structured level hierarchy of Femlisp's uniformly refined n-cube
    (meshgen.lisp:180-183) with Lagrange Q1/Q2 (lagrange.lisp:176-202)."""

    def __init__(self, dim, order, level, base_level=0, ncomp=1, n0=1, dirichlet_mask=None):
        self.dim, self.order, self.top, self.base, self.nc = dim, order, level, base_level, ncomp
        if dirichlet_mask is None:
            dirichlet_mask = (1 << (2 * dim)) - 1
        self.h = lib().ora_create(dim, order, ncomp, n0, level, base_level, dirichlet_mask)
        if not self.h:
            raise ValueError("invalid oracle hierarchy")
        self.n_cells = n0 << level

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_destroy(self.h)
            self.h = None

    def set_coefficient(self, kind, vals):
        v = np.ascontiguousarray(np.atleast_1d(np.asarray(vals, dtype=np.float64)).ravel())
        rc = lib().ora_set_coefficient(self.h, kind, _p(v), v.size)
        if rc:
            raise ValueError(f"ora_set_coefficient rc={rc}")

    def assemble(self, galerkin=False):
        rc = lib().ora_assemble_levels(self.h, 1 if galerkin else 0)
        if rc:
            raise RuntimeError(f"ora_assemble rc={rc}")
        return self

    def set_levels(self, mats, rhs):
        """Level matrices given in the ``matrix()`` layout (a dict level ->
        array) and the top-level rhs, then the coarse inverse."""
        for level, a in mats.items():
            a = np.ascontiguousarray(a, dtype=np.float64).ravel()
            assert a.size == self.nslots * self.nc * self.nc * self.nnodes(level)
            assert lib().ora_set_matrix(self.h, level, _p(a)) == 0
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        assert b.size == self.nnodes() * self.nc
        assert lib().ora_set_rhs(self.h, _p(b)) == 0
        rc = lib().ora_finish_levels(self.h)
        if rc:
            raise RuntimeError(f"ora_finish_levels rc={rc}")
        return self

    @classmethod
    def algebraic(cls, sizes):
        """An algebraic hierarchy (levels 0 .. len(sizes)-1 without geometry)."""
        o = cls.__new__(cls)
        sz = np.ascontiguousarray(sizes, dtype=np.int64)
        o.h = lib().ora_create_algebraic(int(sz.size), sz.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
        assert o.h
        o.dim, o.order, o.nc, o.top, o.base = 0, 1, 1, sz.size - 1, 0
        return o

    @staticmethod
    def _csr_args(start, index, value):
        st = np.ascontiguousarray(start, dtype=np.int64)
        ix = np.ascontiguousarray(index, dtype=np.int32)
        va = np.ascontiguousarray(value, dtype=np.float64)
        return (st, ix, va), (st.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                              ix.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _p(va))

    def set_csr_matrix(self, level, start, index, value):
        keep, args = self._csr_args(start, index, value)
        assert lib().ora_set_csr_matrix(self.h, level, *args) == 0

    def set_interpolation(self, fine_level, start, index, value):
        keep, args = self._csr_args(start, index, value)
        assert lib().ora_set_interpolation(self.h, fine_level, *args) == 0

    def finish(self, rhs):
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        assert lib().ora_set_rhs(self.h, _p(b)) == 0
        rc = lib().ora_finish_levels(self.h)
        if rc:
            raise RuntimeError(f"ora_finish_levels rc={rc}")
        return self

    def nnodes(self, level=None):
        return lib().ora_nnodes(self.h, self.top if level is None else level)

    @property
    def nslots(self):
        return lib().ora_nslots(self.h)

    def matrix(self, level=None):
        level = self.top if level is None else level
        out = np.zeros(self.nslots * self.nc * self.nc * self.nnodes(level))
        assert lib().ora_get_matrix(self.h, level, _p(out)) == 0
        return out.reshape(self.nslots * self.nc * self.nc, -1)

    def rhs(self):
        out = np.zeros(self.nnodes() * self.nc)
        assert lib().ora_get_rhs(self.h, _p(out)) == 0
        return out

    def coarse_inverse(self):
        n = self.nnodes(self.base) * self.nc
        out = np.zeros(n * n)
        assert lib().ora_get_coarse_inverse(self.h, _p(out)) == 0
        return out.reshape(n, n)

    def set_node_damping(self, level, w):
        if w is None:
            lib().ora_set_node_damping(self.h, level, None, self.nnodes(level))
            return
        w = np.ascontiguousarray(w, dtype=np.float64)
        assert lib().ora_set_node_damping(self.h, level, _p(w), w.size) == 0

    def matvec(self, x, level=None):
        level = self.top if level is None else level
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        lib().ora_matvec(self.h, level, _p(x), _p(y))
        return y

    def residual(self, x, b, level=None):
        level = self.top if level is None else level
        x = np.ascontiguousarray(x, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        r = np.zeros_like(x)
        lib().ora_residual(self.h, level, _p(x), _p(b), _p(r))
        return r

    def restrict(self, rf, fine_level):
        rf = np.ascontiguousarray(rf, dtype=np.float64)
        rc = np.zeros(self.nnodes(fine_level - 1) * self.nc)
        lib().ora_restrict(self.h, fine_level, _p(rf), _p(rc))
        return rc

    def prolongate(self, xc, xf, coarse_level, constrained=True):
        xc = np.ascontiguousarray(xc, dtype=np.float64)
        xf = np.array(xf, dtype=np.float64, copy=True)
        lib().ora_prolongate(self.h, coarse_level, _p(xc), _p(xf), 1 if constrained else 0)
        return xf

    def inject(self, xf, coarse_level):
        xf = np.ascontiguousarray(xf, dtype=np.float64)
        xc = np.zeros(self.nnodes(coarse_level))
        lib().ora_inject(self.h, coarse_level, _p(xf), _p(xc))
        return xc

    def jacobi(self, x, r, damp, level=None):
        level = self.top if level is None else level
        x = np.array(x, dtype=np.float64, copy=True)
        r = np.array(r, dtype=np.float64, copy=True)
        lib().ora_jacobi(self.h, level, damp, _p(x), _p(r))
        return x, r

    def sor(self, x, b, r, omega, level=None):
        level = self.top if level is None else level
        x = np.array(x, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(b, dtype=np.float64)
        r = np.array(r, dtype=np.float64, copy=True)
        lib().ora_sor(self.h, level, omega, _p(x), _p(b), _p(r))
        return x, r

    def ssc(self, x, b, r, omega=1.0, level=None):
        """One <geometric-ssc> sweep (vertex-centred blocks); b may be r."""
        level = self.top if level is None else level
        alias = b is r
        x = np.array(x, dtype=np.float64, copy=True)
        r = np.array(r, dtype=np.float64, copy=True)
        bb = r if alias else np.ascontiguousarray(b, dtype=np.float64)
        lib().ora_ssc(self.h, level, omega, _p(x), _p(bb), _p(r))
        return x, r

    def psc(self, x, r, damp=1.0, level=None):
        """One <geometric-psc> sweep (vertex-centred blocks, corrections added
        in block order); r is read, not written."""
        level = self.top if level is None else level
        x = np.array(x, dtype=np.float64, copy=True)
        r = np.ascontiguousarray(r, dtype=np.float64)
        lib().ora_psc(self.h, level, damp, _p(x), _p(r))
        return x

    def coarse_solve(self, x, r, damp=1.0):
        x = np.array(x, dtype=np.float64, copy=True)
        r = np.array(r, dtype=np.float64, copy=True)
        lib().ora_coarse_solve(self.h, damp, _p(x), _p(r))
        return x, r

    def vcycle(self, cfg: SolveCfg, x, b, r=None):
        """One multigrid iterator application; r=None aliases r to b."""
        x = np.array(x, dtype=np.float64, copy=True)
        b = np.array(b, dtype=np.float64, copy=True)
        if r is None:
            lib().ora_vcycle(self.h, ctypes.byref(cfg), _p(x), _p(b), _p(b))
            return x, b, b
        r = np.array(r, dtype=np.float64, copy=True)
        lib().ora_vcycle(self.h, ctypes.byref(cfg), _p(x), _p(b), _p(r))
        return x, b, r

    def solve(self, cfg: SolveCfg, x0=None) -> SolveResult:
        n = self.nnodes() * self.nc
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        hist = np.zeros(cfg.maxsteps + 2)
        steps = ctypes.c_int(0)
        st = lib().ora_solve(self.h, ctypes.byref(cfg), _p(x), _p(hist), hist.size,
                             ctypes.byref(steps))
        if st < 0:
            raise RuntimeError(f"ora_solve rc={st}")
        return SolveResult(x, hist[: steps.value + 1].copy(), steps.value, st)


def dot(x, y) -> float:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().ora_dot(_p(x), _p(y), x.size)


def dot_par(x, y) -> float:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().ora_dot_par(_p(x), _p(y), x.size)


def mf_apply(M, dmask, kcell, x, b=None, fp32=False):
    """The 3D Q1 operator of a cell-wise coefficient applied matrix-free in the
    GPU's operation order (y = A x, or b - A x); see ora_mf_apply.  fp32:
    False (FP64), True (FP32 throughout) or 2 (x rounded to FP32, FP64
    arithmetic)."""
    k = np.ascontiguousarray(kcell, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
    mode = 2 if fp32 == 2 else (1 if fp32 else 0)
    lib().ora_mf_apply(int(M), int(dmask), _p(k), mode, _p(x), None if bb is None else _p(bb), _p(y))
    return y


def num_threads() -> int:
    return lib().ora_num_threads()


def set_num_threads(n: int) -> None:
    L = lib()
    L.ora_set_num_threads.argtypes = [ctypes.c_int]
    L.ora_set_num_threads(int(n))
