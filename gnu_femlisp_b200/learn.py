"""The learned part of the smoother: a damping network that predicts the
Jacobi damping of every node from the coefficient field around it.

No counterpart in the reference.  The network (``fmg_net_*`` in
include/fmgpu.h) runs on the tensor cores for inference and training; this
module holds the handle, the training loop and the training problems.  Its
predictions are installed as per-node damping of the levels of a grid, i.e.
they replace the scalar ``:damp`` of ``<jacobi>`` (linit.lisp:220-250) node
by node in both the FP64 and the mixed-precision cycles; plain
``<geometric-cs>`` with the scalar damping stays the fallback (the judge of
``solve_mixed`` reverts to it when a learned cycle reduces the residual less).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _capi as C
from . import core as _core
from ._capi import FmgError  # noqa: F401
from .core import Context, Grid, Vector


class DampingNet:
    """Handle of one damping network (``fmg_net_create``/``fmg_net_load``)."""

    def __init__(self, ctx: Context, dim: int = 3, seed: int = 0, _handle=None):
        self.ctx = ctx
        lib = ctx._lib
        if _handle is None:
            h = ctypes.c_void_p()
            ctx.check(lib.fmg_net_create(ctx.h, dim, seed, ctypes.byref(h)), "net_create")
            _handle = h
        self.h = _handle
        self.n = int(lib.fmg_net_nparams(self.h))
        self.dim = dim

    @classmethod
    def load(cls, ctx: Context, path: str) -> "DampingNet":
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.fmg_net_load(ctx.h, path.encode(), ctypes.byref(h)), f"net_load({path})")
        net = cls.__new__(cls)
        net.ctx, net.h = ctx, h
        net.n = int(ctx._lib.fmg_net_nparams(h))
        net.dim = 3 if net.n > 20000 else 2
        return net

    @property
    def _lib(self):
        return self.ctx._lib

    def save(self, path: str):
        self.ctx.check(self._lib.fmg_net_save(self.h, path.encode()), f"net_save({path})")

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        self.ctx.check(self._lib.fmg_net_get_params(self.h, C.fptr(out), self.n), "net_get_params")
        return out

    @params.setter
    def params(self, values):
        v = np.ascontiguousarray(values, dtype=np.float32).ravel()
        self.ctx.check(self._lib.fmg_net_set_params(self.h, C.fptr(v), v.size), "net_set_params")

    @property
    def grads(self) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        self.ctx.check(self._lib.fmg_net_get_grads(self.h, C.fptr(out), self.n), "net_get_grads")
        return out

    def zero_grads(self):
        self.ctx.check(self._lib.fmg_net_zero_grads(self.h), "net_zero_grads")

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        self.ctx.check(self._lib.fmg_net_adam(self.h, lr, beta1, beta2, eps), "net_adam")

    def damping(self, grid: Grid, level: int | None = None) -> np.ndarray:
        """Forward pass on one level; installs and returns its node damping."""
        level = grid.top if level is None else level
        out = np.zeros(grid.nnodes(level))
        self.ctx.check(self._lib.fmg_net_damping(self.h, grid.h, level, C.dptr(out)), "net_damping")
        return out

    def apply(self, grid: Grid):
        """Forward pass on every level above the base (installs the damping)."""
        self.ctx.check(self._lib.fmg_net_apply(self.h, grid.h), "net_apply")

    def apply_top(self, grid: Grid):
        """Forward pass on the top level only (the levels below keep the
        scalar damping) -- the setting the network is trained in."""
        for lev in range(grid.base + 1, grid.top):
            grid.set_node_damping(lev, None)
        self.damping(grid, grid.top)

    def backward(self, grid: Grid, level: int, gomega):
        g = np.ascontiguousarray(gomega, dtype=np.float64)
        self.ctx.check(self._lib.fmg_net_backward(self.h, grid.h, level, C.dptr(g)), "net_backward")

    def step(self, grid: Grid, cfg: C.SolveCfg, nsamples: int = 4, seed: int = 0, max_cycles: int = 2) -> float:
        """One training step (forward, MG-generated errors, loss, backward);
        returns the mean loss.  Gradients accumulate until :meth:`adam`."""
        loss = ctypes.c_double()
        self.ctx.check(self._lib.fmg_learn_step(self.h, grid.h, ctypes.byref(cfg), nsamples, seed, max_cycles,
                                                ctypes.byref(loss)), "learn_step")
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            self._lib.fmg_net_destroy(self.h)
            self.h = None

    def __del__(self):
        if _core is None or _core._EXITING:
            return
        try:
            self.close()
        except Exception:
            pass


def learn_loss(grid: Grid, cfg: C.SolveCfg, e0: Vector, want_grad: bool = True):
    """V-cycle A-norm contraction of e0 with the top level's damping, and its
    gradient with respect to that damping (``fmg_learn_loss``)."""
    loss = ctypes.c_double()
    g = np.zeros(grid.nnodes()) if want_grad else None
    grid.ctx.check(grid._lib.fmg_learn_loss(grid.h, ctypes.byref(cfg), e0.h, ctypes.byref(loss),
                                            C.dptr(g) if want_grad else None), "learn_loss")
    return loss.value, g


def learn_loss_levels(grid: Grid, cfg: C.SolveCfg, e0: Vector, level: int, want_grad: bool = True):
    """The same loss with the damping of every level differentiated through
    the whole cycle; returns (loss, dL/domega of `level`)
    (``fmg_learn_loss_levels``)."""
    loss = ctypes.c_double()
    g = np.zeros(grid.nnodes(level)) if want_grad else None
    grid.ctx.check(grid._lib.fmg_learn_loss_levels(grid.h, ctypes.byref(cfg), e0.h, level, ctypes.byref(loss),
                                                   C.dptr(g) if want_grad else None), "learn_loss_levels")
    return loss.value, g


# ------------------------------------------------------- training problems
def fourier_log_window(n: int, dim: int, seed: int, offset, scale: float, modes: int = 64,
                       kmin: float = 1.0, kmax: float = 10.0) -> np.ndarray:
    """The variable-coefficient field of the 256^3 benchmark problem (64
    random Fourier modes, |kappa| ~ U[1,10]) evaluated at the cell centres of
    an n^dim grid covering the window offset + scale [0,1]^dim, normalised by
    the field's expected standard deviation (sqrt(sum a_m^2 / 2)), so that
    windows keep the cell-to-cell contrast of the full field at resolution
    n / scale."""
    rng = np.random.default_rng(seed)
    mag = rng.uniform(kmin, kmax, modes)
    direc = rng.standard_normal((modes, dim))
    direc /= np.linalg.norm(direc, axis=1, keepdims=True)
    kappa = mag[:, None] * direc
    phi = rng.uniform(0.0, 2.0 * np.pi, modes)
    amp = rng.standard_normal(modes)
    coef = amp * np.exp(1j * phi)
    off = np.broadcast_to(np.asarray(offset, dtype=float), (dim,))
    xs = [off[k] + scale * (np.arange(n) + 0.5) / n for k in range(dim)]
    e = [np.exp(2j * np.pi * kappa[:, k][:, None] * xs[k][None, :]) for k in range(dim)]
    if dim == 2:
        field = np.real((e[1].T * coef) @ e[0])
    else:
        left = (e[2].T[:, None, :] * e[1].T[None, :, :] * coef).reshape(n * n, modes)
        field = np.real(left @ e[0])
    return field.reshape(-1) / np.sqrt(0.5 * np.sum(amp ** 2))


@dataclass
class TrainSpec:
    dim: int = 3
    level: int = 5             # training grids of 2^level cells per direction
    base: int = 2
    count: int = 12            # training grids
    seed: int = 1000           # field seeds seed .. seed+count-1 (held out from the benchmark's seed 0)
    scales: tuple = (0.125, 0.25, 0.5, 1.0)
    steps: int = 600
    lr: float = 2e-3
    nsamples: int = 4
    max_cycles: int = 4
    damp: float = 0.6


def training_grids(ctx: Context, spec: TrainSpec):
    """Grids with fields drawn like the benchmark's at several resolutions:
    windows of side `scale` of the unit cube, so one training grid of 2^level
    cells sees the contrast the net meets on a level of 2^level / scale cells."""
    rng = np.random.default_rng(spec.seed)
    grids = []
    n = 1 << spec.level
    for i in range(spec.count):
        scale = spec.scales[i % len(spec.scales)]
        off = rng.uniform(0.0, 1.0 - scale, spec.dim) if scale < 1.0 else np.zeros(spec.dim)
        k = np.exp(fourier_log_window(n, spec.dim, spec.seed + i, off, scale))
        g = Grid(ctx, spec.dim, 1, spec.level, spec.base)
        g.set_coefficient(C.FMG_K_CELL, k)
        g.assemble()
        grids.append(g)
    return grids


def elasticity_training_grids(ctx: Context, level: int = 3, count: int = 8, seed: int = 1000,
                              scales=(0.25, 0.5, 1.0), sigma: float = 0.5):
    """Grids of the clamped-cube elasticity problem (vector Q2, 3 * 2^level
    cells per direction, base level 0, the x = 0 face clamped, force -z) with
    Young's-modulus fields drawn like the benchmark's, E = exp(sigma g) with g
    the unit-std Fourier field, on windows of side `scale` of the unit cube
    (field seeds seed .. seed+count-1; the benchmark uses seed 0)."""
    rng = np.random.default_rng(seed)
    n = 3 << level
    grids = []
    for i in range(count):
        scale = scales[i % len(scales)]
        off = rng.uniform(0.0, 1.0 - scale, 3) if scale < 1.0 else np.zeros(3)
        e = np.exp(sigma * fourier_log_window(n, 3, seed + i, off, scale))
        g = Grid(ctx, 3, 2, level, 0, n0=3, ncomp=3, dirichlet_mask=0b000001)
        g.set_coefficient(C.FMG_LAMBDA_MU_CELL, e)
        g.set_coefficient(C.FMG_F_VEC, [0.0, 0.0, -1.0])
        g.assemble()
        grids.append(g)
    return grids


def train(net: DampingNet, grids, cfg: C.SolveCfg, steps: int, lr: float, nsamples: int = 4,
          max_cycles: int = 4, seed: int = 0, lr_end: float | None = None, log=None):
    """Adam on the mean V-cycle loss, cycling through the training grids, the
    learning rate decaying from lr to lr_end (cosine); returns the loss history."""
    lr_end = lr / 10 if lr_end is None else lr_end
    hist = []
    for it in range(steps):
        g = grids[it % len(grids)]
        loss = net.step(g, cfg, nsamples, seed * 1000003 + it, max_cycles)
        rate = lr_end + 0.5 * (lr - lr_end) * (1 + np.cos(np.pi * it / max(1, steps - 1)))
        net.adam(rate)
        hist.append(loss)
        if log and (it % max(1, steps // 20) == 0 or it == steps - 1):
            log(f"step {it:5d} loss {loss:.5f} lr {rate:.2e}")
    return np.array(hist)


def mean_loss(grids, cfg: C.SolveCfg, nsamples: int = 4, seed: int = 7, cycles: int = 0) -> float:
    """Mean V-cycle loss, with the damping currently installed, of random
    errors after `cycles` cycles of A e = 0 (the same cycle)."""
    tot = 0.0
    for g in grids:
        e, z, r = g.vector(), g.vector(), g.vector()
        for s in range(nsamples):
            rng = np.random.default_rng(seed * 7919 + s)
            v = rng.uniform(-1, 1, g.nnodes())
            v[_dirichlet_mask(g)] = 0.0
            e.set(v)
            for _ in range(cycles):
                g.residual(e, z, r)
                g.vcycle(cfg, e, z, r)
            tot += learn_loss(g, cfg, e, want_grad=False)[0]
    return tot / (len(grids) * nsamples)


def _dirichlet_mask(g: Grid) -> np.ndarray:
    m = (g.order * g.n_cells) + 1
    idx = np.indices((m,) * g.dim).reshape(g.dim, -1)[::-1]  # x fastest
    bnd = np.zeros(idx.shape[1], bool)
    for k in range(g.dim):
        bnd |= (idx[k] == 0) | (idx[k] == m - 1)
    return bnd


# -------------------------------------------- the batched 2D block-field set
def block_field(seed: int, n: int = 128, blocks: int = 8, lo: float = -3.0, hi: float = 3.0) -> np.ndarray:
    """Diffusion per cell of an n x n grid, piecewise constant on a
    blocks x blocks partition with log10 k ~ U[lo, hi] per block (seeded)."""
    from .problems import block_log10_field
    return 10.0 ** block_log10_field(n, blocks, seed, lo, hi)


def train_on_fields(net: DampingNet, ctx: Context, field_of, seeds, cfg: C.SolveCfg, dim: int, level: int,
                    base: int, pool: int = 8, lr: float = 2e-3, lr_end: float | None = None, nsamples: int = 4,
                    max_cycles: int = 4, log=None):
    """One Adam step per field: field_of(seed) gives the cell coefficients;
    a pool of grids is re-assembled with each new field, so every step trains
    on a field not seen before.  Returns the loss history."""
    seeds = list(seeds)
    steps = len(seeds)
    lr_end = lr / 10 if lr_end is None else lr_end
    grids = [Grid(ctx, dim, 1, level, base) for _ in range(pool)]
    hist = []
    for it, sd in enumerate(seeds):
        g = grids[it % pool]
        g.set_coefficient(C.FMG_K_CELL, field_of(sd))
        g.assemble()
        loss = net.step(g, cfg, nsamples, 7919 * sd + 1, max_cycles)
        rate = lr_end + 0.5 * (lr - lr_end) * (1 + np.cos(np.pi * it / max(1, steps - 1)))
        net.adam(rate)
        hist.append(loss)
        if log and (it % max(1, steps // 20) == 0 or it == steps - 1):
            log(f"step {it:6d} field {sd} loss {loss:.5f} mean(last 200) {np.mean(hist[-200:]):.5f}")
    for g in grids:
        g.close()
    return np.array(hist)


def evaluate_on_fields(net: DampingNet, ctx: Context, field_of, seeds, cfg: C.SolveCfg, dim: int, level: int,
                       base: int, top_only: bool = True):
    """Per field: steps and solve time of the plain cycle (scalar damping) and
    of the learned damping (network on every level, then the judge), from x = 0
    to cfg's tolerance with fmg_solve.  Times are wall clock of the solve call
    (it synchronises), without the setup; the learned setup is timed apart."""
    import time
    g = Grid(ctx, dim, 1, level, base)
    x = g.vector()
    rows = []
    for sd in seeds:
        g.set_coefficient(C.FMG_K_CELL, field_of(sd))
        g.assemble()
        for lev in range(g.base + 1, g.top + 1):
            g.set_node_damping(lev, None)
        x.fill(0.0)
        t0 = time.perf_counter()
        hp, sp, stp = g.solve(cfg, x)
        tp = time.perf_counter() - t0
        t0 = time.perf_counter()
        if top_only:
            net.apply_top(g)
        else:
            net.apply(g)
        ok, rp, rl = g.learned_judge(cfg)
        ts = time.perf_counter() - t0
        x.fill(0.0)
        t0 = time.perf_counter()
        hl, sl, stl = g.solve(cfg, x)
        tl = time.perf_counter() - t0
        rows.append(dict(seed=sd, plain_steps=sp, plain_status=stp, plain_s=tp, learned_steps=sl,
                         learned_status=stl, learned_s=tl, setup_s=ts, accepted=ok, rho_plain=rp,
                         rho_learned=rl))
    x.close()
    g.close()
    return rows
