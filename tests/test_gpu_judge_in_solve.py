"""The plain <geometric-cs> cycle as the judge of the learned one inside the
mixed solve (fmg_mixed_cfg.judge): on the first CG steps after each
(re)start both cycles are applied to the same residual and a step along each
direction is scored by its energy decrease; a learned cycle that does worse
is reverted to the plain one for the rest of the solve.  A damping that is
merely worse than the plain :damp (uniformly too small, CG still converges
with it) is caught, which the divergence rule alone does not do; a divergent
one is caught; the trained network on a held-out field is kept and solves in
fewer iterations than the plain cycle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "gnu_femlisp_b200", "weights", "damping3d.fmgnet")


@pytest.fixture(scope="module")
def G():
    import gnu_femlisp_b200 as G
    return G


@pytest.fixture(scope="module")
def ctx(G):
    return G.Context(0)


def _cfg(G, rtol=1e-10, damp=0.6, maxsteps=200):
    C = G._capi
    return G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, damp, 1, 1, 1, 0, 1.0, rtol, 0.0, maxsteps,
                      C.FMG_MULTIPLICATIVE)


def _grid(G, ctx, level, seed):
    from gnu_femlisp_b200 import problems
    n = 1 << level
    g = G.Grid(ctx, 3, 1, level, base_level=2)
    g.set_coefficient(G._capi.FMG_K_CELL, np.exp(problems.fourier_log_field(n, 3, seed)))
    return g.assemble()


def _uniform_damping(g, w):
    for lev in range(g.base + 1, g.top + 1):
        g.set_node_damping(lev, np.full(g.nnodes(lev), w))


def test_merely_worse_damping_reverts_inside_cg(G, ctx):
    g = _grid(G, ctx, 6, 7)
    cfg = _cfg(G)
    _uniform_damping(g, 0.2)                         # converges, but slower than the plain 0.6
    x0 = g.vector()
    _, _, ni_worse, st = g.solve_mixed(cfg, x0)      # no judge: the divergence rule keeps it
    assert st == 0 and g.learned_status()["reverts"] == 0
    x1 = g.vector()
    h, _, ni, st = g.solve_mixed(cfg, x1, judge=2)
    s = g.learned_status()
    assert st == 0 and h[-1] / h[0] < 1e-10
    assert s["reverts"] == 1 and s["rho_plain"] > s["rho_learned"], s
    assert ni < ni_worse, (ni, ni_worse)
    b = x1.get()
    _uniform_damping(g, 0.6)                         # the same solution as the plain cycle's
    x2 = g.vector()
    g.solve_mixed(cfg, x2)
    assert np.linalg.norm(b - x2.get()) <= 1e-9 * np.linalg.norm(x2.get())


def test_divergent_damping_reverts_inside_cg(G, ctx):
    g = _grid(G, ctx, 5, 3)
    _uniform_damping(g, 1.3)
    x = g.vector()
    h, _, _, st = g.solve_mixed(_cfg(G), x, judge=2)
    assert st == 0 and h[-1] / h[0] < 1e-10 and g.learned_status()["reverts"] == 1


def test_trained_net_is_kept_by_the_in_solve_judge(G, ctx):
    from gnu_femlisp_b200.learn import DampingNet
    g = _grid(G, ctx, 6, 0)
    cfg = _cfg(G)
    xp = g.vector()
    _, _, ni_plain, st = g.solve_mixed(cfg, xp)
    assert st == 0
    net = DampingNet.load(ctx, WEIGHTS)
    net.apply(g)
    xl = g.vector()
    h, _, ni_l, st = g.solve_mixed(cfg, xl, judge=2)
    s = g.learned_status()
    assert st == 0 and h[-1] / h[0] < 1e-10
    assert s["reverts"] == 0 and s["rho_learned"] >= s["rho_plain"], s
    assert ni_l < ni_plain, (ni_l, ni_plain)
    net.close()
