"""The trained damping network inside the solver: what it gains over the
plain <geometric-cs> cycle it replaces, and the judge that falls back to that
plain cycle when a learned cycle does worse (a forced divergence)."""
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


def test_trained_net_beats_the_plain_cycle(G, ctx):
    # the benchmark's field recipe with its seed 0 (training used seeds 1000+) at 64^3
    from gnu_femlisp_b200.learn import DampingNet
    g = _grid(G, ctx, 6, 0)
    cfg = _cfg(G)
    xp = g.vector()
    hp, ns_p, st = g.solve(cfg, xp)
    assert st == 0
    xmp = g.vector()
    _, _, ni_p, st = g.solve_mixed(cfg, xmp)
    assert st == 0
    net = DampingNet.load(ctx, WEIGHTS)
    net.apply(g)
    ok, rho_p, rho_l = g.learned_judge(cfg)
    assert ok and rho_l < rho_p, (rho_p, rho_l)
    xl = g.vector()
    hl, ns_l, st = g.solve(cfg, xl)
    assert st == 0 and hl[-1] / hl[0] < 1e-10
    xml = g.vector()
    hml, _, ni_l, st = g.solve_mixed(cfg, xml)
    assert st == 0 and hml[-1] / hml[0] < 1e-10
    assert g.learned_status()["reverts"] == 0
    # at least two CG steps fewer than the plain cycle, FP64 and mixed
    assert ns_l <= ns_p - 2, (ns_p, ns_l)
    assert ni_l <= ni_p - 2, (ni_p, ni_l)
    # same discrete solution
    a, b = xl.get(), xp.get()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8
    a = xml.get()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8


def _divergent_net(G, ctx):
    from gnu_femlisp_b200.learn import DampingNet
    net = DampingNet(ctx, 3, seed=2)
    p = net.params
    p[-1] = 20.0  # output bias: damping 1.3 at every node, beyond Jacobi's stability limit
    net.params = p
    return net


def test_judge_rejects_a_divergent_net(G, ctx):
    g = _grid(G, ctx, 5, 4)
    cfg = _cfg(G)
    net = _divergent_net(G, ctx)
    om = net.damping(g, g.top)
    assert np.all(om[np.abs(om - 1.3) < 1e-3].size > 0.99 * om.size)
    net.apply(g)
    ok, rho_p, rho_l = g.learned_judge(cfg)
    assert not ok and rho_l > rho_p, (rho_p, rho_l)
    assert not g.learned_status()["active"]
    x = g.vector()
    hist, _, ni, st = g.solve_mixed(cfg, x)
    assert st == 0 and hist[-1] / hist[0] < 1e-10


def test_runtime_judge_reverts_to_the_plain_cycle(G, ctx):
    # the multigrid iteration (stationary), where per-cycle residual reductions
    # are meaningful: the setup judge measures the plain cycle, then a
    # divergent damping is installed behind its back; the first cycles grow
    # the residual, the judge drops the damping and the iteration converges
    from gnu_femlisp_b200.learn import DampingNet
    g = _grid(G, ctx, 5, 5)
    C = G._capi
    mg = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 300, C.FMG_MULTIPLICATIVE)
    x0 = g.vector()
    _, ns_plain, st = g.solve(mg, x0)
    assert st == 0
    good = DampingNet.load(ctx, WEIGHTS)
    good.apply(g)
    g.learned_judge(mg)
    net = _divergent_net(G, ctx)
    net.apply(g)
    before = g.learned_status()["reverts"]
    x = g.vector()
    hist, ns, st = g.solve(mg, x)
    rates = (hist[1:] / hist[:-1]).round(3).tolist()
    assert st == 0 and hist[-1] / hist[0] < 1e-10, rates[:10]
    assert g.learned_status()["reverts"] == before + 1, rates[:10]
    assert ns <= ns_plain + 6, (ns_plain, ns)
    b = x0.get()
    assert np.linalg.norm(x.get() - b) / np.linalg.norm(b) < 1e-8


def test_mixed_solve_survives_a_divergent_damping(G, ctx):
    # the same damping inside the mixed flexible CG: it must still reach the
    # FP64 tolerance and the FP64 solution (reverting only if it diverges)
    g = _grid(G, ctx, 5, 6)
    cfg = _cfg(G)
    x0 = g.vector()
    _, _, _, st = g.solve_mixed(cfg, x0)
    assert st == 0
    net = _divergent_net(G, ctx)
    net.apply(g)
    x = g.vector()
    hist, _, ni, st = g.solve_mixed(cfg, x)
    assert st == 0 and hist[-1] / hist[0] < 1e-10
    b = x0.get()
    assert np.linalg.norm(x.get() - b) / np.linalg.norm(b) < 1e-8


def test_2d_net_gains_on_held_out_block_fields(G, ctx):
    # the block-field set (2D Q1 128^2, 8x8 blocks, log10 k ~ U[-3,3]): on
    # held-out seeds, CG preconditioned by the cycle with the learned damping
    # (network on every level, then the judge) needs fewer steps than with the
    # plain w = 0.6 cycle, and never fails
    from gnu_femlisp_b200 import learn
    C = G._capi
    net = learn.DampingNet.load(ctx, os.path.join(ROOT, "gnu_femlisp_b200", "weights", "damping2d.fmgnet"))
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 200,
                     C.FMG_MULTIPLICATIVE)
    rows = learn.evaluate_on_fields(net, ctx, learn.block_field, range(1000000, 1000008), cfg, 2, 7, 2,
                                    top_only=False)
    plain = np.array([r["plain_steps"] for r in rows])
    lrn = np.array([r["learned_steps"] for r in rows])
    assert all(r["plain_status"] == 0 and r["learned_status"] == 0 for r in rows)
    assert lrn.mean() <= 0.85 * plain.mean(), (plain, lrn)
    assert np.all(lrn <= plain + 1), (plain, lrn)


def test_mixed_judge_agrees_with_the_fp64_judge(G, ctx):
    # the judge's CG probe run with the mixed cycle: same verdicts, contraction
    # figures close to the FP64 cycle's (the FP32/BF16 cycle is a slightly
    # different preconditioner), and the divergent damping is still rejected
    from gnu_femlisp_b200.learn import DampingNet
    g = _grid(G, ctx, 6, 0)
    cfg = _cfg(G)
    net = DampingNet.load(ctx, WEIGHTS)
    net.apply(g)
    ok64, rp64, rl64 = g.learned_judge(cfg)
    net.apply(g)
    ok, rp, rl = g.learned_judge_mixed(cfg)
    assert ok64 and ok and rl < 0.98 * rp, (rp, rl)
    assert abs(rp - rp64) < 0.1 * rp64 and abs(rl - rl64) < 0.1 * rl64, (rp64, rl64, rp, rl)
    assert g.learned_status()["active"]
    x = g.vector()
    hist, _, _, st = g.solve_mixed(cfg, x)
    assert st == 0 and hist[-1] / hist[0] < 1e-10
    bad = _divergent_net(G, ctx)
    bad.apply(g)
    ok, rp2, rl2 = g.learned_judge_mixed(cfg)
    assert not ok and rl2 > rp2 and not g.learned_status()["active"], (rp2, rl2)
    assert abs(rp2 - rp) < 1e-9 * rp  # the plain probe is deterministic
    C = G._capi
    mg = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 10, C.FMG_MULTIPLICATIVE)
    bad.apply(g)
    with pytest.raises(G.FmgError):
        g.learned_judge_mixed(mg)
