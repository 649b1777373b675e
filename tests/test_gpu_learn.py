"""Damping network on the GPU: the tensor-core forward and backward kernels
against the CPU oracle (oracle/net_oracle.py), the training-loss gradient
against finite differences, training, and the weight file."""
import os

import numpy as np
import pytest

from oracle import net_oracle as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gnu_femlisp_b200 as G
    return G


@pytest.fixture(scope="module")
def ctx(G):
    return G.Context(0)


def _cfg(G, damp=0.6):
    C = G._capi
    return G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, damp, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 100,
                      C.FMG_MULTIPLICATIVE)


def _grid(G, ctx, dim, level, base, seed):
    from gnu_femlisp_b200 import problems
    n = 1 << level
    k = np.exp(problems.fourier_log_field(n, dim, seed))
    g = G.Grid(ctx, dim, 1, level, base_level=base)
    g.set_coefficient(G._capi.FMG_K_CELL, k)
    return g.assemble(), k


CASES = [(2, 5, 2), (3, 4, 1)]


@pytest.mark.parametrize("dim,level,base", CASES)
def test_forward_matches_oracle(G, ctx, dim, level, base):
    from gnu_femlisp_b200.learn import DampingNet
    g, k = _grid(G, ctx, dim, level, base, seed=11)
    net = DampingNet(ctx, dim, seed=0)
    p = N.init_params(dim, seed=3, scale=1.5)
    net.params = p
    n_top = 1 << level
    for lev in (level, level - 1):
        om = net.damping(g, lev)
        X0 = N.features(k, dim, n_top, 1 << lev)
        ref, _ = N.forward(p, X0, dim)
        err = np.abs(om - ref)
        assert err.max() < 5e-3 and err.mean() < 5e-4, (lev, err.max(), err.mean())
        assert om.std() > 1e-2  # the random net is not constant


@pytest.mark.parametrize("dim,level,base", CASES)
def test_backward_matches_oracle(G, ctx, dim, level, base):
    from gnu_femlisp_b200.learn import DampingNet
    g, k = _grid(G, ctx, dim, level, base, seed=12)
    net = DampingNet(ctx, dim, seed=0)
    p = N.init_params(dim, seed=4, scale=1.5)
    net.params = p
    om = net.damping(g, level)
    gw = np.random.default_rng(1).standard_normal(om.size)
    net.zero_grads()
    net.backward(g, level, gw)
    got = net.grads
    X0 = N.features(k, dim, 1 << level, 1 << level)
    _, cache = N.forward(p, X0, dim)
    ref = N.backward(p, cache, gw, dim)
    L = N.layout(dim)
    for key in ("w1", "b1", "w2", "b2", "w3", "b3"):
        a, b = got[L[key][0]:L[key][1]], ref[L[key][0]:L[key][1]]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 3e-2, (key, rel)
    # accumulation: a second backward doubles the gradient
    net.backward(g, level, gw)
    assert np.allclose(net.grads, 2 * got, rtol=1e-5, atol=1e-7)


def test_loss_gradient_matches_finite_differences(G, ctx):
    from gnu_femlisp_b200.learn import learn_loss
    g, _ = _grid(G, ctx, 3, 4, 1, seed=13)
    cfg = _cfg(G)
    rng = np.random.default_rng(2)
    n = g.nnodes()
    w = rng.uniform(0.4, 1.0, n)
    e0 = rng.uniform(-1, 1, n)
    m = (1 << 4) + 1
    idx = np.indices((m, m, m)).reshape(3, -1)
    e0[((idx == 0) | (idx == m - 1)).any(0)] = 0.0
    ev = g.vector(values=e0)
    g.set_node_damping(g.top, w)
    L0, grad = learn_loss(g, cfg, ev)
    assert 0.0 < L0 < 1.0
    d = rng.standard_normal(n)
    eps = 1e-5
    g.set_node_damping(g.top, w + eps * d)
    Lp, _ = learn_loss(g, cfg, ev, want_grad=False)
    g.set_node_damping(g.top, w - eps * d)
    Lm, _ = learn_loss(g, cfg, ev, want_grad=False)
    fd = (Lp - Lm) / (2 * eps)
    assert abs(fd - grad @ d) <= 1e-6 * max(1.0, abs(fd)), (fd, grad @ d)


def test_all_level_gradient_matches_finite_differences(G, ctx):
    # dL/domega of a coarse level and of the top level through the whole
    # V-cycle, against central differences; the loss equals fmg_learn_loss's
    from gnu_femlisp_b200.learn import learn_loss, learn_loss_levels
    g, _ = _grid(G, ctx, 3, 4, 1, seed=14)
    cfg = _cfg(G)
    rng = np.random.default_rng(3)
    ws = {}
    for lev in range(g.base + 1, g.top + 1):
        ws[lev] = rng.uniform(0.4, 1.0, g.nnodes(lev))
        g.set_node_damping(lev, ws[lev])
    n = g.nnodes()
    e0 = rng.uniform(-1, 1, n)
    m = (1 << 4) + 1
    idx = np.indices((m, m, m)).reshape(3, -1)
    e0[((idx == 0) | (idx == m - 1)).any(0)] = 0.0
    ev = g.vector(values=e0)
    L_old, _ = learn_loss(g, cfg, ev, want_grad=False)
    for lev in (g.top - 1, g.top):
        L0, grad = learn_loss_levels(g, cfg, ev, lev)
        assert abs(L0 - L_old) <= 1e-12 * L_old, (L0, L_old)
        d = rng.standard_normal(ws[lev].size)
        eps = 1e-5
        g.set_node_damping(lev, ws[lev] + eps * d)
        Lp, _ = learn_loss_levels(g, cfg, ev, lev, want_grad=False)
        g.set_node_damping(lev, ws[lev] - eps * d)
        Lm, _ = learn_loss_levels(g, cfg, ev, lev, want_grad=False)
        g.set_node_damping(lev, ws[lev])
        fd = (Lp - Lm) / (2 * eps)
        assert abs(fd - grad @ d) <= 1e-6 * max(1e-3, abs(fd)), (lev, fd, grad @ d)


def test_training_lowers_the_loss(G, ctx):
    from gnu_femlisp_b200.learn import DampingNet, TrainSpec, mean_loss, train, training_grids
    spec = TrainSpec(dim=3, level=4, base=1, count=3)
    grids = training_grids(ctx, spec)
    cfg = _cfg(G)
    for g in grids:  # plain damping
        g.set_node_damping(g.top, np.full(g.nnodes(), 0.6))
    plain = mean_loss(grids, cfg)
    net = DampingNet(ctx, 3, seed=1)
    hist = train(net, grids, cfg, steps=60, lr=3e-3, nsamples=2, max_cycles=1)
    assert np.all(np.isfinite(hist))
    for g in grids:
        net.apply(g)
    learned = mean_loss(grids, cfg)
    assert learned < 0.9 * plain, (plain, learned, hist[:3], hist[-3:])


def test_weight_file_roundtrip_and_corruption(G, ctx, tmp_path):
    from gnu_femlisp_b200.learn import DampingNet
    net = DampingNet(ctx, 2, seed=9)
    p = N.init_params(2, seed=9)
    net.params = p
    path = str(tmp_path / "net.bin")
    net.save(path)
    back = DampingNet.load(ctx, path)
    assert np.array_equal(back.params, p)
    raw = bytearray(open(path, "rb").read())
    raw[100] ^= 0x40
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(G.FmgError) as ei:
        DampingNet.load(ctx, bad)
    assert ei.value.code == -7 and "checksum" in str(ei.value)
    open(bad, "wb").write(bytes(raw[:50]))
    with pytest.raises(G.FmgError):
        DampingNet.load(ctx, bad)
