"""CPU checks of the damping-network oracle (oracle/net_oracle.py): its BF16
rounding and its backward pass against central finite differences of its own
float64 forward pass.  The network has no counterpart in the reference, so
these checks pin the oracle the GPU kernels are compared with."""
import numpy as np
import pytest

from oracle import net_oracle as N


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e-3, 0.0], np.float32)
    y = N.bf16(x)
    assert y[0] == 1.0
    assert y[1] == 1.0                      # tie -> even mantissa
    assert y[2] == 1.0 + 2.0 ** -6          # tie -> even mantissa (up)
    assert y[3] == -2.5
    assert abs(y[4] - 3.0e-3) <= 3.0e-3 * 2.0 ** -8
    assert y[5] == 0.0


def test_layout_sizes():
    assert N.layout(3)["n"] == 27 * 512 + 32 + 27 * 1024 + 32 + 27 * 32 + 1
    assert N.layout(2)["n"] == 9 * 512 + 32 + 9 * 1024 + 32 + 9 * 32 + 1


@pytest.mark.parametrize("dim,level_n", [(2, 6), (3, 3)])
def test_oracle_backward_matches_finite_differences(dim, level_n):
    rng = np.random.default_rng(dim)
    kcell = np.exp(rng.standard_normal(level_n ** dim))
    X0 = N.features(kcell, dim, level_n, level_n, emulate=False)
    p = N.init_params(dim, seed=5, scale=2.0).astype(np.float64)
    om, cache = N.forward(p, X0, dim, emulate=False)
    gw = rng.standard_normal(om.size)
    grad = N.backward(p, cache, gw, dim, emulate=False)
    L = N.layout(dim)
    eps = 1e-6
    idx = np.concatenate([rng.choice(np.arange(*L[k]), size=min(6, L[k][1] - L[k][0]), replace=False)
                          for k in ("w1", "b1", "w2", "b2", "w3", "b3")])
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (gw @ N.forward(pp, X0, dim, emulate=False)[0] - gw @ N.forward(pm, X0, dim, emulate=False)[0]) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_features_coarse_level_averages_gauss_samples():
    # on a coarse level each cell feature is the mean log k over the fine cells
    # hit by its Gauss points: with k constant per 2x2 block the coarse feature
    # equals the block value
    dim, n_top = 2, 8
    blocks = np.arange(16, dtype=float).reshape(4, 4)
    lk = np.kron(blocks, np.ones((2, 2)))
    X = N.features(np.exp(lk.ravel()), dim, n_top, 4, emulate=False)
    mu = lk.mean()
    # node (1,1) of the coarse level: cells (0,0),(1,0),(0,1),(1,1) -> channels 0..3
    assert np.allclose(X[0, 1, 1, :4], (np.array([blocks[0, 0], blocks[0, 1], blocks[1, 0], blocks[1, 1]]) - mu) / 2)
    assert np.allclose(X[0, 1, 1, 4:8], 1.0)
    assert np.allclose(X[0, 0, 0, 4:8], [0, 0, 0, 1])   # corner node: only cell (0,0) present
