"""The vector (elasticity) form of the oracle, checked on the CPU against
properties the discretisation must have, since the reference ships no
golden vectors for its elasticity path: rigid-body modes in the kernel of
the unconstrained operator, symmetry and positive definiteness with the
x = 0 face clamped, linear displacements reproduced exactly (zero interior
rows), and CG preconditioned by the block-Jacobi V(2,2) cycle reaching the
dense solution."""
import numpy as np
import pytest

from oracle import oracle as O


def dense(o, level):
    """The level matrix as a dense (3N x 3N) array from the [slot][k][l][node] storage."""
    nc, dim = o.nc, o.dim
    A = o.matrix(level).reshape(o.nslots, nc, nc, -1)
    N = A.shape[-1]
    M = round(N ** (1.0 / dim))
    w = 2 * o.order + 1
    D = np.zeros((N * nc, N * nc))
    idx = np.arange(N)
    c = np.stack([idx % M, (idx // M) % M, idx // (M * M)], 1)
    for s in range(o.nslots):
        off = np.array([s % w, (s // w) % w, s // (w * w)]) - o.order
        cj = c + off
        ok = np.all((cj >= 0) & (cj < M), 1)
        j = cj[:, 0] + M * (cj[:, 1] + M * cj[:, 2])
        for k in range(nc):
            for m in range(nc):
                D[idx[ok] * nc + k, j[ok] * nc + m] += A[s, k, m, ok]
    return D, c, M


def make(level=1, n0=1, dmask=0, ecell=None, order=2, base=0):
    o = O.Oracle(3, order, level, base_level=base, ncomp=3, n0=n0, dirichlet_mask=dmask)
    if ecell is not None:
        o.set_coefficient(O.LAMBDA_MU_CELL, ecell)
    o.set_coefficient(O.F_VEC, [0.0, 0.0, -1.0])
    return o.assemble()


@pytest.mark.parametrize("order", [1, 2])
def test_rigid_body_modes_in_the_kernel(order):
    rng = np.random.default_rng(0)
    ncell = 2 ** 3
    o = make(level=1, dmask=0, ecell=np.exp(0.5 * rng.standard_normal(ncell)), order=order)
    D, c, M = dense(o, 1)
    x = c / (M - 1)
    modes = [np.tile([1.0, 0, 0], (len(x), 1)), np.tile([0, 1.0, 0], (len(x), 1)), np.tile([0, 0, 1.0], (len(x), 1)),
             np.stack([-x[:, 1], x[:, 0], 0 * x[:, 0]], 1), np.stack([0 * x[:, 0], -x[:, 2], x[:, 1]], 1),
             np.stack([x[:, 2], 0 * x[:, 0], -x[:, 0]], 1)]
    scale = np.abs(D).max()
    for u in modes:
        assert np.abs(D @ u.reshape(-1)).max() < 1e-12 * scale


def test_clamped_operator_is_spd():
    rng = np.random.default_rng(1)
    o = make(level=1, n0=1, dmask=0b000001, ecell=np.exp(0.5 * rng.standard_normal(8)))
    D, _, _ = dense(o, 1)
    assert np.abs(D - D.T).max() < 1e-14 * np.abs(D).max()
    assert np.linalg.eigvalsh(D).min() > 0


def test_linear_displacement_gives_zero_interior_rows():
    o = make(level=2, dmask=0)  # E = 1
    D, c, M = dense(o, 2)
    x = c / (M - 1)
    u = np.stack([0.3 * x[:, 0] + 0.1 * x[:, 1], -0.2 * x[:, 2], 0.5 * x[:, 0] + 0.7 * x[:, 2]], 1).reshape(-1)
    y = (D @ u).reshape(-1, 3)
    interior = np.all((c > 0) & (c < M - 1), 1)
    assert np.abs(y[interior]).max() < 1e-12 * np.abs(D).max()


def test_cg_block_jacobi_vcycle_reaches_the_dense_solution():
    # the benchmark's shape at a small size: 3^3 base cells, x = 0 face clamped
    rng = np.random.default_rng(2)
    ncell = (3 * 2) ** 3
    o = make(level=1, n0=3, dmask=0b000001, ecell=np.exp(0.5 * rng.standard_normal(ncell)), base=0)
    cfg = O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.JACOBI, damp=0.5, pre=2, post=2, compat=False,
                      rtol=1e-10, maxsteps=200)
    r = o.solve(cfg)
    assert r.status == 0 and r.steps < 60, (r.status, r.steps)
    D, _, _ = dense(o, 1)
    xd = np.linalg.solve(D, o.rhs())
    assert np.linalg.norm(r.x - xd) / np.linalg.norm(xd) < 1e-8
    # the body force pulls the free end down
    assert xd.reshape(-1, 3)[:, 2].min() < 0
