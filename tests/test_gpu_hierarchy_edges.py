"""Edge cases of the hierarchy on the GPU against the oracle: a grid whose
base level is its top level (the coarse LU is the whole solve, so the top
level's matrix must be formed before the LU, not deferred)."""
import numpy as np
import pytest

from test_gpu_parity import G, ctx, assert_same, make_pair  # noqa: F401  (fixtures and helpers)

pytestmark = pytest.mark.gpu


def test_single_level_grid_3d_q1(oracle_mod, G, ctx):
    # base level = top level: the coarse LU is the whole solve; the top
    # level's matrix must be in place when the LU is formed
    O = oracle_mod
    o, g = make_pair(O, G, ctx, 3, 1, 2, 2, kcell=True, seed=31)
    assert_same(g.matrix(2), o.matrix(2), "A")
    C = G._capi
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-12, 0.0, 20,
                     C.FMG_MULTIPLICATIVE, 0)
    x = g.vector()
    hist, steps, st = g.solve(cfg, x)
    r = o.solve(O.solve_cfg(damp=0.6, compat=False, rtol=1e-12, maxsteps=20))
    assert st == 0 and np.array_equal(hist, r.history) and np.array_equal(x.get(), r.x)
