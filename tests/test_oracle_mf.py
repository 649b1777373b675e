"""The oracle's matrix-free restatement of the 3D Q1 operator (the order of
operations of the GPU's matrix-free top level) against its assembled matrix
(assemble-interior, fedisc.lisp:108-206; eliminated Dirichlet columns,
constraints.lisp:323-411): equal up to rounding in FP64, within FP32 rounding
in FP32, for full and partial Dirichlet masks."""
import numpy as np
import pytest


@pytest.mark.parametrize("level,dmask", [(3, 63), (4, 63), (4, 0), (4, 1 | 8 | 32), (4, 2 | 4 | 16)])
def test_mf_apply_is_the_assembled_operator(oracle_mod, level, dmask):
    O = oracle_mod
    rng = np.random.default_rng(level * 64 + dmask)
    n = 2 ** level
    M = n + 1
    kcell = np.exp(rng.standard_normal(n ** 3))
    o = O.Oracle(3, 1, level, base_level=1, dirichlet_mask=dmask)
    o.set_coefficient(O.K_CELL, kcell)
    o.assemble()
    x = rng.uniform(-1, 1, M ** 3)
    b = rng.uniform(-1, 1, M ** 3)
    ya = o.matvec(x)
    scale = np.max(np.abs(ya))
    assert np.max(np.abs(O.mf_apply(M, dmask, kcell, x) - ya)) <= 1e-13 * scale
    assert np.max(np.abs(O.mf_apply(M, dmask, kcell, x, b) - (b - ya))) <= 1e-13 * scale
    assert np.max(np.abs(O.mf_apply(M, dmask, kcell, x, fp32=True) - ya)) <= 1e-5 * scale
