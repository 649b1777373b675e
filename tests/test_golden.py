"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py
from the oracle): the oracle must still reproduce them bit for bit, and the
GPU path must match them -- assembled top-level matrix and right-hand side
bitwise, :defnorm history and solution to 1e-12 relative."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

import sys  # noqa: E402
sys.path.insert(0, GOLD)
import make_golden as MG  # noqa: E402

NAMES = sorted(MG.CASES)


def _fixture(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(oracle_mod, name):
    ref = _fixture(name)
    got = MG.make(name)
    for key in ("matrix", "rhs", "history", "x", "steps"):
        assert np.array_equal(got[key], ref[key]), key


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_fixture(name):
    import gnu_femlisp_b200 as G
    C = G._capi
    ref = _fixture(name)
    dim, order, level, base, seed, kw = MG.CASES[name]
    ctx = G.Context(0)
    g = G.Grid(ctx, dim, order, level, base_level=base)
    if "k" in ref:
        g.set_coefficient(C.FMG_K_CELL, ref["k"])
    g.assemble()
    assert np.array_equal(g.matrix(), ref["matrix"].reshape(g.nslots, -1))
    assert np.array_equal(g.rhs(), ref["rhs"])
    smoother = kw.get("smoother", MG.O.JACOBI)  # the oracle numbers the smoothers as the C-ABI does
    cfg = G.SolveCfg(kw["method"], smoother, kw["damp"], kw.get("pre", 1), kw.get("post", 1), 1, 0, 1.0,
                     kw.get("rtol", 0.0), kw.get("atol", 0.0), kw["maxsteps"], C.FMG_MULTIPLICATIVE)
    x = g.vector()
    hist, steps, status = g.solve(cfg, x)
    assert steps == int(ref["steps"])
    assert np.max(np.abs(hist - ref["history"]) / ref["history"]) <= 1e-12
    xs = ref["x"]
    assert np.max(np.abs(x.get() - xs)) <= 1e-12 * np.max(np.abs(xs))
