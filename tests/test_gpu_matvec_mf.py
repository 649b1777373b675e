"""The matrix-free top-level operator (fmg_matvec_mf: the operator the mixed
solve applies on a 3D Q1 top level) against the oracle's restatement of its
operation order, bit for bit, in FP64 and FP32, as y = A x and as the
residual b - A x; and against the assembled matrix of assemble-interior
(fedisc.lisp:108-206, sparse-matrix.lisp:392-405) within rounding.

The sizes cover both halves of the kernel: 17^3 nodes has no whole tile and
runs entirely on the face CTAs; 33^3, 65^3 and 129^3 have tiled boxes with
faces beside them.  The Dirichlet masks cover all faces, none, and the mixed
cases that put eliminated columns inside the staged rows (x = 0, x = M - 1)
and on the rows and planes the copies fetch as zeros."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gnu_femlisp_b200 as G
    return G


@pytest.fixture(scope="module")
def ctx(G):
    return G.Context(0)


CASES = [(4, 63), (5, 63), (5, 0), (5, 1 | 8 | 32), (5, 2 | 4 | 16), (6, 63), (6, 1 | 2), (6, 3 | 12), (7, 63)]


@pytest.mark.parametrize("level,dmask", CASES)
def test_matvec_mf_bitwise_with_oracle(oracle_mod, G, ctx, level, dmask):
    O = oracle_mod
    rng = np.random.default_rng(100 * level + dmask)
    n = 2 ** level
    M = n + 1
    kcell = np.exp(rng.standard_normal(n ** 3))
    g = G.Grid(ctx, 3, 1, level, base_level=min(2, level - 1), dirichlet_mask=dmask)
    g.set_coefficient(G._capi.FMG_K_CELL, kcell)
    g.assemble()
    xv, bv, yv = g.vector(), g.vector(), g.vector()
    x = rng.uniform(-1, 1, M ** 3)
    b = rng.uniform(-1, 1, M ** 3)
    xv.set(x)
    bv.set(b)
    for fp32 in (False, True, 2):
        for with_b in ((False, True) if fp32 != 2 else (False,)):
            g.matvec_mf(xv, yv, b=bv if with_b else None, fp32=fp32)
            got = yv.get()
            want = O.mf_apply(M, dmask, kcell, x, b if with_b else None, fp32=fp32)
            assert np.array_equal(got, want), (fp32, with_b, np.max(np.abs(got - want)))
    # the FP64 form is the assembled operator up to rounding
    g.matvec_mf(xv, yv)
    ymf = yv.get()
    g.matvec(xv, yv)
    yas = yv.get()
    scale = np.max(np.abs(yas))
    assert np.max(np.abs(ymf - yas)) <= 1e-13 * scale


def test_matvec_mf_two_calls_and_large(oracle_mod, G, ctx):
    """257^3 (the benchmark's top level, 1024 tiles and 197,377 face nodes):
    FP64 residual bitwise with the oracle, twice in a row."""
    O = oracle_mod
    level = 8
    n = 2 ** level
    M = n + 1
    rng = np.random.default_rng(8)
    kcell = np.exp(rng.standard_normal(n ** 3))
    g = G.Grid(ctx, 3, 1, level, base_level=2)
    g.set_coefficient(G._capi.FMG_K_CELL, kcell)
    g.assemble()
    xv, bv, yv = g.vector(), g.vector(), g.vector()
    x = rng.uniform(-1, 1, M ** 3)
    b = rng.uniform(-1, 1, M ** 3)
    xv.set(x)
    bv.set(b)
    want = O.mf_apply(M, 63, kcell, x, b)
    for _ in range(2):
        g.matvec_mf(xv, yv, b=bv)
        assert np.array_equal(yv.get(), want)
    for fp32 in (True, 2):
        want32 = O.mf_apply(M, 63, kcell, x, None, fp32=fp32)
        g.matvec_mf(xv, yv, fp32=fp32)
        assert np.array_equal(yv.get(), want32), fp32


def test_matvec_mf_refuses_other_grids(G, ctx):
    g = G.Grid(ctx, 2, 1, 4, base_level=1)
    g.assemble()
    xv, yv = g.vector(), g.vector()
    with pytest.raises(Exception):
        g.matvec_mf(xv, yv)
