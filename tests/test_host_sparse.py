"""Host-side sparse conversions (no GPU): the stencil-slot storage of a level
matrix to the compressed rows that fmg_set_matrix takes back, checked against
the oracle's own matrix-vector product on scalar Q1/Q2 and the 3 x 3 block
(elasticity) levels."""
import numpy as np
import pytest

from gnu_femlisp_b200.core import slots_to_csr


def _apply(start, index, values, x):
    y = np.zeros(start.size - 1)
    for i in range(start.size - 1):
        s, e = start[i], start[i + 1]
        y[i] = np.dot(values[s:e], x[index[s:e]])
    return y


@pytest.mark.parametrize("dim,order,level,ncomp,n0", [(2, 1, 4, 1, 1), (3, 1, 3, 1, 1), (2, 2, 3, 1, 1),
                                                      (3, 2, 2, 1, 1), (3, 2, 1, 3, 2)])
def test_slots_to_csr_matches_the_oracle_matvec(oracle_mod, dim, order, level, ncomp, n0):
    O = oracle_mod
    dmask = 0b000001 if ncomp == 3 else None
    o = O.Oracle(dim, order, level, base_level=0, ncomp=ncomp, n0=n0, dirichlet_mask=dmask)
    rng = np.random.default_rng(dim * 10 + order)
    ncell = (n0 << level) ** dim
    if ncomp == 3:
        o.set_coefficient(O.LAMBDA_MU_CELL, np.exp(0.5 * rng.standard_normal(ncell)))
        o.set_coefficient(O.F_VEC, [0.0, 0.0, -1.0])
    else:
        o.set_coefficient(O.K_CELL, np.exp(rng.standard_normal(ncell)))
    o.assemble()
    start, index, values = slots_to_csr(o.matrix(), dim, order, ncomp)
    n = o.nnodes() * ncomp
    assert start.size == n + 1 and start[0] == 0 and np.all(np.diff(start) >= 0)
    assert np.all((index >= 0) & (index < n)) and np.all(values != 0.0)
    for i in range(n):  # columns ascending within a row
        assert np.all(np.diff(index[start[i]:start[i + 1]]) > 0)
    x = rng.standard_normal(n)
    y = _apply(start, index, values, x)
    ref = o.matvec(x)
    assert np.max(np.abs(y - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("start,index,values,msg", [
    ([0, 2, 5], [0, 1, 0, 1], [1.0, 2.0, 3.0, 4.0, 5.0], "index holds 4"),
    ([0, 2, 5], [0, 1, 0, 1, 2], [1.0, 2.0], "values hold 2"),
    ([0, 3, 2], [0, 1, 2], [1.0, 2.0, 3.0], "nondecreasing"),
    ([1, 2, 3], [0, 1, 2], [1.0, 2.0, 3.0], "begin at 0"),
])
def test_compressed_arrays_are_checked_before_the_c_call(start, index, values, msg):
    # a short index or value array would make the library read past the end
    # of host memory: the host wrapper refuses it before any C call
    from gnu_femlisp_b200.core import _compressed
    with pytest.raises(ValueError, match=msg):
        _compressed(start, index, values)
    st, ix, va = _compressed([0, 1, 3], [0, 0, 1], [2.0, -1.0, 2.0])
    assert st.dtype == np.int32 and ix.dtype == np.int32 and va.dtype == np.float64
