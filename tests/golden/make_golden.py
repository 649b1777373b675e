"""Generate the golden fixtures of tests/golden from the oracle.

    python tests/golden/make_golden.py

Femlisp cannot run here and ships no golden vectors of its own (its tests
assert known answers, which tests/test_oracle_kat.py checks against the
oracle).  These fixtures freeze the oracle's outputs -- assembled top-level
matrix, right-hand side, :defnorm history and solution -- on small seeded
problems, so that the GPU path is compared with fixed data and any change of
the oracle itself shows up as a failing test.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# name -> (dim, order, level, base, k-field seed or None, solve_cfg kwargs)
CASES = {
    # config C1: 2D Poisson, Q1 64^2, CG + V(1,1) Jacobi(0.6)
    "c1_q1_2d_cg": (2, 1, 6, 0, None, dict(method=O.METHOD_CG_MG, damp=0.6, compat=False, rtol=1e-10,
                                           maxsteps=100)),
    # the Femlisp known answer: 1D Q1, level 3, base 2, V(1,0) Jacobi(0.5), 10 steps
    "kat_1d_vcycle": (1, 1, 3, 2, None, dict(method=O.METHOD_MG, smoother=O.JACOBI, damp=0.5, pre=1, post=0,
                                             rtol=0.0, atol=1e-12, maxsteps=10)),
    # variable coefficient, 3D Q1 8^3 cells, CG + V(1,1) Jacobi(0.6)
    "q1_3d_vark_cg": (3, 1, 3, 1, 7, dict(method=O.METHOD_CG_MG, damp=0.6, compat=False, rtol=1e-10,
                                          maxsteps=100)),
    # 2D Q2 with multicolour SOR(1.2) V(2,2) as the iteration (config C2's smoother)
    "q2_2d_sor_mg": (2, 2, 3, 1, 3, dict(method=O.METHOD_MG, smoother=O.SOR, damp=1.2, pre=2, post=2,
                                         rtol=1e-10, maxsteps=60)),
    # the vertex-centred SSC of higher-order discretisations as the iteration, V(1,0)
    "q2_2d_ssc_mg": (2, 2, 3, 1, 5, dict(method=O.METHOD_MG, smoother=O.SSC, damp=1.0, pre=1, post=0,
                                         rtol=1e-10, maxsteps=60)),
    # 3D Q2, CG + V(1,1) PSC(0.2) (additive vertex blocks)
    "q2_3d_psc_cg": (3, 2, 2, 0, 9, dict(method=O.METHOD_CG_MG, smoother=O.PSC, damp=0.2, compat=False,
                                         rtol=1e-10, maxsteps=100)),
}


def kfield(dim, level, seed):
    n = 1 << level
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(-2.0, 2.0, n ** dim))


def make(name):
    dim, order, level, base, seed, kw = CASES[name]
    o = O.Oracle(dim, order, level, base_level=base)
    k = None
    if seed is not None:
        k = kfield(dim, level, seed)
        o.set_coefficient(O.K_CELL, k)
    o.assemble()
    r = o.solve(O.solve_cfg(**kw))
    out = dict(matrix=o.matrix(), rhs=o.rhs(), history=np.asarray(r.history), x=np.asarray(r.x),
               steps=np.int64(r.steps))
    if k is not None:
        out["k"] = k
    return out


def main():
    O.build()
    for name in CASES:
        d = make(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print(name, "steps", int(d["steps"]), "reduction", d["history"][-1] / d["history"][0])


if __name__ == "__main__":
    main()
