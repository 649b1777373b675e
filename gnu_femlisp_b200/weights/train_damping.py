"""Train the damping network shipped with the package.

    python -m gnu_femlisp_b200.weights.train_damping [--dim 3] [--out PATH]

3D: twelve 32^3-cell grids whose coefficient is the 256^3 benchmark problem's
field recipe (64 random Fourier modes, |kappa| in [1, 10], unit standard
deviation) on windows of side 1/8, 1/4, 1/2 and 1 of the unit cube, field
seeds 1000-1011 (the benchmark uses seed 0), so the net sees the cell-to-cell
contrast of every level of the 256^3 hierarchy.  1500 Adam steps, learning
rate 2e-3 -> 2e-4 (cosine), 4 samples per step, each a random error after 4
cycles of the current network's V(1,1) cycle.  Takes about 15 s on one B200.
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(argv=None):
    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import learn
    ap = argparse.ArgumentParser()
    ap.add_argument("--dim", type=int, default=3)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    C = G._capi
    ctx = G.Context(0)
    spec = learn.TrainSpec(dim=a.dim, level=5 if a.dim == 3 else 7, base=2, count=12, steps=a.steps, lr=2e-3,
                           nsamples=4, max_cycles=4)
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, spec.damp, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 100,
                     C.FMG_MULTIPLICATIVE)
    grids = learn.training_grids(ctx, spec)
    net = learn.DampingNet(ctx, a.dim, seed=1)
    t0 = time.time()
    hist = learn.train(net, grids, cfg, spec.steps, spec.lr, spec.nsamples, spec.max_cycles, log=print)
    ctx.synchronize()
    print(f"trained {spec.steps} steps in {time.time() - t0:.1f} s, final mean loss "
          f"{np.mean(hist[-50:]):.4f}")
    out = a.out or os.path.join(HERE, f"damping{a.dim}d.fmgnet")
    net.save(out)
    print("wrote", out)


if __name__ == "__main__":
    main()
