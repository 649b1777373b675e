"""Train the damping networks shipped with the package.

    python -m gnu_femlisp_b200.weights.train_damping --dim 3 [--out PATH]
    python -m gnu_femlisp_b200.weights.train_damping --dim 2 [--out PATH]
    python -m gnu_femlisp_b200.weights.train_damping --dim 3 --elastic [--out PATH]

Both minimise the A-norm contraction of one V(1,1) Jacobi cycle on errors the
multigrid itself makes (random vectors after 4 cycles of A e = 0 with the
current damping), differentiated through the whole cycle with respect to
the damping of every level (fmg_learn_step); Adam, learning rate decaying
from lr to lr/10 (cosine), 4 samples per step.  Deterministic.

3D (the 256^3 benchmark problem's class): twelve 32^3-cell grids whose
coefficient is the benchmark field's recipe (64 random Fourier modes,
|kappa| in [1, 10], unit standard deviation) on windows of side 1/8, 1/4,
1/2 and 1 of the unit cube, field seeds 1000-1011 (the benchmark uses seed
0); 1500 steps, lr 2e-3; about 15 s on one B200.

3D elasticity (--elastic; the clamped-cube vector-Q2 problem of 48^3 cells):
eight grids of 24^3 cells, Young's modulus E = exp(0.5 g) with g the same
Fourier recipe on windows of side 1/4, 1/2 and 1 (seeds 1000-1007; the
benchmark uses seed 0), the per-node damping of the 3 x 3 block Jacobi
differentiated through the block V(1,1) cycle; 800 steps, lr 2e-3.

2D (the block-field set): 128^2-cell grids, k piecewise constant on an 8 x 8
block partition with log10 k ~ U[-3, 3]; one new field per step, seeds
0 .. steps-1 (20,000 by default; held-out evaluation seeds start at
1,000,000); lr 1e-3; about 2.5 min on one B200.
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
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--elastic", action="store_true", help="the 3D elasticity net (vector Q2, block Jacobi)")
    a = ap.parse_args(argv)
    C = G._capi
    ctx = G.Context(0)
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 100,
                     C.FMG_MULTIPLICATIVE)
    net = learn.DampingNet(ctx, a.dim, seed=1)
    t0 = time.time()
    if a.elastic:
        grids = learn.elasticity_training_grids(ctx, level=3, count=8)
        hist = learn.train(net, grids, cfg, a.steps or 800, 2e-3, 4, 4, log=print)
    elif a.dim == 3:
        spec = learn.TrainSpec(dim=3, level=5, base=2, count=12, steps=a.steps or 1500, lr=2e-3, nsamples=4,
                               max_cycles=4)
        grids = learn.training_grids(ctx, spec)
        hist = learn.train(net, grids, cfg, spec.steps, spec.lr, spec.nsamples, spec.max_cycles, log=print)
    else:
        steps = a.steps or 20000
        hist = learn.train_on_fields(net, ctx, learn.block_field, range(steps), cfg, 2, 7, 2, lr=1e-3,
                                     nsamples=4, max_cycles=4, log=print)
    ctx.synchronize()
    print(f"trained {len(hist)} steps in {time.time() - t0:.1f} s, mean loss first 50 {np.mean(hist[:50]):.4f}, "
          f"last 50 {np.mean(hist[-50:]):.4f}")
    out = a.out or os.path.join(HERE, "damping3d_elastic.fmgnet" if a.elastic else f"damping{a.dim}d.fmgnet")
    net.save(out)
    print("wrote", out)


if __name__ == "__main__":
    main()
