"""B200-native multigrid solve path for Femlisp (libfmgpu).

Conjugate gradients preconditioned by a geometric correction-scheme V-cycle
with damped-Jacobi / multicolour-SOR smoothing on Lagrange Q1/Q2 level
matrices, all on one GPU behind the C-ABI in ``include/fmgpu.h``.
"""
from ._capi import FmgError, MixedCfg, SolveCfg  # noqa: F401
from .core import Context, Grid, Vector, slots_to_csr  # noqa: F401
from .iteration import (CG, LU, SOR, AlgebraicSystem, CdrProblem, GaussSeidel, GeometricCS, GeometricPSC, GeometricSSC, Jacobi,  # noqa: F401
                        LagrangeFE, LinearSolver, LocalMG, Mesh, cdr_model_problem, discretize_globally,
                        geometric_cs, geometric_psc, geometric_ssc, lagrange_fe, local_mg, sample_at_gauss_points, solve,
                        uniformly_refined_hierarchical_mesh)

__all__ = [
    "FmgError", "MixedCfg", "SolveCfg", "Context", "Grid", "Vector", "slots_to_csr", "AlgebraicSystem", "CG", "LU", "SOR", "GaussSeidel",
    "GeometricCS", "GeometricPSC", "GeometricSSC", "Jacobi", "CdrProblem", "LagrangeFE", "LinearSolver", "LocalMG", "Mesh",
    "cdr_model_problem", "discretize_globally", "geometric_cs", "geometric_psc", "geometric_ssc", "lagrange_fe",
    "local_mg", "sample_at_gauss_points", "solve", "uniformly_refined_hierarchical_mesh",
]
