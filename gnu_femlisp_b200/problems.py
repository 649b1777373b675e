"""Seeded synthetic inputs of the benchmark configurations.

There is no public dataset for this path; each configuration is
self-describing.  All fields are generated on the host with numpy's PCG64
generator so that the GPU path, the oracle and the CPU baseline all receive
the same arrays.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def fourier_log_field(n: int, dim: int, seed: int = 0, modes: int = 64, kmin: float = 1.0,
                      kmax: float = 10.0) -> np.ndarray:
    """log k at the centres of the n^dim cells (x fastest): a sum of `modes`
    cosines a_m cos(2 pi kappa_m . x + phi_m) with |kappa_m| ~ U[kmin, kmax],
    uniformly random direction, phi ~ U[0, 2 pi), a ~ N(0, 1), normalised to
    mean 0 and standard deviation 1 over the cells."""
    rng = np.random.default_rng(seed)
    mag = rng.uniform(kmin, kmax, modes)
    direc = rng.standard_normal((modes, dim))
    direc /= np.linalg.norm(direc, axis=1, keepdims=True)
    kappa = mag[:, None] * direc
    phi = rng.uniform(0.0, 2.0 * np.pi, modes)
    amp = rng.standard_normal(modes)
    xc = (np.arange(n) + 0.5) / n
    # sum_m a_m Re(exp(i phi_m) prod_k exp(2 pi i kappa_mk x_k)), with the
    # x factor contracted as one complex matrix product (axes z, y, x)
    e = [np.exp(2j * np.pi * kappa[:, k][:, None] * xc[None, :]) for k in range(dim)]  # [m, n]
    coef = amp * np.exp(1j * phi)
    if dim == 1:
        field = np.real(coef @ e[0])
    elif dim == 2:
        field = np.real((e[1].T * coef) @ e[0])
    else:
        left = (e[2].T[:, None, :] * e[1].T[None, :, :] * coef).reshape(n * n, modes)
        field = np.real(left @ e[0])
    field = field.reshape(-1)
    field -= field.mean()
    field /= field.std()
    return field


def block_log10_field(n: int, blocks: int, seed: int, lo: float = -3.0, hi: float = 3.0) -> np.ndarray:
    """log10 k piecewise constant on a blocks x blocks partition of an n x n
    cell grid (x fastest), log10 k ~ U[lo, hi] per block."""
    rng = np.random.default_rng(seed)
    vals = rng.uniform(lo, hi, (blocks, blocks))
    bs = n // blocks
    return np.kron(vals, np.ones((bs, bs))).reshape(-1)


@dataclass
class Workload:
    name: str
    dim: int
    order: int
    level: int
    base_level: int
    kcell: np.ndarray | None      # diffusion per top-level cell, or None for k = 1
    source: object                # float or callable(points) -> f
    smoother: int                 # 0 Jacobi, 1 SOR
    damp: float
    pre: int
    post: int
    rtol: float = 1e-10

    @property
    def n_cells(self) -> int:
        return 1 << self.level

    @property
    def nodes(self) -> int:
        return (self.order * self.n_cells + 1) ** self.dim


def c1() -> Workload:
    """2D Poisson -Lap u = 1, Q1 on 64x64 cells, CG + V(1,1) Jacobi(0.6), base level 0."""
    return Workload("C1 2D Q1 64^2 Poisson", 2, 1, 6, 0, None, 1.0, 0, 0.6, 1, 1)


def c2() -> Workload:
    """3D Poisson with f = sin(pi x) sin(pi y) sin(pi z), Q2 on 64^3 cells,
    V(2,2) multicolour SOR(1.2), base level 2 (4^3 cells, dense LU)."""
    def f(p):
        return np.sin(np.pi * p[..., 0]) * np.sin(np.pi * p[..., 1]) * np.sin(np.pi * p[..., 2])
    return Workload("C2 3D Q2 64^3 Poisson sin-source", 3, 2, 6, 2, None, f, 1, 1.2, 2, 2)


def c3(seed: int = 0, level: int = 8) -> Workload:
    """3D -div(k grad u) = 1, Q1 on 256^3 cells, log k a seeded 64-mode
    Fourier field (std 1), CG + V(1,1) Jacobi(0.6), base level 2."""
    n = 1 << level
    k = np.exp(fourier_log_field(n, 3, seed))
    return Workload(f"C3 3D Q1 {n}^3 variable-k diffusion", 3, 1, level, 2, k, 1.0, 0, 0.6, 1, 1)


@dataclass
class ElasticityWorkload:
    name: str
    order: int
    n0: int
    level: int
    base_level: int
    ecell: np.ndarray             # lambda = mu = E per top-level cell
    force: tuple
    dirichlet_mask: int           # bit 0: the x = 0 face clamped (all components)
    damp: float
    pre: int
    post: int
    rtol: float = 1e-10

    @property
    def n_cells(self) -> int:
        return self.n0 << self.level

    @property
    def nodes(self) -> int:
        return (self.order * self.n_cells + 1) ** 3

    @property
    def dofs(self) -> int:
        return 3 * self.nodes


def c5(seed: int = 0, level: int = 4) -> ElasticityWorkload:
    """3D linear elasticity, vector Q2 on (3 * 2^level)^3 cells (48^3 at
    level 4: 97^3 nodes, 2,738,019 DoF), lambda = mu = E = exp(0.5 g) per
    cell with g the seeded 64-mode Fourier field of unit standard deviation
    (log-normal, sigma 0.5), body force (0, 0, -1), the x = 0 face clamped;
    CG + V(2,2) block Jacobi(0.6), base level 0 (3^3 cells, dense LU)."""
    n = 3 << level
    e = np.exp(0.5 * fourier_log_field(n, 3, seed))
    return ElasticityWorkload(f"C5 3D vector-Q2 elasticity {n}^3 cells", 2, 3, level, 0, e, (0.0, 0.0, -1.0),
                              0b000001, 0.6, 2, 2)

