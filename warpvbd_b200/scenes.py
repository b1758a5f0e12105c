"""Procedural test scenes (cantilever beam, hanging mass-spring, env batches).

Geometry and boundary conditions follow the reference's scene scripts:

* cantilever: ``examples/run_cantilever.py:27-46`` -- a voxelised beam, the
  vertices with x < 1e-3 fixed, the vertices with x > L - 1e-3 the tip face;
* mass-spring: ``examples/run_mass_spring.py:30-54`` -- a cube hanging from a
  one-voxel column, the top face of the column fixed, the bottom face of the
  cube the tip.  Here the cube edge and column length are free parameters and
  the voxel edge is fixed (1 cm), so the default (11, 20) is an 11x11x11 cube
  under a 1x1x20 column;
* batches: several mass-springs of different sizes and materials drawn from a
  seeded generator (the reference draws unseeded moduli,
  ``examples/run_mass_spring_parallel.py:70``).
"""
from dataclasses import dataclass, field

import numpy as np

from .mesh import voxel2hex, hex2tets


@dataclass
class Scene:
    name: str
    vertices: np.ndarray          # float64 [V, 3] rest positions
    tets: np.ndarray              # int32 [T, 4]
    active: np.ndarray            # bool [V]
    tip: np.ndarray               # int64 [n_tip] tip-face vertex ids
    density: np.ndarray           # float64 [T]
    youngs: np.ndarray            # float64 [T]
    poisson: np.ndarray           # float64 [T]
    meta: dict = field(default_factory=dict)

    @property
    def n_vertices(self):
        return self.vertices.shape[0]

    @property
    def n_tets(self):
        return self.tets.shape[0]

    def solver_kwargs(self):
        return dict(initial_positions=self.vertices, elements=self.tets,
                    densities=self.density, youngs_modulus=self.youngs,
                    poissons_ratio=self.poisson, active_mask=self.active)


def cantilever(nx=20, ny=None, nz=None, length=1.0, youngs=1e6, poisson=0.45, density=1000.0):
    """Beam of ``length`` x length/10 x length/10 voxelised nx x ny x nz; x=0 face fixed."""
    ny = nx // 10 if ny is None else ny
    nz = nx // 10 if nz is None else nz
    h = length / nx
    vox = np.ones((nx, ny, nz), dtype=bool)
    X, hexes = voxel2hex(vox, h, h, h)
    tets = hex2tets(hexes).astype(np.int32)
    active = ~(X[:, 0] < 1e-3)
    tip = np.nonzero(active & (X[:, 0] > nx * h - 1e-3))[0]
    T = tets.shape[0]
    return Scene(f"cantilever_{nx}x{ny}x{nz}", X, tets, active, tip,
                 np.full(T, density), np.full(T, youngs), np.full(T, poisson),
                 {"voxel": h, "shape": (nx, ny, nz)})


def mass_spring(cube=11, column=20, voxel=0.01, youngs=5e5, poisson=0.4, density=1000.0):
    """cube^3 voxels hanging from a 1x1xcolumn column whose top face is fixed."""
    vox = np.zeros((cube, cube, cube + column), dtype=bool)
    vox[:, :, :cube] = True
    vox[cube // 2, cube // 2, cube:] = True
    X, hexes = voxel2hex(vox, voxel, voxel, voxel)
    tets = hex2tets(hexes).astype(np.int32)
    top = (cube + column) * voxel
    active = ~(X[:, 2] > top - 1e-4)
    tip = np.nonzero(X[:, 2] < 1e-4)[0]
    T = tets.shape[0]
    return Scene(f"massspring_{cube}_{column}", X, tets, active, tip,
                 np.full(T, density), np.full(T, youngs), np.full(T, poisson),
                 {"voxel": voxel, "cube": cube, "column": column})


def env_batch(n_env=256, seed=0, cube=(7, 15), column=(5, 30), youngs=(1e5, 1e6),
              poisson=(0.35, 0.48), density=1000.0):
    """Seeded batch of uneven mass-spring environments: cube edge and column
    length uniform integers, E log-uniform, nu uniform."""
    rng = np.random.default_rng(seed)
    envs = []
    for _ in range(n_env):
        c = int(rng.integers(cube[0], cube[1] + 1))
        L = int(rng.integers(column[0], column[1] + 1))
        E = float(np.exp(rng.uniform(np.log(youngs[0]), np.log(youngs[1]))))
        nu = float(rng.uniform(poisson[0], poisson[1]))
        envs.append(mass_spring(c, L, youngs=E, poisson=nu, density=density))
    return envs
