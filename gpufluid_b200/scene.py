"""Host-side scene set-up: particle seeding and analytic SDFs.

These run once per scene on the host, as they do in the reference:

* ``seed_box_positions`` -- ``FlipSolver3D.seed_box`` (solver3d.py:2826-2850):
  jittered lattice, ``per_axis = round(ppc ** (1/3))`` sub-positions per axis,
  one fresh ``np.random.default_rng(0)`` stream per call with three draws per
  particle (x, y, z) in loop order i, j, k, sx, sy, sz; float64 arithmetic,
  float32 result.  Vectorised: a single ``rng.random(3 * n)`` call yields the
  same stream as the reference's per-particle ``rng.random()`` calls.
* ``seed_sphere_positions`` -- the same lattice restricted to cells whose
  centre lies inside a sphere (a seeder the reference does not have).
* ``cell_centers``, ``sdf_sphere``, ``sdf_box``, ``sdf_cylinder_y``,
  ``sdf_plane`` -- the analytic SDFs of primitives/sdf.py:31-80 (the obstacle
  shapes of the scene TOML; a cell is solid where the SDF is <= 0).
"""
from __future__ import annotations

import numpy as np


def cell_centers(nx: int, ny: int, nz: int, dx: float) -> np.ndarray:
    i = (np.arange(nx) + 0.5) * dx
    j = (np.arange(ny) + 0.5) * dx
    k = (np.arange(nz) + 0.5) * dx
    X, Y, Z = np.meshgrid(i, j, k, indexing="ij")
    return np.stack([X, Y, Z], axis=-1).astype(np.float32)


def sdf_sphere(grid_xyz: np.ndarray, center, radius: float) -> np.ndarray:
    c = np.asarray(center, dtype=np.float32)
    return np.linalg.norm(grid_xyz - c, axis=-1) - float(radius)


def sdf_box(grid_xyz: np.ndarray, center, half_size) -> np.ndarray:
    c = np.asarray(center, dtype=np.float32)
    h = np.asarray(half_size, dtype=np.float32)
    d = np.abs(grid_xyz - c) - h
    outside = np.linalg.norm(np.maximum(d, 0.0), axis=-1)
    inside = np.minimum(np.max(d, axis=-1), 0.0)
    return outside + inside


def sdf_cylinder_y(grid_xyz: np.ndarray, center, radius: float, half_height: float) -> np.ndarray:
    """Capped cylinder with its axis along y."""
    q = grid_xyz - np.asarray(center, dtype=np.float32)
    d_rad = np.sqrt(q[..., 0] ** 2 + q[..., 2] ** 2) - float(radius)
    d_ax = np.abs(q[..., 1]) - float(half_height)
    return (np.sqrt(np.maximum(d_rad, 0.0) ** 2 + np.maximum(d_ax, 0.0) ** 2)
            + np.minimum(np.maximum(d_rad, d_ax), 0.0))


def sdf_plane(grid_xyz: np.ndarray, point, normal) -> np.ndarray:
    """Half-space, negative on the -normal side of ``point``."""
    nrm = np.asarray(normal, dtype=np.float32)
    nrm = nrm / (np.linalg.norm(nrm) + 1e-12)
    return ((grid_xyz - np.asarray(point, dtype=np.float32)) * nrm).sum(axis=-1)


def _lattice(cells: np.ndarray, per_axis: int, dx: float) -> np.ndarray:
    n_cells = cells.shape[0]
    n = n_cells * per_axis ** 3
    if n == 0:
        return np.zeros((0, 3), np.float32)
    r = np.random.default_rng(0).random(3 * n).reshape(n, 3)
    sub = np.stack(np.meshgrid(np.arange(per_axis), np.arange(per_axis), np.arange(per_axis),
                               indexing="ij"), axis=-1).reshape(-1, 3).astype(np.float64)
    cell = np.repeat(cells.astype(np.float64), per_axis ** 3, axis=0)
    subs = np.tile(sub, (n_cells, 1))
    pos = (cell + (subs + 0.5 + 0.3 * (r - 0.5)) / per_axis) * dx
    return pos.astype(np.float32)


def seed_box_positions(dx: float, lo, hi, ppc: int = 8) -> np.ndarray:
    i0, i1 = int(lo[0] / dx), int(hi[0] / dx)
    j0, j1 = int(lo[1] / dx), int(hi[1] / dx)
    k0, k1 = int(lo[2] / dx), int(hi[2] / dx)
    per_axis = int(round(ppc ** (1.0 / 3.0)))
    I, J, K = np.meshgrid(np.arange(i0, i1), np.arange(j0, j1), np.arange(k0, k1), indexing="ij")
    cells = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1)
    return _lattice(cells, per_axis, dx)


def seed_sphere_positions(nx: int, ny: int, nz: int, dx: float, center, radius: float,
                          ppc: int = 8) -> np.ndarray:
    per_axis = int(round(ppc ** (1.0 / 3.0)))
    inside = sdf_sphere(cell_centers(nx, ny, nz, dx), center, radius) <= 0.0
    cells = np.argwhere(inside)
    return _lattice(cells, per_axis, dx)


def wall_labels(nx: int, ny: int, nz: int) -> np.ndarray:
    """One-cell solid shell (solver3d.py:2475-2482) as uint8 labels."""
    m = np.zeros((nx, ny, nz), dtype=np.uint8)
    m[0, :, :] = 2; m[-1, :, :] = 2
    m[:, 0, :] = 2; m[:, -1, :] = 2
    m[:, :, 0] = 2; m[:, :, -1] = 2
    return m
