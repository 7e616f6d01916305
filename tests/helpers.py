"""Shared helpers for the GPU parity tests (scene construction, comparisons)."""
from __future__ import annotations

import numpy as np


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def assert_bitexact(name, got, want):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    if got.dtype == np.float32:
        gb, wb = got.view(np.uint32), want.astype(np.float32).view(np.uint32)
    else:
        gb, wb = got, want.astype(got.dtype)
    bad = np.flatnonzero(gb.ravel() != wb.ravel())
    assert bad.size == 0, (f"{name}: {bad.size}/{got.size} differ, first {bad[:5]}: "
                           f"got {got.ravel()[bad[:5]]} want {want.ravel()[bad[:5]]}")


def random_particles(nx, ny, nz, dx, n, seed=0, outside=0.02, vel_sigma=1.0):
    """Seeded positions over the domain, a few just outside it (the reference
    clamps their cell index), and Gaussian velocities."""
    rng = np.random.default_rng(seed)
    dom = np.array([nx, ny, nz], np.float64) * dx
    pos = rng.random((n, 3)) * dom
    k = int(n * outside)
    if k:
        pos[:k] = rng.uniform(-0.5, 1.5, size=(k, 3)) * dx + rng.choice([0.0, 1.0], size=(k, 3)) * (dom - dx)
    vel = rng.normal(0.0, vel_sigma, size=(n, 3))
    C = rng.normal(0.0, 2.0, size=(n, 3, 3))
    return pos.astype(np.float32), vel.astype(np.float32), C.astype(np.float32)


def dam_break(solver_cls, n, transfer="flip", sphere=None, box=((0.0, 0.0, 0.0), (0.4, 0.6, 1.0)),
              **kw):
    from gpufluid_b200 import scene
    s = solver_cls(n[0], n[1], n[2], transfer_mode=transfer, **kw)
    if sphere is not None:
        s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), *sphere))
    s.seed_box(*box)
    return s
