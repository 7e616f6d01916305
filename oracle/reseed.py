"""CPU oracle for GPU particle reseeding -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import this module, as the checker; the product
(``gpufluid_b200``) never does.

NumPy restatement of ``reseed_particles_gpu`` (src/gpufluid/sim/reseed.py:
275-396) with its kernels ``k_count_particles_per_cell`` (:161-181),
``k_mark_keep_by_rank`` (:185-222) and ``k_scatter_alive_pv`` (:226-243):

* each particle's cell is floor(p/dx) clamped to the grid (float32 divide);
* a particle in a solid cell (marker 2) is dropped; otherwise it is kept when
  its rank among its cell's particles is below ``max_per_cell``.  The
  reference takes the rank from an atomic counter, so any arrival order is
  valid; this restatement (like the GPU path here) ranks by particle index,
  the order sequential threads produce;
* survivors keep their order; then every fluid cell ((marker 1 or counted
  particles) and not solid) with fewer than ``min_per_cell`` particles gets
  the deficit, placed at (cell + 0.5 + jitter * (U - 0.5)) * dx with U from
  ``rng`` in C order of the cells, velocity 0.

Parity pin: ``tests/golden/reseed/reseed.npz`` holds the reference function's
own outputs run on the sequential Warp stand-in
(``tests/golden/make_reseed_golden.py``); ``tests/test_reseed.py`` checks this
restatement against them.
"""
from __future__ import annotations

import numpy as np


def cells_of(pos, dx, shape):
    nx, ny, nz = shape
    f = (pos / np.float32(dx)).astype(np.float32)
    i = np.clip(np.floor(f[:, 0]).astype(np.int64), 0, nx - 1)
    j = np.clip(np.floor(f[:, 1]).astype(np.int64), 0, ny - 1)
    k = np.clip(np.floor(f[:, 2]).astype(np.int64), 0, nz - 1)
    return i, j, k


def reseed(pos, vel, marker, dx, min_per_cell, max_per_cell, jitter, rng):
    """(new_pos, new_vel, n_emit, n_cull)."""
    nx, ny, nz = marker.shape
    n = len(pos)
    counts = np.zeros(marker.shape, np.int64)
    alive = np.zeros(n, bool)
    if n:
        i, j, k = cells_of(pos, dx, marker.shape)
        flat = (i * ny + j) * nz + k
        np.add.at(counts.reshape(-1), flat, 1)
        seen = np.zeros(nx * ny * nz, np.int64)
        solid = marker.reshape(-1) == 2
        for p in range(n):  # ranks in index order
            c = flat[p]
            if solid[c]:
                continue
            alive[p] = seen[c] < max_per_cell
            seen[c] += 1
    kept_p, kept_v = pos[alive], vel[alive]
    n_cull = n - int(alive.sum())
    solid = marker == 2
    fluid = ((marker == 1) | (counts > 0)) & ~solid
    deficit = np.clip(min_per_cell - counts, 0, None)
    deficit[~fluid] = 0
    n_emit = int(deficit.sum())
    if n_emit == 0:
        return kept_p, kept_v, 0, n_cull
    idx = np.argwhere(deficit > 0)
    rep = deficit[deficit > 0]
    cells = np.repeat(idx, rep, axis=0).astype(np.float32)
    jit = (rng.random((n_emit, 3)) - 0.5).astype(np.float32) * jitter
    emit = (cells + 0.5 + jit) * dx
    return (np.concatenate([kept_p, emit]), np.concatenate([kept_v, np.zeros_like(emit)]),
            n_emit, n_cull)
