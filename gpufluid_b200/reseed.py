"""Particle reseeding (src/gpufluid/sim/reseed.py, S2.11.GPU).

Keeps the particle density per cell bounded: in every non-solid cell the
particles beyond ``max_per_cell`` are removed, particles in solid cells are
removed, and every fluid cell (marked fluid by the last substep, or holding
particles) with fewer than ``min_per_cell`` gets the deficit at jittered cell
centres with zero velocity.  ``FlipSolver3D.reseed`` runs it on the GPU
(binning, ranking, stream compaction) with the emission list built on the
host from the per-cell counts, as the reference's ``reseed_particles_gpu``
does; the command line calls it every ``reseed_every_n_frames`` frames.

The reference switches to a host implementation below 100,000 particles
(``reseed_particles``), which picks the culled particles with the generator;
this package always follows the device semantics, whose culled set (the
first ``max_per_cell`` of each cell by particle order) is one the reference's
device path produces.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class ReseedConfig:
    """reseed.py:31-36."""
    min_per_cell: int = 4
    max_per_cell: int = 16
    jitter: float = 0.3
    every_n_frames: int = 5
