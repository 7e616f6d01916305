"""Inflow and outflow regions (src/gpufluid/domain/regions.py:23-119).

``InflowBox`` emits particles inside a box every frame at a rate; the
positions come from the solver's own seeded generator on the host, as in the
reference (``emit``, regions.py:42-51).  ``OutflowBox`` removes every particle
inside its box; the solver does that on the GPU (``gf_outflow_compact``, a
mark / scan / scatter stream compaction that keeps the survivors' order).
Both are active for frames in [frame_start, frame_end].

Register them with ``FlipSolver3D.add_inflow`` / ``add_outflow``; they act in
``FlipSolver3D.prepare_frame`` (outflows first, then inflows), which the
command line calls once per frame.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np


@dataclass
class InflowBox:
    """A box that emits ``round(rate_per_sec * frame_dt)`` particles per frame
    with velocity ``velocity``.  ``color`` / ``temperature`` are accepted for
    scene-file compatibility; this build carries no particle attributes, so,
    like the reference's solver without attribute arrays, it ignores them."""
    lo: Tuple[float, float, float]
    hi: Tuple[float, float, float]
    velocity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rate_per_sec: float = 5000.0
    frame_start: int = 0
    frame_end: int = 10_000
    color: Optional[Tuple[float, float, float]] = None
    temperature: Optional[float] = None

    def active(self, frame_idx: int) -> bool:
        return self.frame_start <= frame_idx <= self.frame_end

    def emit(self, frame_idx: int, frame_dt: float,
             rng: np.random.Generator) -> Optional[np.ndarray]:
        """(N, 3) float32 positions, or None when not emitting this frame:
        lo + (hi - lo) * U[0,1) in float32, drawn from ``rng`` (regions.py:42-51)."""
        if not self.active(frame_idx):
            return None
        n = int(round(self.rate_per_sec * frame_dt))
        if n <= 0:
            return None
        lo = np.asarray(self.lo, dtype=np.float32)
        hi = np.asarray(self.hi, dtype=np.float32)
        return lo + (hi - lo) * rng.random((n, 3)).astype(np.float32)


@dataclass
class OutflowBox:
    """A box that removes every particle with lo <= p <= hi on all axes."""
    lo: Tuple[float, float, float]
    hi: Tuple[float, float, float]
    frame_start: int = 0
    frame_end: int = 10_000

    def __post_init__(self):
        for axis, (lo_v, hi_v) in enumerate(zip(self.lo, self.hi)):
            if hi_v < lo_v:
                name = "xyz"[axis]
                raise ValueError(f"OutflowBox: hi[{name}]={hi_v} < lo[{name}]={lo_v}; an outflow "
                                 f"box needs hi >= lo on every axis (got lo={self.lo}, "
                                 f"hi={self.hi}).")

    def active(self, frame_idx: int) -> bool:
        return self.frame_start <= frame_idx <= self.frame_end


def apply_inflows(inflows: List[InflowBox], frame_idx: int, frame_dt: float,
                  rng: np.random.Generator) -> Tuple[np.ndarray, np.ndarray]:
    """Positions and velocities emitted by all inflows this frame, in list
    order (regions.py:131-150)."""
    pos, vel = [], []
    for inf in inflows:
        p = inf.emit(frame_idx, frame_dt, rng)
        if p is None or len(p) == 0:
            continue
        pos.append(p)
        vel.append(np.broadcast_to(np.asarray(inf.velocity, dtype=np.float32),
                                   (len(p), 3)).copy())
    if not pos:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32)
    return np.concatenate(pos, axis=0), np.concatenate(vel, axis=0)


def outflow_box_array(outflows: List[OutflowBox], frame_idx: int) -> np.ndarray:
    """(k, 6) float32 {lo, hi} rows of the outflows active this frame, the
    box table ``gf_outflow_compact`` takes."""
    rows = [[*o.lo, *o.hi] for o in outflows if o.active(frame_idx)]
    return np.asarray(rows, dtype=np.float32).reshape(-1, 6)
