"""CPU oracle for inflow / outflow regions -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import this module, as the checker; the product
(``gpufluid_b200``) never does.

NumPy restatement of the reference's region logic:

* ``outflow_keep``  -- ``apply_outflows`` (src/gpufluid/domain/regions.py:
  113-128) and the kernel pair ``k3_mark_alive_outflows`` /
  ``k3_scatter_alive`` (solver3d.py:1945-1985): a particle is dropped when
  lo <= p <= hi on all axes for any active box; survivors keep their order.
* ``emit``          -- ``InflowBox.emit`` (regions.py:42-51).
* ``inflows``       -- ``apply_inflows`` (regions.py:131-150).
* ``solid_filter``  -- the emit filter of ``prepare_frame`` (solver3d.py:
  3985-4012): drop emitted positions whose cell (clipped int(p/dx)) is solid.
* ``prepare_frame`` -- outflows, then inflows, then the filter and the append
  (solver3d.py:3946-4040).

Parity pin: ``tests/golden/regions/regions.npz`` holds the reference module's own
outputs (``tests/golden/make_regions_golden.py``); ``tests/test_regions.py``
checks this restatement against them.
"""
from __future__ import annotations

import numpy as np


def outflow_keep(pos, boxes):
    """Boolean mask of the particles inside no box; boxes: (k, 6) lo, hi."""
    keep = np.ones(len(pos), dtype=bool)
    for b in np.asarray(boxes, np.float32).reshape(-1, 6):
        lo, hi = b[:3], b[3:]
        keep &= ~np.all((pos >= lo) & (pos <= hi), axis=1)
    return keep


def emit(lo, hi, rate_per_sec, frame_start, frame_end, frame_idx, frame_dt, rng):
    if frame_idx < frame_start or frame_idx > frame_end:
        return None
    n = int(round(rate_per_sec * frame_dt))
    if n <= 0:
        return None
    lo = np.asarray(lo, dtype=np.float32)
    hi = np.asarray(hi, dtype=np.float32)
    return lo + (hi - lo) * rng.random((n, 3)).astype(np.float32)


def inflows(boxes, frame_idx, frame_dt, rng):
    """boxes: list of dicts with lo, hi, velocity, rate_per_sec, frame_start, frame_end."""
    ps, vs = [], []
    for b in boxes:
        p = emit(b["lo"], b["hi"], b["rate_per_sec"], b["frame_start"], b["frame_end"],
                 frame_idx, frame_dt, rng)
        if p is None or len(p) == 0:
            continue
        ps.append(p)
        vs.append(np.broadcast_to(np.asarray(b["velocity"], dtype=np.float32),
                                  (len(p), 3)).copy())
    if not ps:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32)
    return np.concatenate(ps), np.concatenate(vs)


def solid_filter(pos, marker, dx):
    ix = np.clip((pos[:, 0] / dx).astype(np.int32), 0, marker.shape[0] - 1)
    iy = np.clip((pos[:, 1] / dx).astype(np.int32), 0, marker.shape[1] - 1)
    iz = np.clip((pos[:, 2] / dx).astype(np.int32), 0, marker.shape[2] - 1)
    return marker[ix, iy, iz] != 2


def prepare_frame(pos, vel, out_boxes, in_boxes, frame_idx, frame_dt, rng, marker, dx):
    """Particles (original order) after one frame's outflows and inflows.
    out_boxes: list of (lo, hi, frame_start, frame_end)."""
    active = [[*lo, *hi] for lo, hi, a, b in out_boxes if a <= frame_idx <= b]
    if active and len(pos):
        keep = outflow_keep(pos, active)
        pos, vel = pos[keep], vel[keep]
    ep, ev = inflows(in_boxes, frame_idx, frame_dt, rng)
    if len(ep):
        keep = solid_filter(ep, marker, dx)
        ep, ev = ep[keep], ev[keep]
    if len(ep):
        pos = np.concatenate([pos, ep])
        vel = np.concatenate([vel, ev])
    return pos, vel
