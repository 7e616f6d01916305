"""Generate golden vectors for inflow / outflow regions from the reference's
own ``gpufluid.domain.regions`` (src/gpufluid/domain/regions.py).

Test-fixture generator (run by hand, in a container that holds the reference
checkout; nothing at test or bench time reads the reference):

    python tests/golden/make_regions_golden.py --reference <path of the GPUFLUID checkout>

It imports the reference module unmodified (pure NumPy, no Warp needed) and
records:

* ``apply_outflows`` on 4,096 seeded particles plus 12 placed exactly on box
  faces, edges and corners, against three boxes (one outside its frame range);
* ``apply_inflows`` from two boxes over frames 0-3 at 1/24 s with the solver's
  generator (``default_rng(0)``, solver3d.py:2494), one box starting at frame 2.

Writes ``tests/golden/regions/regions.npz`` (its own folder: the solver fixtures are
globbed from ``tests/golden/*.npz``).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

OUT_BOXES = [((0.0, 0.0, 0.0), (0.25, 0.25, 0.25), 0, 10),
             ((0.5, 0.1, 0.6), (0.75, 0.9, 1.0), 0, 10),
             ((0.3, 0.3, 0.3), (0.6, 0.6, 0.6), 5, 10)]   # inactive at frame 2
OUT_FRAME = 2
IN_BOXES = [dict(lo=(0.1, 0.6, 0.1), hi=(0.3, 0.8, 0.3), velocity=(0.0, -2.0, 0.5),
                 rate_per_sec=2400.0, frame_start=0, frame_end=10),
            dict(lo=(0.55, 0.5, 0.55), hi=(0.9, 0.6, 0.9), velocity=(1.0, 0.0, 0.0),
                 rate_per_sec=1000.0, frame_start=2, frame_end=10)]
IN_FRAMES = 4
IN_DT = 1.0 / 24.0


def outflow_inputs():
    rng = np.random.default_rng(123)
    pos = rng.random((4096, 3)).astype(np.float32)
    edge = np.array([[0.25, 0.25, 0.25], [0.0, 0.0, 0.0], [0.25, 0.1, 0.2],
                     [0.2500001, 0.1, 0.1], [0.5, 0.1, 0.6], [0.75, 0.9, 1.0],
                     [0.75, 0.5, 0.8], [0.7500001, 0.5, 0.8], [0.6, 0.1, 0.6],
                     [0.3, 0.3, 0.3], [0.45, 0.45, 0.45], [0.1, 0.2, 0.2500001]],
                    dtype=np.float32)
    pos = np.concatenate([pos, edge])
    vel = rng.normal(size=pos.shape).astype(np.float32)
    return pos, vel


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GPUFLUID_REFERENCE"),
                    required="GPUFLUID_REFERENCE" not in os.environ,
                    help="GPUFLUID source checkout (or set GPUFLUID_REFERENCE)")
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(args.reference, "src"))
    from gpufluid.domain.regions import InflowBox, OutflowBox, apply_inflows, apply_outflows

    pos, vel = outflow_inputs()
    outs = [OutflowBox(lo=lo, hi=hi, frame_start=a, frame_end=b) for lo, hi, a, b in OUT_BOXES]
    kept_pos, kept_vel = apply_outflows(pos, vel, outs, frame_idx=OUT_FRAME)

    infs = [InflowBox(**d) for d in IN_BOXES]
    rng = np.random.default_rng(0)
    em_pos, em_vel, em_frame = [], [], []
    for f in range(IN_FRAMES):
        p, v = apply_inflows(infs, f, IN_DT, rng)
        em_pos.append(p)
        em_vel.append(v)
        em_frame.append(np.full(len(p), f, np.int32))
    np.savez_compressed(
        os.path.join(HERE, "regions", "regions.npz"),
        out_pos=pos, out_vel=vel, kept_pos=kept_pos, kept_vel=kept_vel,
        emit_pos=np.concatenate(em_pos), emit_vel=np.concatenate(em_vel),
        emit_frame=np.concatenate(em_frame))
    print("kept", len(kept_pos), "of", len(pos), "; emitted", sum(len(p) for p in em_pos))


if __name__ == "__main__":
    main()
